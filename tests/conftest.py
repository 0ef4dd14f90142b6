import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _build_all():
    import importlib.util
    spec = importlib.util.spec_from_file_location("fmx_build", os.path.join(ROOT, "flashx_b200", "build.py"))
    fb = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(fb)
    fb.build()
    import oracle
    oracle.build(ref=None)


_build_all()


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch
