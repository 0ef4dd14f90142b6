"""The FlashMatrix-side binding (include/fmx_flashmatrix.hpp) is compiled
code, not prose: it is built here against stand-ins that carry the
reference's declarations of matrix_store, mem_matrix_store, scalar_type and
BOOST_LOG_TRIVIAL (tests/shim/flashmatrix_standin.h) and linked with
libfmx.so.  Without a GPU, loading reports the missing device the way
sparse_matrix::create's callers see a failure (null plus a log line); on a
GPU the binding's multiply refuses what sparse_matrix::multiply refuses
(sparse_matrix.cpp:709-771) and its result equals the oracle's bit for bit."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from flashx_b200 import _lib, matrix_image
from flashx_b200.graphs import rmat_edges

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    exe = str(tmp_path / "shim_check")
    libdir = os.path.dirname(_lib.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "tests", "shim"), os.path.join(ROOT, "tests", "shim", "shim_check.cpp"),
                    "-L", libdir, "-lfmx", f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    return exe


def _files(tmp_path, scale=12, k=8):
    src, dst = rmat_edges(scale, seed=4)
    n = 1 << scale
    img = matrix_image.build(src, dst, None, nrows=n, ncols=n, block_size=(1024, 1024), dedup=True)
    idx_p, mat_p = str(tmp_path / "a.mat_idx"), str(tmp_path / "a.mat")
    img.dump(idx_p, mat_p)
    X = np.random.default_rng(2).integers(-8, 9, (n, k)).astype(np.float32)
    x_p = str(tmp_path / "x.f32")
    X.tofile(x_p)
    return img, idx_p, mat_p, X, x_p


def test_binding_compiles_and_reports_a_failed_load(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe, str(tmp_path / "missing.mat_idx"), str(tmp_path / "missing.mat"), "4", "x", "y"],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 2
    assert r.stderr.startswith("[error] ") and r.stderr.strip()


def test_binding_without_gpu_logs_the_device_error(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the no-GPU error path")
    exe = _build(tmp_path)
    _, idx_p, mat_p, _, x_p = _files(tmp_path)
    r = subprocess.run([exe, idx_p, mat_p, "8", x_p, str(tmp_path / "y.f32")], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 2
    assert "device" in r.stderr


@pytest.mark.gpu
def test_binding_multiply_matches_the_oracle(tmp_path, torch_cuda):
    exe = _build(tmp_path)
    img, idx_p, mat_p, X, x_p = _files(tmp_path)
    y_p = str(tmp_path / "y.f32")
    r = subprocess.run([exe, idx_p, mat_p, "8", x_p, y_p], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    # the three refused calls each logged one line
    assert r.stderr.count("[error] ") == 3
    idx, mat = img.bytes()
    want = oracle.spmm(idx, mat, X)
    got = np.fromfile(y_p, dtype=np.float32).reshape(want.shape)
    assert np.array_equal(got, want)
