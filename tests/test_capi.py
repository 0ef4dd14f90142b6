"""The C ABI: libfmx.so loads without a GPU, exports every function that
include/fmx.h declares, and reports errors through status codes."""
import ctypes as C
import os
import re
import subprocess

import pytest
import torch

from flashx_b200 import _lib, matrix_image, FmxError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fmx.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fmx_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_functions():
    names = declared_functions()
    assert "fmx_spmm" in names and "fmx_matrix_create" in names and "fmx_image_build" in names
    assert len(names) >= 20


def test_library_exports_every_declared_function():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (fmx_[a-z0-9_]+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, f"declared in include/fmx.h but not exported: {missing}"
    for n in declared_functions():
        getattr(_lib.lib, n)


def test_python_binding_covers_the_header():
    assert set(declared_functions()) <= set(_lib.exported_symbols())


def test_header_compiles_as_c_and_cpp(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "fmx.h"\nint main(void) { return fmx_strerror(0) == 0; }\n')
    for cc, flags in (("gcc", ["-std=c99"]), ("g++", ["-x", "c++", "-std=c++11"])):
        subprocess.run([cc, *flags, "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-c", str(src),
                        "-o", str(tmp_path / "t.o")], check=True)


def test_status_strings():
    for code in range(0, -9, -1):
        assert _lib.lib.fmx_strerror(code)
    assert _lib.lib.fmx_strerror(-99) == b"unknown status"
    assert _lib.lib.fmx_version().startswith(b"fmx")


def test_null_arguments_are_rejected():
    assert _lib.lib.fmx_matrix_create(None, None, 0, None) == _lib.FMX_ERR_INVAL
    assert _lib.lib.fmx_spmm(None, 0, None, 1, 0, None, 1, 1, None, None, None) == _lib.FMX_ERR_INVAL
    assert _lib.lib.fmx_spmm_host(None, 0, None, 1, 0, None, 1, 1) == _lib.FMX_ERR_INVAL
    assert _lib.lib.fmx_spmm_host_async(None, 0, None, 1, 0, None, 1, 1, None) == _lib.FMX_ERR_INVAL
    assert _lib.lib.fmx_image_free(None) == _lib.FMX_OK
    assert _lib.lib.fmx_matrix_free(None) == _lib.FMX_OK


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU error path")
def test_matrix_create_without_gpu_reports_cuda_error():
    img = matrix_image.build([0, 1], [1, 0], None, block_size=(16, 16))
    h = C.c_void_p()
    rc = _lib.lib.fmx_matrix_create(img._h, None, 0, C.byref(h))
    assert rc == _lib.FMX_ERR_CUDA
    assert "device" in _lib.last_error()


def test_eigen_structs_match_the_header(tmp_path):
    """The ctypes mirrors of fmx_eigen_options / fmx_eigen_status have the C
    layout, and fmx_eigen_default_options fills the reference's defaults
    (eigen_options(), eigensolver.cpp:82-91) without touching a GPU."""
    src = tmp_path / "s.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "fmx.h"\n'
                   'int main(void) { printf("%zu %zu %zu %zu %zu\\n", sizeof(fmx_eigen_options),'
                   ' offsetof(fmx_eigen_options, tol), offsetof(fmx_eigen_options, seed),'
                   ' offsetof(fmx_eigen_options, ldx0), sizeof(fmx_eigen_status)); return 0; }\n')
    exe = tmp_path / "s"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    O, S = _lib.eigen_options_t, _lib.eigen_status_t
    assert got == [C.sizeof(O), O.tol.offset, O.seed.offset, O.ldx0.offset, C.sizeof(S)]
    o = O()
    _lib.lib.fmx_eigen_default_options(C.byref(o), 8)
    assert (o.nev, o.block_size, o.max_iters, o.which, o.precision) == (8, 16, 500, _lib.EIGEN_LA, _lib.EIGEN_PLAIN)
    assert o.tol == 1e-8 and (o.lower, o.upper) == (-1.0, 1.0)
    from flashx_b200.eigen import eigen_options
    e = eigen_options()
    assert (e.tol, e.max_iters, e.which, e.max_restarts) == (1e-8, 500, "LM", 100)
    assert e.init(8) and e.block_size == 16 and not e.init(8, "Lanczos")
