"""fmx_spmm_noalloc: the SpMM entry point that allocates nothing.

It exists for callers that cannot allocate device memory while they run
(inside a memory pool or arena that owns the device's memory, in allocator
callbacks, on real-time paths).  It keeps its scratch in a fixed array
compiled into libfmx.  These tests call it through the C ABI, twice in a
row (the second call sees the first call's leftovers in the shared array),
and require results identical to fmx_spmm's bit for bit (the two run the
same kernels in the same order) and to the CPU oracle's (bit for bit with
integer-valued inputs, within the 1e-5 parity tolerance otherwise).

This file is collected last on purpose, so that a run which stops at the
first failure has already run every other test.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from flashx_b200 import _lib, matrix_image, sparse_matrix
from flashx_b200.graphs import rmat_edges

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402

pytestmark = pytest.mark.gpu

RTOL = 1e-5
SCRATCH = 32 << 20


def _scratch_need(m):
    """The fixed-scratch bytes fmx_spmm_noalloc needs for this matrix: the
    hot pack, (n_hot + 1) rows of 128 bytes rounded up to 256 bytes, plus
    4-byte chunk sums, 256 per partial slot.  fmx_matrix_hot's scratch count
    holds the partial slots at 8 bytes: (n_hot + 1) * 128 + slots * 2048."""
    n_hot, _, scratch = m.hot()
    hot = (n_hot + 1) * 128
    slots = (scratch - hot) // 2048
    return (hot + 255) // 256 * 256 + slots * 256 * 4


def _noalloc(torch, m, x, y):
    st = torch.cuda.current_stream(x.device).cuda_stream
    return _lib.lib.fmx_spmm_noalloc(m.handle, x.data_ptr(), x.stride(0) if x.shape[0] > 1 else x.shape[1],
                                     y.data_ptr(), y.stride(0) if y.shape[0] > 1 else y.shape[1], x.shape[1], st)


@pytest.mark.parametrize("weighted", [False, True])
def test_noalloc_matches_fmx_spmm_twice(torch_cuda, weighted):
    torch = torch_cuda
    n = 1 << 16
    src, dst = rmat_edges(16, seed=5)
    vals = None
    if weighted:
        vals = (1.0 - np.random.default_rng(1).random(len(src))).astype(np.float32)
    img = matrix_image.build(src, dst, vals, nrows=n, ncols=n, block_size=(16384, 16384), dedup=True)
    m = sparse_matrix.create(img, None)
    assert 0 < _scratch_need(m) <= SCRATCH
    g = torch.Generator(device="cuda").manual_seed(3)
    for k in (16, 1, 130, 32):
        x = torch.randn((n, k), generator=g, device="cuda")
        ref = torch.empty((n, k), device="cuda")
        assert m.multiply(x, ref)
        for _ in range(2):
            y = torch.full((n, k), float("nan"), device="cuda")
            assert _noalloc(torch, m, x, y) == _lib.FMX_OK, _lib.last_error()
            torch.cuda.synchronize()
            assert torch.equal(y, ref), f"k={k}: differs from fmx_spmm"
    # against the CPU oracle: bit for bit for the binary matrix with
    # integer-valued X (every sum exact), else within the parity tolerance
    idx, mat = img.bytes()
    xi = np.random.default_rng(4).integers(-8, 9, (n, 16)).astype(np.float32)
    xf = np.random.default_rng(5).standard_normal((n, 16)).astype(np.float32)
    for xh, exact in ((xi, not weighted), (xf, False)):
        want = oracle.spmm(idx, mat, xh)
        for _ in range(2):
            y = torch.full((n, 16), float("nan"), device="cuda")
            assert _noalloc(torch, m, torch.from_numpy(xh).cuda(), y) == _lib.FMX_OK, _lib.last_error()
            torch.cuda.synchronize()
            got = y.cpu().numpy()
            if exact:
                assert np.array_equal(got, want)
            else:
                np.testing.assert_allclose(got, want, rtol=RTOL, atol=RTOL * float(np.abs(want).max()))


def test_noalloc_rejects_matrices_beyond_its_scratch(torch_cuda):
    torch = torch_cuda
    n = 1 << 20
    src, dst = rmat_edges(20, seed=2)
    m = sparse_matrix.create(matrix_image.build(src, dst, None, nrows=n, ncols=n, dedup=True), None)
    assert _scratch_need(m) > SCRATCH
    x = torch.zeros((n, 16), device="cuda")
    y = torch.zeros((n, 16), device="cuda")
    assert _noalloc(torch, m, x, y) == _lib.FMX_ERR_UNSUPPORTED
    assert "fixed scratch" in _lib.last_error()
    # wrong entry types are refused with a type error
    img = matrix_image.build([0, 1], [1, 0], np.array([1.0, 2.0]), nrows=2, ncols=2, block_size=(2, 2))
    md = sparse_matrix.create(img, None)
    x2 = torch.zeros((2, 4), device="cuda")
    y2 = torch.zeros((2, 4), device="cuda")
    assert _noalloc(torch, md, x2, y2) == _lib.FMX_ERR_TYPE
