"""The semi-external form (fmx_matrix_create_streamed): the entry stream in
pinned host memory, streamed to the GPU slice by slice during every SpMM.
Each range runs the same kernel code on the same entries as in the resident
matrix, so every product must be bit-identical to the resident one, for any
slice size (many slices, ranges of one slice split over the two device
slots, one slice), dense type, k, row scales and orientation."""
import numpy as np
import pytest

from flashx_b200 import FmxError, _lib, matrix_image, sparse_matrix
from flashx_b200.algs import PageRank
from flashx_b200.graphs import rmat_edges

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rmat16():
    n = 1 << 16
    s, d = rmat_edges(16, seed=3)
    rng = np.random.default_rng(0)
    w = rng.uniform(-1, 1, len(s)).astype(np.float32)
    out = {}
    for weighted in (False, True):
        v = w if weighted else None
        img = matrix_image.build(s, d, v, nrows=n, ncols=n, block_size=(16384, 16384), dedup=True)
        timg = matrix_image.build(d, s, v, nrows=n, ncols=n, block_size=(16384, 16384), dedup=True)
        out[weighted] = (img, timg)
    return n, out


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("slice_entries", [512, 40000, 1 << 24])
def test_streamed_matches_resident(torch_cuda, rmat16, weighted, slice_entries):
    torch = torch_cuda
    n, imgs = rmat16
    img, timg = imgs[weighted]
    res = sparse_matrix.create(img, timg)
    st = sparse_matrix.create_streamed(img, timg, slice_entries=slice_entries)
    slices, host = st.stream_info()
    assert host >= 4 * res.get_nnz() and (slices > 1) == (slice_entries < (1 << 20))
    assert res.stream_info() == (0, 0)
    g = torch.Generator(device="cuda").manual_seed(slice_entries)
    for a, b in ((res, st), (res.transpose(), st.transpose())):
        for k, dt in ((1, torch.float32), (4, torch.float32), (16, torch.float32), (40, torch.float32),
                      (1, torch.float64), (8, torch.float64)):
            X = torch.randn((n, k), generator=g, device="cuda", dtype=dt)
            assert torch.equal(a.multiply(X), b.multiply(X)), (k, dt)
        Xb = torch.randn((n, 16), generator=g, device="cuda").to(torch.bfloat16)
        Yr = torch.empty((n, 16), device="cuda")
        Ys = torch.empty((n, 16), device="cuda")
        assert a.multiply(Xb, Yr) and b.multiply(Xb, Ys)
        assert torch.equal(Yr, Ys)
        sc = torch.rand(n, device="cuda") + 0.5
        X = torch.randn((n, 16), generator=g, device="cuda")
        Yr, Ys = torch.empty_like(X), torch.empty_like(X)
        assert a.multiply(X, Yr, row_scale_in=sc, row_scale_out=sc)
        assert b.multiply(X, Ys, row_scale_in=sc, row_scale_out=sc)
        assert torch.equal(Yr, Ys)


def test_streamed_pagerank_and_host_buffers(torch_cuda, rmat16):
    torch = torch_cuda
    n, imgs = rmat16
    img, timg = imgs[False]
    res = sparse_matrix.create(img, timg)
    st = sparse_matrix.create_streamed(img, timg, slice_entries=20000)
    p1, i1 = PageRank(res, 30, 0.85)
    p2, i2 = PageRank(st, 30, 0.85)
    assert i1 == i2 and torch.equal(p1, p2)
    X = np.random.default_rng(1).standard_normal((n, 16)).astype(np.float32)
    assert np.array_equal(res.multiply_host(X), st.multiply_host(X))


def test_streamed_rejected_by_noalloc(torch_cuda, rmat16):
    torch = torch_cuda
    n, imgs = rmat16
    st = sparse_matrix.create_streamed(imgs[False][0], None, slice_entries=4096)
    X = torch.randn((n, 16), device="cuda")
    Y = torch.empty_like(X)
    rc = _lib.lib.fmx_spmm_noalloc(st.handle, X.data_ptr(), 16, Y.data_ptr(), 16, 16,
                                   torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.FMX_ERR_UNSUPPORTED
