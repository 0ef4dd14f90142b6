"""GPU PageRank (fmx_pagerank) against the oracle's restatement of
fm::alg::PageRank (matrix/libmatrix-algs/PageRank.cpp:63-133).

Bar: bit-identical ranks and the same iteration count when every vertex's
in-degree row has at most EXACT_ROW_MAX entries (all sums in the reference's
order); otherwise rows above that are summed in chunks, so ranks match within
RTOL = 1e-5 relative and the iteration count may differ by one.
"""
import numpy as np
import pytest

import oracle
from flashx_b200 import _lib, create_2d_matrix
from flashx_b200.algs import PageRank
from flashx_b200.graphs import rmat_edges

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def _directed(n, m, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(0, n, m).astype(np.uint32), rng.integers(0, n, m).astype(np.uint32)


@pytest.mark.parametrize("iters,damping", [(30, 0.85), (5, 0.5), (200, 0.85)])
def test_pagerank_bit_exact_on_short_rows(torch_cuda, iters, damping):
    n = 6000
    src, dst = _directed(n, 50000, 11)
    m, img, timg = create_2d_matrix(src, dst, None, block_size=(1024, 1024), is_sym=False, nrows=n, ncols=n,
                                    return_images=True)
    (idx, mat), (tidx, tmat) = img.bytes(), timg.bytes()
    assert np.bincount(dst, minlength=n).max() <= _lib.EXACT_ROW_MAX
    pr, it = PageRank(m, iters, damping)
    ref, rit = oracle.pagerank(idx, mat, tidx, tmat, iters, damping, nthreads=4)
    assert it == rit
    assert np.array_equal(pr.cpu().numpy(), ref)


def test_pagerank_rmat_s16_configuration(torch_cuda):
    """The reference's CPU configuration: R-MAT scale 16, 30 iterations at
    damping 0.85 (hub rows longer than EXACT_ROW_MAX are summed in chunks)."""
    from flashx_b200 import set_deduplicate
    n = 1 << 16
    src, dst = rmat_edges(16, seed=1)
    set_deduplicate(True)
    try:
        m, img, timg = create_2d_matrix(src, dst, None, block_size=(16384, 16384), is_sym=False, nrows=n, ncols=n,
                                        return_images=True)
    finally:
        set_deduplicate(False)
    (idx, mat), (tidx, tmat) = img.bytes(), timg.bytes()
    pr, it = PageRank(m, 30, 0.85)
    ref, rit = oracle.pagerank(idx, mat, tidx, tmat, 30, 0.85, nthreads=8)
    assert abs(it - rit) <= 1
    p = pr.cpu().numpy()
    np.testing.assert_allclose(p, ref, rtol=RTOL, atol=RTOL * float(ref.max()))
    assert abs(float(p.astype(np.float64).sum()) - float(ref.astype(np.float64).sum())) < 1e-4


def test_pagerank_errors(torch_cuda):
    from flashx_b200 import FmxError, matrix_image, sparse_matrix
    rect = sparse_matrix.create(matrix_image.build([0, 1], [1, 0], None, nrows=4, ncols=2, block_size=(2, 2)), None)
    with pytest.raises(FmxError) as e:
        PageRank(rect, 10, 0.85)
    assert e.value.code == _lib.FMX_ERR_DIM


def test_pagerank_fused_matches_stepwise_loop(torch_cuda):
    """The fused iteration (update applied where the SpMV closes a row, and
    in the fixup for chunked hub rows) against a host-driven loop of plain
    SpMVs on the transpose with the update in float32 numpy (one rounding per
    operation, as PageRank.cpp:100-123): bit-identical at R-MAT scale 16,
    whose hub rows go through the fixup, for an iteration cap below, at and
    above the point of convergence."""
    torch = torch_cuda
    from flashx_b200 import set_deduplicate
    n = 1 << 16
    src, dst = rmat_edges(16, seed=2)
    set_deduplicate(True)
    try:
        m = create_2d_matrix(src, dst, None, block_size=(16384, 16384), is_sym=False, nrows=n, ncols=n)
    finally:
        set_deduplicate(False)
    mt = m.transpose()
    assert mt.schedule()[2] > 0                   # heavy rows take the fixup path
    d = np.float32(0.85)
    deg = m.multiply(torch.ones((n, 1), device="cuda")).cpu().numpy()[:, 0]
    deg = np.maximum(deg, np.float32(1))
    tele = np.float32((1.0 - float(d)) / n)     # (1 - d) / n in double from the float d
    eps = np.float32(0.001 / n)
    pr = np.full(n, np.float32(1.0 / n), dtype=np.float32)
    x = pr / deg
    pr1 = x * deg
    ref_iters, ref = [], []
    it, conv = 0, 0
    while conv < n and it < 60:
        out = mt.multiply(torch.from_numpy(x).cuda().reshape(n, 1)).cpu().numpy()[:, 0]
        p2 = out * d + tele
        conv = int(np.count_nonzero(np.abs(pr1 - p2) < eps))
        pr = p2
        x = p2 / deg
        pr1 = x * deg
        it += 1
        ref.append(pr.copy())
    for cap in (3, 17, 60):
        got, git = PageRank(m, cap, 0.85)
        assert git == min(cap, it)
        assert np.array_equal(got.cpu().numpy(), ref[git - 1])


def test_workspace_pool_release(torch_cuda):
    """The solvers' workspace pool keeps freed memory for the next call;
    release_cached hands it back, and later calls still run."""
    torch = torch_cuda
    from flashx_b200 import release_cached
    n = 6000
    src, dst = _directed(n, 50000, 11)
    m = create_2d_matrix(src, dst, None, block_size=(1024, 1024), is_sym=False, nrows=n, ncols=n)
    p1, i1 = PageRank(m, 30, 0.85)
    release_cached(0)
    p2, i2 = PageRank(m, 30, 0.85)
    assert i1 == i2 and torch.equal(p1, p2)
    release_cached(0)
