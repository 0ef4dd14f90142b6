"""GPU SpMM over the FlashGraph 1D format (fmx_matrix_from_fg /
fmx_matrix_load_fg) against the oracle's restatement of
fg_row_spmm_task::run_on_row (flash-graph/fg_sparse_matrix.cpp:83-106),
which is pinned to FlashGraph's own record classes in
tests/test_fg_format.py.

Bar: bit-exact for every row of at most EXACT_ROW_MAX stored neighbors (the
record order, one rounding per multiply and add); hub rows within RTOL.
A FlashGraph matrix and the 2D image of the same unique edges give
identical products (the reference unit test's equivalence).
"""
import numpy as np
import pytest

import oracle
from flashx_b200 import FmxError, _lib, matrix_image, sparse_matrix
from flashx_b200.fg import FG_graph, create_sparse_matrix

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def _graph(seed, n, m, undirected, weighted, hub=True):
    rng = np.random.default_rng(seed)
    s = rng.integers(0, n, m).astype(np.uint32)
    d = rng.integers(0, n, m).astype(np.uint32)
    if hub:                                   # a hub row, a hub column, self-loops, duplicates
        s = np.concatenate([s, np.full(900, 3, np.uint32), rng.integers(0, n, 700).astype(np.uint32),
                            np.arange(20, dtype=np.uint32), s[:50]])
        d = np.concatenate([d, rng.integers(0, n, 900).astype(np.uint32), np.full(700, 9, np.uint32),
                            np.arange(20, dtype=np.uint32), d[:50]])
    w = rng.uniform(-1, 1, len(s)).astype(np.float32) if weighted else None
    if undirected:
        s, d = np.concatenate([s, d]), np.concatenate([d, s])
        w = None if w is None else np.concatenate([w, w])
    return s, d, w


def _degrees(s, n):
    return np.bincount(s.astype(np.int64), minlength=n)


@pytest.mark.parametrize("undirected", [False, True])
@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_fg_spmm_parity(torch_cuda, undirected, weighted, dtype):
    torch = torch_cuda
    n = 5000
    s, d, w = _graph(3, n, 40000, undirected, weighted)
    adj = oracle.fg_build(s, d, w, n, directed=not undirected)
    m = create_sparse_matrix(FG_graph.from_bytes(adj), "float" if weighted else None)
    assert m.is_symmetric() == undirected and m.get_nnz() == (len(s) if not undirected else len(s))
    prim = oracle.P_FLOAT if weighted else oracle.P_BOOL
    rng = np.random.default_rng(5)
    for transpose in (False, True):
        mm = m.transpose() if transpose else m
        light = _degrees(d if transpose else s, n) <= _lib.EXACT_ROW_MAX
        assert not light.all()
        for k in (1, 4, 10, 16):
            X = rng.standard_normal((n, k)).astype(dtype)
            Y = mm.multiply(torch.from_numpy(X).cuda()).cpu().numpy()
            R = oracle.fg_spmm(adj, X, transpose, prim)
            assert np.array_equal(Y[light], R[light])
            np.testing.assert_allclose(Y, R, rtol=RTOL, atol=RTOL * np.abs(R).max())


def test_fg_matches_2d_matrix(torch_cuda):
    """Unique edges over 16K vertices, X[i][j] = 10 i + j, k = 10, as in
    flash-graph/unit-test/test-sparse_matrix.cpp: the FlashGraph matrix and
    the 2D image of the same edges give identical products on the GPU, hub
    rows included (the same rows in the same order reach the same kernels)."""
    torch = torch_cuda
    n = 1024 * 16
    rng = np.random.default_rng(11)
    key = np.unique(rng.integers(0, n, 100000).astype(np.int64) * n + rng.integers(0, n, 100000))
    key = np.concatenate([key, 7 * n + np.arange(0, n, 40)])          # one hub row
    key = np.unique(key)
    s, d = (key // n).astype(np.uint32), (key % n).astype(np.uint32)
    vals = np.arange(len(s), dtype=np.float32)
    fgm = create_sparse_matrix(FG_graph.from_bytes(oracle.fg_build(s, d, vals, n, directed=True)), "float")
    img = matrix_image.build(s, d, vals, nrows=n, ncols=n, block_size=(1024, 1024), dedup=True, remove_self=False)
    timg = matrix_image.build(d, s, vals, nrows=n, ncols=n, block_size=(1024, 1024), dedup=True, remove_self=False)
    m2 = sparse_matrix.create(img, timg)
    X = torch.arange(n * 10, dtype=torch.float64, device="cuda").reshape(n, 10).float()
    assert torch.equal(fgm.multiply(X), m2.multiply(X))
    assert torch.equal(fgm.transpose().multiply(X), m2.transpose().multiply(X))
    assert fgm.schedule() == m2.schedule()


def test_fg_load_from_file(torch_cuda, tmp_path):
    torch = torch_cuda
    n = 2000
    s, d, w = _graph(9, n, 10000, False, True, hub=False)
    adj = oracle.fg_build(s, d, w, n, directed=True)
    p = tmp_path / "g.adj"
    p.write_bytes(adj)
    a = create_sparse_matrix(FG_graph.create(str(p)), "float")
    b = create_sparse_matrix(FG_graph.from_bytes(adj), "float")
    X = torch.randn((n, 16), device="cuda")
    assert torch.equal(a.multiply(X), b.multiply(X))
    assert np.array_equal(a.multiply(X).cpu().numpy(), oracle.fg_spmm(adj, X.cpu().numpy(), False, oracle.P_FLOAT))


def test_fg_errors(torch_cuda):
    n = 100
    s, d, w = _graph(1, n, 500, False, True, hub=False)
    adj = bytearray(oracle.fg_build(s, d, w, n, directed=True))
    with pytest.raises(FmxError) as e:                 # edge data of 4 bytes, no entry type
        create_sparse_matrix(FG_graph.from_bytes(adj), None)
    assert e.value.code == _lib.FMX_ERR_TYPE
    with pytest.raises(FmxError) as e:
        create_sparse_matrix(FG_graph.from_bytes(adj), "double")
    assert e.value.code == _lib.FMX_ERR_TYPE
    with pytest.raises(FmxError) as e:                 # truncated inside the records
        create_sparse_matrix(FG_graph.from_bytes(adj[:-8]), "float")
    assert e.value.code == _lib.FMX_ERR_IMAGE
    bad = bytearray(adj)
    bad[0] ^= 1
    with pytest.raises(FmxError) as e:
        create_sparse_matrix(FG_graph.from_bytes(bad), "float")
    assert e.value.code == _lib.FMX_ERR_IMAGE
    ts = bytearray(adj)
    ts[12:16] = (2).to_bytes(4, "little")               # TS_DIRECTED
    with pytest.raises(FmxError) as e:
        create_sparse_matrix(FG_graph.from_bytes(ts), "float")
    assert e.value.code == _lib.FMX_ERR_UNSUPPORTED
    with pytest.raises(FileNotFoundError):
        FG_graph.create("/nonexistent/graph.adj")
