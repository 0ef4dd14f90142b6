"""Pins the oracle's FlashGraph 1D pieces (CPU only).

1. The record layout of the oracle's writer and reader against FlashGraph's
   OWN record class (ext_mem_undirected_vertex::num_edges2vsize and
   get_edge_data_offset, flash-graph/vertex.h:482-506, compiled in place into
   oracle/_ref/libfmx_reffg.so where the reference tree exists).
2. The oracle's row SpMM (fg_row_spmm_task::run_on_row,
   flash-graph/fg_sparse_matrix.cpp:83-106) against the same product walked
   with the reference's record and header classes: bit for bit.
3. The equivalence the reference unit test
   flash-graph/unit-test/test-sparse_matrix.cpp exercises: one edge list of
   unique edges over 16K vertices, multiplied as a FlashGraph matrix and as a
   2D-tiled matrix (1024 x 1024 tiles) by X[i][j] = 10 i + j, k = 10, gives
   the same result (both sum each row in ascending neighbor order).
"""
import numpy as np
import pytest

import oracle

needs_reffg = pytest.mark.skipif(oracle.reffg() is None,
                                 reason="FlashGraph walker not built (needs the reference tree)")


def _edges(seed, n, m, undirected=False, weighted=False):
    rng = np.random.default_rng(seed)
    s = rng.integers(0, n, m).astype(np.uint32)
    d = rng.integers(0, n, m).astype(np.uint32)
    w = rng.standard_normal(m).astype(np.float32) if weighted else None
    if undirected:
        s, d = np.concatenate([s, d]), np.concatenate([d, s])
        w = None if w is None else np.concatenate([w, w])
    return s, d, w


@needs_reffg
def test_record_layout_matches_flashgraph():
    r = oracle.reffg()
    assert r.ref_fg_header_size() == 4096
    for eds in (0, 1, 2, 4, 8, 16):
        for ne in range(0, 300):
            assert oracle.fg_vsize(ne, eds) == r.ref_fg_vsize(ne, eds), (ne, eds)
            if eds:
                assert oracle.fg_data_off(ne, eds) == r.ref_fg_data_off(ne, eds), (ne, eds)


@needs_reffg
@pytest.mark.parametrize("undirected", [False, True])
@pytest.mark.parametrize("weighted", [False, True])
def test_row_spmm_matches_flashgraph_walker(undirected, weighted):
    import ctypes as C
    n = 3000
    s, d, w = _edges(7, n, 20000, undirected, weighted)
    # a hub and a self-loop or two
    s = np.concatenate([s, np.full(600, 5, np.uint32), np.arange(10, dtype=np.uint32)])
    d = np.concatenate([d, np.random.default_rng(1).integers(0, n, 600).astype(np.uint32),
                        np.arange(10, dtype=np.uint32)])
    if w is not None:
        w = np.concatenate([w, np.linspace(-1, 1, 610, dtype=np.float32)])
    adj = oracle.fg_build(s, d, w, n, directed=not undirected)
    nv, ne, eds, dr = C.c_uint64(), C.c_uint64(), C.c_int(), C.c_int()
    assert oracle.reffg().ref_fg_header(adj, C.byref(nv), C.byref(ne), C.byref(eds), C.byref(dr)) == 0
    assert (nv.value, eds.value, dr.value) == (n, 4 if weighted else 0, 0 if undirected else 1)
    prim = oracle.P_FLOAT if weighted else oracle.P_BOOL
    rng = np.random.default_rng(2)
    for dt in (np.float32, np.float64):
        X = rng.standard_normal((n, 5)).astype(dt)
        for t in (False, True):
            assert np.array_equal(oracle.fg_spmm(adj, X, t, prim), oracle.ref_fg_spmm(adj, X, t))


@pytest.mark.parametrize("directed", [True, False])
@pytest.mark.parametrize("with_attr", [False, True])
def test_fg_matches_2d_like_the_reference_unit_test(directed, with_attr):
    n = 1024 * 16
    rng = np.random.default_rng(11)
    key = np.unique(rng.integers(0, n, 100000).astype(np.int64) * n + rng.integers(0, n, 100000))
    s, d = (key // n).astype(np.uint32), (key % n).astype(np.uint32)
    vals = np.arange(len(s), dtype=np.float32) if with_attr else None
    if not directed:
        s, d = np.concatenate([s, d]), np.concatenate([d, s])
        vals = None if vals is None else np.concatenate([vals, vals])
        key2 = s.astype(np.int64) * n + d
        first = np.unique(key2, return_index=True)[1]          # an edge and its mirror may coincide
        s, d = s[first], d[first]
        vals = None if vals is None else vals[first]
    adj = oracle.fg_build(s, d, vals, n, directed=directed)
    idx, mat = oracle.build_image(s, d, vals, nrows=n, ncols=n, block=(1024, 1024), dedup=True,
                                  keep_self=True)
    X = (np.arange(n * 10, dtype=np.float64).reshape(n, 10)).astype(np.float32)   # in_mat[i][j] = 10 i + j
    prim = oracle.P_FLOAT if with_attr else oracle.P_BOOL
    assert np.array_equal(oracle.fg_spmm(adj, X, False, prim), oracle.spmm(idx, mat, X))


def _from_fg(adj, prim):
    import ctypes as C
    from flashx_b200 import _lib
    h = C.c_void_p()
    rc = _lib.lib.fmx_matrix_from_fg(adj, len(adj), prim, 0, C.byref(h))
    return rc, h


def test_product_loader_validates_on_the_host():
    """fmx_matrix_from_fg parses and checks the image before it needs a GPU:
    malformed images are rejected here with the reference's error classes,
    and a valid one gets as far as the device (FMX_ERR_CUDA without one)."""
    import torch
    from flashx_b200 import _lib
    n = 300
    s, d, w = _edges(3, n, 2000, False, True)
    adj = oracle.fg_build(s, d, w, n, directed=True)
    bad = bytearray(adj)
    bad[0] ^= 1                                          # magic
    assert _from_fg(bytes(bad), _lib.P_FLOAT)[0] == _lib.FMX_ERR_IMAGE
    ver = bytearray(adj)
    ver[8:12] = (3).to_bytes(4, "little")                # version
    assert _from_fg(bytes(ver), _lib.P_FLOAT)[0] == _lib.FMX_ERR_IMAGE
    ts = bytearray(adj)
    ts[12:16] = (3).to_bytes(4, "little")                # TS_UNDIRECTED
    assert _from_fg(bytes(ts), _lib.P_FLOAT)[0] == _lib.FMX_ERR_UNSUPPORTED
    assert _from_fg(adj, _lib.P_BOOL)[0] == _lib.FMX_ERR_TYPE      # 4-byte edge data
    assert _from_fg(adj, _lib.P_DOUBLE)[0] == _lib.FMX_ERR_TYPE
    assert _from_fg(adj[:-4], _lib.P_FLOAT)[0] == _lib.FMX_ERR_IMAGE   # truncated
    assert _from_fg(adj[:100], _lib.P_FLOAT)[0] == _lib.FMX_ERR_IMAGE  # no header page
    nb = bytearray(adj)
    first = 4096 + 12                                    # first neighbor of vertex 0's in-record
    nb[first:first + 4] = (n + 5).to_bytes(4, "little")
    if int.from_bytes(adj[4096 + 8:4096 + 12], "little"):          # vertex 0 has in-edges
        assert _from_fg(bytes(nb), _lib.P_FLOAT)[0] == _lib.FMX_ERR_IMAGE
    ids = bytearray(adj)
    ids[4096:4100] = (7).to_bytes(4, "little")           # record 0 names vertex 7
    assert _from_fg(bytes(ids), _lib.P_FLOAT)[0] == _lib.FMX_ERR_IMAGE
    if not torch.cuda.is_available():
        assert _from_fg(adj, _lib.P_FLOAT)[0] == _lib.FMX_ERR_CUDA


def test_device_entry_points_check_arguments_on_the_host():
    """The device builder and the streamed form reject bad arguments before
    they touch a GPU."""
    import ctypes as C
    from flashx_b200 import _lib
    h = C.c_void_p()
    L = _lib.lib
    # flags outside DEDUP | KEEP_SELF_LOOPS | TRANSPOSE
    assert L.fmx_matrix_build_device(None, None, None, _lib.P_BOOL, 0, 4, 4, 0x4, 0, None, C.byref(h)) \
        == _lib.FMX_ERR_INVAL
    # edges without arrays, values of a weighted type without a value array
    assert L.fmx_matrix_build_device(None, None, None, _lib.P_BOOL, 10, 4, 4, 0, 0, None, C.byref(h)) \
        == _lib.FMX_ERR_INVAL
    assert L.fmx_matrix_create_streamed(None, None, 0, 0, C.byref(h)) == _lib.FMX_ERR_INVAL
    assert L.fmx_matrix_stream_info(None, None, None) == _lib.FMX_ERR_INVAL
    assert L.fmx_release_cached(-1) == _lib.FMX_ERR_INVAL
