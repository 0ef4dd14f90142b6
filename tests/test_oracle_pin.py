"""Pins the CPU oracle (oracle/fmx_oracle.c) before it is trusted.

1. Against the reference's OWN tile classes (matrix/sparse_matrix_format.h,
   compiled in place into oracle/_ref/libfmx_refwalk.so where the reference
   tree exists): same non-zeros, bit-identical SpMM for every dense type.
2. Against the golden fixtures of the reference unit test
   matrix/unit-test/test-sparse_matrix.cpp (tests/golden/, made by
   make_golden.py with the reference walker).
3. Against the known answer of matrix/test/rand_mat_gen.cpp:178-199.
4. Hilbert order against matrix/hilbert_curve.cpp.
5. The oracle's R-MAT stream against the library's generator (the CPU arm
   of the benchmark makes its workload without the GPU library).
"""
import hashlib
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="reference walker not built (needs the reference tree)")


def _rand_graph(seed, n, m):
    rng = np.random.default_rng(seed)
    return rng.integers(0, n, m).astype(np.uint32), rng.integers(0, n, m).astype(np.uint32)


GRAPHS = [
    # seed, n, m, block, value dtype, dedup, keep self loops
    (1, 1000, 6000, (64, 128), None, False, False),
    (2, 5000, 40000, (256, 256), np.float32, True, False),
    (3, 3000, 30000, (1024, 512), np.float64, False, True),
    (4, 2000, 12000, (2, 4), np.int32, True, False),
    (5, 40000, 120000, (32768, 32768), np.int64, False, False),
    (6, 700, 50000, (128, 64), np.float32, False, False),
]


@needs_ref
@pytest.mark.parametrize("g", range(len(GRAPHS)))
def test_oracle_matches_reference_walk(g):
    seed, n, m, block, vdt, dedup, keep_self = GRAPHS[g]
    src, dst = _rand_graph(seed, n, m)
    vals = None if vdt is None else np.random.default_rng(seed).integers(-5, 6, m).astype(vdt)
    idx, mat = oracle.build_image(src, dst, vals, block=block, dedup=dedup, keep_self=keep_self)
    assert oracle.verify(idx, mat) == 0
    r1, c1 = oracle.nonzeros(idx, mat)
    r2, c2 = oracle.ref_nonzeros(idx, mat)
    assert np.array_equal(r1, r2) and np.array_equal(c1, c2)
    h = oracle.header(idx)
    rng = np.random.default_rng(seed + 100)
    dense = [np.float32, np.float64, np.int32, np.int64] if vdt is None else [vdt]
    for dt in dense:
        for k in (1, 3, 8, 16):
            if np.issubdtype(dt, np.floating):
                X = rng.standard_normal((h["ncols"], k)).astype(dt)
            else:
                X = rng.integers(-1000, 1000, (h["ncols"], k)).astype(dt)
            Y = oracle.spmm(idx, mat, X, nthreads=3)
            R = oracle.ref_spmm(idx, mat, X)
            assert np.array_equal(Y.view(np.uint8), R.view(np.uint8))


@needs_ref
def test_oracle_double_dense_float_entries():
    """spmm_creator<double, float> (matrix/test/test-eigen.cpp:47)."""
    src, dst = _rand_graph(7, 3000, 20000)
    vals = np.random.default_rng(7).random(20000).astype(np.float32)
    idx, mat = oracle.build_image(src, dst, vals, block=(512, 512))
    X = np.random.default_rng(8).standard_normal((3000, 8))
    # the oracle converts float entries to double, as the reference does
    # (dest += src * data with data promoted)
    Y = oracle.spmm(idx, mat, X)
    R = oracle.ref_spmm(idx, mat, X, dense_double_sparse_float=True)
    assert np.array_equal(Y, R)


def test_golden_reference_unit_test():
    """matrix/unit-test/test-sparse_matrix.cpp: 16K x 16K, 100,000 glibc random()
    draws, 1024 x 1024 blocks, X[i][j] = i * 10 + j, binary and weighted."""
    g = np.load(os.path.join(GOLDEN, "test_sparse_matrix.npz"))
    src, dst, n = g["src"].astype(np.uint32), g["dst"].astype(np.uint32), int(g["n"])
    X = (np.arange(n)[:, None] * 10 + np.arange(10)[None, :]).astype(np.float32)
    for name, vals in (("binary", None), ("weighted", np.arange(len(src), dtype=np.float32))):
        idx, mat = oracle.build_image(src, dst, vals, block=(1024, 1024), ref_value_layout=True)
        assert hashlib.sha256(idx).digest() == g[f"{name}_idx_sha256"].tobytes()
        assert hashlib.sha256(mat).digest() == g[f"{name}_mat_sha256"].tobytes()
        Y = oracle.spmm(idx, mat, X, nthreads=4)
        assert hashlib.sha256(Y.tobytes()).digest() == g[f"{name}_y_sha256"].tobytes()
        np.testing.assert_array_equal(Y.astype(np.float64).sum(axis=0), g[f"{name}_colsum"])
        tidx, tmat = oracle.build_image(dst, src, vals, nrows=n, ncols=n, block=(1024, 1024),
                                        ref_value_layout=True)
        Yt = oracle.spmm(tidx, tmat, X)
        assert hashlib.sha256(Yt.tobytes()).digest() == g[f"{name}_t_y_sha256"].tobytes()


def test_rand_mat_gen_known_answer_oracle():
    """matrix/test/rand_mat_gen.cpp:178-199 on the oracle: binary A times
    [0..ncol-1] is each row's sum of column ids (duplicates kept)."""
    rng = np.random.default_rng(3)
    nrow, ncol = 20000, 12000
    deg = rng.integers(0, 40, nrow)
    src = np.repeat(np.arange(nrow, dtype=np.uint32), deg)
    dst = rng.integers(0, ncol, len(src)).astype(np.uint32)
    idx, mat = oracle.build_image(src, dst, None, nrows=nrow, ncols=ncol, block=(4096, 2048))
    Y = oracle.spmm(idx, mat, np.arange(ncol, dtype=np.int64), nthreads=4)[:, 0]
    keep = src != dst
    expect = np.bincount(src[keep], weights=dst[keep].astype(np.float64), minlength=nrow).astype(np.int64)
    assert np.array_equal(Y, expect)


def test_oracle_threads_and_super_blocks_agree():
    src, dst = _rand_graph(11, 9000, 90000)
    idx, mat = oracle.build_image(src, dst, None, block=(512, 512), dedup=True)
    X = np.random.default_rng(1).standard_normal((9000, 8)).astype(np.float32)
    base = oracle.spmm(idx, mat, X, nthreads=1)
    for t in (2, 5, 8):
        for cache in (1 << 16, 1 << 20, 1 << 24):
            assert np.array_equal(oracle.spmm(idx, mat, X, nthreads=t, cpu_cache_size=cache), base)


def test_hilbert_matches_reference():
    g = np.load(os.path.join(GOLDEN, "hilbert.npz"))
    L = oracle.orc()
    for nn in (2, 4, 8, 16):
        mine = np.array([[L.orc_hilbert_xy2d(nn, x, y) for y in range(nn)] for x in range(nn)])
        assert np.array_equal(mine, g[f"n{nn}"])
        # every cell gets a distinct position on the curve
        assert sorted(mine.ravel().tolist()) == list(range(nn * nn))


def test_oracle_pagerank_matches_restatement():
    """PageRank.cpp:63-133 semantics against a numpy restatement."""
    rng = np.random.default_rng(5)
    n = 3000
    src = rng.integers(0, n, 20000).astype(np.uint32)
    dst = rng.integers(0, n, 20000).astype(np.uint32)
    idx, mat = oracle.build_image(src, dst, None, nrows=n, ncols=n, block=(1024, 1024), dedup=True)
    tidx, tmat = oracle.build_image(dst, src, None, nrows=n, ncols=n, block=(1024, 1024), dedup=True)
    pr, iters = oracle.pagerank(idx, mat, tidx, tmat, max_iters=30, damping=0.85)
    r, c = oracle.nonzeros(idx, mat)
    deg = np.maximum(np.bincount(r.astype(np.int64), minlength=n).astype(np.float32), np.float32(1))
    p = np.full(n, np.float32(1.0) / np.float32(n), dtype=np.float32)
    teleport = np.float32((1.0 - 0.85) / n)
    for _ in range(iters):
        x = (p / deg).astype(np.float32)
        out = np.zeros(n, dtype=np.float64)
        np.add.at(out, c.astype(np.int64), x[r.astype(np.int64)].astype(np.float64))
        p = (out.astype(np.float32) * np.float32(0.85) + teleport).astype(np.float32)
    np.testing.assert_allclose(pr, p, rtol=1e-5, atol=1e-9)


@pytest.mark.parametrize("scale,seed,permute", [(8, 1, True), (14, 1, True), (12, 3, False), (17, 9, True)])
def test_oracle_rmat_stream_matches_the_library(scale, seed, permute):
    from flashx_b200.graphs import rmat_edges
    a = rmat_edges(scale, seed=seed, permute=permute)
    b = oracle.rmat_edges(scale, seed=seed, permute=permute, nthreads=3)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_oracle_builder_sort_keeps_first_duplicates():
    """The builder's parallel radix sort: duplicates keep the first
    occurrence's value, exactly as the library's builder does."""
    from flashx_b200 import matrix_image
    rng = np.random.default_rng(8)
    n, m = 3000, 3_000_000            # several sort threads, many duplicates
    src = rng.integers(0, n, m).astype(np.uint32)
    dst = rng.integers(0, n, m).astype(np.uint32)
    vals = rng.standard_normal(m).astype(np.float32)
    idx, mat = oracle.build_image(src, dst, vals, nrows=n, ncols=n, block=(1024, 512), dedup=True)
    i2, m2 = matrix_image.build(src, dst, vals, nrows=n, ncols=n, block_size=(1024, 512), dedup=True).bytes()
    assert bytes(idx) == bytes(i2) and bytes(mat) == bytes(m2)
