"""The block eigensolver (fmx_eigen_solve) against FP64 references.

There is no eigensolver in the reference tree to pin against (its iterations
live in the external Trilinos Anasazi), so each result is checked by:
  * the residual ||A x - l x|| / ||A|| of every returned pair, recomputed here
    in FP64 with scipy (not with the library's SpMM): <= tol (1e-6) x 2;
  * eigenvalues against scipy's ARPACK (FP64): |l - l_ref| <= 1e-6;
  * the largest principal angle between the returned subspace and the FP64
    eigenvectors of the same eigenvalues: sin <= 1e-4 (residual / gap);
  * on R-MAT graphs, whose top eigenvalue 1 has one eigenvector per
    connected component (D^1/2 1_C), the angle to that exact eigenspace.
"""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import connected_components
from scipy.sparse.linalg import eigsh

from flashx_b200 import _lib, FmxError, matrix_image, sparse_matrix
from flashx_b200.eigen import NA_operator, compute_eigen, eigen_options
from flashx_b200.graphs import rmat_edges, sbm_edges, symmetrize

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _na(n, src, dst):
    keep = src != dst
    A = sp.csr_matrix((np.ones(int(keep.sum())), (src[keep], dst[keep])), shape=(n, n))
    A.data[:] = 1.0
    deg = np.asarray(A.sum(1)).ravel()
    s = np.where(deg > 0, 1.0 / np.sqrt(np.maximum(deg, 1)), 0.0)
    return (sp.diags(s) @ A @ sp.diags(s)).tocsr(), A, deg


def _matrix(n, src, dst, block=4096):
    img = matrix_image.build(src, dst, None, nrows=n, ncols=n, block_size=(block, block), dedup=True)
    return sparse_matrix.create(img, None)


def _residuals(N, vals, X):
    R = N @ X - X * vals
    return np.linalg.norm(R, axis=0) / np.linalg.norm(X, axis=0)


def _sin_angle(X, U):
    """Largest principal angle (sine) between span(X) and span(U)."""
    Qx, _ = np.linalg.qr(X)
    Qu, _ = np.linalg.qr(U)
    s = np.linalg.svd(Qu.T @ Qx, compute_uv=False)
    return float(np.sqrt(max(0.0, 1.0 - s.min() ** 2)))


@pytest.mark.parametrize("precision", ["plain", "mixed"])
@pytest.mark.parametrize("n,B,ratio", [(6000, 4, 20.0), (12000, 8, 30.0)])
def test_sbm_top_blocks(torch_cuda, precision, n, B, ratio):
    src, dst, _ = sbm_edges(n, B, 20.0, ratio, seed=n + B)
    n = n // B * B
    N, _, _ = _na(n, src, dst)
    m = _matrix(n, src, dst)
    opts = eigen_options()
    opts.init(B)
    opts.which = "LA"
    opts.tol = TOL
    opts.precision = precision
    res = compute_eigen(NA_operator(m), True, opts)
    assert res.status.converged == B and res.status.max_residual <= TOL
    assert res.status.num_ops == res.status.spmm_calls * opts.block_size
    X = res.vecs.double().cpu().numpy()
    r = _residuals(N, res.vals, X)
    assert r.max() <= 2 * TOL, r
    # the library's explicit residuals agree with FP64 ones down to the FP32
    # storage floor of the vectors (about 1e-7)
    np.testing.assert_allclose(res.residuals, r, rtol=0.05, atol=2e-7)
    w, U = eigsh(N, k=B + 4, which="LA", tol=1e-12)
    order = np.argsort(-w)
    w, U = w[order], U[:, order]
    assert w[B - 1] - w[B] > 0.05                   # a separated block subspace
    assert np.abs(res.vals - w[:B]).max() <= 1e-6
    assert _sin_angle(X, U[:, :B]) <= 1e-4


def test_largest_magnitude_on_bipartite_graph(torch_cuda):
    """which = "LM" (the reference's default) finds the pairs +-l of a
    bipartite graph."""
    rng = np.random.default_rng(5)
    n, half = 4000, 2000
    u = rng.integers(0, half, 40000)
    v = half + rng.integers(0, half, 40000)
    # plant structure: a denser corner so that the second pair is separated
    u2 = rng.integers(0, 300, 6000)
    v2 = half + rng.integers(0, 300, 6000)
    s, d = symmetrize(np.concatenate([u, u2]).astype(np.uint32), np.concatenate([v, v2]).astype(np.uint32))
    N, _, _ = _na(n, s, d)
    m = _matrix(n, s, d, block=1024)
    opts = eigen_options()
    opts.init(4)
    opts.which = "LM"
    opts.tol = TOL
    res = compute_eigen(NA_operator(m), True, opts)
    assert res.status.converged == 4
    X = res.vecs.double().cpu().numpy()
    assert _residuals(N, res.vals, X).max() <= 2 * TOL
    w, U = eigsh(N, k=8, which="LM", tol=1e-12)
    order = np.argsort(-np.abs(w))
    w, U = w[order], U[:, order]
    np.testing.assert_allclose(np.sort(res.vals), np.sort(w[:4]), atol=1e-6)
    assert np.abs(np.abs(res.vals) - np.abs(w[:4])).max() <= 1e-6
    assert _sin_angle(X, U[:, :4]) <= 1e-4


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_rmat_top8_in_component_eigenspace(torch_cuda, precision):
    """Symmetrised R-MAT scale 18 (the eigensolver configuration at a smaller
    scale): the top-8 eigenvalue is 1 with one eigenvector D^1/2 1_C per
    connected component, so the FP64 answer is known exactly."""
    scale = 18
    n = 1 << scale
    src, dst = rmat_edges(scale, seed=1)
    s, d = symmetrize(src, dst)
    N, A, deg = _na(n, s, d)
    m = _matrix(n, s, d, block=16384)
    ncomp, lab = connected_components(A, directed=False)
    nontrivial = np.bincount(lab, weights=deg) > 0
    assert nontrivial.sum() >= 8
    opts = eigen_options()
    opts.init(8)
    opts.which = "LA"
    opts.tol = TOL
    opts.precision = precision
    res = compute_eigen(NA_operator(m), True, opts)
    assert res.status.converged == 8
    X = res.vecs.double().cpu().numpy()
    assert _residuals(N, res.vals, X).max() <= 2 * TOL
    assert np.abs(res.vals - 1.0).max() <= 1e-6
    # projection onto span{D^1/2 1_C}: coefficient per component
    sq = np.sqrt(deg)
    for j in range(8):
        x = X[:, j]
        coef = np.bincount(lab, weights=sq * x, minlength=ncomp) / np.maximum(np.bincount(lab, weights=deg,
                                                                                          minlength=ncomp), 1e-300)
        px = coef[lab] * sq
        assert np.linalg.norm(x - px) / np.linalg.norm(x) <= 1e-4


def test_warm_start_needs_fewer_passes(torch_cuda):
    """A start block close to the answer (X0) converges in fewer filter
    passes than the random start, to the same eigenvalues."""
    import torch
    n, B = 8000, 6
    src, dst, _ = sbm_edges(n, B, 20.0, 25.0, seed=77)
    n = n // B * B
    N, _, _ = _na(n, src, dst)
    m = _matrix(n, src, dst)
    op = NA_operator(m)
    opts = eigen_options()
    opts.init(B)
    opts.which = "LA"
    opts.tol = TOL
    cold = compute_eigen(op, True, opts)
    w, U = eigsh(N, k=opts.block_size, which="LA", tol=1e-10)
    rng = np.random.default_rng(1)
    X0 = U + 1e-3 * rng.standard_normal(U.shape)
    warm = compute_eigen(op, True, opts, X0=torch.from_numpy(X0.astype(np.float32)).cuda())
    assert warm.status.converged == B and cold.status.converged == B
    assert warm.status.num_ops < cold.status.num_ops
    np.testing.assert_allclose(warm.vals, cold.vals, atol=1e-6)


def test_argument_errors(torch_cuda):
    n = 1000
    rng = np.random.default_rng(3)
    s, d = symmetrize(rng.integers(0, n, 5000).astype(np.uint32), rng.integers(0, n, 5000).astype(np.uint32))
    m = _matrix(n, s, d, block=256)
    opts = eigen_options()
    opts.init(4)
    opts.block_size = 2                     # nev > block_size
    with pytest.raises(FmxError) as e:
        compute_eigen(m, True, opts)
    assert e.value.code == _lib.FMX_ERR_INVAL
    opts.init(4)
    opts.block_size = 65
    with pytest.raises(FmxError) as e:
        compute_eigen(m, True, opts)
    assert e.value.code == _lib.FMX_ERR_UNSUPPORTED
    rect = sparse_matrix.create(matrix_image.build(s, d % 500, None, nrows=n, ncols=500, block_size=(256, 256)), None)
    opts.init(4)
    with pytest.raises(FmxError) as e:
        compute_eigen(rect, True, opts)
    assert e.value.code == _lib.FMX_ERR_DIM


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_svd_operator_rectangular(torch_cuda, precision):
    """A^T A of a rectangular weighted matrix through its transpose
    (SVD_Operator, test-eigen.cpp:138-177): eigenvalues are the squared
    singular values (scipy svds, FP64), vectors the right singular vectors."""
    from scipy.sparse.linalg import svds
    from flashx_b200 import create_2d_matrix
    from flashx_b200.eigen import SVD_operator
    rng = np.random.default_rng(21)
    nr, nc, m = 5000, 3000, 60000
    src = rng.integers(0, nr, m).astype(np.uint32)
    dst = rng.integers(0, nc, m).astype(np.uint32)
    # a planted low-rank part so that the top singular values are separated
    src = np.concatenate([src, rng.integers(0, 200, 8000).astype(np.uint32)])
    dst = np.concatenate([dst, rng.integers(0, 150, 8000).astype(np.uint32)])
    vals = rng.uniform(0.5, 1.5, len(src)).astype(np.float32)
    mat = create_2d_matrix(src, dst, vals, block_size=(1024, 1024), is_sym=False, nrows=nr, ncols=nc)
    keep = src != dst                      # the builder drops (i, i) entries (set_remove_self_edge default)
    A = sp.csr_matrix((vals[keep].astype(np.float64), (src[keep], dst[keep])), shape=(nr, nc))
    A.sum_duplicates()
    opts = eigen_options()
    opts.init(4)
    opts.which = "LA"
    opts.tol = TOL
    opts.precision = precision
    op = SVD_operator(mat)
    res = compute_eigen(op, True, opts)
    assert res.status.converged == 4
    X = res.vecs.double().cpu().numpy()
    N = (A.T @ A).tocsr()
    norm = float(svds(A, k=1, return_singular_vectors=False)[0]) ** 2
    assert norm <= op.upper * (1 + 1e-6)       # the filter's bound holds
    # residuals relative to the bound the solver normalises by
    r = np.linalg.norm(N @ X - X * res.vals, axis=0) / np.linalg.norm(X, axis=0) / op.upper
    assert r.max() <= 2 * TOL
    u, sv, vt = svds(A, k=6)
    order = np.argsort(-sv)
    sv, vt = sv[order], vt[order]
    np.testing.assert_allclose(res.vals, sv[:4] ** 2, rtol=1e-6)
    assert _sin_angle(X, vt[:4].T) <= 1e-4


@pytest.mark.parametrize("block", [10, 12, 20, 24, 32])
def test_block_sizes_off_sixteen(torch_cuda, block):
    """Blocks of up to 32 columns take the FP64 tensor-path basis update (one
    or two 16-column halves, guarded loads past b); the Gram takes the FP64
    MMA kernel up to 16 columns and the CUDA-core kernel beyond."""
    n, B = 8000, 4
    src, dst, _ = sbm_edges(n, B, 20.0, 20.0, seed=5)
    N, _, _ = _na(n, src, dst)
    m = _matrix(n, src, dst)
    opts = eigen_options()
    opts.init(B)
    opts.block_size = block
    opts.which = "LA"
    opts.tol = TOL
    res = compute_eigen(NA_operator(m), True, opts)
    assert res.status.converged == B and res.status.max_residual <= TOL
    vals = np.asarray(res.vals, dtype=np.float64)
    X = res.vecs.double().cpu().numpy()
    assert float(_residuals(N, vals, X).max()) <= 2 * TOL
    w = eigsh(N, k=B, which="LA", tol=1e-10, return_eigenvectors=False)
    assert np.allclose(np.sort(vals), np.sort(w), atol=1e-6)
