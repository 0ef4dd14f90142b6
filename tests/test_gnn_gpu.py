"""The learned warm start: libfmx's GNN forward/backward kernels against a
torch FP64 autograd oracle on the CPU, finite differences, and what the
trained network gains over the random start.

Tolerances (norm-wise relative error of the full gradient vector):
  FMX_DENSE_TF32X3 (3xTF32 products, FP32 accumulation)     2e-3
  FMX_DENSE_BF16   (BF16 operands, FP32 accumulation)       6e-2
Finite differences (3xTF32, central, step 1e-2 along the gradient): 2e-2.
"""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.linalg import eigsh

from flashx_b200 import _lib, matrix_image, sparse_matrix
from flashx_b200.eigen import NA_operator
from flashx_b200.graphs import sbm_edges
from flashx_b200.warmstart import compare_starts, sbm_instance, warm_start_net

pytestmark = pytest.mark.gpu


class _graph:
    """An SBM graph on the GPU plus its FP64 operator and top eigenvectors."""

    def __init__(self, torch, n=3000, B=4, ratio=15.0, seed=3):
        src, dst, _ = sbm_edges(n, B, 20.0, ratio, seed)
        n = n // B * B
        self.mat = sparse_matrix.create(
            matrix_image.build(src, dst, None, nrows=n, ncols=n, block_size=(4096, 4096), dedup=True), None)
        self.op = NA_operator(self.mat)
        keep = src != dst
        A = sp.csr_matrix((np.ones(int(keep.sum())), (src[keep], dst[keep])), shape=(n, n))
        A.data[:] = 1.0
        deg = np.asarray(A.sum(1)).ravel()
        s = np.where(deg > 0, 1 / np.sqrt(np.maximum(deg, 1)), 0.0)
        self.N = (sp.diags(s) @ A @ sp.diags(s)).tocsr()
        w, U = eigsh(self.N, k=B, which="LA", tol=1e-10)
        self.U64 = U
        self.U = torch.from_numpy(U.astype(np.float32)).cuda()
        self.nev = B


def _torch_loss_grad(torch, params, Z, N, U):
    """The same network and loss in torch FP64 on the CPU (autograd)."""
    p = torch.tensor(params, dtype=torch.float64, requires_grad=True)
    W1 = p[:4096].view(64, 64)
    b1 = p[4096:4160]
    W2 = p[4160:].view(64, 16)
    Zt = torch.tensor(Z, dtype=torch.float64)
    Nt = torch.sparse_csr_tensor(torch.tensor(N.indptr, dtype=torch.int64), torch.tensor(N.indices, dtype=torch.int64),
                                 torch.tensor(N.data, dtype=torch.float64), size=N.shape)
    H = torch.relu(Zt @ W1 + b1)
    Y = Nt @ (H @ W2)
    Ut = torch.tensor(U, dtype=torch.float64)
    G = Y.T @ Y
    M = Ut.T @ Y
    f = torch.trace(M @ torch.linalg.solve(G, M.T))
    loss = 1.0 - f / U.shape[1]
    loss.backward()
    return float(loss), p.grad.numpy()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("precision,tol", [("tf32x3", 2e-3), ("bf16", 6e-2)])
def test_gradient_matches_torch_fp64(torch_cuda, precision, tol):
    torch = torch_cuda
    g = _graph(torch)
    net = warm_start_net(seed=1)
    Z = net.features(g.op, 7)
    loss, grad = net.loss_grad(g.op, Z, g.U, precision=precision, want_grad=True)
    ref_loss, ref_grad = _torch_loss_grad(torch, net.get_params(), Z.cpu().numpy(), g.N, g.U64)
    assert abs(loss - ref_loss) <= (1e-4 if precision == "tf32x3" else 1e-2)
    assert _rel(grad, ref_grad) <= tol
    # each block (dW1, db1, dW2) on its own
    for lo, hi in ((0, 4096), (4096, 4160), (4160, 5184)):
        assert _rel(grad[lo:hi], ref_grad[lo:hi]) <= 2 * tol


def test_gradient_matches_finite_differences(torch_cuda):
    torch = torch_cuda
    g = _graph(torch, seed=5)
    net = warm_start_net(seed=2)
    Z = net.features(g.op, 11)
    p0 = net.get_params()
    _, grad = net.loss_grad(g.op, Z, g.U, precision="tf32x3", want_grad=True)
    rng = np.random.default_rng(0)
    for d in (grad / np.linalg.norm(grad), rng.standard_normal(grad.size).astype(np.float32)):
        d = d / np.linalg.norm(d)
        eps = 1e-2
        net.set_params(p0 + eps * d)
        lp = net.loss_grad(g.op, Z, g.U, precision="tf32x3")
        net.set_params(p0 - eps * d)
        lm = net.loss_grad(g.op, Z, g.U, precision="tf32x3")
        fd = (lp - lm) / (2 * eps)
        an = float(np.dot(grad, d))
        assert abs(fd - an) <= 2e-2 * max(abs(an), 1e-3), (fd, an)
    net.set_params(p0)


def test_features_match_their_definition(torch_cuda):
    """Z = [F, N F, N^2 F, N^3 F] with F[:, 0] the standardised log(1 + degree)
    and F[:, 1:] N(0, 1) channels (N = D^-1/2 A D^-1/2, FP64 on the CPU)."""
    torch = torch_cuda
    g = _graph(torch, n=6000, B=6)
    Z = warm_start_net.features(g.op, 5).double().cpu().numpy()
    A = g.N
    sc = g.op.scale.double().cpu().numpy()
    ld = np.where(sc > 0, np.log1p(1.0 / np.maximum(sc, 1e-30) ** 2), 0.0)
    np.testing.assert_allclose(Z[:, 0], (ld - ld.mean()) / ld.std(), atol=1e-4)
    R = Z[:, 1:16].ravel()
    assert abs(R.mean()) < 0.02 and abs(R.std() - 1.0) < 0.02
    F = Z[:, :16]
    for h in range(1, 4):
        F = A @ F
        np.testing.assert_allclose(Z[:, 16 * h:16 * (h + 1)], F, atol=1e-4 * max(1.0, float(np.abs(F).max())))


def test_params_roundtrip_and_determinism(torch_cuda, tmp_path):
    torch = torch_cuda
    g = _graph(torch, n=2000)
    net = warm_start_net(seed=4)
    path = str(tmp_path / "w.f32")
    net.save(path)
    back = warm_start_net.load(path)
    assert np.array_equal(back.get_params(), net.get_params())
    Z1 = net.features(g.op, 3)
    Z2 = net.features(g.op, 3)
    assert torch.equal(Z1, Z2)
    assert torch.equal(net.forward(g.op, Z1), back.forward(g.op, Z2))
    assert not torch.equal(Z1, net.features(g.op, 4))


def test_training_improves_the_start_block(torch_cuda):
    """Trained on the plain solver's eigenvectors of 24 small SBM graphs, the
    network's start block aligns with the wanted eigenvectors of 6 held-out
    graphs far better than a random block does, and the solver started from
    it needs fewer SpMMs in total than from a random block, with the
    network's own 4 per graph counted."""
    torch = torch_cuda
    train = [sbm_instance(s, n_range=(3000, 6000)) for s in range(24)]
    held = [sbm_instance(1000 + s, n_range=(3000, 6000)) for s in range(6)]
    net = warm_start_net(seed=0)
    before = np.mean([net.loss_grad(h.op, net.features(h.op, 99), h.U) for h in held])
    hist = net.train(train, epochs=6, lr=3e-3)
    after = np.mean([net.loss_grad(h.op, net.features(h.op, 99), h.U) for h in held])
    rows = [compare_starts(net, h) for h in held]
    print("train loss", np.round(hist, 4), "held-out loss before", round(before, 4), "after", round(after, 4))
    for r in rows:
        print(r)
    assert all(r["converged"] for r in rows)
    assert after < before - 0.1 and after < 0.75
    assert np.median([r["spmm_warm"] for r in rows]) <= np.median([r["spmm_random"] for r in rows])
    assert sum(r["spmm_warm"] for r in rows) < sum(r["spmm_random"] for r in rows)
