"""The closed-form gradient of the warm-start loss that libfmx's loss_kernel
and dy_kernel implement, checked against torch autograd in FP64 (CPU only):

  L = 1 - tr(M G^-1 M^T) / nev,  G = Y^T Y,  M = U^T Y
  dL/dY = U P1 + Y P2,  P1 = -(2/nev) M G^-1,  P2 = (2/nev) G^-1 M^T M G^-1
"""
import numpy as np
import pytest
import torch


@pytest.mark.parametrize("n,nev", [(500, 4), (2000, 16), (300, 1)])
def test_subspace_loss_gradient_closed_form(n, nev):
    rng = np.random.default_rng(n + nev)
    U, _ = np.linalg.qr(rng.standard_normal((n, nev)))
    Y = torch.tensor(rng.standard_normal((n, 16)), dtype=torch.float64, requires_grad=True)
    Ut = torch.tensor(U)
    G = Y.T @ Y
    M = Ut.T @ Y
    L = 1 - torch.trace(M @ torch.linalg.solve(G, M.T)) / nev
    L.backward()
    Yn = Y.detach().numpy()
    Gn = Yn.T @ Yn
    Mn = U.T @ Yn
    K = Mn @ np.linalg.inv(Gn)
    P1 = -(2 / nev) * K
    P2 = (2 / nev) * K.T @ K
    dY = U @ P1 + Yn @ P2
    np.testing.assert_allclose(dY, Y.grad.numpy(), rtol=1e-9, atol=1e-12)
    # the loss is 0 exactly when span(Y) contains span(U)
    Yc = np.hstack([U, rng.standard_normal((n, 16 - nev))])
    Gc, Mc = Yc.T @ Yc, U.T @ Yc
    assert abs(1 - np.trace(Mc @ np.linalg.solve(Gc, Mc.T)) / nev) < 1e-12
