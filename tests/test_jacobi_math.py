"""CPU: the arithmetic of jacobi_fast_kernel (flashx_b200/csrc/dense.cu),
restated in numpy, against numpy.linalg.eigh.

The kernel's steps, as written there:
- round-robin pairing of 0..m-1 (m = b rounded up to even; a padding index
  has a zero row and column);
- each step applies J^T A J one 2 x 2 block at a time, where block (P, R)
  holds the rows of pair P and the columns of pair R: columns mixed by pair
  R's rotation, then rows by pair P's (new a = c a - s q, new q = s a + c q);
- the angle t = sign(d) e / (|d| + sqrt(d^2 + e^2)), d = a_qq - a_pp,
  e = 2 a_pq, in FP32, then c = 1/sqrt(1 + t^2), s = t c renormalised in
  FP64 by two Newton steps for c^2 + s^2 = 1;
- the sweep loop stops when off-diagonal over diagonal, squared, is below
  1e-24.

This checks the method: the eigenvalues to 1e-12 of the largest and the
eigenvectors orthonormal to 1e-13 despite the FP32 angles, and the number of
sweeps. The GPU tests check the kernel itself (tests/test_dense_gpu.py).
"""
import numpy as np
import pytest


def _rotation(app, aqq, apq):
    if apq == 0.0:
        return 1.0, 0.0
    d, e = aqq - app, 2.0 * apq
    M = max(abs(d), abs(e))
    scale = 2.0 ** -np.frexp(M)[1]
    df, ef = np.float32(d * scale), np.float32(e * scale)
    if ef == 0:
        return 1.0, 0.0
    r = np.sqrt(np.float32(df * df + ef * ef), dtype=np.float32)
    t = np.float32(ef / (np.float32(abs(df)) + r))
    if df < 0:
        t = -t
    c32 = np.float32(1.0) / np.sqrt(np.float32(1.0) + t * t, dtype=np.float32)
    c, s = float(c32), float(t) * float(c32)
    for _ in range(2):
        f = 1.5 - 0.5 * (c * c + s * s)
        c, s = c * f, s * f
    return c, s


def _pairs(m, step):
    out = []
    for k in range(m // 2):
        a = 0 if k == 0 else 1 + (k - 1 + step) % (m - 1)
        q = 1 + (m - 2 - k + step) % (m - 1)
        out.append((min(a, q), max(a, q)))
    return out


def _jacobi(H, max_sweeps=30):
    b = H.shape[0]
    m = b + (b & 1)
    A = np.zeros((m, m))
    A[:b, :b] = 0.5 * (H + H.T)
    Q = np.eye(m)
    sweeps = 0
    for sweep in range(max_sweeps):
        # the squares summed apart, as the kernel does (the total minus the
        # diagonal's cancels to rounding noise near convergence)
        d2 = float(np.sum(np.diag(A) ** 2))
        off2 = float(np.sum((A - np.diag(np.diag(A))) ** 2))
        if off2 / (d2 if d2 > 0 else 1.0) < 1e-24:
            break
        sweeps += 1
        for step in range(m - 1):
            pairs = _pairs(m, step)
            rot = [_rotation(A[a, a], A[q, q], A[a, q]) for a, q in pairs]
            An, Qn = A.copy(), Q.copy()
            for P, (aP, qP) in enumerate(pairs):
                cP, sP = rot[P]
                for R, (aR, qR) in enumerate(pairs):
                    cR, sR = rot[R]
                    x = A[np.ix_([aP, qP], [aR, qR])]
                    y = np.array([[cR * x[0, 0] - sR * x[0, 1], sR * x[0, 0] + cR * x[0, 1]],
                                  [cR * x[1, 0] - sR * x[1, 1], sR * x[1, 0] + cR * x[1, 1]]])
                    z = np.array([[cP * y[0, 0] - sP * y[1, 0], cP * y[0, 1] - sP * y[1, 1]],
                                  [sP * y[0, 0] + cP * y[1, 0], sP * y[0, 1] + cP * y[1, 1]]])
                    An[np.ix_([aP, qP], [aR, qR])] = z
                    u = Q[np.ix_([aP, qP], [aR, qR])]
                    Qn[np.ix_([aP, qP], [aR, qR])] = np.array(
                        [[cR * u[0, 0] - sR * u[0, 1], sR * u[0, 0] + cR * u[0, 1]],
                         [cR * u[1, 0] - sR * u[1, 1], sR * u[1, 0] + cR * u[1, 1]]])
            A, Q = An, Qn
    w = np.diag(A)[:b] if m == b else np.array([A[j, j] for j in range(m) if abs(Q[b, j]) <= 0.5])
    V = Q[:b][:, [j for j in range(m) if m == b or abs(Q[b, j]) <= 0.5]]
    order = np.argsort(-w, kind="stable")
    return w[order], V[:, order], sweeps


@pytest.mark.parametrize("b", [16, 24, 7])
def test_jacobi_method_matches_eigh(b):
    rng = np.random.default_rng(b)
    X = rng.standard_normal((b, b))
    H = X + X.T
    w, V, sweeps = _jacobi(H)
    ref = np.sort(np.linalg.eigvalsh(H))[::-1]
    scale = np.abs(ref).max()
    assert np.max(np.abs(w - ref)) <= 1e-12 * scale
    assert np.max(np.abs(V.T @ V - np.eye(b))) <= 1e-13
    assert np.max(np.abs(H @ V - V * w)) <= 1e-11 * scale
    assert sweeps <= 8
