"""Dense eigensolver kernels against plain PyTorch FP64 references.

Tolerances (relative to the result's max magnitude):
  BF16 tensor cores      3e-2  (8-bit mantissa operands, FP32 accumulate)
  TF32x3 tensor cores    1e-5  (split operands: FP32-level accuracy)
  FP64 CUDA-core Gram    1e-12
"""
import ctypes as C

import numpy as np
import pytest

from flashx_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = {_lib.DENSE_BF16: 3e-2, _lib.DENSE_TF32X3: 1e-5, _lib.DENSE_F64: 1e-12}


def _stream(torch):
    return torch.cuda.current_stream().cuda_stream


@pytest.mark.parametrize("prec", [_lib.DENSE_BF16, _lib.DENSE_TF32X3])
@pytest.mark.parametrize("n,K,N,ldx", [(1000, 16, 16, 16), (100003, 16, 16, 16), (100, 16, 16, 16), (50000, 32, 16, 32),
                                       (7777, 48, 32, 48), (300, 8, 64, 8), (130, 64, 48, 64),
                                       # K padded to the MMA step; rows wider than K
                                       (999, 12, 24, 12), (4097, 20, 16, 24), (70000, 16, 16, 20),
                                       # K % 4 != 0: the thread-staged kernel
                                       (5000, 10, 16, 10), (333, 3, 8, 7)])
def test_tc_gemm(torch_cuda, prec, n, K, N, ldx):
    torch = torch_cuda
    g = torch.Generator(device="cuda").manual_seed(n + K)
    Xf = torch.randn((n, ldx), generator=g, device="cuda")
    X = Xf[:, :K]
    B = torch.randn((K, N), generator=g, device="cuda")
    Y = torch.full((n, N), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = _lib.lib.fmx_dense_gemm(prec, Xf.data_ptr(), ldx, n, K, B.data_ptr(), N, N, Y.data_ptr(), N, err.data_ptr(),
                                 _stream(torch))
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = X.double() @ B.double()
    scale = float(ref.abs().max())
    assert float((Y.double() - ref).abs().max()) <= TOL[prec] * scale


@pytest.mark.parametrize("prec", [_lib.DENSE_BF16, _lib.DENSE_TF32X3, _lib.DENSE_F64])
@pytest.mark.parametrize("n,M,N", [(1000, 16, 16), (200001, 16, 16), (100, 16, 16), (65536, 32, 32), (4097, 48, 16), (129, 64, 64),
                                   (50, 16, 48), (777, 12, 5), (3, 1, 16), (99999, 8, 8), (100003, 16, 9)])
def test_gram(torch_cuda, prec, n, M, N):
    _gram_case(torch_cuda, prec, n, M, N, M, N)


# strided rows and row lengths that are not whole 16-byte units: the
# pipelined kernel takes rows of up to 64 floats in whole units, the older
# kernels the rest
@pytest.mark.parametrize("prec", [_lib.DENSE_BF16, _lib.DENSE_TF32X3])
@pytest.mark.parametrize("n,M,N,ldx,ldw", [(70001, 16, 16, 20, 32), (5000, 10, 6, 12, 8), (3333, 7, 16, 7, 16),
                                           (40000, 24, 20, 24, 20), (1000, 16, 16, 100, 16)])
def test_gram_strided(torch_cuda, prec, n, M, N, ldx, ldw):
    _gram_case(torch_cuda, prec, n, M, N, ldx, ldw)


def _gram_case(torch_cuda, prec, n, M, N, ldx, ldw):
    torch = torch_cuda
    g = torch.Generator(device="cuda").manual_seed(n + M + N)
    Xf = torch.randn((n, ldx), generator=g, device="cuda")
    Wf = torch.randn((n, ldw), generator=g, device="cuda")
    X, W = Xf[:, :M], Wf[:, :N]
    parts = _lib.lib.fmx_dense_gram_parts(prec, n)
    dt = torch.float64 if prec == _lib.DENSE_F64 else torch.float32
    part = torch.empty(parts * M * N, dtype=dt, device="cuda")
    G = torch.full((M, N), float("nan"), dtype=dt, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    for _ in range(2):                      # deterministic: same bits twice
        rc = _lib.lib.fmx_dense_gram(prec, Xf.data_ptr(), ldx, M, Wf.data_ptr(), ldw, N, n, part.data_ptr(),
                                     G.data_ptr(), err.data_ptr(), _stream(torch))
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        if _ == 0:
            first = G.clone()
    assert torch.equal(first, G)
    assert int(err.item()) == 0
    ref = X.double().T @ W.double()
    scale = float(ref.abs().max())
    assert float((G.double() - ref).abs().max()) <= TOL[prec] * scale * (1 if prec != _lib.DENSE_F64 else 10)


@pytest.mark.parametrize("b", [1, 4, 16, 33, 64])
def test_chol_inv(torch_cuda, b):
    torch = torch_cuda
    g = torch.Generator(device="cuda").manual_seed(b)
    A = torch.randn((b + 5, b), generator=g, device="cuda", dtype=torch.float64)
    G = A.T @ A + 0.1 * torch.eye(b, device="cuda", dtype=torch.float64)
    T = torch.empty((b, b), dtype=torch.float64, device="cuda")
    info = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    assert _lib.lib.fmx_dense_chol_inv(G.data_ptr(), b, T.data_ptr(), info.data_ptr(), _stream(torch)) == 0
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    assert torch.allclose(torch.triu(T), T)
    I = T.T @ G @ T
    assert float((I - torch.eye(b, device="cuda", dtype=torch.float64)).abs().max()) < 1e-10
    # a non-positive pivot is reported
    Gbad = G.clone()
    Gbad[b // 2, b // 2] = -1.0
    assert _lib.lib.fmx_dense_chol_inv(Gbad.data_ptr(), b, T.data_ptr(), info.data_ptr(), _stream(torch)) == 0
    torch.cuda.synchronize()
    assert int(info.item()) > 0


@pytest.mark.parametrize("b", [1, 2, 7, 16, 24, 31, 32, 33, 48, 64])
def test_sym_eig(torch_cuda, b):
    torch = torch_cuda
    g = torch.Generator(device="cuda").manual_seed(100 + b)
    A = torch.randn((b, b), generator=g, device="cuda", dtype=torch.float64)
    H = A + A.T
    w = torch.empty(b, dtype=torch.float64, device="cuda")
    V = torch.empty((b, b), dtype=torch.float64, device="cuda")
    assert _lib.lib.fmx_dense_sym_eig(H.data_ptr(), b, w.data_ptr(), V.data_ptr(), _stream(torch)) == 0
    torch.cuda.synchronize()
    ref = torch.linalg.eigvalsh(H).flip(0)
    assert float((w - ref).abs().max()) < 1e-10 * max(1.0, float(ref.abs().max()))
    assert float((V.T @ V - torch.eye(b, device="cuda", dtype=torch.float64)).abs().max()) < 1e-10
    assert float((H @ V - V * w).abs().max()) < 1e-9 * max(1.0, float(ref.abs().max()))
