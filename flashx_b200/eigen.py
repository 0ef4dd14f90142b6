"""Block eigensolver on the B200 SpMM: the mirror of fm::eigen
(matrix/eigensolver/eigensolver.h:35-80, eigensolver.cpp:82-308).

    op = NA_operator(mat)                 # D^-1/2 A D^-1/2 (test-eigen.cpp:88-136)
    opts = eigen_options(); opts.init(8)  # nev = 8
    res = compute_eigen(op, True, opts)   # res.vals, res.vecs, res.status

The iteration (Chebyshev-filtered subspace iteration with FP64 CholQR2 and
Rayleigh-Ritz) runs in libfmx.so (fmx_eigen_solve); this module only fills
the option struct and wraps the device arrays.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib

_SOLVERS = ("KrylovSchur", "Davidson", "LOBPCG", "ChFSI")


class eigen_options:
    """eigen_options (eigensolver.h:57-73): same field names and defaults
    (tol 1e-8, max_iters 500, which "LM").  The reference picks an Anasazi
    solver by name; here every name runs the same block Chebyshev iteration,
    with block_size >= nev.  Extra fields: degree (the largest number of SpMMs
    per filter pass; each pass picks what its slowest residual needs),
    precision ("plain" or "mixed"), tensor_until, lower/upper (spectrum bounds;
    [-1, 1] holds for D^-1/2 A D^-1/2), seed."""

    def __init__(self):
        self.tol = 1.0e-8
        self.num_blocks = 0
        self.max_restarts = 100
        self.max_iters = 500
        self.block_size = 0
        self.nev = 1
        self.solver = "KrylovSchur"
        self.which = "LM"
        self.in_mem = True
        self.degree = 16
        self.precision = "plain"
        self.tensor_until = 1e-3
        self.lower = -1.0
        self.upper = 1.0
        self.seed = 1

    def init(self, nev, solver="KrylovSchur"):
        """eigen_options::init (eigensolver.cpp:93-116): False for an unknown solver."""
        if solver not in _SOLVERS:
            return False
        self.nev = nev
        self.solver = solver
        self.block_size = min(64, max(2 * nev, 16))
        return True

    def _struct(self):
        o = _lib.eigen_options_t()
        lib.fmx_eigen_default_options(C.byref(o), int(self.nev))
        o.nev = int(self.nev)
        o.block_size = int(self.block_size or min(64, max(2 * self.nev, 16)))
        o.degree = int(self.degree)
        o.max_iters = int(self.max_iters)
        if self.which not in ("LA", "LM"):
            raise ValueError(f"which must be 'LA' or 'LM' (got {self.which!r})")
        o.which = _lib.EIGEN_LA if self.which == "LA" else _lib.EIGEN_LM
        if self.precision not in ("plain", "mixed"):
            raise ValueError(f"precision must be 'plain' or 'mixed' (got {self.precision!r})")
        o.precision = _lib.EIGEN_PLAIN if self.precision == "plain" else _lib.EIGEN_MIXED
        o.tol = float(self.tol)
        o.lower = float(self.lower)
        o.upper = float(self.upper)
        o.tensor_until = float(self.tensor_until)
        o.seed = int(self.seed)
        return o


class eigen_status:
    def __init__(self, st):
        self.num_iters = st.iters
        self.num_ops = st.num_ops
        self.spmm_calls = st.spmm_calls
        self.converged = st.converged
        self.max_residual = st.max_residual
        self.seconds = st.seconds


class eigen_res:
    """eigen_res (eigensolver.h:49-55): vals (numpy FP64), vecs (n x nev
    FP32 CUDA tensor), status (num_iters, num_ops, ...), residuals (FP64,
    ||A x - l x|| / ||A|| of each returned pair)."""

    def __init__(self, vals, vecs, status, residuals):
        self.vals = vals
        self.vecs = vecs
        self.status = status
        self.residuals = residuals


class NA_operator:
    """D^-1/2 A D^-1/2 with D = A 1 (NA_eigen_Operator, test-eigen.cpp:88-136):
    the scaling is computed once on the GPU and fused into every SpMM."""

    def __init__(self, mat, device=0):
        import torch
        self.mat = mat
        self.scale = torch.empty(mat.get_num_rows(), dtype=torch.float32, device=f"cuda:{device}")
        st = torch.cuda.current_stream(self.scale.device).cuda_stream
        check(lib.fmx_na_scale(mat.handle, self.scale.data_ptr(), st))

    def get_num_rows(self):
        return self.mat.get_num_rows()

    def get_num_cols(self):
        return self.mat.get_num_cols()

    def run(self, x):
        """y = D^-1/2 A D^-1/2 x (spm_function::run)."""
        return self.mat.multiply(x, None, self.scale, self.scale)


class SVD_operator:
    """A^T A through the transpose (SVD_Operator, test-eigen.cpp:138-177):
    its top eigenpairs are the squared singular values and the right
    singular vectors of A.  The spectrum bound the Chebyshev filter needs is
    ||A^T A|| <= ||A||_1 ||A||_inf = (max column sum) (max row sum), from two
    SpMMs with a ones vector (exact as a bound for nonnegative entries)."""

    def __init__(self, mat):
        import torch
        self.mat = mat
        dev = f"cuda:{mat.device}"
        r = mat.multiply(torch.ones((mat.get_num_cols(), 1), device=dev))
        c = mat.transpose().multiply(torch.ones((mat.get_num_rows(), 1), device=dev))
        self.upper = float(r.abs().max()) * float(c.abs().max())

    def get_num_rows(self):
        return self.mat.get_num_cols()

    def get_num_cols(self):
        return self.mat.get_num_cols()


def compute_eigen(op, sym, opts, X0=None, stream=None):
    """compute_eigen(func, sym, opts) (eigensolver.h:74-75).  `op` is an
    NA_operator, an SVD_operator or a symmetric sparse_matrix; X0 an optional
    start block (n x block_size CUDA FP32 tensor, e.g. a learned warm
    start)."""
    import torch
    if not sym:
        raise ValueError("the block eigensolver handles symmetric operators")
    gram = isinstance(op, SVD_operator)
    mat = op.mat if isinstance(op, (NA_operator, SVD_operator)) else op
    scale = op.scale if isinstance(op, NA_operator) else None
    n = mat.get_num_cols() if gram else mat.get_num_rows()
    o = opts._struct()
    if gram:
        o.op = _lib.EIGEN_OP_GRAM
        o.lower, o.upper = 0.0, max(op.upper, 1e-30)
    dev = scale.device if scale is not None else torch.device("cuda", mat.device)
    if X0 is not None:
        if X0.dtype != torch.float32 or not X0.is_cuda or X0.shape != (n, o.block_size) or X0.stride(1) != 1:
            raise ValueError(f"X0 must be a row-major CUDA float32 tensor of shape ({n}, {o.block_size})")
        o.X0 = X0.data_ptr()
        o.ldx0 = X0.stride(0)
    vecs = torch.empty((n, o.nev), dtype=torch.float32, device=dev)
    vals = np.zeros(o.nev)
    res = np.zeros(o.nev)
    st = _lib.eigen_status_t()
    stream = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    check(lib.fmx_eigen_solve(mat.handle, scale.data_ptr() if scale is not None else None, C.byref(o),
                              vals.ctypes.data, vecs.data_ptr(), o.nev, res.ctypes.data, C.byref(st), stream))
    return eigen_res(vals, vecs, eigen_status(st), res)
