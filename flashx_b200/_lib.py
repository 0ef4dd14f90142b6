"""ctypes binding of libfmx.so (the C ABI declared in include/fmx.h).

The library must exist (built in-tree by flashx_b200.build); there is no
fallback implementation: importing this module without it raises.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfmx.so")

FMX_OK = 0
FMX_ERR_INVAL = -1
FMX_ERR_DIM = -2
FMX_ERR_TYPE = -3
FMX_ERR_IMAGE = -4
FMX_ERR_OOM = -5
FMX_ERR_CUDA = -6
FMX_ERR_IO = -7
FMX_ERR_UNSUPPORTED = -8

F32, F64, BF16, I32, I64 = 0, 1, 2, 3, 4
P_BOOL, P_INTEGER, P_LONG, P_FLOAT, P_DOUBLE = 0, 4, 6, 8, 9

EXACT_ROW_MAX = 256   # FMX_EXACT_ROW_MAX: rows summed in the reference's order

DENSE_BF16, DENSE_TF32X3, DENSE_F64 = 0, 1, 2

EIGEN_LA, EIGEN_LM = 0, 1
GNN_FEATURES, GNN_OUT, GNN_PARAMS = 64, 16, 5184
EIGEN_PLAIN, EIGEN_MIXED = 0, 1
EIGEN_OP_SCALED, EIGEN_OP_GRAM = 0, 1

BUILD_DEDUP = 0x1
BUILD_KEEP_SELF_LOOPS = 0x2
BUILD_REF_VALUE_LAYOUT = 0x4
BUILD_TRANSPOSE = 0x8


class FmxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{msg} [status {code}]")
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python flashx_b200/build.py` "
            "(the CUDA library is required; there is no CPU fallback)")
    return C.CDLL(LIB_PATH)


lib = _load()

_vp, _sz, _u64, _i64, _u32, _int, _d = C.c_void_p, C.c_size_t, C.c_uint64, C.c_int64, C.c_uint32, C.c_int, C.c_double
_P = C.POINTER



class eigen_options_t(C.Structure):
    """struct fmx_eigen_options (include/fmx.h)."""
    _fields_ = [("nev", C.c_int), ("block_size", C.c_int), ("degree", C.c_int), ("max_iters", C.c_int),
                ("which", C.c_int), ("precision", C.c_int), ("tol", C.c_double), ("lower", C.c_double),
                ("upper", C.c_double), ("tensor_until", C.c_double), ("seed", C.c_uint64), ("X0", C.c_void_p),
                ("ldx0", C.c_int64), ("op", C.c_int)]


class eigen_status_t(C.Structure):
    """struct fmx_eigen_status (include/fmx.h)."""
    _fields_ = [("iters", C.c_int), ("converged", C.c_int), ("num_ops", C.c_int64), ("spmm_calls", C.c_int64),
                ("max_residual", C.c_double), ("seconds", C.c_double)]


_SIGS = {
    "fmx_strerror": (C.c_char_p, [_int]),
    "fmx_last_error": (C.c_char_p, []),
    "fmx_version": (C.c_char_p, []),
    "fmx_image_build": (_int, [_vp, _vp, _vp, _int, _u64, _u64, _u64, _u32, _u32, _int, _int, _P(_vp)]),
    "fmx_image_from_bytes": (_int, [_vp, _sz, _vp, _sz, _P(_vp)]),
    "fmx_image_load": (_int, [C.c_char_p, C.c_char_p, _P(_vp)]),
    "fmx_image_dump": (_int, [_vp, C.c_char_p, C.c_char_p]),
    "fmx_image_bytes": (_int, [_vp, _P(_vp), _P(_sz), _P(_vp), _P(_sz)]),
    "fmx_image_info": (_int, [_vp, _P(_u64), _P(_u64), _P(_u64), _P(_u32), _P(_int), _P(_u32), _P(_u32)]),
    "fmx_image_verify": (_int, [_vp]),
    "fmx_image_free": (_int, [_vp]),
    "fmx_matrix_create": (_int, [_vp, _vp, _int, _P(_vp)]),
    "fmx_matrix_load": (_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, _int, _P(_vp)]),
    "fmx_matrix_info": (_int, [_vp, _P(_u64), _P(_u64), _P(_u64), _P(_int), _P(_int)]),
    "fmx_matrix_device_bytes": (_int, [_vp, _P(_u64)]),
    "fmx_matrix_transpose": (_int, [_vp, _P(_vp)]),
    "fmx_matrix_free": (_int, [_vp]),
    "fmx_spmm": (_int, [_vp, _int, _vp, _i64, _int, _vp, _i64, _i64, _vp, _vp, _vp]),
    "fmx_spmm_host": (_int, [_vp, _int, _vp, _i64, _int, _vp, _i64, _i64]),
    "fmx_spmm_host_async": (_int, [_vp, _int, _vp, _i64, _int, _vp, _i64, _i64, _vp]),
    "fmx_spmm_noalloc": (_int, [_vp, _vp, _i64, _vp, _i64, _i64, _vp]),
    "fmx_matrix_schedule": (_int, [_vp, _P(_u64), _P(_u64), _P(_u64), _P(_u64)]),
    "fmx_matrix_hot": (_int, [_vp, _P(_u64), _P(_u64), _P(_u64)]),
    "fmx_matrix_layout_digest": (_int, [_vp, _int, _P(_u64)]),
    "fmx_dense_gemm": (_int, [_int, _vp, _i64, _i64, _int, _vp, _int, _int, _vp, _i64, _vp, _vp]),
    "fmx_dense_gram_parts": (_int, [_int, _i64]),
    "fmx_dense_gram": (_int, [_int, _vp, _i64, _int, _vp, _i64, _int, _i64, _vp, _vp, _vp, _vp]),
    "fmx_dense_chol_inv": (_int, [_vp, _int, _vp, _vp, _vp]),
    "fmx_dense_sym_eig": (_int, [_vp, _int, _vp, _vp, _vp]),
    "fmx_matrix_build_device": (_int, [_vp, _vp, _vp, _int, _u64, _u64, _u64, _int, _int, _vp, _P(_vp)]),
    "fmx_matrix_from_fg": (_int, [_vp, _sz, _int, _int, _P(_vp)]),
    "fmx_matrix_create_streamed": (_int, [_vp, _vp, _int, _u64, _P(_vp)]),
    "fmx_release_cached": (_int, [_int]),
    "fmx_matrix_stream_info": (_int, [_vp, _P(_u64), _P(_u64)]),
    "fmx_matrix_load_fg": (_int, [C.c_char_p, _int, _int, _P(_vp)]),
    "fmx_eigen_default_options": (None, [_P(eigen_options_t), _int]),
    "fmx_eigen_solve": (_int, [_vp, _vp, _P(eigen_options_t), _vp, _vp, _i64, _vp, _P(eigen_status_t), _vp]),
    "fmx_na_scale": (_int, [_vp, _vp, _vp]),
    "fmx_pagerank": (_int, [_vp, _u64, C.c_float, _vp, _P(_u64), _vp]),
    "fmx_gnn_create": (_int, [_int, _u64, _P(_vp)]),
    "fmx_gnn_free": (_int, [_vp]),
    "fmx_gnn_set_params": (_int, [_vp, _vp]),
    "fmx_gnn_get_params": (_int, [_vp, _vp]),
    "fmx_gnn_features": (_int, [_vp, _vp, _u64, _vp, _vp]),
    "fmx_gnn_forward": (_int, [_vp, _vp, _vp, _vp, _int, _vp, _vp]),
    "fmx_gnn_loss_grad": (_int, [_vp, _vp, _vp, _vp, _vp, _i64, _int, _int, _vp, _vp, _vp]),
    "fmx_gnn_adam_step": (_int, [_vp, C.c_float, _vp]),
    "fmx_rmat_edges_host": (_int, [_int, _u64, _d, _d, _d, _u64, _int, _vp, _vp, _int]),
    "fmx_rmat_edges_device": (_int, [_int, _u64, _d, _d, _d, _u64, _int, _vp, _vp, _vp]),
}

for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def last_error():
    s = lib.fmx_last_error()
    return s.decode() if s else ""


def check(code):
    """Raise FmxError for a non-zero status of a C-ABI call."""
    if code != FMX_OK:
        raise FmxError(code, last_error() or lib.fmx_strerror(code).decode())
    return code


def exported_symbols():
    return list(_SIGS)
