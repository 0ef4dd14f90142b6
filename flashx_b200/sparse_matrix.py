"""Host-side mirror of FlashMatrix's sparse-matrix interface over libfmx.

Names and argument meaning follow the reference:
  SpM_2d_index / SpM_2d_storage  matrix/sparse_matrix_format.h:441-532
  sparse_matrix.create           matrix/sparse_matrix.h:522-539
  sparse_matrix.multiply         matrix/sparse_matrix.h:629-650
  sparse_matrix.transpose        matrix/sparse_matrix.h:627
  create_2d_matrix               matrix/fm_utils.h:37-39
  set_deduplicate / set_remove_self_edge   matrix/fm_utils.h:34-35
Error behaviour follows it too: multiply(in, out) returns False and logs the
reason (sparse_matrix.cpp:712-718,754-766); loaders raise (the reference
throws io_exception / wrong_format on load, sparse_matrix_format.cpp:241-258).

Dense operands are torch CUDA tensors, row-major (stride(1) == 1), resident
on the matrix's device.  All compute runs in libfmx's CUDA kernels.
"""
import ctypes as C
import logging

import numpy as np

from . import _lib
from ._lib import lib, check, FmxError

log = logging.getLogger("flashx_b200")

_dedup = False
_remove_self = True


def set_deduplicate(v):
    """fm::set_deduplicate (matrix/fm_utils.cpp:41-44); off by default."""
    global _dedup
    _dedup = bool(v)


def set_remove_self_edge(v):
    """fm::set_remove_self_edge (matrix/fm_utils.cpp:46-49); on by default."""
    global _remove_self
    _remove_self = bool(v)


_PRIM_OF = {None: _lib.P_BOOL, "bool": _lib.P_BOOL, "float": _lib.P_FLOAT, "float32": _lib.P_FLOAT,
            "double": _lib.P_DOUBLE, "float64": _lib.P_DOUBLE, "int": _lib.P_INTEGER,
            "int32": _lib.P_INTEGER, "long": _lib.P_LONG, "int64": _lib.P_LONG}
_NP_OF_PRIM = {_lib.P_FLOAT: np.float32, _lib.P_DOUBLE: np.float64, _lib.P_INTEGER: np.int32,
               _lib.P_LONG: np.int64}
_ESIZE = {_lib.P_BOOL: 0, _lib.P_FLOAT: 4, _lib.P_INTEGER: 4, _lib.P_DOUBLE: 8, _lib.P_LONG: 8}


class matrix_image:
    """A .mat_idx / .mat byte pair (SpM_2d_index + SpM_2d_storage), host side."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.fmx_image_free(h)
            self._h = C.c_void_p(None)

    @classmethod
    def load(cls, mat_idx_file, mat_file):
        h = C.c_void_p()
        check(lib.fmx_image_load(mat_idx_file.encode(), mat_file.encode(), C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_bytes(cls, idx, mat):
        idx = bytes(idx)
        mat = bytes(mat)
        h = C.c_void_p()
        check(lib.fmx_image_from_bytes(idx, len(idx), mat, len(mat), C.byref(h)))
        return cls(h.value)

    @classmethod
    def build(cls, src, dst, vals=None, nrows=0, ncols=0, block_size=(16384, 16384),
              dedup=None, remove_self=None, ref_value_layout=False, nthreads=0):
        """Edge list -> image (fm::create_2d_matrix, fm_utils.cpp:617-715)."""
        src = np.ascontiguousarray(src, dtype=np.uint32)
        dst = np.ascontiguousarray(dst, dtype=np.uint32)
        if src.shape != dst.shape:
            raise ValueError("src and dst differ in length")
        prim = _lib.P_BOOL
        vptr = None
        if vals is not None:
            vals = np.ascontiguousarray(vals)
            prim = {np.dtype(np.float32): _lib.P_FLOAT, np.dtype(np.float64): _lib.P_DOUBLE,
                    np.dtype(np.int32): _lib.P_INTEGER, np.dtype(np.int64): _lib.P_LONG}.get(vals.dtype)
            if prim is None:
                raise TypeError(f"unsupported value dtype {vals.dtype}")
            if vals.shape != src.shape:
                raise ValueError("values differ in length from the edges")
            vptr = vals.ctypes.data
        flags = 0
        if (_dedup if dedup is None else dedup):
            flags |= _lib.BUILD_DEDUP
        if not (_remove_self if remove_self is None else remove_self):
            flags |= _lib.BUILD_KEEP_SELF_LOOPS
        if ref_value_layout:
            flags |= _lib.BUILD_REF_VALUE_LAYOUT
        h = C.c_void_p()
        check(lib.fmx_image_build(src.ctypes.data, dst.ctypes.data, vptr, prim, len(src), nrows, ncols,
                                  block_size[0], block_size[1], flags, nthreads, C.byref(h)))
        return cls(h.value)

    def dump(self, mat_idx_file, mat_file):
        check(lib.fmx_image_dump(self._h, mat_idx_file.encode(), mat_file.encode()))

    def bytes(self):
        ip, il, mp, ml = C.c_void_p(), C.c_size_t(), C.c_void_p(), C.c_size_t()
        check(lib.fmx_image_bytes(self._h, C.byref(ip), C.byref(il), C.byref(mp), C.byref(ml)))
        return C.string_at(ip, il.value), C.string_at(mp, ml.value)

    def info(self):
        nr, nc, nz = C.c_uint64(), C.c_uint64(), C.c_uint64()
        es, pt, bh, bw = C.c_uint32(), C.c_int(), C.c_uint32(), C.c_uint32()
        check(lib.fmx_image_info(self._h, C.byref(nr), C.byref(nc), C.byref(nz), C.byref(es),
                                 C.byref(pt), C.byref(bh), C.byref(bw)))
        return dict(nrows=nr.value, ncols=nc.value, nnz=nz.value, entry_size=es.value,
                    prim=pt.value, block_h=bh.value, block_w=bw.value)

    def verify(self):
        check(lib.fmx_image_verify(self._h))


class SpM_2d_index:
    """The .mat_idx half (header page + block-row offsets)."""

    def __init__(self, data):
        self.data = bytes(data)

    @classmethod
    def load(cls, idx_file):
        with open(idx_file, "rb") as f:
            return cls(f.read())


class SpM_2d_storage:
    """The .mat half (header page + packed tiles)."""

    def __init__(self, data):
        self.data = bytes(data)

    @classmethod
    def load(cls, mat_file, index=None):
        with open(mat_file, "rb") as f:
            return cls(f.read())


def _dtype_code(t):
    import torch
    return {torch.float32: _lib.F32, torch.float64: _lib.F64, torch.bfloat16: _lib.BF16,
            torch.int32: _lib.I32, torch.int64: _lib.I64}.get(t.dtype)


def _as_2d(t):
    return t.unsqueeze(1) if t.dim() == 1 else t


class sparse_matrix:
    """A 2D-tiled sparse matrix resident in one GPU's HBM."""

    def __init__(self, handle, device, owner=None):
        self._h = C.c_void_p(handle)
        self.device = device
        self._owner = owner
        nr, nc, nz, pt, sym = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_int(), C.c_int()
        check(lib.fmx_matrix_info(self._h, C.byref(nr), C.byref(nc), C.byref(nz), C.byref(pt), C.byref(sym)))
        self._nrows, self._ncols, self._nnz = nr.value, nc.value, nz.value
        self._prim, self._sym = pt.value, bool(sym.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.fmx_matrix_free(h)
            self._h = C.c_void_p(None)

    @property
    def handle(self):
        return self._h

    # -- construction (sparse_matrix::create, sparse_matrix.cpp:679-707) --
    @classmethod
    def create(cls, index, storage, t_index=None, t_storage=None, device=0):
        """create(SpM_2d_index, SpM_2d_storage[, t_index, t_storage]) or
        create(matrix_image[, None, t_image])."""
        if isinstance(index, matrix_image):
            img, timg = index, t_storage if isinstance(t_storage, matrix_image) else storage
        else:
            img = matrix_image.from_bytes(index.data, storage.data)
            timg = None
            if t_index is not None:
                timg = matrix_image.from_bytes(t_index.data, t_storage.data)
        if not isinstance(timg, matrix_image):
            timg = None
        h = C.c_void_p()
        check(lib.fmx_matrix_create(img._h, timg._h if timg is not None else None, device, C.byref(h)))
        return cls(h.value, device)

    @classmethod
    def create_streamed(cls, index, t_index=None, device=0, slice_entries=0):
        """The semi-external form (sparse_matrix::create(index, mat_io_factory),
        sparse_matrix.cpp:693-707): from matrix_image(s), the entry stream kept
        in pinned host memory and streamed to the GPU in slices of about
        slice_entries entries (0: 2^26) during every multiply."""
        h = C.c_void_p()
        check(lib.fmx_matrix_create_streamed(index._h, t_index._h if t_index is not None else None, device,
                                             int(slice_entries), C.byref(h)))
        return cls(h.value, device)

    def stream_info(self):
        """(slices per SpMM, pinned host bytes); (0, 0) for a resident matrix."""
        a, b = C.c_uint64(), C.c_uint64()
        check(lib.fmx_matrix_stream_info(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    @classmethod
    def load(cls, mat_idx_file, mat_file, t_mat_idx_file=None, t_mat_file=None, device=0):
        h = C.c_void_p()
        enc = lambda s: s.encode() if s is not None else None
        check(lib.fmx_matrix_load(enc(mat_idx_file), enc(mat_file), enc(t_mat_idx_file), enc(t_mat_file),
                                  device, C.byref(h)))
        return cls(h.value, device)

    @classmethod
    def from_device_edges(cls, src, dst, vals=None, nrows=0, ncols=0, dedup=None, remove_self=None,
                          transpose=False, stream=None):
        """The matrix straight from an edge list already on a GPU (int32 or
        uint32-valued CUDA tensors; vals: a float32/float64/int32/int64 CUDA
        tensor or None): fmx_matrix_build_device sorts and deduplicates on
        that GPU, with the same result as create_2d_matrix on the host.
        transpose=True also builds A^T (a directed graph's asymmetric pair)."""
        import torch
        if src.shape != dst.shape or not src.is_cuda or src.device != dst.device:
            raise ValueError("src and dst must be CUDA tensors of one shape on one device")
        if src.dtype != torch.int32 or dst.dtype != torch.int32:
            raise ValueError("src and dst must be int32 tensors (ids < 2^31)")
        src, dst = src.contiguous(), dst.contiguous()
        prim, vptr = _lib.P_BOOL, None
        if vals is not None:
            prim = {torch.float32: _lib.P_FLOAT, torch.float64: _lib.P_DOUBLE, torch.int32: _lib.P_INTEGER,
                    torch.int64: _lib.P_LONG}.get(vals.dtype)
            if prim is None or vals.shape != src.shape or vals.device != src.device:
                raise ValueError("vals must be a float32/float64/int32/int64 CUDA tensor like src")
            vals = vals.contiguous()
            vptr = vals.data_ptr()
        flags = 0
        if (_dedup if dedup is None else dedup):
            flags |= _lib.BUILD_DEDUP
        if not (_remove_self if remove_self is None else remove_self):
            flags |= _lib.BUILD_KEEP_SELF_LOOPS
        if transpose:
            flags |= _lib.BUILD_TRANSPOSE
        dev = src.device.index
        st = stream if stream is not None else torch.cuda.current_stream(src.device).cuda_stream
        h = C.c_void_p()
        check(lib.fmx_matrix_build_device(src.data_ptr(), dst.data_ptr(), vptr, prim, src.numel(), nrows, ncols,
                                          flags, dev, st, C.byref(h)))
        return cls(h.value, dev)

    # -- reference accessors --
    def get_num_rows(self):
        return self._nrows

    def get_num_cols(self):
        return self._ncols

    def get_nnz(self):
        return self._nnz

    def is_symmetric(self):
        return self._sym

    def get_entry_size(self):
        return _ESIZE[self._prim]

    def get_type(self):
        return {_lib.P_BOOL: "bool", _lib.P_FLOAT: "float", _lib.P_DOUBLE: "double",
                _lib.P_INTEGER: "int", _lib.P_LONG: "long"}[self._prim]

    def device_bytes(self):
        b = C.c_uint64()
        check(lib.fmx_matrix_device_bytes(self._h, C.byref(b)))
        return b.value

    def schedule(self):
        """(light rows, warp tasks, heavy rows, kernels per SpMM panel)."""
        v = [C.c_uint64() for _ in range(4)]
        check(lib.fmx_matrix_schedule(self._h, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def hot(self):
        """(hot columns packed per SpMM, entries reading the pack, scratch bytes)."""
        v = [C.c_uint64() for _ in range(3)]
        check(lib.fmx_matrix_hot(self._h, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def layout_digest(self, transpose=False):
        """64-bit digest of the resident layout of A (or of A^T): equal for two
        builds exactly when they lay the matrix out identically."""
        v = C.c_uint64()
        check(lib.fmx_matrix_layout_digest(self._h, 1 if transpose else 0, C.byref(v)))
        return v.value

    def transpose(self):
        h = C.c_void_p()
        check(lib.fmx_matrix_transpose(self._h, C.byref(h)))
        return sparse_matrix(h.value, self.device, owner=self)

    # -- SpMM --
    def multiply(self, in_mat, out=None, row_scale_in=None, row_scale_out=None, stream=None):
        """multiply(in, out) -> bool (sparse_matrix.cpp:751-771); Y is overwritten.
        multiply(in) -> a new output tensor (sparse_matrix.cpp:773-795)."""
        import torch
        if out is None:
            res = torch.empty((self._nrows,) + tuple(in_mat.shape[1:]), dtype=in_mat.dtype, device=in_mat.device)
            if not self.multiply(in_mat, res, row_scale_in, row_scale_out, stream):
                raise FmxError(_lib.FMX_ERR_INVAL, _lib.last_error())
            return res
        x, y = _as_2d(in_mat), _as_2d(out)
        if x.shape[0] != self._ncols or y.shape[0] != self._nrows or x.shape[1] != y.shape[1]:
            log.error("the input and output matrix have incompatible dimensions")
            return False
        xt, yt = _dtype_code(x), _dtype_code(y)
        if xt is None or yt is None:
            log.error("unsupported dense type %s -> %s", x.dtype, y.dtype)
            return False
        def rowmajor(t):
            return t.shape[1] == 1 or t.stride(1) == 1

        if not (rowmajor(x) and rowmajor(y)) or not x.is_cuda or not y.is_cuda:
            log.error("dense matrices must be row-major CUDA tensors")
            return False
        ldx = x.stride(0) if x.shape[0] > 1 else x.shape[1]
        ldy = y.stride(0) if y.shape[0] > 1 else y.shape[1]
        sin = row_scale_in.data_ptr() if row_scale_in is not None else None
        sout = row_scale_out.data_ptr() if row_scale_out is not None else None
        st = stream if stream is not None else torch.cuda.current_stream(x.device).cuda_stream
        rc = lib.fmx_spmm(self._h, xt, x.data_ptr(), ldx, yt, y.data_ptr(), ldy, x.shape[1],
                          sin, sout, st)
        if rc != _lib.FMX_OK:
            log.error("fmx_spmm: %s", _lib.last_error())
            return False
        return True

    def multiply_host(self, X, Y=None):
        """SpMM on host (numpy) buffers: copies X in and Y out (synchronous)."""
        X = np.ascontiguousarray(X)
        X2 = X.reshape(X.shape[0], -1)
        code = {np.dtype(np.float32): _lib.F32, np.dtype(np.float64): _lib.F64,
                np.dtype(np.int32): _lib.I32, np.dtype(np.int64): _lib.I64}[X.dtype]
        if Y is None:
            Y = np.empty((self._nrows, X2.shape[1]), dtype=X.dtype)
        check(lib.fmx_spmm_host(self._h, code, X2.ctypes.data, X2.shape[1], code, Y.ctypes.data, Y.shape[1],
                                X2.shape[1]))
        return Y


    def multiply_host_async(self, X, Y, stream):
        """SpMM on host (numpy) buffers, asynchronous on `stream` (a CUDA
        stream handle): X is copied in and Y out when the stream gets there.
        Keep X and Y alive (and pinned, for asynchronous copies) until the
        stream is synchronised."""
        X2 = X.reshape(X.shape[0], -1)
        Y2 = Y.reshape(Y.shape[0], -1)
        if not (X2.flags.c_contiguous and Y2.flags.c_contiguous):
            raise ValueError("multiply_host_async takes C-contiguous arrays")
        code = {np.dtype(np.float32): _lib.F32, np.dtype(np.float64): _lib.F64,
                np.dtype(np.int32): _lib.I32, np.dtype(np.int64): _lib.I64}[X.dtype]
        check(lib.fmx_spmm_host_async(self._h, code, X2.ctypes.data, X2.shape[1], code, Y2.ctypes.data,
                                      Y2.shape[1], X2.shape[1], stream))
        return Y


def create_2d_matrix(src, dst, vals=None, block_size=(16384, 16384), is_sym=True, device=0,
                     nrows=0, ncols=0, ref_value_layout=False, return_images=False):
    """fm::create_2d_matrix (matrix/fm_utils.cpp:726-841): edge list -> matrix.
    Non-symmetric input also builds the transpose image (:790-823)."""
    img = matrix_image.build(src, dst, vals, nrows, ncols, block_size, ref_value_layout=ref_value_layout)
    timg = None
    if not is_sym:
        inf = img.info()
        timg = matrix_image.build(dst, src, vals, inf["ncols"], inf["nrows"], block_size,
                                  ref_value_layout=ref_value_layout)
    m = sparse_matrix.create(img, None, None, timg, device=device)
    if return_images:
        return m, img, timg
    return m
