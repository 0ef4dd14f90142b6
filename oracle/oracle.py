"""ctypes wrapper of the CPU ORACLE (test infrastructure only).

Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
and reference legs -- never by the flashx_b200 package.

  liboracle.so       oracle/fmx_oracle.c, the C restatement of the reference's
                     builder, SpMM traversal and PageRank (built by `make -C oracle`).
  libfmx_refwalk.so  oracle/ref_walk.cpp compiled against the reference's own
                     tile headers in place (`make -C oracle ref`, only where the
                     reference tree exists); optional.
  libfmx_reffg.so    oracle/ref_fg_walk.cpp compiled against FlashGraph's own
                     vertex record and header classes in place (same rule).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REFWALK_SO = os.path.join(HERE, "_ref", "libfmx_refwalk.so")
REFFG_SO = os.path.join(HERE, "_ref", "libfmx_reffg.so")
# Where the FlashX source tree lies, for building the reference walkers
# (`make ref`); unset means "not available" and the walkers are not built.
REFERENCE_TREE = os.environ.get("FMX_REFERENCE_TREE") or None

D_F32, D_F64, D_I32, D_I64 = 0, 1, 3, 4
P_BOOL, P_INTEGER, P_LONG, P_FLOAT, P_DOUBLE = 0, 4, 6, 8, 9
_NP = {D_F32: np.float32, D_F64: np.float64, D_I32: np.int32, D_I64: np.int64}
_D_OF = {np.dtype(v): k for k, v in _NP.items()}


def build(ref=None, tree=None):
    """Compile the oracle, and the reference walkers when the FlashX tree is
    given (`tree`, else the FMX_REFERENCE_TREE environment variable) and
    holds matrix/."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    tree = tree or REFERENCE_TREE
    if ref is None:
        ref = bool(tree) and os.path.isdir(os.path.join(tree, "matrix"))
    if ref:
        if not tree:
            raise ValueError("building the reference walkers needs the FlashX tree (FMX_REFERENCE_TREE)")
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={tree}"], check=True)


_orc = None
_ref = None


def orc():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        L = C.CDLL(ORACLE_SO)
        vp, sz, u64, i64, i32 = C.c_void_p, C.c_size_t, C.c_uint64, C.c_int64, C.c_int
        L.orc_build_image.restype = i32
        L.orc_build_image.argtypes = [vp, vp, vp, i32, u64, u64, u64, C.c_uint32, C.c_uint32, i32, i32, i32,
                                      C.POINTER(vp), C.POINTER(sz), C.POINTER(vp), C.POINTER(sz)]
        L.orc_free.argtypes = [vp]
        L.orc_nonzeros.restype = i64
        L.orc_nonzeros.argtypes = [vp, sz, vp, sz, vp, vp, u64]
        L.orc_spmm.restype = i32
        L.orc_spmm.argtypes = [vp, sz, vp, sz, i32, vp, vp, u64, i32, i32, u64, i32, u64, u64]
        L.orc_num_block_rows.restype = i64
        L.orc_num_block_rows.argtypes = [vp, sz]
        L.orc_block_rows_nnz.restype = i64
        L.orc_block_rows_nnz.argtypes = [vp, sz, vp, sz, u64, u64]
        L.orc_verify.restype = i32
        L.orc_verify.argtypes = [vp, sz, vp, sz]
        L.orc_pagerank.restype = i32
        L.orc_pagerank.argtypes = [vp, sz, vp, sz, vp, sz, vp, sz, u64, C.c_float, i32, vp, C.POINTER(u64)]
        L.orc_hilbert_xy2d.restype = i32
        L.orc_hilbert_xy2d.argtypes = [i32, i32, i32]
        L.orc_now.restype = C.c_double
        L.orc_rmat_edges.restype = i32
        L.orc_rmat_edges.argtypes = [i32, u64, C.c_double, C.c_double, C.c_double, u64, i32, vp, vp, i32]
        L.orc_fg_build.restype = i32
        L.orc_fg_build.argtypes = [vp, vp, vp, C.c_uint32, u64, u64, i32, C.POINTER(vp), C.POINTER(u64)]
        L.orc_fg_spmm.restype = i32
        L.orc_fg_spmm.argtypes = [vp, u64, i32, i32, i32, vp, vp, u64]
        L.orc_fg_vsize.restype = u64
        L.orc_fg_vsize.argtypes = [C.c_uint32, C.c_uint32]
        L.orc_fg_data_off.restype = u64
        L.orc_fg_data_off.argtypes = [C.c_uint32, C.c_uint32]
        _orc = L
    return _orc


def ref_available():
    return os.path.exists(REFWALK_SO)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REFWALK_SO):
            return None
        L = C.CDLL(REFWALK_SO)
        vp, u64, i64, i32 = C.c_void_p, C.c_uint64, C.c_int64, C.c_int
        L.ref_spmm.restype = i32
        L.ref_spmm.argtypes = [vp, vp, i32, vp, vp, u64]
        L.ref_nonzeros.restype = i64
        L.ref_nonzeros.argtypes = [vp, vp, vp, vp, u64]
        L.ref_hilbert_xy2d.restype = i32
        L.ref_hilbert_xy2d.argtypes = [i32, i32, i32]
        L.ref_header.restype = i32
        L.ref_header.argtypes = [vp] + [C.POINTER(u64)] * 5 + [C.POINTER(i32)] * 3
        _ref = L
    return _ref


def build_image(src, dst, vals=None, nrows=0, ncols=0, block=(16384, 16384), dedup=False,
                keep_self=False, ref_value_layout=False):
    """Oracle builder -> (idx bytes, mat bytes)."""
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    prim, vp = P_BOOL, None
    if vals is not None:
        vals = np.ascontiguousarray(vals)
        prim = {np.dtype(np.float32): P_FLOAT, np.dtype(np.float64): P_DOUBLE,
                np.dtype(np.int32): P_INTEGER, np.dtype(np.int64): P_LONG}[vals.dtype]
        vp = vals.ctypes.data
    ip, il, mp, ml = C.c_void_p(), C.c_size_t(), C.c_void_p(), C.c_size_t()
    rc = orc().orc_build_image(src.ctypes.data, dst.ctypes.data, vp, prim, len(src), nrows, ncols,
                               block[0], block[1], int(dedup), int(keep_self), int(ref_value_layout),
                               C.byref(ip), C.byref(il), C.byref(mp), C.byref(ml))
    if rc:
        raise ValueError("oracle builder rejected the edge list")
    idx = C.string_at(ip, il.value)
    mat = C.string_at(mp, ml.value)
    orc().orc_free(ip)
    orc().orc_free(mp)
    return idx, mat


def nonzeros(idx, mat):
    n = orc().orc_nonzeros(idx, len(idx), mat, len(mat), None, None, 0)
    if n < 0:
        raise ValueError("malformed image")
    r = np.empty(n, dtype=np.uint64)
    c = np.empty(n, dtype=np.uint64)
    orc().orc_nonzeros(idx, len(idx), mat, len(mat), r.ctypes.data, c.ctypes.data, n)
    return r, c


def header(idx):
    h = np.frombuffer(idx[:64], dtype=np.uint8)
    nrows = int(np.frombuffer(idx[24:32], dtype=np.uint64)[0])
    ncols = int(np.frombuffer(idx[32:40], dtype=np.uint64)[0])
    esize = int(np.frombuffer(idx[16:24], dtype=np.uint64)[0])
    prim = int(np.frombuffer(idx[44:48], dtype=np.int32)[0])
    bh = int(np.frombuffer(idx[48:56], dtype=np.uint64)[0])
    bw = int(np.frombuffer(idx[56:64], dtype=np.uint64)[0])
    del h
    return dict(nrows=nrows, ncols=ncols, entry_size=esize, prim=prim, block_h=bh, block_w=bw)


def spmm(idx, mat, X, nthreads=1, hilbert=False, cpu_cache_size=0, copy_task=True, brows=None, out=None):
    """Oracle SpMM Y = A X (X: 2-D numpy array, ncols x k, row-major).

    `out`, when given, is the C-contiguous nrows x k result array of X's
    dtype (rows outside `brows` are left as they are)."""
    X = np.ascontiguousarray(X)
    if X.ndim == 1:
        X = X[:, None]
    d = _D_OF[X.dtype]
    h = header(idx)
    if out is not None:
        if out.shape != (h["nrows"], X.shape[1]) or out.dtype != X.dtype or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous nrows x k array of X's dtype")
        Y = out
    else:
        Y = np.zeros((h["nrows"], X.shape[1]), dtype=X.dtype)
    b0, b1 = (0, 0) if brows is None else brows
    rc = orc().orc_spmm(idx, len(idx), mat, len(mat), d, X.ctypes.data, Y.ctypes.data, X.shape[1],
                        nthreads, int(hilbert), cpu_cache_size, int(copy_task), b0, b1)
    if rc:
        raise ValueError("oracle SpMM failed")
    return Y


def ref_spmm(idx, mat, X, dense_double_sparse_float=False):
    """SpMM through the reference's own tile iterators (None if not built)."""
    L = ref()
    if L is None:
        return None
    X = np.ascontiguousarray(X)
    if X.ndim == 1:
        X = X[:, None]
    d = 5 if dense_double_sparse_float else _D_OF[X.dtype]
    h = header(idx)
    Y = np.zeros((h["nrows"], X.shape[1]), dtype=X.dtype)
    if L.ref_spmm(idx, mat, d, X.ctypes.data, Y.ctypes.data, X.shape[1]):
        raise ValueError("reference walk failed")
    return Y


def ref_nonzeros(idx, mat):
    L = ref()
    if L is None:
        return None
    n = L.ref_nonzeros(idx, mat, None, None, 0)
    r = np.empty(n, dtype=np.uint64)
    c = np.empty(n, dtype=np.uint64)
    L.ref_nonzeros(idx, mat, r.ctypes.data, c.ctypes.data, n)
    return r, c


def verify(idx, mat):
    return orc().orc_verify(idx, len(idx), mat, len(mat))


def pagerank(idx, mat, t_idx, t_mat, max_iters=30, damping=0.85, nthreads=1):
    n = header(idx)["nrows"]
    pr = np.empty(n, dtype=np.float32)
    it = C.c_uint64()
    rc = orc().orc_pagerank(idx, len(idx), mat, len(mat), t_idx, len(t_idx), t_mat, len(t_mat), max_iters,
                            damping, nthreads, pr.ctypes.data, C.byref(it))
    if rc:
        raise ValueError("oracle PageRank failed")
    return pr, it.value


def rmat_edges(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1, permute=True, nedges=None, nthreads=0):
    """The benchmark's R-MAT edge stream (uint32 src, dst), generated on the
    CPU without the GPU library: the same edges as
    flashx_b200.graphs.rmat_edges for the same arguments."""
    m = int(nedges if nedges is not None else edge_factor * (1 << scale))
    src = np.empty(m, dtype=np.uint32)
    dst = np.empty(m, dtype=np.uint32)
    if orc().orc_rmat_edges(scale, m, a, b, c, seed, int(permute), src.ctypes.data, dst.ctypes.data, nthreads):
        raise ValueError("oracle R-MAT: bad arguments")
    return src, dst


def num_block_rows(idx):
    return orc().orc_num_block_rows(idx, len(idx))


def block_rows_nnz(idx, mat, b0, b1):
    return orc().orc_block_rows_nnz(idx, len(idx), mat, len(mat), b0, b1)


def now():
    return orc().orc_now()


# ---- the FlashGraph 1D format ------------------------------------------------

def fg_build(src, dst, vals=None, num_vertices=0, directed=True):
    """FlashGraph adjacency image (bytes) of an edge list: neighbor lists
    sorted by id, duplicates and self-loops kept; vals (one per edge, any
    fixed-size dtype) become the edge data.  For an undirected graph list
    both directions of every edge."""
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    if not num_vertices:
        num_vertices = int(max(src.max(initial=0), dst.max(initial=0))) + 1 if len(src) else 0
    eds, vp = 0, None
    if vals is not None:
        vals = np.ascontiguousarray(vals)
        eds, vp = vals.dtype.itemsize, vals.ctypes.data
    out, n = C.c_void_p(), C.c_uint64()
    if orc().orc_fg_build(src.ctypes.data, dst.ctypes.data, vp, eds, len(src), num_vertices, int(directed),
                          C.byref(out), C.byref(n)):
        raise ValueError("oracle fg_build failed")
    b = C.string_at(out, n.value)
    orc().orc_free(out)
    return b


def fg_spmm(adj, X, transpose=False, edge_prim=P_BOOL):
    """fg_row_spmm_task over an adjacency image: Y = A X (A^T X)."""
    X = np.ascontiguousarray(X)
    X2 = X.reshape(X.shape[0], -1)
    Y = np.empty_like(X2)
    if orc().orc_fg_spmm(adj, len(adj), int(transpose), edge_prim, _D_OF[X.dtype], X2.ctypes.data, Y.ctypes.data,
                         X2.shape[1]):
        raise ValueError("oracle fg_spmm failed")
    return Y.reshape(X.shape)


def fg_vsize(ne, eds):
    return orc().orc_fg_vsize(ne, eds)


def fg_data_off(ne, eds):
    return orc().orc_fg_data_off(ne, eds)


_reffg = None


def reffg():
    """The walker built from FlashGraph's own headers, or None."""
    global _reffg
    if _reffg is None:
        if not os.path.exists(REFFG_SO):
            return None
        L = C.CDLL(REFFG_SO)
        u64 = C.c_uint64
        L.ref_fg_header_size.restype = u64
        L.ref_fg_vsize.restype = u64
        L.ref_fg_vsize.argtypes = [C.c_uint32, C.c_uint32]
        L.ref_fg_data_off.restype = u64
        L.ref_fg_data_off.argtypes = [C.c_uint32, C.c_uint32]
        L.ref_fg_header.restype = C.c_int
        L.ref_fg_header.argtypes = [C.c_void_p, C.POINTER(u64), C.POINTER(u64), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.ref_fg_spmm.restype = C.c_int
        L.ref_fg_spmm.argtypes = [C.c_void_p, u64, C.c_int, C.c_int, C.c_void_p, C.c_void_p, u64]
        _reffg = L
    return _reffg


def ref_fg_spmm(adj, X, transpose=False):
    """The same product through FlashGraph's own record classes (float edge
    data, FP32 or FP64 operands)."""
    X = np.ascontiguousarray(X)
    Y = np.empty_like(X)
    if reffg().ref_fg_spmm(adj, len(adj), int(transpose), 0 if X.dtype == np.float32 else 1, X.ctypes.data,
                           Y.ctypes.data, X.shape[1]):
        raise ValueError("reference FlashGraph walker failed")
    return Y
