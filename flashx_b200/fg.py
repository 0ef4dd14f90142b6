"""The FlashGraph 1D format (flash-graph/fg_sparse_matrix.cpp).

  g = FG_graph.create("graph.adj")               # or FG_graph.from_bytes(b)
  m = create_sparse_matrix(g, entry_type=None)   # fg::create_sparse_matrix
  m.multiply(X, Y)

create_sparse_matrix(fg, entry_type) (fg_sparse_matrix.cpp:577-590) makes a
matrix whose row i is vertex i's out-edge list (its in-edge list in the
transpose; an undirected graph is symmetric), summed in record order as
fg_row_spmm_task::run_on_row does (:83-106).  entry_type: None for a graph
without edge data, else "float", "double", "int" or "long", whose size must
equal the graph's edge data size.  The vertex index file that
FG_graph::create also takes is not needed: the adjacency records are read
in order.
"""
import ctypes as C
import os

from . import _lib
from ._lib import check, lib
from .sparse_matrix import sparse_matrix

_PRIM = {None: _lib.P_BOOL, "bool": _lib.P_BOOL, "float": _lib.P_FLOAT, "double": _lib.P_DOUBLE,
         "int": _lib.P_INTEGER, "long": _lib.P_LONG}


class FG_graph:
    """A FlashGraph graph image: the adjacency file's bytes or its path."""

    def __init__(self, path=None, data=None):
        self.path, self.data = path, data

    @classmethod
    def create(cls, graph_file, index_file=None):
        if not os.path.exists(graph_file):
            raise FileNotFoundError(graph_file)
        return cls(path=graph_file)

    @classmethod
    def from_bytes(cls, data):
        return cls(data=bytes(data))


def create_sparse_matrix(fg, entry_type=None, device=0):
    prim = _PRIM.get(entry_type)
    if prim is None:
        raise ValueError(f"unsupported entry type {entry_type!r}")
    h = C.c_void_p()
    if fg.data is not None:
        check(lib.fmx_matrix_from_fg(fg.data, len(fg.data), prim, device, C.byref(h)))
    else:
        check(lib.fmx_matrix_load_fg(fg.path.encode(), prim, device, C.byref(h)))
    return sparse_matrix(h.value, device)
