"""Algorithms on the GPU SpMM: the mirror of fm::alg (matrix/libmatrix-algs)."""
import ctypes as C

from ._lib import check, lib


def PageRank(mat, max_niters=30, damping_factor=0.85, stream=None):
    """fm::alg::PageRank(mat, max_niters, damping_factor, num_in_mem)
    (matrix/libmatrix-algs/PageRank.cpp:63-133): returns (pr, iterations), pr
    an n-element float32 CUDA tensor.  `mat` needs its transpose (built by
    create_2d_matrix(..., is_sym=False) for a directed graph)."""
    import torch
    pr = torch.empty(mat.get_num_rows(), dtype=torch.float32, device=f"cuda:{mat.device}")
    it = C.c_uint64()
    st = stream if stream is not None else torch.cuda.current_stream(pr.device).cuda_stream
    check(lib.fmx_pagerank(mat.handle, int(max_niters), float(damping_factor), pr.data_ptr(), C.byref(it), st))
    return pr, it.value
