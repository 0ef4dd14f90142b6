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


def main(argv=None):
    """PageRank on a seeded R-MAT graph (edge factor 16, deduplicated,
    directed, as the reference's PageRank driver takes a directed graph):
    python -m flashx_b200.algs --scale 16 --iters 30 --damping 0.85 --reps 3
    prints one JSON line with the iterations and the time per iteration."""
    import argparse
    import json
    import time

    import torch

    from .graphs import rmat_edges
    from .sparse_matrix import create_2d_matrix, set_deduplicate
    p = argparse.ArgumentParser(description=main.__doc__)
    p.add_argument("--scale", type=int, default=16)
    p.add_argument("--iters", type=int, default=30)
    p.add_argument("--damping", type=float, default=0.85)
    p.add_argument("--reps", type=int, default=3)
    p.add_argument("--seed", type=int, default=1)
    a = p.parse_args(argv)
    n = 1 << a.scale
    s, d = rmat_edges(a.scale, seed=a.seed)
    set_deduplicate(True)
    try:
        m = create_2d_matrix(s, d, None, block_size=(16384, 16384), is_sym=False, nrows=n, ncols=n)
    finally:
        set_deduplicate(False)
    times, it = [], 0
    for _ in range(max(1, a.reps)):
        torch.cuda.synchronize()
        t = time.perf_counter()
        _, it = PageRank(m, a.iters, a.damping)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t)
    best = min(times)
    print(json.dumps({"scale": a.scale, "n": n, "nnz": int(m.get_nnz()), "iters": int(it),
                      "ms_per_iter": round(best * 1e3 / max(it, 1), 4)}), flush=True)


if __name__ == "__main__":
    main()
