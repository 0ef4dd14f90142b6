"""Seeded synthetic graphs: R-MAT and stochastic block models.

R-MAT follows the quadrant recursion of Chakrabarti et al. with the
probabilities FlashX's generator uses (flash-graph/tools/rmat-gen.cpp:43-44:
a,b,c,d = 0.57/0.19/0.19/0.05, vertex labels permuted).  The edge stream is
counter-based (edge i depends only on (seed, i)), so libfmx's host and device
generators produce the same edges.

The SBM follows flash-graph/utils/sbm.cpp's model (equal blocks, in-block
probability p_in, between-block p_out, vertex ids randomly permuted,
sbm.cpp:87-115,199-202) with this library's own sampler: each undirected edge
picks "inside a block" with probability r/(r + B - 1) for r = p_in/p_out and
then two endpoints uniformly inside that block (or in two distinct blocks).
"""
import numpy as np

from . import _lib
from ._lib import lib, check

RMAT_ABC = (0.57, 0.19, 0.19)


def rmat_edges(scale, edge_factor=16, a=RMAT_ABC[0], b=RMAT_ABC[1], c=RMAT_ABC[2], seed=1,
               permute=True, nedges=None, nthreads=0):
    """Host R-MAT edge list (uint32 src, dst) of 2^scale vertices."""
    m = int(nedges if nedges is not None else edge_factor * (1 << scale))
    src = np.empty(m, dtype=np.uint32)
    dst = np.empty(m, dtype=np.uint32)
    check(lib.fmx_rmat_edges_host(scale, m, a, b, c, seed, int(permute), src.ctypes.data, dst.ctypes.data,
                                  nthreads))
    return src, dst


def rmat_edges_device(scale, edge_factor=16, a=RMAT_ABC[0], b=RMAT_ABC[1], c=RMAT_ABC[2], seed=1,
                      permute=True, nedges=None, device=0):
    """Device R-MAT edge list as two int32 torch tensors (same stream as the host one)."""
    import torch
    m = int(nedges if nedges is not None else edge_factor * (1 << scale))
    src = torch.empty(m, dtype=torch.int32, device=f"cuda:{device}")
    dst = torch.empty(m, dtype=torch.int32, device=f"cuda:{device}")
    st = torch.cuda.current_stream(src.device).cuda_stream
    check(lib.fmx_rmat_edges_device(scale, m, a, b, c, seed, int(permute), src.data_ptr(), dst.data_ptr(), st))
    return src, dst


def symmetrize(src, dst):
    """Both directions of every edge (the caller dedups through the builder)."""
    return np.concatenate([src, dst]), np.concatenate([dst, src])


def sbm_edges(n, nblocks, avg_degree, ratio, seed):
    """Undirected SBM as a symmetric directed edge list plus block labels.

    Returns (src, dst, labels) with labels[v] the block of vertex v (after
    the random relabelling)."""
    rng = np.random.default_rng(seed)
    bsize = n // nblocks
    n = bsize * nblocks
    m = int(round(n * avg_degree / 2))
    p_in = ratio / (ratio + nblocks - 1)
    inside = rng.random(m) < p_in
    b1 = rng.integers(0, nblocks, m)
    shift = rng.integers(1, nblocks, m) if nblocks > 1 else np.zeros(m, dtype=np.int64)
    b2 = np.where(inside, b1, (b1 + shift) % nblocks)
    u = b1 * bsize + rng.integers(0, bsize, m)
    v = b2 * bsize + rng.integers(0, bsize, m)
    perm = rng.permutation(n).astype(np.uint32)
    u = perm[u]
    v = perm[v]
    labels = np.empty(n, dtype=np.int32)
    labels[perm] = np.repeat(np.arange(nblocks, dtype=np.int32), bsize)
    s, d = symmetrize(u.astype(np.uint32), v.astype(np.uint32))
    return s, d, labels
