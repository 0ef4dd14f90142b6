"""flashx_b200: FlashMatrix's 2D-tiled sparse-times-dense multiply on B200.

The compute runs in libfmx.so (hand-written CUDA for sm_100a behind the C ABI
in include/fmx.h).  This package is the host-side mirror of the reference's
interface plus the workloads built on the SpMM.
"""
from ._lib import FmxError, lib  # noqa: F401  (raises if libfmx.so is missing)
from .sparse_matrix import (  # noqa: F401
    SpM_2d_index, SpM_2d_storage, create_2d_matrix, matrix_image, set_deduplicate,
    set_remove_self_edge, sparse_matrix)



def release_cached(device=0):
    """Hand the solvers' reserved device workspace back to the driver
    (fmx_release_cached; as torch.cuda.empty_cache does for torch's cache)."""
    from ._lib import check
    check(lib.fmx_release_cached(int(device)))


__all__ = ["FmxError", "SpM_2d_index", "SpM_2d_storage", "create_2d_matrix", "matrix_image",
           "release_cached", "set_deduplicate", "set_remove_self_edge", "sparse_matrix"]
