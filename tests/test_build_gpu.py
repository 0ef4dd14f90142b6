"""The GPU builder (fmx_matrix_build_device): an edge list on the device
sorted, deduplicated and scheduled without a host image, against the host
builder's image of the same edges (matrix_image.build, the restated
fm::create_2d_matrix): same non-zeros, same schedule, bit-identical SpMMs on
both orientations."""
import numpy as np
import pytest

from flashx_b200 import FmxError, _lib, matrix_image, sparse_matrix
from flashx_b200.graphs import rmat_edges, rmat_edges_device

pytestmark = pytest.mark.gpu


def _pair(torch, src, dst, vals, n, dedup, keep_self, block=(1024, 1024)):
    host = sparse_matrix.create(
        matrix_image.build(src, dst, vals, nrows=n, ncols=n, block_size=block, dedup=dedup, remove_self=not keep_self),
        matrix_image.build(dst, src, vals, nrows=n, ncols=n, block_size=block, dedup=dedup,
                                 remove_self=not keep_self))
    assert not host.is_symmetric()
    tv = None if vals is None else torch.from_numpy(vals).cuda()
    dev = sparse_matrix.from_device_edges(torch.from_numpy(src.astype(np.int32)).cuda(),
                                          torch.from_numpy(dst.astype(np.int32)).cuda(), tv, nrows=n, ncols=n,
                                          dedup=dedup, remove_self=not keep_self, transpose=True)
    return host, dev


def _same_products(torch, a, b, k, dtype):
    g = torch.Generator(device="cuda").manual_seed(k)
    X = torch.randn((a.get_num_cols(), k), generator=g, device="cuda").to(dtype)
    ya, yb = a.multiply(X), b.multiply(X)
    assert torch.equal(ya, yb)
    at, bt = a.transpose(), b.transpose()
    assert torch.equal(at.multiply(X), bt.multiply(X))


@pytest.mark.parametrize("dedup,keep_self,weighted", [(True, False, False), (False, False, True),
                                                      (True, True, True), (False, True, False)])
def test_device_build_matches_host_build(torch_cuda, dedup, keep_self, weighted):
    torch = torch_cuda
    rng = np.random.default_rng(3)
    n, m = 20000, 200000
    src = rng.integers(0, n, m).astype(np.uint32)
    dst = rng.integers(0, n, m).astype(np.uint32)
    src[:5000] = dst[:5000]                      # self-loops
    src[5000:9000], dst[5000:9000] = src[9000:13000], dst[9000:13000]    # duplicates
    src = np.concatenate([src, np.full(3000, 7, np.uint32)])            # a long row
    dst = np.concatenate([dst, rng.integers(0, n, 3000).astype(np.uint32)])
    vals = rng.uniform(-1, 1, len(src)).astype(np.float32) if weighted else None
    host, dev = _pair(torch, src, dst, vals, n, dedup, keep_self)
    assert host.get_nnz() == dev.get_nnz()
    assert host.schedule() == dev.schedule()
    # the GPU scheduler lays out both orientations byte for byte as the host one
    assert host.layout_digest() == dev.layout_digest()
    assert host.layout_digest(transpose=True) == dev.layout_digest(transpose=True)
    for k in (1, 16, 33):
        _same_products(torch, host, dev, k, torch.float32)


def test_device_schedule_edge_rows(torch_cuda):
    """Rows at the scheduler's boundaries: exactly 256 entries (summed whole),
    257 (two chunks), 9 chunks (a warp each in the fixup), more than 64
    chunks (a block each), empty rows first and last, FP64 values."""
    torch = torch_cuda
    rng = np.random.default_rng(11)
    n = 50000
    parts_s, parts_d = [], []
    for row, deg in ((5, 20000), (6, 257), (7, 256), (8, 2100), (9, 1)):
        parts_s.append(np.full(deg, row, np.uint32))
        parts_d.append(rng.choice(np.arange(10, n - 10, dtype=np.uint32), deg, replace=False))
    m = 300000
    parts_s.append(rng.integers(10, n - 10, m).astype(np.uint32))
    parts_d.append(rng.integers(0, n, m).astype(np.uint32))
    src, dst = np.concatenate(parts_s), np.concatenate(parts_d)
    vals = rng.uniform(-1, 1, len(src))
    host, dev = _pair(torch, src, dst, vals, n, True, False, block=(4096, 4096))
    assert host.schedule() == dev.schedule() and host.hot() == dev.hot()
    assert host.layout_digest() == dev.layout_digest()
    assert host.layout_digest(transpose=True) == dev.layout_digest(transpose=True)
    for k in (1, 16):
        _same_products(torch, host, dev, k, torch.float64)


def test_device_rmat_matches_host_rmat(torch_cuda):
    """R-MAT scale 20 generated on the device and built there, against the
    host generator's identical stream built on the host."""
    torch = torch_cuda
    n = 1 << 20
    s, d = rmat_edges(20, seed=1)
    host = sparse_matrix.create(matrix_image.build(s, d, None, nrows=n, ncols=n, block_size=(16384, 16384),
                                                   dedup=True), None)
    ds, dd = rmat_edges_device(20, seed=1)
    assert np.array_equal(ds.cpu().numpy().view(np.uint32), s)
    dev = sparse_matrix.from_device_edges(ds, dd, nrows=n, ncols=n, dedup=True)
    assert host.get_nnz() == dev.get_nnz() and host.hot() == dev.hot()
    assert host.schedule() == dev.schedule()
    assert host.layout_digest() == dev.layout_digest()
    for dt in (torch.float32, torch.bfloat16):
        X = torch.randn((n, 16), device="cuda").to(dt)
        Y1 = torch.empty((n, 16), device="cuda")
        Y2 = torch.empty((n, 16), device="cuda")
        assert host.multiply(X, Y1) and dev.multiply(X, Y2)
        assert torch.equal(Y1, Y2)


def test_device_build_errors(torch_cuda):
    torch = torch_cuda
    s = torch.tensor([0, 1, 5], dtype=torch.int32, device="cuda")
    d = torch.tensor([1, 0, 2], dtype=torch.int32, device="cuda")
    with pytest.raises(FmxError) as e:
        sparse_matrix.from_device_edges(s, d, nrows=4, ncols=4)
    assert e.value.code == _lib.FMX_ERR_INVAL
    m = sparse_matrix.from_device_edges(s, d)                 # both dimensions from the largest id
    assert (m.get_num_rows(), m.get_num_cols()) == (6, 6)
    empty = torch.zeros(0, dtype=torch.int32, device="cuda")
    m0 = sparse_matrix.from_device_edges(empty, empty, nrows=8, ncols=8)
    assert m0.get_nnz() == 0
    assert not m0.multiply(torch.ones((8, 4), device="cuda")).any()
