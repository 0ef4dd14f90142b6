"""GPU parity: libfmx's CUDA SpMM against the CPU oracle on the same image.

Bar: bit-exact for integer types and for every row summed by one lane group
(rows of <= EXACT_ROW_MAX = 256 entries are summed in the reference's ascending-column order
with separate multiply and add roundings); bit-exact for split rows when the
inputs are integer-valued (all partial sums exact); otherwise within
RTOL = 1e-5 relative (FP32) of the oracle.
"""
import numpy as np
import pytest

import oracle
from flashx_b200 import _lib, matrix_image, sparse_matrix, create_2d_matrix
from flashx_b200.graphs import rmat_edges

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def _graph(n, m, seed, heavy=()):
    rng = np.random.default_rng(seed)
    src = rng.integers(0, n, m).astype(np.uint32)
    dst = rng.integers(0, n, m).astype(np.uint32)
    extra_s, extra_d = [], []
    for row, deg in heavy:
        assert deg <= n, "a row cannot hold more distinct columns than the matrix has"
        extra_s.append(np.full(deg, row, dtype=np.uint32))
        extra_d.append(rng.choice(n, deg, replace=False).astype(np.uint32))
    if heavy:
        src = np.concatenate([src] + extra_s)
        dst = np.concatenate([dst] + extra_d)
    return src, dst


def _dense(rng, shape, dt, integer=False):
    if dt in (np.int32, np.int64) or integer:
        return rng.integers(-8, 9, shape).astype(dt)
    return rng.standard_normal(shape).astype(dt)


def _to_torch(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _gpu_spmm(torch, m, X, out_dtype=None, s_in=None, s_out=None):
    x = _to_torch(torch, X)
    y = torch.empty((m.get_num_rows(), X.shape[1]), dtype=out_dtype or x.dtype, device="cuda")
    y.fill_(float("nan") if y.dtype.is_floating_point else -7)
    si = _to_torch(torch, s_in) if s_in is not None else None
    so = _to_torch(torch, s_out) if s_out is not None else None
    assert m.multiply(x, y, si, so), _lib.last_error()
    torch.cuda.synchronize()
    return y.float().cpu().numpy() if y.dtype == torch.bfloat16 else y.cpu().numpy()


CASES = [
    # n, m, block, weighted dtype, dedup, heavy rows (row, degree)
    (1000, 6000, (64, 128), None, False, ()),
    (5000, 60000, (1024, 1024), np.float32, True, ()),
    (20000, 100000, (16384, 16384), None, True, ((7, 20000), (11, 900), (13, 600))),
    (20000, 100000, (4096, 2048), np.float32, False, ((3, 17000), (5, 5000))),
    (3000, 20000, (256, 256), np.float64, True, ((1, 2999),)),
]


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("k", [1, 2, 3, 4, 8, 10, 16, 32, 64, 130])
def test_parity_float(torch_cuda, case, k):
    torch = torch_cuda
    n, mm, block, wdt, dedup, heavy = CASES[case]
    src, dst = _graph(n, mm, 100 + case, heavy)
    rng = np.random.default_rng(case * 1000 + k)
    vals = None if wdt is None else rng.uniform(0.0, 1.0, len(src)).astype(wdt)
    idx, mat = oracle.build_image(src, dst, vals, block=block, dedup=dedup)
    img = matrix_image.from_bytes(idx, mat)
    m = sparse_matrix.create(img, None, device=0)
    dt = np.float64 if wdt is np.float64 else np.float32
    has_split = any(d > _lib.EXACT_ROW_MAX for _, d in heavy)
    for integer in (True, False):
        X = _dense(rng, (n, k), dt, integer)
        Y = _gpu_spmm(torch, m, X)
        R = oracle.spmm(idx, mat, X, nthreads=4)
        if not has_split or (integer and wdt is None):
            bad = np.argwhere(Y.view(np.uint32 if Y.dtype == np.float32 else np.uint64)
                              != R.view(np.uint32 if R.dtype == np.float32 else np.uint64))
            assert len(bad) == 0, (
                f"not bit-exact at {len(bad)} elements (first {bad[:5].tolist()}): "
                f"max diff {np.max(np.abs(Y - R))}")
        else:
            np.testing.assert_allclose(Y, R, rtol=RTOL, atol=RTOL * np.abs(R).max())


@pytest.mark.parametrize("dt", [np.int32, np.int64])
@pytest.mark.parametrize("k", [1, 4, 5, 16])
def test_parity_integer(torch_cuda, dt, k):
    torch = torch_cuda
    src, dst = _graph(30000, 150000, 7, ((2, 20000), (9, 3000)))
    rng = np.random.default_rng(k)
    vals = rng.integers(-3, 4, len(src)).astype(np.int32 if dt is np.int32 else np.int64)
    for w in (None, vals):
        idx, mat = oracle.build_image(src, dst, w, block=(2048, 2048), dedup=True)
        m = sparse_matrix.create(matrix_image.from_bytes(idx, mat), None)
        X = rng.integers(-1000, 1000, (30000, k)).astype(dt)
        assert np.array_equal(_gpu_spmm(torch, m, X), oracle.spmm(idx, mat, X))


def test_rand_mat_gen_known_answer(torch_cuda):
    """matrix/test/rand_mat_gen.cpp:178-199: a binary matrix times
    [0, 1, ..., ncol-1] equals each row's sum of column ids (duplicates kept)."""
    torch = torch_cuda
    rng = np.random.default_rng(11)
    nrow, ncol = 30000, 20000
    deg = rng.integers(0, 60, nrow)
    src = np.repeat(np.arange(nrow, dtype=np.uint32), deg)
    dst = rng.integers(0, ncol, len(src)).astype(np.uint32)
    m = create_2d_matrix(src, dst, None, block_size=(4096, 4096), nrows=nrow, ncols=ncol)
    X = np.arange(ncol, dtype=np.int64)[:, None]
    Y = _gpu_spmm(torch, m, X)[:, 0]
    keep = src != dst
    expect = np.bincount(src[keep], weights=dst[keep].astype(np.float64), minlength=nrow).astype(np.int64)
    assert np.array_equal(Y, expect)


def test_bf16_input(torch_cuda):
    torch = torch_cuda
    src, dst = _graph(8000, 80000, 3)
    idx, mat = oracle.build_image(src, dst, None, block=(4096, 4096), dedup=True)
    m = sparse_matrix.create(matrix_image.from_bytes(idx, mat), None)
    rng = np.random.default_rng(5)
    for k in (8, 16, 32, 6):
        Xf = rng.standard_normal((8000, k)).astype(np.float32)
        xb = torch.from_numpy(Xf).to(torch.bfloat16).cuda()
        Xr = xb.float().cpu().numpy()          # the bf16-rounded operand
        y = torch.empty((8000, k), dtype=torch.float32, device="cuda")
        assert m.multiply(xb, y)
        R = oracle.spmm(idx, mat, Xr)
        assert np.array_equal(y.cpu().numpy(), R)
        yb = torch.empty((8000, k), dtype=torch.bfloat16, device="cuda")
        assert m.multiply(xb, yb)
        assert torch.equal(yb.cpu(), torch.from_numpy(R).to(torch.bfloat16))


def test_row_scales(torch_cuda):
    """y = D_out A D_in x, the normalised-adjacency operator of
    matrix/test/test-eigen.cpp:88-136 (scale_rows, SpMM, scale_rows)."""
    torch = torch_cuda
    n = 30000
    src, dst = _graph(n, 200000, 9, ((4, 18000), (8, 2000)))
    idx, mat = oracle.build_image(src, dst, None, block=(8192, 8192), dedup=True)
    m = sparse_matrix.create(matrix_image.from_bytes(idx, mat), None)
    rng = np.random.default_rng(2)
    for dt in (np.float32, np.float64):
        X = rng.standard_normal((n, 16)).astype(dt)
        s_in = rng.uniform(0.1, 2.0, n).astype(dt)
        s_out = rng.uniform(0.1, 2.0, n).astype(dt)
        Y = _gpu_spmm(torch, m, X, s_in=s_in, s_out=s_out)
        R = oracle.spmm(idx, mat, (X * s_in[:, None]).astype(dt)) * s_out[:, None]
        np.testing.assert_allclose(Y, R, rtol=RTOL if dt == np.float32 else 1e-12,
                                   atol=(RTOL if dt == np.float32 else 1e-12) * np.abs(R).max())
    # BF16 in and out with both scales (the eigensolver's correction SpMMs):
    # FP32 accumulation of the BF16-rounded operand, one BF16 rounding at the end
    s_in = rng.uniform(0.1, 2.0, n).astype(np.float32)
    s_out = rng.uniform(0.1, 2.0, n).astype(np.float32)
    for k in (16, 32, 8):
        xb = torch.from_numpy(rng.standard_normal((n, k)).astype(np.float32)).to(torch.bfloat16).cuda()
        yb = torch.empty((n, k), dtype=torch.bfloat16, device="cuda")
        assert m.multiply(xb, yb, torch.from_numpy(s_in).cuda(), torch.from_numpy(s_out).cuda())
        Xr = xb.float().cpu().numpy()
        R = (oracle.spmm(idx, mat, (Xr * s_in[:, None]).astype(np.float32)) * s_out[:, None]).astype(np.float32)
        got = yb.float().cpu().numpy()
        np.testing.assert_allclose(got, R, rtol=1e-2, atol=1e-2 * np.abs(R).max())


def test_asymmetric_transpose(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(4)
    src = rng.integers(0, 4000, 30000).astype(np.uint32)
    dst = rng.integers(0, 4000, 30000).astype(np.uint32)
    m, img, timg = create_2d_matrix(src, dst, None, block_size=(1024, 1024), is_sym=False, return_images=True)
    assert not m.is_symmetric()
    X = rng.integers(-8, 9, (m.get_num_cols(), 8)).astype(np.float32)
    t = m.transpose()
    i, a = img.bytes()
    ti, ta = timg.bytes()
    assert np.array_equal(_gpu_spmm(torch, m, X), oracle.spmm(i, a, X))
    assert np.array_equal(_gpu_spmm(torch, t, X), oracle.spmm(ti, ta, X))


def test_rmat_s18_parity(torch_cuda):
    torch = torch_cuda
    src, dst = rmat_edges(18, seed=1)
    rng = np.random.default_rng(0)
    for weighted in (False, True):
        vals = rng.uniform(0.0, 1.0, len(src)).astype(np.float32) if weighted else None
        vals = None if vals is None else np.where(vals == 0, np.float32(1.0), vals)
        img = matrix_image.build(src, dst, vals, nrows=1 << 18, ncols=1 << 18, block_size=(16384, 16384),
                                 dedup=True)
        idx, mat = img.bytes()
        m = sparse_matrix.create(img, None)
        rows, _ = oracle.nonzeros(idx, mat)
        light = np.bincount(rows.astype(np.int64), minlength=1 << 18) <= _lib.EXACT_ROW_MAX
        assert not light.all()     # the hubs exercise the split paths
        for k in (1, 4, 16, 32):
            Xi = rng.integers(-8, 9, (1 << 18, k)).astype(np.float32)
            Y, R = _gpu_spmm(torch, m, Xi), oracle.spmm(idx, mat, Xi, nthreads=8)
            if weighted:   # split rows re-associate non-integer products
                assert np.array_equal(Y[light], R[light])
                np.testing.assert_allclose(Y, R, rtol=RTOL, atol=RTOL * np.abs(R).max())
            else:
                assert np.array_equal(Y, R)
            Xf = rng.standard_normal((1 << 18, k)).astype(np.float32)
            Y, R = _gpu_spmm(torch, m, Xf), oracle.spmm(idx, mat, Xf, nthreads=8)
            assert np.array_equal(Y[light], R[light])
            np.testing.assert_allclose(Y, R, rtol=RTOL, atol=RTOL * np.abs(R).max())


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_spmv_kernel_matches_lane_group_kernel(torch_cuda, dtype):
    """k = 1 without row scales runs the warp-per-range SpMV kernel; with row
    scales of exactly 1 (x * 1 and y * 1 are exact) it runs the lane-group
    kernel.  Rows of up to EXACT_ROW_MAX entries have the same arithmetic in
    both and must agree bit for bit; hub rows (chunks added up in another
    association) within RTOL."""
    torch = torch_cuda
    tdt = getattr(torch, dtype)
    n = 1 << 17
    src, dst = rmat_edges(17, seed=4)
    rng = np.random.default_rng(1)
    ones = torch.ones(n, device="cuda", dtype=tdt)
    for weighted in (False, True):
        vals = rng.uniform(0.0, 1.0, len(src)).astype(np.float32) if weighted else None
        m = sparse_matrix.create(matrix_image.build(src, dst, vals, nrows=n, ncols=n, block_size=(16384, 16384),
                                                    dedup=True), None)
        assert m.schedule()[2] > 0
        light = torch.from_numpy(np.bincount(src[src != dst].astype(np.int64), minlength=n) <= _lib.EXACT_ROW_MAX)
        X = torch.randn((n, 1), device="cuda", dtype=tdt)
        Y1 = m.multiply(X)
        Ys = torch.empty_like(Y1)
        assert m.multiply(X, Ys, row_scale_in=ones, row_scale_out=ones)
        y1, ys = Y1.cpu()[:, 0], Ys.cpu()[:, 0]
        assert torch.equal(y1[light], ys[light]) and not bool(light.all())
        torch.testing.assert_close(y1, ys, rtol=RTOL, atol=RTOL * float(ys.abs().max()))
        # a strided single column (ldx = ldy = 3)
        X3 = torch.zeros((n, 3), device="cuda", dtype=tdt)
        X3[:, :1] = X
        Y3 = torch.full((n, 3), 7.0, device="cuda", dtype=tdt)
        assert m.multiply(X3[:, :1], Y3[:, :1])
        assert torch.equal(Y3[:, :1], Y1) and bool((Y3[:, 1:] == 7).all())


def test_host_buffers_e2e(torch_cuda):
    src, dst = _graph(5000, 40000, 21)
    idx, mat = oracle.build_image(src, dst, None, block=(1024, 1024), dedup=True)
    m = sparse_matrix.create(matrix_image.from_bytes(idx, mat), None)
    X = np.random.default_rng(1).integers(-8, 9, (5000, 16)).astype(np.float32)
    assert np.array_equal(m.multiply_host(X), oracle.spmm(idx, mat, X))


def test_host_buffers_async_two_streams(torch_cuda):
    """fmx_spmm_host_async: six calls in flight on two streams, each with its
    own pinned X and Y, through the matrix's two staging slots; every Y equals
    the oracle's (integer-valued X, so exact), and so does a later call on a
    third stream."""
    torch = torch_cuda
    src, dst = _graph(20000, 100000, 23, ((7, 15000), (11, 900)))
    idx, mat = oracle.build_image(src, dst, None, block=(4096, 4096), dedup=True)
    m = sparse_matrix.create(matrix_image.from_bytes(idx, mat), None)
    rng = np.random.default_rng(5)
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    xs, ys, want = [], [], []
    for i in range(6):
        x = torch.from_numpy(rng.integers(-8, 9, (20000, 16)).astype(np.float32)).pin_memory()
        y = torch.full((20000, 16), float("nan")).pin_memory()
        xs.append(x)
        ys.append(y)
        want.append(oracle.spmm(idx, mat, x.numpy()))
    for i in range(6):
        m.multiply_host_async(xs[i].numpy(), ys[i].numpy(), streams[i % 2].cuda_stream)
    for s in streams:
        s.synchronize()
    for i in range(6):
        assert np.array_equal(ys[i].numpy(), want[i]), i
    del streams
    s3 = torch.cuda.Stream()
    y3 = torch.full((20000, 16), float("nan")).pin_memory()
    m.multiply_host_async(xs[0].numpy(), y3.numpy(), s3.cuda_stream)
    s3.synchronize()
    assert np.array_equal(y3.numpy(), want[0])


def test_multiply_errors(torch_cuda):
    """Dimension and type mismatches return False, like the reference."""
    torch = torch_cuda
    src, dst = _graph(1000, 5000, 1)
    m = create_2d_matrix(src, dst, None, block_size=(256, 256), nrows=1000, ncols=1000)
    x = torch.zeros((999, 4), device="cuda")
    y = torch.zeros((1000, 4), device="cuda")
    assert not m.multiply(x, y)
    x = torch.zeros((1000, 4), device="cuda")
    assert not m.multiply(x, torch.zeros((1000, 4), dtype=torch.float64, device="cuda"))
    assert m.multiply(x, y)


def test_repeated_calls_varying_k(torch_cuda):
    """Scratch reuse: one matrix multiplied repeatedly with panel widths that
    shrink and grow (k = 130 ends with a 2-column panel) stays exact."""
    torch = torch_cuda
    src, dst = _graph(3000, 30000, 17)
    idx, mat = oracle.build_image(src, dst, None, block=(512, 1024), dedup=False)
    m = sparse_matrix.create(matrix_image.from_bytes(idx, mat), None)
    rng = np.random.default_rng(9)
    for k in (130, 32, 2, 64, 130, 16, 1, 33, 16):
        X = rng.integers(-8, 9, (3000, k)).astype(np.float32)
        for _ in range(2):
            assert np.array_equal(_gpu_spmm(torch, m, X), oracle.spmm(idx, mat, X))


def test_empty_matrix(torch_cuda):
    """A matrix without edges (every block row stored as one empty tile) gives
    Y = 0, overwriting whatever Y held."""
    torch = torch_cuda
    e = np.zeros(0, dtype=np.uint32)
    idx, mat = oracle.build_image(e, e, None, nrows=64, ncols=64, block=(16, 16))
    m = sparse_matrix.create(matrix_image.from_bytes(idx, mat), None)
    assert m.get_nnz() == 0
    for k in (1, 16):
        X = np.ones((64, k), dtype=np.float32)
        Y = _gpu_spmm(torch, m, X)
        assert np.array_equal(Y, oracle.spmm(idx, mat, X)) and not Y.any()


@pytest.fixture(scope="module")
def rmat_s24():
    """The bench graph: R-MAT scale 24, edge factor 16, seed 1, deduplicated,
    self-loops removed, 16384 x 16384 tiles; unweighted and uniform(0,1]
    weighted images of the same edges."""
    src, dst = rmat_edges(24, seed=1)
    n = 1 << 24
    vals = np.random.default_rng(24).uniform(0.0, 1.0, len(src)).astype(np.float32)
    vals[vals == 0] = 1.0
    out = {}
    for name, v in (("binary", None), ("weighted", vals)):
        img = matrix_image.build(src, dst, v, nrows=n, ncols=n, block_size=(16384, 16384), dedup=True)
        out[name] = img
    del src, dst, vals
    idx, mat = out["binary"].bytes()
    rows, cols = oracle.nonzeros(idx, mat)
    out["outdeg"] = np.bincount(rows.astype(np.int64), minlength=n)
    out["indeg"] = np.bincount(cols.astype(np.int64), minlength=n)
    return out


@pytest.mark.parametrize("k", [1, 4, 16, 32])
def test_rmat_s24_properties(torch_cuda, rmat_s24, k):
    """Full-size checks on the bench graph, unweighted: A 1 = out-degrees;
    A (X + Z) = A X + A Z bit for bit (integer-valued operands keep every
    partial sum exact); the checksum of checksums 1^T (A X) = indeg^T X; and
    bit-exact agreement with the oracle on a sample of block rows."""
    torch = torch_cuda
    img = rmat_s24["binary"]
    m = sparse_matrix.create(img, None)
    n = m.get_num_rows()
    assert m.get_nnz() == int(rmat_s24["outdeg"].sum())
    assert 8 * int(rmat_s24["outdeg"].max()) < (1 << 24)
    ones = torch.ones((n, k), device="cuda")
    y = torch.empty((n, k), device="cuda")
    assert m.multiply(ones, y)
    deg = torch.from_numpy(rmat_s24["outdeg"].astype(np.float32)).cuda()
    assert torch.equal(y, deg[:, None].expand(n, k))
    g = torch.Generator(device="cuda").manual_seed(k)
    X = torch.randint(-4, 5, (n, k), generator=g, device="cuda").float()
    Z = torch.randint(-4, 5, (n, k), generator=g, device="cuda").float()
    yx, yz, ys = (torch.empty((n, k), device="cuda") for _ in range(3))
    assert m.multiply(X, yx) and m.multiply(Z, yz) and m.multiply(X + Z, ys)
    assert torch.equal(ys, yx + yz)
    indeg = torch.from_numpy(rmat_s24["indeg"].astype(np.float64)).cuda()
    assert torch.equal(yx.double().sum(0), (indeg[:, None] * X.double()).sum(0))
    idx, mat = img.bytes()
    Xh = X.cpu().numpy()
    R = oracle.spmm(idx, mat, Xh, nthreads=16, brows=(0, 4))
    assert np.array_equal(yx[: 4 * 16384].cpu().numpy(), R[: 4 * 16384])


@pytest.mark.parametrize("k", [1, 16, 32])
def test_rmat_s24_weighted(torch_cuda, rmat_s24, k):
    """Full-size weighted image with N(0,1) operands: rows of at most
    EXACT_ROW_MAX entries match the oracle bit for bit on a sample of block
    rows, every sampled row within RTOL, and A 1 equals the oracle's row
    sums of the weights within RTOL."""
    torch = torch_cuda
    img = rmat_s24["weighted"]
    m = sparse_matrix.create(img, None)
    n = m.get_num_rows()
    g = torch.Generator(device="cuda").manual_seed(100 + k)
    X = torch.randn((n, k), generator=g, device="cuda")
    y = torch.empty((n, k), device="cuda")
    assert m.multiply(X, y)
    idx, mat = img.bytes()
    R = oracle.spmm(idx, mat, X.cpu().numpy(), nthreads=16, brows=(0, 4))[: 4 * 16384]
    Y = y[: 4 * 16384].cpu().numpy()
    light = rmat_s24["outdeg"][: 4 * 16384] <= _lib.EXACT_ROW_MAX
    assert np.array_equal(Y[light], R[light])
    np.testing.assert_allclose(Y, R, rtol=RTOL, atol=RTOL * np.abs(R).max())
