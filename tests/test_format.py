"""Host side of libfmx against the oracle: the image builder produces the
same bytes as the restated reference builder (matrix/fm_utils.cpp), the
loader rejects malformed images, images round-trip through files, and the
R-MAT generator is deterministic with the configured quadrant mix.
No GPU is needed."""
import os
import struct

import numpy as np
import pytest

import oracle
from flashx_b200 import _lib, matrix_image, FmxError
from flashx_b200.graphs import rmat_edges, sbm_edges, symmetrize


def _rand_graph(seed, n, m):
    rng = np.random.default_rng(seed)
    return rng.integers(0, n, m).astype(np.uint32), rng.integers(0, n, m).astype(np.uint32)


BUILDS = [
    # seed, n, m, block, value dtype, dedup, keep self, ref value layout, nrows/ncols
    (1, 1000, 6000, (64, 128), None, False, False, False, 0),
    (2, 5000, 60000, (256, 256), np.float32, True, False, False, 0),
    (3, 5000, 60000, (256, 256), np.float32, True, False, True, 0),
    (4, 3000, 30000, (1024, 512), np.float64, False, True, True, 0),
    (5, 2000, 12000, (2, 4), np.int32, True, False, False, 2500),
    (6, 40000, 90000, (32768, 32768), np.int64, False, False, False, 0),
    (7, 300, 40000, (32, 16), None, True, True, False, 0),
    (8, 10, 0, (16, 16), None, False, False, False, 64),          # no edges at all
]


@pytest.mark.parametrize("b", range(len(BUILDS)))
def test_builder_matches_oracle_bytes(b):
    seed, n, m, block, vdt, dedup, keep_self, refv, size = BUILDS[b]
    src, dst = _rand_graph(seed, n, m)
    vals = None if vdt is None else np.random.default_rng(seed).integers(-9, 10, m).astype(vdt)
    oi, om = oracle.build_image(src, dst, vals, nrows=size, ncols=size, block=block, dedup=dedup,
                                keep_self=keep_self, ref_value_layout=refv)
    img = matrix_image.build(src, dst, vals, nrows=size, ncols=size, block_size=block, dedup=dedup,
                             remove_self=not keep_self, ref_value_layout=refv, nthreads=3)
    pi, pm = img.bytes()
    assert pi == oi and pm == om
    img.verify()
    info = img.info()
    assert info["nnz"] == oracle.nonzeros(oi, om)[0].size
    assert (info["block_h"], info["block_w"]) == block


def test_builder_thread_counts_agree():
    src, dst = _rand_graph(9, 20000, 200000)
    vals = np.random.default_rng(1).random(len(src)).astype(np.float32)
    ref = matrix_image.build(src, dst, vals, block_size=(1024, 1024), dedup=True, nthreads=1).bytes()
    for t in (2, 7, 16):
        assert matrix_image.build(src, dst, vals, block_size=(1024, 1024), dedup=True, nthreads=t).bytes() == ref


def test_golden_reference_unit_test_images():
    """The builder reproduces the reference unit test's images byte for byte
    (matrix/unit-test/test-sparse_matrix.cpp, 1024 x 1024 blocks)."""
    import hashlib
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "test_sparse_matrix.npz"))
    src, dst = g["src"].astype(np.uint32), g["dst"].astype(np.uint32)
    for name, vals in (("binary", None), ("weighted", np.arange(len(src), dtype=np.float32))):
        idx, mat = matrix_image.build(src, dst, vals, block_size=(1024, 1024), ref_value_layout=True).bytes()
        assert hashlib.sha256(idx).digest() == g[f"{name}_idx_sha256"].tobytes()
        assert hashlib.sha256(mat).digest() == g[f"{name}_mat_sha256"].tobytes()


def test_dump_load_roundtrip(tmp_path):
    src, dst = _rand_graph(10, 4000, 30000)
    img = matrix_image.build(src, dst, None, block_size=(512, 512), dedup=True)
    ip, mp = str(tmp_path / "a.mat_idx"), str(tmp_path / "a.mat")
    img.dump(ip, mp)
    back = matrix_image.load(ip, mp)
    assert back.bytes() == img.bytes()
    assert back.info() == img.info()


def _corrupt(idx, mat, what):
    idx, mat = bytearray(idx), bytearray(mat)
    if what == "magic":
        idx[0] ^= 1
    elif what == "version":
        idx[8] = 3
    elif what == "header_mismatch":
        mat[24] ^= 1                                  # nrows differs
    elif what == "block_not_pow2":
        struct.pack_into("<Q", idx, 48, 1000)
        struct.pack_into("<Q", mat, 48, 1000)
    elif what == "offsets":
        struct.pack_into("<q", idx, 4096 + 8, 4096)   # block row 0 empty
    elif what == "truncated":
        mat = mat[: len(mat) // 2]
    elif what == "column":
        # first tile: overwrite its first column id with one past the block
        nrow_part = struct.unpack_from("<H", mat, 4096 + 16)[0]
        assert nrow_part & 0x8000
        struct.pack_into("<H", mat, 4096 + 18, 0x7FFF)
    elif what == "end_marker":
        # the first tile's end-of-row-parts marker
        nnz, nrow, ncoo = struct.unpack_from("<IHH", mat, 4096 + 8)
        rhead = (nrow - ncoo) * 2 + (nnz - ncoo) * 2 + 2
        struct.pack_into("<H", mat, 4096 + 16 + rhead - 2, 0x0001)
    return bytes(idx), bytes(mat)


@pytest.mark.parametrize("what", ["magic", "version", "header_mismatch", "block_not_pow2", "offsets",
                                  "truncated", "column", "end_marker"])
def test_loader_rejects_malformed_images(what):
    src, dst = _rand_graph(12, 300, 5000)
    idx, mat = matrix_image.build(src, dst, None, nrows=300, ncols=300, block_size=(256, 256)).bytes()
    bi, bm = _corrupt(idx, mat, what)
    with pytest.raises(FmxError) as e:
        matrix_image.from_bytes(bi, bm)
    assert e.value.code in (_lib.FMX_ERR_IMAGE, _lib.FMX_ERR_UNSUPPORTED)


def test_builder_rejects_bad_arguments():
    src, dst = _rand_graph(13, 100, 1000)
    with pytest.raises(FmxError) as e:
        matrix_image.build(src, dst, None, block_size=(100, 128))
    assert e.value.code == _lib.FMX_ERR_INVAL
    with pytest.raises(FmxError) as e:
        matrix_image.build(src, dst, None, nrows=50, ncols=50, block_size=(64, 64))
    assert e.value.code == _lib.FMX_ERR_INVAL
    with pytest.raises(FmxError):
        matrix_image.build(src, dst, None, block_size=(65536, 64))


def test_load_missing_file(tmp_path):
    with pytest.raises(FmxError) as e:
        matrix_image.load(str(tmp_path / "no.mat_idx"), str(tmp_path / "no.mat"))
    assert e.value.code == _lib.FMX_ERR_IO


def test_rmat_deterministic_and_quadrant_mix():
    s1, d1 = rmat_edges(14, seed=3, permute=False)
    s2, d2 = rmat_edges(14, seed=3, permute=False, nthreads=5)
    assert np.array_equal(s1, s2) and np.array_equal(d1, d2)
    assert len(s1) == 16 << 14
    # per bit level, (row bit, col bit) follows a/b/c/d = .57/.19/.19/.05
    counts = np.zeros(4)
    for bit in range(14):
        rb = (s1 >> bit) & 1
        cb = (d1 >> bit) & 1
        counts += np.bincount(rb * 2 + cb, minlength=4)
    frac = counts / counts.sum()
    np.testing.assert_allclose(frac, [0.57, 0.19, 0.19, 0.05], atol=0.003)
    # the relabelling is a bijection applied to both ends
    sp, dp = rmat_edges(14, seed=3, permute=True)
    perm = {}
    for a, b in zip(s1[:20000].tolist(), sp[:20000].tolist()):
        assert perm.setdefault(a, b) == b
    assert len(set(perm.values())) == len(perm)
    assert not np.array_equal(s1, sp)


def test_sbm_edges_symmetric_and_blocky():
    src, dst, labels = sbm_edges(20000, 8, 20.0, 10.0, seed=4)
    assert len(src) == len(dst) and len(src) % 2 == 0
    half = len(src) // 2
    assert np.array_equal(src[:half], dst[half:]) and np.array_equal(dst[:half], src[half:])
    same = labels[src] == labels[dst]
    expect = 10.0 / (10.0 + 7)
    assert abs(same.mean() - expect) < 0.01
    s, d = symmetrize(np.array([1, 2], np.uint32), np.array([3, 4], np.uint32))
    assert s.tolist() == [1, 2, 3, 4] and d.tolist() == [3, 4, 1, 2]
