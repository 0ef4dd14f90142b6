"""Generates the golden fixtures in tests/golden/ (run where the reference
tree and g++ exist; the fixtures are committed).

test_sparse_matrix.npz -- the reference unit test matrix/unit-test/
    test-sparse_matrix.cpp:40-146 restated: its glibc-random() edge list (via
    gen_test_sparse_matrix.cpp), the 2D images the reference builder makes of
    it with 1024x1024 blocks (binary, and float-weighted with the reference's
    value placement), and Y = A X for its X[i][j] = i * 10 + j (float, 10
    columns), computed by walking the image with the reference's own tile
    classes (oracle/_ref/libfmx_refwalk.so).
hilbert.npz -- hilbert_xy2d(n, x, y) from the reference's
    matrix/hilbert_curve.cpp for n = 2, 4, 8, 16.
"""
import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402


def edges():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "gen")
        subprocess.run(["g++", "-O2", "-o", exe, os.path.join(HERE, "gen_test_sparse_matrix.cpp")], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    a = np.array([list(map(int, line.split())) for line in out.splitlines()], dtype=np.uint32)
    return a[:, 0].copy(), a[:, 1].copy()


def main():
    oracle.build(ref=True)
    assert oracle.ref_available(), "the reference walker is needed to make the fixtures"
    src, dst = edges()
    vals = np.arange(len(src), dtype=np.float32)
    n = int(max(src.max(), dst.max())) + 1
    X = (np.arange(n)[:, None] * 10 + np.arange(10)[None, :]).astype(np.float32)
    out = {"src": src.astype(np.uint16), "dst": dst.astype(np.uint16), "n": np.int64(n)}
    for name, v in (("binary", None), ("weighted", vals)):
        idx, mat = oracle.build_image(src, dst, v, block=(1024, 1024), ref_value_layout=True)
        Y = oracle.ref_spmm(idx, mat, X)
        out[f"{name}_idx_sha256"] = np.frombuffer(hashlib.sha256(idx).digest(), np.uint8)
        out[f"{name}_mat_sha256"] = np.frombuffer(hashlib.sha256(mat).digest(), np.uint8)
        out[f"{name}_y_sha256"] = np.frombuffer(hashlib.sha256(Y.tobytes()).digest(), np.uint8)
        out[f"{name}_colsum"] = Y.astype(np.float64).sum(axis=0)
        out[f"{name}_nnz"] = np.int64(oracle.nonzeros(idx, mat)[0].size)
        tidx, tmat = oracle.build_image(dst, src, v, nrows=n, ncols=n, block=(1024, 1024), ref_value_layout=True)
        Yt = oracle.ref_spmm(tidx, tmat, X)
        out[f"{name}_t_y_sha256"] = np.frombuffer(hashlib.sha256(Yt.tobytes()).digest(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "test_sparse_matrix.npz"), **out)
    L = oracle.ref()
    h = {}
    for nn in (2, 4, 8, 16):
        h[f"n{nn}"] = np.array([[L.ref_hilbert_xy2d(nn, x, y) for y in range(nn)] for x in range(nn)], dtype=np.int32)
    np.savez_compressed(os.path.join(HERE, "hilbert.npz"), **h)
    print("edges", len(src), "n", n, {k: int(out[k]) for k in out if k.endswith("_nnz")})


if __name__ == "__main__":
    main()
