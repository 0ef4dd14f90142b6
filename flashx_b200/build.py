"""Builds libfmx.so in-tree with nvcc for sm_100a (no JIT cache).

    python flashx_b200/build.py [--force]

(run as a file, not as `-m flashx_b200.build`, so that a stale library is
never loaded by the package import while it is being rebuilt)

The library is written next to this file (flashx_b200/libfmx.so) so that a
copy of the tree carries it.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfmx.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith((".cu", ".cpp")))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(os.path.dirname(HERE), "include", "fmx.h"))
    return hs


def nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found; libfmx.so cannot be built")
    return p


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources() + headers())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [nvcc(), "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-pthread",
               "--expt-relaxed-constexpr", "-I", os.path.join(os.path.dirname(HERE), "include"),
               *ARCH, "-c", src, "-o", obj]
        procs.append((src, cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for src, cmd, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode:
            sys.stderr.write(out.decode())
        if p.returncode:
            failed.append(src)
    if failed:
        raise RuntimeError("nvcc failed on: " + ", ".join(failed))
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-shared", *ARCH, "-Xcompiler", "-fPIC,-pthread", "-o", tmp, *objs]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode:
        sys.stderr.write(r.stdout.decode())
        raise RuntimeError("linking libfmx.so failed")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
