"""SpMM throughput of the B200 FlashMatrix drop-in on synthetic R-MAT.

Workload (one step = one SpMM over the whole matrix): R-MAT scale 24
(16,777,216 vertices, edge factor 16, a/b/c/d = 0.57/0.19/0.19/0.05, seed 1,
vertex labels permuted, duplicates and self-loops removed, unweighted) in the
2D tile format, times a dense FP32 n x 16 matrix with N(0,1) entries.

Metric: GB/s of algorithmic traffic per SpMM,
    B_alg = 4 (n_rows + 1) + 4 nnz (1 + weighted) + n_cols k s + n_rows k s,
divided by the device time (CUDA events, max over ranks).  Inputs (X 1.07 GB,
column indices ~1 GB) are larger than the 126 MB L2, so no flush is needed.

  python bench.py [--gpus N --steps K --warmup W] [--impl fmx|reference]
      [--scale 24 --k 16 --weighted]

The line's "eigen" object (rank 0, after the SpMM timing; --skip-eigen
leaves it out) times the block eigensolver on its configuration: top 8
eigenpairs of D^-1/2 A D^-1/2 of the symmetrised R-MAT scale 22 graph, block
16, residual 1e-6, plain against mixed precision and against mixed precision
started from the learned warm start (weights in
flashx_b200/warmstart_weights.f32), plus that comparison on held-out SBM
graphs.  The "pagerank" object times fm::alg::PageRank (30 iterations, damping
0.85) at the reference's CPU configuration (R-MAT scale 16) on the GPU next
to the oracle's CPU restatement, and at scale 22 on the GPU.

--impl reference times the reference's CPU SpMM algorithm (the oracle's C
restatement of FlashMatrix's 2D traversal; the reference library itself
cannot be built here) on all host cores, one whole-matrix SpMM per step, in a
process that loads only the oracle (its own R-MAT stream and image builder).
Under torchrun every rank runs an independent replica (the path does not
need a data exchange); value = all ranks' bytes / max rank time.
"""
import argparse
import datetime
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2000)
    p.add_argument("--warmup", type=int, default=20)
    p.add_argument("--impl", default="fmx", choices=["fmx", "reference"])
    p.add_argument("--scale", type=int, default=24)
    p.add_argument("--k", type=int, default=16)
    p.add_argument("--weighted", action="store_true")
    p.add_argument("--no-permute", action="store_true")
    p.add_argument("--block", type=int, default=16384)
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU-baseline sample time")
    p.add_argument("--e2e-steps", type=int, default=16)
    p.add_argument("--skip-cpu", action="store_true")
    p.add_argument("--skip-eigen", action="store_true")
    p.add_argument("--skip-streamed", action="store_true")
    p.add_argument("--eig-scale", type=int, default=22, help="R-MAT scale of the eigensolver workload")
    p.add_argument("--eig-sbm", type=int, default=20, help="held-out SBM graphs for the learned warm start")
    p.add_argument("--eig-reps", type=int, default=5, help="timed solves per mode (after one warm-up)")
    p.add_argument("--large", action="store_true",
                   help="run only the large single-GPU configuration (R-MAT scale 26: SpMM k=16 and 32, top-16 "
                        "eigensolve plain / mixed / learned start) and print its JSON line")
    p.add_argument("--skip-sweep", action="store_true")
    p.add_argument("--skip-dense", action="store_true")
    p.add_argument("--dense-only", action="store_true",
                   help="run only the eigensolver's dense tensor-core kernels (n = 2^22, 16 columns) and print "
                        "their JSON object")
    p.add_argument("--eigen-only", action="store_true",
                   help="run only the eigensolver configuration (and --eig-sbm held-out SBM graphs) and print "
                        "its JSON object")
    p.add_argument("--skip-large", action="store_true")
    p.add_argument("--large-scale", type=int, default=26)
    return p.parse_args()


def workload_name(a):
    return (f"rmat-s{a.scale}-ef16-k{a.k}-f32-{'weighted' if a.weighted else 'unweighted'}"
            f"{'' if a.no_permute else '-permuted'}")


def build_graph(a):
    from flashx_b200 import matrix_image
    from flashx_b200.graphs import rmat_edges
    t0 = time.time()
    src, dst = rmat_edges(a.scale, seed=1, permute=not a.no_permute)
    vals = None
    if a.weighted:
        rng = np.random.default_rng(7)
        vals = (1.0 - rng.random(len(src), dtype=np.float32)).astype(np.float32)  # (0, 1]
    n = 1 << a.scale
    img = matrix_image.build(src, dst, vals, nrows=n, ncols=n, block_size=(a.block, a.block), dedup=True)
    del src, dst, vals
    return img, time.time() - t0


def max_over_ranks(x, world, device):
    """The largest value of x over the ranks (the slowest replica's time);
    x itself when the job has one rank.  `device` holds the reduction tensor:
    the rank's GPU under NCCL, the CPU under gloo."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_gbs(bytes_per_step, steps, world, seconds):
    """Whole-job GB/s: every replica's bytes over the slowest replica's time."""
    return bytes_per_step * steps * world / seconds / 1e9


def b_alg(n_rows, n_cols, nnz, k, weighted, s=4):
    return 4 * (n_rows + 1) + 4 * nnz * (1 + int(weighted)) + n_cols * k * s + n_rows * k * s


def cpu_info():
    model = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return os.cpu_count() or 1, model


def oracle_mod():
    """The CPU oracle (test infrastructure): the reference's CPU SpMM, builder
    and PageRank restated in C; loaded only by the CPU legs of this bench."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def oracle_image(a):
    """The bench workload's 2D image made by the oracle alone: its own R-MAT
    stream (the same edges as the library's generator) and its own builder
    (the restatement of matrix/fm_utils.cpp:228-433,617-715), so that no GPU
    library is loaded in the process."""
    oracle = oracle_mod()
    src, dst = oracle.rmat_edges(a.scale, seed=1, permute=not a.no_permute)
    vals = None
    if a.weighted:
        rng = np.random.default_rng(7)
        vals = (1.0 - rng.random(len(src), dtype=np.float32)).astype(np.float32)  # (0, 1]
    n = 1 << a.scale
    idx, mat = oracle.build_image(src, dst, vals, nrows=n, ncols=n, block=(a.block, a.block), dedup=True)
    return idx, mat


def cpu_spmm_times(idx, mat, X, nthreads, runs, brows=None, Y=None):
    """Wall times of `runs` oracle SpMMs (each as the reference's
    sparse_matrix::multiply runs it: block-row tasks pulled by `nthreads`
    workers, per-task copy of the tiles, thread-local output band copied into
    Y) into one preallocated, already touched Y."""
    oracle = oracle_mod()
    h = oracle.header(idx)
    if Y is None:
        Y = np.zeros((h["nrows"], X.shape[1]), dtype=X.dtype)
        Y.fill(0)
    times = []
    for _ in range(runs):
        t = time.perf_counter()
        oracle.spmm(idx, mat, X, nthreads=nthreads, brows=brows, out=Y)
        times.append(time.perf_counter() - t)
    return times, Y


def cpu_plan(idx, mat, X, nthreads, steps, budget_s):
    """How much of the matrix one CPU step covers: the whole matrix when
    `steps` whole-matrix SpMMs fit in `budget_s` seconds, else the first block
    rows that do (a multiple of the thread count, at least four block rows
    per thread).  Returns (brows or None, nnz covered, one calibration time)."""
    oracle = oracle_mod()
    nb = oracle.num_block_rows(idx)
    nnz = oracle.block_rows_nnz(idx, mat, 0, nb)
    (t_full,), Y = cpu_spmm_times(idx, mat, X, nthreads, 1)
    if t_full * steps <= budget_s:
        return None, nnz, t_full, Y
    per = budget_s / steps
    b1 = int(nb * per / t_full) // nthreads * nthreads
    b1 = int(min(nb, max(4 * nthreads, b1)))
    return (0, b1), oracle.block_rows_nnz(idx, mat, 0, b1), t_full, Y


def cpu_workload_x(a, ncols):
    rng = np.random.default_rng(3)
    return rng.standard_normal((ncols, a.k)).astype(np.float32)


def cpu_sample_desc(a, brows, nnz_s, nnz, nb, nthreads, model):
    what = (f"the whole matrix ({nb} block rows, {nnz} non-zeros)" if brows is None else
            f"block rows [0,{brows[1]}) of {nb} ({nnz_s} of {nnz} non-zeros)")
    return (f"{what}, {a.block}x{a.block} tiles, FP32 k={a.k}, {nthreads} threads, sequential order, "
            f"cpu_cache_size 1 MiB, per-task tile copy; GB/s = B_alg per nnz x nnz covered / time; CPU: {model}")


def cpu_config_s16(nthreads, reps=5):
    """The reference's CPU configuration: R-MAT scale 16 (edge factor 16,
    seed 1, deduplicated, no self-loops, unweighted) times FP64 X (uniform in
    [-1, 1]) with k in {1, 8}; tiles 16384^2 and 32768^2; sequential and
    Hilbert order (matrix/sparse_matrix.cpp:120-186, matrix_config.h:88);
    median of `reps` timed SpMMs after one warm-up, on `nthreads` threads."""
    oracle = oracle_mod()
    n = 1 << 16
    src, dst = oracle.rmat_edges(16, seed=1)
    rng = np.random.default_rng(11)
    out = {"workload": "rmat-s16-ef16-unweighted, X FP64 uniform[-1,1]", "threads": nthreads,
           "timing": f"median of {reps} after 1 warm-up, oracle (C restatement of the reference's CPU SpMM)"}
    for tile in (16384, 32768):
        idx, mat = oracle.build_image(src, dst, None, nrows=n, ncols=n, block=(tile, tile), dedup=True)
        nnz = oracle.block_rows_nnz(idx, mat, 0, oracle.num_block_rows(idx))
        for k in (1, 8):
            X = rng.uniform(-1.0, 1.0, (n, k))
            Y = np.zeros((n, k))
            for order in ("seq", "hilbert"):
                times = []
                for i in range(reps + 1):
                    t = time.perf_counter()
                    oracle.spmm(idx, mat, X, nthreads=nthreads, hilbert=order == "hilbert", out=Y)
                    if i:
                        times.append(time.perf_counter() - t)
                ms = float(np.median(times)) * 1e3
                out[f"tile{tile}_k{k}_{order}"] = {"ms": round(ms, 4), "nnz": int(nnz),
                                                   "gbs": round(b_alg(n, n, nnz, k, False, 8) / ms / 1e6, 3)}
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5:
                time.sleep(0.05)
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


class NvmlSampler:
    """SM clock and clock-event reasons polled through NVML every ~1 ms while
    the timed region runs (a region of tens of ms gets tens of samples; the
    nvidia-smi sampler's 200 ms period would see at most one).  Falls back to
    ClockSampler when NVML is unavailable."""
    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, gpu):
        self.gpu = gpu
        self.samples = []
        self.fallback = None
        self.stop_flag = threading.Event()

    def _handle(self, nv):
        import torch
        try:
            pr = torch.cuda.get_device_properties(self.gpu)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.gpu)

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv = nv
            self.h = self._handle(nv)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
        except Exception:
            self.fallback = ClockSampler(self.gpu)
            self.fallback.start()
            return
        self.th = threading.Thread(target=self._poll, daemon=True)
        self.th.start()

    def _poll(self):
        nv = self.nv
        while not self.stop_flag.is_set():
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                reasons = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                self.samples.append((mhz, reasons))
            except Exception:
                pass
            time.sleep(0.001)

    def stop(self):
        if self.fallback is not None:
            return self.fallback.stop()
        self.stop_flag.set()
        self.th.join(timeout=5)
        try:
            self.nv.nvmlShutdown()
        except Exception:
            pass
        sm = [x for x, _ in self.samples]
        reasons = sorted(nm for nm, bit in self.REASONS.items() if any(r & bit for _, r in self.samples))
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(sm), "sampler": "NVML, every ~1 ms during the timed region"}


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def read_traffic(name):
    """Per-launch DRAM bytes of the SpMM kernel from a committed ncu summary."""
    p = os.path.join(ROOT, "profiles", f"{name}.traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return d
    except (OSError, ValueError):
        return None


def _timed_solve(torch, dev, fn, reps=5):
    """Median wall time (ms, CUDA events on the current stream) of `fn`,
    after one untimed call; returns (ms, last result)."""
    fn()
    times, res = [], None
    stream = torch.cuda.current_stream(dev)
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        res = fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        times.append(e0.elapsed_time(e1))
    _timed_solve.last_times = [round(t, 2) for t in times]
    return float(np.median(times)), res


def eigenspace_errors(rows, cols, n, vals, X):
    """Errors of computed eigenpairs of D^-1/2 A D^-1/2 (A symmetric, binary,
    D = A 1) against the exact FP64 eigenspace of eigenvalue 1: for an
    undirected graph it is span{D^1/2 1_C} over the connected components C
    with edges, one dimension per component.  Per vector x_j (FP64 on the
    host): sin of its angle to that space, ||x - P x|| / ||x||, and
    |lambda_j - 1|; plus the largest principal angle between span(X) and
    the space (X orthonormalised first).  `rows`, `cols`: the matrix's
    non-zeros."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components
    A = sp.csr_matrix((np.ones(len(rows), dtype=np.float32), (rows, cols)), shape=(n, n))
    deg = np.asarray(A.sum(axis=1)).ravel().astype(np.float64)
    ncomp, label = connected_components(A, directed=False)
    del A
    has = deg > 0
    vol = np.bincount(label, weights=deg, minlength=ncomp)
    sq = np.sqrt(deg)
    X = np.asarray(X, dtype=np.float64)

    def resid(Z):
        # Z - P Z with P the orthogonal projector onto span{D^1/2 1_C}
        out = np.empty_like(Z)
        for j in range(Z.shape[1]):
            s = np.bincount(label, weights=sq * Z[:, j], minlength=ncomp)
            coef = np.divide(s, vol, out=np.zeros_like(s), where=vol > 0)
            out[:, j] = Z[:, j] - sq * coef[label]
        return out

    R = resid(X)
    sin_j = np.linalg.norm(R, axis=0) / np.maximum(np.linalg.norm(X, axis=0), 1e-300)
    Q, _ = np.linalg.qr(X)
    RQ = resid(Q)
    s2 = np.linalg.eigvalsh(RQ.T @ RQ)
    mult = int(np.unique(label[has]).size)
    return {"eigenspace": f"eigenvalue 1 of D^-1/2 A D^-1/2: span{{D^1/2 1_C}}, {mult} components with edges",
            "multiplicity_covers_block": mult >= X.shape[1],
            "sin_angle_to_eigenspace": [float(f"{v:.3e}") for v in sin_j],
            "abs_eigenvalue_error": [float(f"{abs(v - 1.0):.3e}") for v in vals],
            "largest_principal_angle_sin": float(f"{np.sqrt(max(s2.max(), 0.0)):.3e}")}


def _solve_summary(ms, r):
    return {"ms": round(ms, 2), "ms_each": list(getattr(_timed_solve, "last_times", [])),
            "spmm_calls": int(r.status.spmm_calls), "num_ops": int(r.status.num_ops),
            "iters": int(r.status.num_iters), "converged": int(r.status.converged),
            "max_residual": float(r.status.max_residual)}


def eigen_measure(a, dev):
    """The eigensolver configuration: top 8 eigenpairs of D^-1/2 A D^-1/2 of
    a symmetrised R-MAT graph (scale a.eig_scale, edge factor 16, seed 1),
    block 16, residual 1e-6: plain (FP32 SpMM, FP64 dense) against mixed
    (BF16 correction-form filter, tensor-core dense early), each with a random
    start and the mixed one also with the learned start; then the learned
    start against the random one on held-out SBM graphs (committed weights)."""
    import torch
    from flashx_b200 import matrix_image, sparse_matrix
    from flashx_b200.eigen import NA_operator, compute_eigen
    from flashx_b200.graphs import rmat_edges, symmetrize
    from flashx_b200 import warmstart as ws
    n = 1 << a.eig_scale
    t0 = time.time()
    s, d = rmat_edges(a.eig_scale, seed=1)
    s, d = symmetrize(s, d)
    img = matrix_image.build(s, d, None, nrows=n, ncols=n, block_size=(16384, 16384), dedup=True)
    m = sparse_matrix.create(img, None, device=dev.index)
    del s, d
    op = NA_operator(m, device=dev.index)
    results = {}
    out = {"workload": f"rmat-s{a.eig_scale}-ef16-symmetrised-na-top8-block16-tol1e-6", "n": n,
           "nnz": int(m.get_nnz()), "build_s": round(time.time() - t0, 2),
           "timing": f"median of {a.eig_reps} after 1 warm-up, CUDA events around the whole solve (host loop included)"}
    for prec in ("plain", "mixed"):
        o = ws.eigen_opts(8, 1e-6, prec)
        torch.cuda.nvtx.range_push(f"eigen_{prec}")     # for profiler filters (ncu --nvtx-include)
        ms, r = _timed_solve(torch, dev, lambda: compute_eigen(op, True, o), reps=a.eig_reps)
        torch.cuda.nvtx.range_pop()
        out[prec] = _solve_summary(ms, r)
        results[prec] = r
    out["speedup_mixed_vs_plain"] = round(out["plain"]["ms"] / out["mixed"]["ms"], 3)
    weights = os.path.join(ROOT, "flashx_b200", "warmstart_weights.f32")
    if not os.path.exists(weights):
        out["learned"] = "no committed weights"
        return out
    net = ws.warm_start_net.load(weights, dev.index)
    o = ws.eigen_opts(8, 1e-6, "mixed")
    torch.cuda.nvtx.range_push("eigen_mixed_learned")
    ms, r = _timed_solve(torch, dev, lambda: compute_eigen(op, True, o, X0=net.start_block(op)), reps=a.eig_reps)
    torch.cuda.nvtx.range_pop()
    out["mixed_learned"] = _solve_summary(ms, r)
    out["mixed_learned"]["spmm_calls"] += ws.SPMM_PER_START
    out["speedup_learned_mixed_vs_plain"] = round(out["plain"]["ms"] / ms, 3)
    results["mixed_learned"] = r
    # per-pair errors against the exact FP64 eigenspace (computed on the host)
    oracle = oracle_mod()
    idx, mat = img.bytes()
    rows, cols = oracle.nonzeros(idx, mat)
    del img, idx, mat
    for name, res in results.items():
        e = eigenspace_errors(rows, cols, n, res.vals, res.vecs.cpu().numpy())
        e["residual"] = [float(f"{v:.3e}") for v in res.residuals]
        out[name]["errors"] = e
    del rows, cols, results, op, m
    if a.eig_sbm <= 0:
        return out
    rows = []
    for i in range(a.eig_sbm):
        inst = ws.sbm_instance(30_000_000 + i, solve=False)
        po, mo = ws.eigen_opts(inst.nev, 1e-6, "plain"), ws.eigen_opts(inst.nev, 1e-6, "mixed")
        ms_p, rp = _timed_solve(torch, dev, lambda: compute_eigen(inst.op, True, po), reps=3)
        ms_m, rm = _timed_solve(torch, dev, lambda: compute_eigen(inst.op, True, mo), reps=3)
        ms_w, rw = _timed_solve(torch, dev, lambda: compute_eigen(inst.op, True, mo,
                                                                  X0=net.start_block(inst.op, 0, mo.block_size)),
                                reps=3)
        rows.append((ms_p, int(rp.status.spmm_calls), ms_m, int(rm.status.spmm_calls), ms_w,
                     int(rw.status.spmm_calls) + ws.SPMM_PER_START,
                     int(all(r.status.converged == inst.nev for r in (rp, rm, rw)))))
        del inst
    R = np.array(rows)
    out["sbm_heldout"] = {
        "graphs": a.eig_sbm, "n": "uniform 10k-200k", "blocks": "4-16 (nev = blocks)", "ratio": "5-20",
        "timing": "median of 3 solves per graph and arm, after one warm-up, CUDA events around the solve",
        "plain_random_ms_median": round(float(np.median(R[:, 0])), 2),
        "mixed_random_ms_median": round(float(np.median(R[:, 2])), 2),
        "mixed_learned_ms_median": round(float(np.median(R[:, 4])), 2),
        "plain_random_spmm_sum": int(R[:, 1].sum()), "mixed_random_spmm_sum": int(R[:, 3].sum()),
        "mixed_learned_spmm_sum": int(R[:, 5].sum()),
        "learned_vs_random_mixed_total_time": round(float(R[:, 2].sum() / R[:, 4].sum()), 3),
        "learned_mixed_vs_random_plain_total_time": round(float(R[:, 0].sum() / R[:, 4].sum()), 3),
        "all_converged": int(R[:, 6].sum())}
    return out


def streamed_measure(img, X, Y, dev, reps=5):
    """The semi-external form at the bench workload: the entry stream in
    pinned host memory, streamed to the GPU in slices of 2^26 entries during
    every SpMM.  Its bound is the host-to-device copy rate, measured here
    as the best of three 1 GiB pinned copies."""
    import torch
    from flashx_b200 import sparse_matrix
    t = time.time()
    m = sparse_matrix.create_streamed(img, None, device=dev.index)
    create_s = time.time() - t
    slices, host_bytes = m.stream_info()
    Ys = torch.empty_like(Y)
    stream = torch.cuda.current_stream(dev)
    for _ in range(2):
        m.multiply(X, Ys, stream=stream.cuda_stream)
    torch.cuda.synchronize(dev)
    identical = bool(torch.equal(Y, Ys))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        m.multiply(X, Ys, stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / reps
    h = torch.empty(1 << 28, dtype=torch.float32, pin_memory=True)
    d = torch.empty(1 << 28, dtype=torch.float32, device=dev)
    d.copy_(h, non_blocking=True)
    torch.cuda.synchronize(dev)
    rates = []
    for _ in range(3):
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        d.copy_(h, non_blocking=True)
        c1.record(stream)
        torch.cuda.synchronize(dev)
        rates.append((1 << 30) / (c0.elapsed_time(c1) / 1e3) / 1e9)
    h2d = max(rates)
    achieved = host_bytes / (ms / 1e3) / 1e9
    del m, h, d
    return {"slice_entries": 1 << 26, "slices": int(slices), "stream_bytes_per_spmm": int(host_bytes),
            "ms_per_spmm": round(ms, 3), "create_s": round(create_s, 2), "identical_to_resident": identical,
            "roofline": {"bound": "pcie_h2d", "achieved": round(achieved, 2), "peak": round(h2d, 2), "unit": "GB/s",
                         "frac": round(achieved / h2d, 4), "peak_kind": "measured here: best of three 1 GiB pinned copies"}}


def pagerank_measure(a, dev):
    """PageRank at the reference's CPU configuration (R-MAT scale 16, edge
    factor 16, seed 1, deduplicated, directed; 30 iterations at damping 0.85)
    on the GPU against the oracle's restatement of the reference on all host
    cores, plus the GPU at scale 22; ms per iteration."""
    import torch
    from flashx_b200 import create_2d_matrix, set_deduplicate
    from flashx_b200.algs import PageRank
    from flashx_b200.graphs import rmat_edges
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    out = {"iterations_max": 30, "damping": 0.85}
    nthreads, _ = cpu_info()
    set_deduplicate(True)
    try:
        for scale in (16, 22):
            n = 1 << scale
            s, d = rmat_edges(scale, seed=1)
            m, img, timg = create_2d_matrix(s, d, None, block_size=(16384, 16384), is_sym=False, nrows=n, ncols=n,
                                            return_images=True, device=dev.index)
            del s, d
            ms, (pr, it) = _timed_solve(torch, dev, lambda: PageRank(m, 30, 0.85), reps=3)
            row = {"n": n, "nnz": int(m.get_nnz()), "iters": int(it), "gpu_ms_per_iter": round(ms / max(it, 1), 4)}
            if scale == 16:
                (idx, mat), (tidx, tmat) = img.bytes(), timg.bytes()
                t = time.perf_counter()
                ref, rit = oracle.pagerank(idx, mat, tidx, tmat, 30, 0.85, nthreads=nthreads)
                cpu_s = time.perf_counter() - t
                row.update({"cpu_ms_per_iter": round(cpu_s * 1e3 / max(rit, 1), 3), "cpu_iters": int(rit),
                            "cpu_cores": nthreads, "cpu_kind": "port",
                            "max_rel_diff_vs_cpu": float(np.max(np.abs(pr.cpu().numpy() - ref)) / float(ref.max()))})
            out[f"rmat-s{scale}"] = row
            del m, img, timg
    finally:
        set_deduplicate(False)
    return out


def _time_spmm(torch, m, X, Y, steps, warmup=3):
    """Mean device time (ms) of `steps` fmx_spmm calls after `warmup`."""
    for _ in range(warmup):
        m.multiply(X, Y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        m.multiply(X, Y)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def sweep_measure(a, m, n, nnz, dev, peak, steps=20):
    """The GPU SpMM sweep of the configuration at the bench's scale: k = 1, 4
    and 32 on the bench matrix (unweighted, FP32 X ~ N(0,1)), and k = 16 on
    the same R-MAT graph with uniform(0,1] FP32 weights (built on the GPU
    from the device R-MAT stream)."""
    import torch
    from flashx_b200 import sparse_matrix
    from flashx_b200.graphs import rmat_edges_device
    g = torch.Generator(device=dev).manual_seed(4321)
    out = {"steps": steps, "timing": "mean of the steps after 3 warm-up calls, CUDA events"}

    def line(ms, k, weighted, nnz_):
        bb = b_alg(n, n, nnz_, k, weighted)
        return {"ms": round(ms, 4), "gbs": round(bb / ms / 1e6, 1), "frac": round(bb / ms / 1e6 / peak, 4),
                "bytes_alg": bb}
    for k in (1, 4, 32):
        X = torch.randn((n, k), generator=g, device=dev)
        Y = torch.empty((n, k), device=dev)
        out[f"k{k}"] = line(_time_spmm(torch, m, X, Y, steps), k, False, nnz)
        del X, Y
    src, dst = rmat_edges_device(a.scale, seed=1, permute=not a.no_permute, device=dev.index)
    vals = 1.0 - torch.rand(src.shape, generator=g, device=dev)            # (0, 1]
    t = time.time()
    mw = sparse_matrix.from_device_edges(src, dst, vals, nrows=n, ncols=n, dedup=True)
    build_s = time.time() - t
    del src, dst, vals
    X = torch.randn((n, 16), generator=g, device=dev)
    Y = torch.empty((n, 16), device=dev)
    out["k16_weighted"] = line(_time_spmm(torch, mw, X, Y, steps), 16, True, mw.get_nnz())
    out["k16_weighted"]["device_build_s"] = round(build_s, 2)
    del mw, X, Y
    torch.cuda.empty_cache()
    return out


def dense_measure(dev, peak, n=1 << 22, b=16, steps=20):
    """The block eigensolver's dense products on the tensor cores and in
    FP64, on tall-skinny FP32 operands (n rows, b columns): Y = X B (basis
    update) and G = X^T W (Gram).  Bytes per call: n (K + N) 4; the bound is
    the measured HBM copy rate."""
    import torch
    from flashx_b200 import _lib
    g = torch.Generator(device=dev).manual_seed(5)
    X = torch.randn((n, b), generator=g, device=dev)
    W = torch.randn((n, b), generator=g, device=dev)
    B = torch.randn((b, b), generator=g, device=dev)
    Y = torch.empty((n, b), device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream(dev).cuda_stream
    out = {"n": n, "columns": b, "bytes_per_call": n * 2 * b * 4,
           "timing": f"mean of {steps} calls after 3, CUDA events", "memory_bound_us": round(n * 2 * b * 4 / peak / 1e3, 1)}

    def timed(fn):
        for _ in range(3):
            if fn():
                raise RuntimeError(_lib.last_error())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps * 1e3
    names = {_lib.DENSE_BF16: "bf16", _lib.DENSE_TF32X3: "tf32x3", _lib.DENSE_F64: "f64"}
    for prec in (_lib.DENSE_TF32X3, _lib.DENSE_BF16):
        us = timed(lambda: _lib.lib.fmx_dense_gemm(prec, X.data_ptr(), b, n, b, B.data_ptr(), b, b, Y.data_ptr(), b,
                                                   err.data_ptr(), st))
        ref = X.double() @ B.double()
        out[f"gemm_{names[prec]}"] = {"us": round(us, 1), "frac": round(n * 2 * b * 4 / us / 1e3 / peak, 4),
                                     "rel_err": float(f"{float((Y.double() - ref).abs().max() / ref.abs().max()):.2e}")}
    ref = X.double().T @ W.double()
    for prec in (_lib.DENSE_TF32X3, _lib.DENSE_BF16, _lib.DENSE_F64):
        parts = _lib.lib.fmx_dense_gram_parts(prec, n)
        dt = torch.float64 if prec == _lib.DENSE_F64 else torch.float32
        part = torch.empty(parts * b * b, dtype=dt, device=dev)
        G = torch.empty((b, b), dtype=dt, device=dev)
        us = timed(lambda: _lib.lib.fmx_dense_gram(prec, X.data_ptr(), b, b, W.data_ptr(), b, b, n, part.data_ptr(),
                                                   G.data_ptr(), err.data_ptr(), st))
        out[f"gram_{names[prec]}"] = {"us": round(us, 1), "frac": round(n * 2 * b * 4 / us / 1e3 / peak, 4),
                                     "rel_err": float(f"{float((G.double() - ref).abs().max() / ref.abs().max()):.2e}")}
    out["tensor_core_errors"] = int(err.item())
    # the Rayleigh-Ritz eigenproblem of the solver (FP64 Jacobi) at the
    # block sizes the eigen and large configurations use
    jac = {}
    for bb in (16, 24):
        A = torch.randn((bb, bb), generator=g, device=dev, dtype=torch.float64)
        H = (A + A.T).contiguous()
        wv = torch.empty(bb, dtype=torch.float64, device=dev)
        V = torch.empty((bb, bb), dtype=torch.float64, device=dev)
        jac[f"b{bb}_us"] = round(timed(lambda: _lib.lib.fmx_dense_sym_eig(H.data_ptr(), bb, wv.data_ptr(), V.data_ptr(),
                                                                         st)), 1)
    out["sym_eig"] = jac
    del X, W, B, Y
    torch.cuda.empty_cache()
    return out


def large_measure(a, dev, peak):
    """The large single-GPU configuration: R-MAT at --large-scale (26: 67M
    vertices, edge factor 16, seed 1, deduplicated, int32 column ids),
    generated and built on the GPU; FP32 SpMM at k = 16 and 32 on the
    directed graph, then the top 16 eigenpairs of D^-1/2 A D^-1/2 of the
    symmetrised graph (block 24, residual 1e-6): plain, mixed, and mixed from
    the learned start (one warm-up solve, then one timed solve each)."""
    import torch
    from flashx_b200 import sparse_matrix
    from flashx_b200.eigen import NA_operator, compute_eigen
    from flashx_b200.graphs import rmat_edges_device
    from flashx_b200 import warmstart as ws
    scale = a.large_scale
    n = 1 << scale
    out = {"workload": f"rmat-s{scale}-ef16", "n": n, "built": "device R-MAT stream + fmx_matrix_build_device"}
    src, dst = rmat_edges_device(scale, seed=1, device=dev.index)
    t = time.time()
    m = sparse_matrix.from_device_edges(src, dst, None, nrows=n, ncols=n, dedup=True)
    torch.cuda.synchronize()
    out["directed_build_s"] = round(time.time() - t, 1)
    nnz = m.get_nnz()
    out["directed_nnz"] = int(nnz)
    g = torch.Generator(device=dev).manual_seed(99)
    for k in (16, 32):
        X = torch.randn((n, k), generator=g, device=dev)
        Y = torch.empty((n, k), device=dev)
        ms = _time_spmm(torch, m, X, Y, 10)
        bb = b_alg(n, n, nnz, k, False)
        out[f"spmm_k{k}"] = {"ms": round(ms, 3), "gbs": round(bb / ms / 1e6, 1), "frac": round(bb / ms / 1e6 / peak, 4)}
        del X, Y
    del m
    torch.cuda.empty_cache()
    t = time.time()
    # both directions of every edge; self-loops go first (the builder drops
    # them anyway), which keeps the list under the builder's 2^31 edges
    keep = src != dst
    src, dst = src[keep], dst[keep]
    del keep
    ssym = torch.cat([src, dst])
    dsym = torch.cat([dst, src])
    del src, dst
    m = sparse_matrix.from_device_edges(ssym, dsym, None, nrows=n, ncols=n, dedup=True)
    del ssym, dsym
    torch.cuda.empty_cache()
    op = NA_operator(m, device=dev.index)
    torch.cuda.synchronize()
    out["symmetrised_build_s"] = round(time.time() - t, 1)
    out["symmetrised_nnz"] = int(m.get_nnz())
    net = ws.warm_start_net.load(os.path.join(ROOT, "flashx_b200", "warmstart_weights.f32"), dev.index)
    for name, prec, learned in (("plain", "plain", False), ("mixed", "mixed", False),
                                ("mixed_learned", "mixed", True)):
        o = ws.eigen_opts(16, 1e-6, prec)
        ms, r = _timed_solve(torch, dev, lambda: compute_eigen(
            op, True, o, X0=net.start_block(op, 0, o.block_size) if learned else None), reps=1)
        out[name] = _solve_summary(ms, r)
        out[name]["block"] = o.block_size
        if learned:
            out[name]["spmm_calls"] += ws.SPMM_PER_START
    out["speedup_mixed_vs_plain"] = round(out["plain"]["ms"] / out["mixed"]["ms"], 3)
    out["speedup_learned_mixed_vs_plain"] = round(out["plain"]["ms"] / out["mixed_learned"]["ms"], 3)
    del op, m
    torch.cuda.empty_cache()
    return out


def repo_libraries():
    """The repository's shared libraries mapped into this process."""
    libs = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.startswith(ROOT) and ".so" in path:
                    libs.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(libs)


def run_reference(a, rank, world):
    """The reference arm: FlashMatrix's CPU SpMM (the oracle's restatement of
    sparse_matrix::multiply over the 2D image, matrix/sparse_matrix.h:219-375,
    sparse_matrix.cpp:251-473) on all host cores, on the same workload as the
    GPU arm.  Only the oracle is loaded: its own R-MAT stream and builder make
    the image.  Each step is one whole-matrix SpMM when --steps + --warmup of
    them fit in about four minutes, else the first block rows that do."""
    if rank != 0:
        return
    oracle = oracle_mod()
    nthreads, model = cpu_info()
    t0 = time.time()
    idx, mat = oracle_image(a)
    build_s = time.time() - t0
    h = oracle.header(idx)
    nb = oracle.num_block_rows(idx)
    X = cpu_workload_x(a, h["ncols"])
    runs = a.steps + a.warmup
    brows, nnz_s, t_cal, Y = cpu_plan(idx, mat, X, nthreads, runs, 240.0)
    nnz = oracle.block_rows_nnz(idx, mat, 0, nb)
    times, _ = cpu_spmm_times(idx, mat, X, nthreads, runs, brows=brows, Y=Y)
    times = times[a.warmup:]
    per_nnz = b_alg(h["nrows"], h["ncols"], nnz, a.k, a.weighted) / nnz
    gbs = [per_nnz * nnz_s / t / 1e9 for t in times]
    value = float(np.median(gbs))
    sample = cpu_sample_desc(a, brows, nnz_s, nnz, nb, nthreads, model)
    line = {
        "metric": "SpMM GB/s (algorithmic bytes / time)", "value": round(value, 3), "unit": "GB/s",
        "impl": "reference", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": round(float(np.median(times)) * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(a), "scale": a.scale, "k": a.k, "nnz": nnz,
                   "block": a.block, "whole_matrix_per_step": brows is None, "sample": sample,
                   "oracle_build_s": round(build_s, 2)},
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": nthreads, "kind": "port",
                         "sample": sample, "cpu_config": cpu_config_s16(nthreads)},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "repo_libraries_loaded": repo_libraries(),
    }
    print(json.dumps(line), flush=True)


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return run_reference(a, rank, world)
    if a.eigen_only:
        if rank == 0:
            import torch
            print(json.dumps(eigen_measure(a, torch.device("cuda", local))), flush=True)
        return
    if a.dense_only:
        if rank == 0:
            import torch
            peak, _ = read_peaks()
            print(json.dumps(dense_measure(torch.device("cuda", local), peak)), flush=True)
        return
    if a.large:
        if rank == 0:
            import torch
            peak, _ = read_peaks()
            print(json.dumps(large_measure(a, torch.device("cuda", local), peak)), flush=True)
        return

    import torch
    import torch.distributed as dist
    from flashx_b200 import sparse_matrix
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=dev)

    img, build_s = build_graph(a)
    inf = img.info()
    t0 = time.time()
    m = sparse_matrix.create(img, None, device=local)
    create_s = time.time() - t0
    n_rows, n_cols, nnz, k = inf["nrows"], inf["ncols"], inf["nnz"], a.k
    light, tasks, heavy, kernels = m.schedule()
    n_hot, hot_entries, scratch_bytes = m.hot()
    cpu_img = img if (rank == 0 and world == 1 and not a.skip_cpu) else None
    keep_img = rank == 0 and world == 1 and not a.skip_streamed
    if cpu_img is None and not keep_img:
        del img

    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    X = torch.randn((n_cols, k), generator=g, device=dev, dtype=torch.float32)
    Y = torch.empty((n_rows, k), device=dev, dtype=torch.float32)
    stream = torch.cuda.current_stream(dev)
    st = stream.cuda_stream

    def step():
        if not m.multiply(X, Y, stream=st):
            raise RuntimeError("fmx_spmm failed")

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize(dev)

    # -- timed region --
    clocks = NvmlSampler(local)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t_begin = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    clocks.start()
    t_begin.record(stream)
    for i in range(a.steps):
        starts[i].record(stream)
        step()
        ends[i].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    total_ms = t_begin.elapsed_time(t_end)
    launch_ms = float(np.mean([s.elapsed_time(e) for s, e in zip(starts, ends)]))
    total_ms = max_over_ranks(total_ms, world, dev)

    per_spmm = b_alg(n_rows, n_cols, nnz, k, a.weighted)
    value = job_gbs(per_spmm, a.steps, world, total_ms / 1e3)
    peak, peak_kind = read_peaks()
    achieved = per_spmm / (launch_ms / 1e3) / 1e9
    tr = read_traffic(workload_name(a))
    traffic = None
    if tr is not None:
        traffic = tr.get("bytes_per_launch")

    # -- end to end through the C ABI with host buffers (pinned) --
    # Every step copies its X from pinned host memory to the device and its Y
    # back.  `value`: fmx_spmm_host_async with two calls in flight on two
    # streams (one call's copy of Y overlaps the next call's copy of X; the
    # link carries both directions at once).  `serial`: the synchronous
    # fmx_spmm_host, one call at a time.
    e2e = None
    if a.e2e_steps > 0:
        Xc = X.cpu()
        Xh = [torch.empty((n_cols, k), dtype=torch.float32, pin_memory=True) for _ in range(2)]
        for xh in Xh:
            xh.copy_(Xc)
        del Xc
        Yh = [torch.empty((n_rows, k), dtype=torch.float32, pin_memory=True) for _ in range(2)]
        Xn, Yn = [xh.numpy() for xh in Xh], [yh.numpy() for yh in Yh]
        m.multiply_host(Xn[0], Yn[0])   # warm-up: staging buffers
        if world > 1:
            dist.barrier()
        t = time.perf_counter()
        for _ in range(a.e2e_steps):
            m.multiply_host(Xn[0], Yn[0])
        serial_s = max_over_ranks(time.perf_counter() - t, world, dev)
        streams = [torch.cuda.Stream(dev), torch.cuda.Stream(dev)]
        for i in range(2):                 # warm-up: each stream's staging buffers
            m.multiply_host_async(Xn[i], Yn[i], streams[i].cuda_stream)
        for sm in streams:
            sm.synchronize()
        if world > 1:
            dist.barrier()
        t = time.perf_counter()
        for i in range(a.e2e_steps):
            m.multiply_host_async(Xn[i % 2], Yn[i % 2], streams[i % 2].cuda_stream)
        for sm in streams:
            sm.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t, world, dev)
        identical = bool(torch.equal(Yh[0], Y.cpu()) and torch.equal(Yh[1], Yh[0]))
        e2e = {"value": round(job_gbs(per_spmm, a.e2e_steps, world, e2e_s), 3), "unit": "GB/s",
               "h2d_bytes_per_step": n_cols * k * 4, "d2h_bytes_per_step": n_rows * k * 4,
               "ms_per_step": round(e2e_s / a.e2e_steps * 1e3, 3),
               "api": "fmx_spmm_host_async, two calls in flight on two streams, pinned host buffers, wall clock "
                      "from the first call to both streams' end",
               "results_identical_to_device_spmm": identical,
               "serial": {"value": round(job_gbs(per_spmm, a.e2e_steps, world, serial_s), 3), "unit": "GB/s",
                          "ms_per_step": round(serial_s / a.e2e_steps * 1e3, 3), "api": "fmx_spmm_host"}}
        del Xh, Yh, Xn, Yn

    streamed = None
    if keep_img:
        streamed = streamed_measure(img, X, Y, dev)
        if cpu_img is None:
            del img

    cpu = None
    if cpu_img is not None:
        nthreads, model = cpu_info()
        cidx, cmat = cpu_img.bytes()
        oracle = oracle_mod()
        nb = oracle.num_block_rows(cidx)
        Xc = cpu_workload_x(a, n_cols)
        # whole-matrix SpMMs totalling about --cpu-seconds (at least 3)
        brows, nnz_s, t_cal, Yc = cpu_plan(cidx, cmat, Xc, nthreads, 3, max(a.cpu_seconds, 3.0))
        reps = max(3, min(9, int(a.cpu_seconds / max(t_cal, 1e-3))))
        times, _ = cpu_spmm_times(cidx, cmat, Xc, nthreads, reps, brows=brows, Y=Yc)
        del Xc, Yc
        gbs = per_spmm / nnz * nnz_s / float(np.median(times)) / 1e9
        cpu = {"value": round(gbs, 3), "unit": "GB/s", "cores": nthreads, "kind": "port",
               "sample": cpu_sample_desc(a, brows, nnz_s, nnz, nb, nthreads, model) + f"; median of {reps}",
               "cpu_config": cpu_config_s16(nthreads)}

    sweep = dense = None
    if rank == 0 and not a.skip_sweep:
        sweep = sweep_measure(a, m, n_rows, nnz, dev, peak)
    if rank == 0 and not a.skip_dense:
        dense = dense_measure(dev, peak)

    eig = prk = large = None
    if rank == 0 and not a.skip_eigen:
        del m, X, Y
        torch.cuda.empty_cache()
        eig = eigen_measure(a, dev)
        prk = pagerank_measure(a, dev)
    if rank == 0 and not a.skip_large:
        torch.cuda.empty_cache()
        large = large_measure(a, dev, peak)

    if rank == 0:
        line = {
            "metric": "SpMM GB/s (algorithmic bytes / time)",
            "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(total_ms / a.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(a), "scale": a.scale, "k": k, "edge_factor": 16,
                       "abcd": [0.57, 0.19, 0.19, 0.05], "nnz": nnz, "n_rows": n_rows,
                       "block": a.block, "bytes_alg_per_step": per_spmm,
                       "l2": "no flush: X (%.2f GB) and indices (%.2f GB) exceed the 126 MB L2"
                             % (n_cols * k * 4 / 1e9, nnz * 4 / 1e9),
                       "parallelism": f"replicas{world}" if world > 1 else "single",
                       "host_build_s": round(build_s, 2), "device_create_s": round(create_s, 2),
                       "schedule": {"exact_rows": light, "ranges": tasks, "long_rows": heavy,
                                    "hot_cols": n_hot, "hot_entry_frac": round(hot_entries / max(nnz, 1), 4),
                                    "scratch_bytes": scratch_bytes}},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                         "kernel": "pack_hot_vec_kernel + spmm_wide_kernel + spmm_fixup kernels, per fmx_spmm call",
                         "traffic": traffic},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": a.steps * kernels,
            "clocks": clk,
            "sweep": sweep,
            "dense": dense,
            "eigen": eig,
            "pagerank": prk,
            "streamed": streamed,
            "large": large,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
