"""Learned warm start for the block eigensolver (no reference counterpart).

A 2-layer graph network (libfmx's fmx_gnn_*: forward and backward on the
SpMM and the tcgen05 dense kernels, BF16 operands, FP32 accumulation) maps
vertex features (standardised log-degree plus 15 N(0,1) channels, propagated
three times by D^-1/2 A D^-1/2) to a 16-column start block.  It is trained on
eigenvectors that the plain solver computes on generated SBM graphs; the
randomly started plain solver stays the fallback, and every residual is
recomputed by the solver itself.

    net = warm_start_net(seed=0)
    net.train(instances, epochs=4)            # instances: sbm_instance(...)
    X0 = net.start_block(op)                  # op: eigen.NA_operator
    res = compute_eigen(op, True, opts, X0=X0)
    net.save("weights.f32"); net = warm_start_net.load("weights.f32")
"""
import ctypes as C
import time

import numpy as np

from . import _lib
from ._lib import check, lib
from .eigen import NA_operator, compute_eigen, eigen_options
from .graphs import sbm_edges
from .sparse_matrix import matrix_image, sparse_matrix

PRECISION = {"bf16": _lib.DENSE_BF16, "tf32x3": _lib.DENSE_TF32X3}
SPMM_PER_START = 4          # three feature propagations + the output propagation


class warm_start_net:
    """The network's weights and optimiser state on one GPU."""

    def __init__(self, seed=0, device=0):
        self._h = C.c_void_p()
        check(lib.fmx_gnn_create(device, seed, C.byref(self._h)))
        self.device = device

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:     # the module may be torn down at exit
            lib.fmx_gnn_free(h)
            self._h = C.c_void_p(None)

    # -- parameters (a flat file of FMX_GNN_PARAMS little-endian floats) --
    def get_params(self):
        p = np.empty(_lib.GNN_PARAMS, dtype=np.float32)
        check(lib.fmx_gnn_get_params(self._h, p.ctypes.data))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != _lib.GNN_PARAMS:
            raise ValueError(f"expected {_lib.GNN_PARAMS} parameters, got {p.size}")
        check(lib.fmx_gnn_set_params(self._h, p.ctypes.data))

    def save(self, path):
        self.get_params().astype("<f4").tofile(path)

    @classmethod
    def load(cls, path, device=0):
        net = cls(0, device)
        net.set_params(np.fromfile(path, dtype="<f4"))
        return net

    # -- network --
    @staticmethod
    def features(op, seed, stream=None):
        import torch
        n = op.get_num_rows()
        Z = torch.empty((n, _lib.GNN_FEATURES), dtype=torch.float32, device=op.scale.device)
        st = stream if stream is not None else torch.cuda.current_stream(Z.device).cuda_stream
        check(lib.fmx_gnn_features(op.mat.handle, op.scale.data_ptr(), seed, Z.data_ptr(), st))
        return Z

    def forward(self, op, Z, precision="bf16", stream=None):
        import torch
        Y = torch.empty((op.get_num_rows(), _lib.GNN_OUT), dtype=torch.float32, device=Z.device)
        st = stream if stream is not None else torch.cuda.current_stream(Z.device).cuda_stream
        check(lib.fmx_gnn_forward(self._h, op.mat.handle, op.scale.data_ptr(), Z.data_ptr(), PRECISION[precision],
                                  Y.data_ptr(), st))
        return Y

    def start_block(self, op, seed=0, block_size=_lib.GNN_OUT):
        """The warm start X0 (n x block_size) for compute_eigen (4 SpMMs):
        the network's 16 columns, then uniform(-1, 1) columns if the block is
        wider."""
        import torch
        Y = self.forward(op, self.features(op, seed))
        if block_size <= _lib.GNN_OUT:
            return Y[:, :block_size].contiguous()
        g = torch.Generator(device=Y.device)
        g.manual_seed(seed)
        extra = torch.rand((Y.shape[0], block_size - _lib.GNN_OUT), generator=g, device=Y.device) * 2 - 1
        return torch.cat([Y, extra], 1).contiguous()

    def loss_grad(self, op, Z, U, precision="bf16", want_grad=False, stream=None):
        import torch
        loss = C.c_double()
        g = np.empty(_lib.GNN_PARAMS, dtype=np.float32) if want_grad else None
        st = stream if stream is not None else torch.cuda.current_stream(Z.device).cuda_stream
        check(lib.fmx_gnn_loss_grad(self._h, op.mat.handle, op.scale.data_ptr(), Z.data_ptr(), U.data_ptr(),
                                    U.stride(0), U.shape[1], PRECISION[precision], C.byref(loss),
                                    g.ctypes.data if want_grad else None, st))
        return (loss.value, g) if want_grad else loss.value

    def adam_step(self, lr, stream=None):
        import torch
        st = stream if stream is not None else torch.cuda.current_stream(torch.device("cuda", self.device)).cuda_stream
        check(lib.fmx_gnn_adam_step(self._h, float(lr), st))

    def train(self, instances, epochs=4, lr=3e-3, seed=0, log=None):
        """Adam on the alignment loss, one graph per step, fresh random
        feature channels every epoch; returns the mean loss of each epoch."""
        hist = []
        for ep in range(epochs):
            tot = 0.0
            for i, inst in enumerate(instances):
                Z = self.features(inst.op, seed * 1000003 + ep * 10007 + i)
                tot += self.loss_grad(inst.op, Z, inst.U)
                self.adam_step(lr)
            hist.append(tot / max(len(instances), 1))
            if log:
                log(f"epoch {ep}: mean loss {hist[-1]:.4f}")
        return hist


class sbm_instance:
    """One generated SBM graph on the GPU with its NA operator and the plain
    solver's top-nev eigenvectors (nev = number of blocks)."""

    def __init__(self, seed, n_range=(10000, 200000), blocks=(4, 16), ratio=(5.0, 20.0), avg_degree=20.0,
                 tol=1e-6, solve=True):
        rng = np.random.default_rng(seed)
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        self.nblocks = int(rng.integers(blocks[0], blocks[1] + 1))
        self.ratio = float(rng.uniform(*ratio))
        src, dst, self.labels = sbm_edges(n, self.nblocks, avg_degree, self.ratio, seed)
        self.n = n // self.nblocks * self.nblocks
        img = matrix_image.build(src, dst, None, nrows=self.n, ncols=self.n, block_size=(16384, 16384), dedup=True)
        self.mat = sparse_matrix.create(img, None)
        self.op = NA_operator(self.mat)
        self.nev = self.nblocks
        self.U = None
        if solve:
            res = compute_eigen(self.op, True, eigen_opts(self.nev, tol))
            self.U = res.vecs
            self.solve_status = res.status


def block_size_for(nev):
    """16 columns (the network's output) while they leave guard vectors
    (nev <= 8); else nev + 8 rounded up to a multiple of 8, the extra columns
    of a learned start being random.  With block_size == nev the filter's cut
    would be a wanted Ritz value and the iteration could not converge."""
    return _lib.GNN_OUT if nev <= 8 else (nev + 15) // 8 * 8


def eigen_opts(nev, tol=1e-6, precision="plain", degree=16, max_iters=300):
    o = eigen_options()
    o.init(nev)
    o.block_size = block_size_for(nev)
    o.which = "LA"
    o.tol = tol
    o.precision = precision
    o.degree = degree
    o.max_iters = max_iters
    return o


def compare_starts(net, inst, tol=1e-6, precision="plain", seed=0):
    """Random start against the network's start on one instance: SpMM counts
    (the warm side includes the network's 4 SpMMs), times and whether both
    converged."""
    import torch
    opts = eigen_opts(inst.nev, tol, precision)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    cold = compute_eigen(inst.op, True, opts)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    X0 = net.start_block(inst.op, seed, opts.block_size)
    warm = compute_eigen(inst.op, True, opts, X0=X0)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    return {"n": inst.n, "blocks": inst.nblocks, "ratio": round(inst.ratio, 2),
            "spmm_random": int(cold.status.spmm_calls), "spmm_warm": int(warm.status.spmm_calls) + SPMM_PER_START,
            "s_random": t1 - t0, "s_warm": t2 - t1,
            "converged": bool(cold.status.converged == inst.nev and warm.status.converged == inst.nev)}


def _median_solve_ms(fn, reps):
    """Median time (ms, CUDA events around the call) of `reps` calls of fn
    after one untimed call, and the last result."""
    import torch
    fn()
    times, res = [], None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        res = fn()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return float(np.median(times)), res


def evaluate(net, n_test=200, n_range=(10000, 200000), tol=1e-6, seed=0, reps=3, log=None):
    """Three starts on `n_test` held-out SBM graphs (the seeds `study` holds
    out): the plain solver from a random block, the mixed solver from a
    random block, and the mixed solver from the network's block (its 4 SpMMs
    and its time included).  Returns per-graph rows and totals."""
    rows = []
    for s in range(n_test):
        inst = sbm_instance(seed * 1000003 + 10_000_000 + s, n_range=n_range, tol=tol, solve=False)
        po, mo = eigen_opts(inst.nev, tol, "plain"), eigen_opts(inst.nev, tol, "mixed")
        tp, rp = _median_solve_ms(lambda: compute_eigen(inst.op, True, po), reps)
        tm, rm = _median_solve_ms(lambda: compute_eigen(inst.op, True, mo), reps)
        tw, rw = _median_solve_ms(lambda: compute_eigen(inst.op, True, mo, X0=net.start_block(inst.op, s, mo.block_size)),
                                  reps)
        rows.append({"n": inst.n, "blocks": inst.nblocks, "ratio": round(inst.ratio, 2),
                     "ms_plain": round(tp, 3), "ms_mixed": round(tm, 3), "ms_learned": round(tw, 3),
                     "spmm_plain": int(rp.status.spmm_calls), "spmm_mixed": int(rm.status.spmm_calls),
                     "spmm_learned": int(rw.status.spmm_calls) + SPMM_PER_START,
                     "converged": bool(all(r.status.converged == inst.nev for r in (rp, rm, rw)))})
        if log and (s + 1) % 50 == 0:
            log(f"evaluated {s + 1} held-out graphs")
        del inst
    ok = [r for r in rows if r["converged"]]
    med = lambda k: float(np.median([r[k] for r in ok])) if ok else float("nan")
    tot = lambda k: float(sum(r[k] for r in ok))
    return {"n_test": n_test, "converged": len(ok), "reps": reps,
            "median_ms": {k: round(med("ms_" + k), 3) for k in ("plain", "mixed", "learned")},
            "total_ms": {k: round(tot("ms_" + k), 1) for k in ("plain", "mixed", "learned")},
            "median_spmm": {k: med("spmm_" + k) for k in ("plain", "mixed", "learned")},
            "total_spmm": {k: int(tot("spmm_" + k)) for k in ("plain", "mixed", "learned")},
            "learned_fewer_spmm_than_mixed": int(sum(r["spmm_learned"] < r["spmm_mixed"] for r in ok)),
            "learned_faster_than_mixed": int(sum(r["ms_learned"] < r["ms_mixed"] for r in ok)),
            "rows": rows}


def study(n_train=2000, n_test=200, epochs=4, lr=3e-3, n_range=(10000, 200000), precision="plain", tol=1e-6,
          weights_out=None, seed=0, log=print):
    """Train on `n_train` generated SBM graphs (n uniform in n_range, 4-16
    equal blocks, average degree 20, p_in/p_out 5-20, seeded, randomly
    relabelled) and compare random and learned starts on `n_test` held-out
    ones; returns a summary dict (medians, sums, per-graph rows)."""
    t0 = time.perf_counter()
    train = []
    for s in range(n_train):
        train.append(sbm_instance(seed * 1000003 + s, n_range=n_range, tol=tol))
        if log and (s + 1) % 200 == 0:
            log(f"generated and solved {s + 1} training graphs ({time.perf_counter() - t0:.0f} s)")
    t1 = time.perf_counter()
    net = warm_start_net(seed=seed)
    hist = net.train(train, epochs=epochs, lr=lr, seed=seed, log=log)
    t2 = time.perf_counter()
    del train
    rows = []
    for s in range(n_test):
        inst = sbm_instance(seed * 1000003 + 10_000_000 + s, n_range=n_range, tol=tol, solve=False)
        rows.append(compare_starts(net, inst, tol=tol, precision=precision, seed=s))
        del inst
    if weights_out:
        net.save(weights_out)
    med = lambda k: float(np.median([r[k] for r in rows]))
    return {"n_train": n_train, "n_test": n_test, "epochs": epochs, "train_loss": [round(h, 4) for h in hist],
            "median_spmm_random": med("spmm_random"), "median_spmm_warm": med("spmm_warm"),
            "sum_spmm_random": int(sum(r["spmm_random"] for r in rows)),
            "sum_spmm_warm": int(sum(r["spmm_warm"] for r in rows)),
            "median_s_random": med("s_random"), "median_s_warm": med("s_warm"),
            "converged": int(sum(r["converged"] for r in rows)), "seconds_data": round(t1 - t0, 1),
            "seconds_train": round(t2 - t1, 1), "rows": rows}


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train the warm-start network and compare it with the random start")
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--test", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--nmin", type=int, default=10000)
    ap.add_argument("--nmax", type=int, default=200000)
    ap.add_argument("--precision", default="plain", choices=["plain", "mixed"])
    ap.add_argument("--weights", default=None, help="write the trained weights (flat little-endian float32)")
    ap.add_argument("--out", default=None, help="write the summary as JSON")
    ap.add_argument("--eval-only", action="store_true",
                    help="load --weights and compare plain-random, mixed-random and mixed-learned starts on the "
                         "--test held-out graphs")
    a = ap.parse_args()
    if a.eval_only:
        res = evaluate(warm_start_net.load(a.weights), a.test, n_range=(a.nmin, a.nmax), log=print)
        print(json.dumps({k: v for k, v in res.items() if k != "rows"}), flush=True)
        if a.out:
            with open(a.out, "w") as f:
                json.dump(res, f)
        raise SystemExit(0)
    res = study(a.train, a.test, a.epochs, n_range=(a.nmin, a.nmax), precision=a.precision, weights_out=a.weights)
    brief = {k: v for k, v in res.items() if k != "rows"}
    print(json.dumps(brief), flush=True)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f)
