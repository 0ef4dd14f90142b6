"""bench.py's replica path on the CPU: two gloo ranks reduce their timings
to the slowest rank's, and the whole-job value counts every replica's bytes
over that time; the reference arm does its work on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t_ms = [12.5, 20.0][rank]
        worst = bench.max_over_ranks(t_ms, world, "cpu")
        value = bench.job_gbs(3.0e9, 100, world, worst / 1e3)
        q.put((rank, worst, value))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, worst, value in got:
        assert worst == 20.0
        assert value == pytest.approx(3.0e9 * 100 * 2 / 0.020 / 1e9)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(7.0, 1, "cpu") == 7.0
    assert bench.job_gbs(1e9, 10, 1, 2.0) == pytest.approx(5.0)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def test_reference_arm_loads_only_the_oracle():
    """Rank 0 of the reference arm times the whole matrix per step in a
    process that maps no library of the GPU path: the oracle's own R-MAT
    stream and builder make the image."""
    import json
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--scale", "14",
                        "--steps", "2", "--warmup", "1"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["repo_libraries_loaded"] == ["oracle/_build/liboracle.so"]
    assert line["config"]["whole_matrix_per_step"] is True
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    cfg = line["cpu_baseline"]["cpu_config"]
    for tile in (16384, 32768):
        for k in (1, 8):
            for order in ("seq", "hilbert"):
                assert cfg[f"tile{tile}_k{k}_{order}"]["gbs"] > 0
