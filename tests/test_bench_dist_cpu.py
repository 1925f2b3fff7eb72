"""bench.py's multi-rank logic on CPU: two gloo ranks (127.0.0.1) run the same
per-rank query sharding, MAX-over-ranks timing and whole-job rate the GPU run
uses with NCCL."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    import bench
    from bbrcit_kde_b200 import workloads as W
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        wl = W.config2(n=64, m=1000)
        q = bench.rank_queries(W, wl, rank, 1000)
        ms = 100.0 + 50.0 * rank          # rank 1 is the slow one
        total = bench.max_over_ranks(dist, ms, "cpu")
        rate = bench.whole_job_rate(2.0 * 64 * 1000, 5, world, total)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), q=q, total=total, rate=rate)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_queries_and_take_max(tmp_path):
    port = 29500 + (os.getpid() % 1000)
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    r0, r1 = (np.load(tmp_path / f"r{i}.npz") for i in range(2))
    sys.path.insert(0, ROOT)
    from bbrcit_kde_b200 import workloads as W
    # rank 0 keeps the configuration's queries; rank 1 has its own seeded batch
    np.testing.assert_array_equal(r0["q"], W.config2(n=64, m=1000).queries)
    assert r1["q"].shape == r0["q"].shape and not np.array_equal(r0["q"], r1["q"])
    assert np.all(np.abs(r1["q"]) <= 3.0)
    # both ranks see the slowest rank's time and the same whole-job rate
    assert float(r0["total"]) == float(r1["total"]) == 150.0
    assert float(r0["rate"]) == pytest.approx(2.0 * 64 * 1000 * 5 * 2 / 0.150)


def test_single_process_helpers():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 12.5, "cpu") == 12.5
    assert bench.whole_job_rate(1e12, 3, 4, 1000.0) == pytest.approx(1.2e13)


def test_reference_arm_line_and_workloads():
    """--impl reference prints one JSON line with the contract's keys for the
    workloads it times (the reference's own CPU direct_eval), and refuses, with a
    message and a non-zero status, the workloads whose line carries its own
    CPU baseline."""
    import json
    import subprocess
    run = lambda *extra: subprocess.run(   # noqa: E731
        [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
         "--warmup", "1", "--cpu-seconds", "1", *extra], capture_output=True, text=True,
        timeout=600, cwd=ROOT)
    r = run("--workload", "plain-small")
    assert r.returncode == 0, r.stderr
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and "plain 2-D Gaussian" in \
        line["config"]["workload"]
    r = run("--workload", "cv-batch")
    assert r.returncode == 2 and "own cpu_baseline" in r.stderr
