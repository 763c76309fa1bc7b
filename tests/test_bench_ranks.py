"""The benchmark's multi-rank host logic on CPU: each rank of a 2-process gloo group
reports its own timings; the job throughput uses the maximum over ranks."""
import json
import os
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def _rank(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    # rank 1 is the slow one on the device leg, rank 0 on the end-to-end leg
    times = [100.0 + 50.0 * rank, 400.0 - 100.0 * rank]
    out[rank] = bench.job_throughput(times, frames_per_rank=300, world=world)
    dist.barrier()
    dist.destroy_process_group()


def test_job_throughput_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, 29517, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        for r in range(2):
            value, e2e, ms, e2e_ms = out[r]
            assert ms == 150.0 and e2e_ms == 400.0          # max over ranks
            assert abs(value - 600 / 0.150) < 1e-6 and abs(e2e - 600 / 0.400) < 1e-6


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    value, e2e, ms, _ = bench.job_throughput([200.0, 250.0], frames_per_rank=30, world=1)
    assert ms == 200.0 and abs(value - 150.0) < 1e-9 and abs(e2e - 120.0) < 1e-9


def test_bench_workload_lists_match_the_package():
    """bench.py restates the tau / lambda list makers so its reference arm imports nothing of
    the product; they must agree with the package's."""
    from cuda_multiddm_b200 import media
    for lo, hi, n in [(1, 500, 64), (1, 300, 48), (1, 400, 64), (1, 20, 20)]:
        assert bench.log_taus(lo, hi, n) == media.log_taus(lo, hi, n)
    for lo, hi, n in [(2, 512, 30), (4, 128, 10), (2, 1024, 40)]:
        assert bench.log_lambdas(lo, hi, n) == media.log_lambdas(lo, hi, n)
    assert bench.frames_elements(bench.WORKLOADS["c2"]) == 2_112_512
    assert sum((2048 // s) ** 2 for s in bench.WORKLOADS["c3"]["scales"]) == 5461


def test_reference_arm_runs_without_the_product_library(tmp_path):
    """The reference arm (FP64 oracle on the host cores) on the smallest workload: one JSON
    line with the same config as the GPU arm's, and libddm_b200.so never loaded."""
    import subprocess
    import sys
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'c1', "
            "'--steps', '2', '--warmup', '3']; runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); print('LOADED' if 'libddm_b200' in maps else 'CLEAN')")
    out = subprocess.run([sys.executable, "-c", code], cwd=bench.ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    line = json.loads(lines[0])
    assert lines[-1] == "CLEAN"
    assert line["impl"] == "reference" and line["steps"] == 2 and line["value"] > 0
    assert line["config"] == bench.config_of(bench.WORKLOADS["c1"], 1)
    assert abs(line["ms_per_step"] * line["steps"] / 1000.0 * line["value"] - 2 * line["frames_per_step"]) < 1e-6
