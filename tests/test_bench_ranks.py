"""The benchmark's multi-rank host logic on CPU: each rank of a 2-process gloo group
reports its own timings; the job throughput uses the maximum over ranks."""
import os
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


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
