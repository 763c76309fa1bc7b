"""Benchmark of the multi-scale DDM hot path on B200.

Workload (the multi-scale FP32 configuration): 1000 frames of 1024x1024 uint8 synthetic
Brownian-particle video (4000 Gaussian spots, sigma 2 px, amplitude 120 on background 20,
steps N(0, 2 px^2) per axis per frame, i.e. D = 1 px^2/frame, Gaussian noise sd 4),
scales {1024, 512, 256, 128}, 64 taus log-spaced 1..500, 30 lambdas log-spaced 2..512 px,
tolerance 1.2, chunks of 30 frames, unbiased estimator (tau_max > chunk).

One step = one chunk of 30 frames through the engine: extraction + 2-D R2C FFT of every
tile at every scale into the device ring, then |F(t) - F(t-tau)|^2 for all 64 taus of the
30 new frames. The ring is pre-filled with ceil(tau_max / chunk) + 1 chunks first, so every
timed frame pairs at all 64 lags (steady state). The video is 1000 frames long and the
steps cycle through it. The timed region ends with the azimuthal average (ISF ready).

  value    frames/s with the video resident in HBM (device pointers submitted)
  e2e      frames/s through the public API from pinned host memory: every step copies its
           30 frames host->device and reads the updated ISF (a live result) device->host
  roofline the lag kernel against HBM, with the algorithmic bytes per analysed frame
           8*E*(T+1) + 16*T*E/C (one F(t) read, one F(t-tau) read per tau, Kahan
           accumulators read+written once per chunk), E = 2,112,512 complex per frame;
           the kernel reads each distinct partner frame of a launch once (0.30 of those
           bytes), so frac is above 1, and traffic / traffic_gbs / traffic_frac give the
           ncu-measured DRAM bytes per launch and their rate over the same launch time

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "frames/s analysed (1024^2, 4 scales, 64 tau)"
UNIT = "frames/s"
SCALES = [1024, 512, 256, 128]
CHUNK = 30
N_FRAMES = 1000
SIDE = 1024
# A 4x smaller frame with the same tau list and chunk (the same lag schedule per element),
# small enough for ncu captures that save and restore device memory (about 3 GB held).
SMALL = dict(SIDE=512, SCALES=[512, 256, 128, 64], N_FRAMES=300)


def workload():
    from cuda_multiddm_b200.media import log_lambdas, log_taus
    return log_taus(1, 500, 64), log_lambdas(2, 512, 30)


def frames_elements() -> int:
    return sum((SIDE // s) ** 2 * s * (s // 2 + 1) for s in SCALES)


def lag_bytes_per_frame(T: int) -> float:
    E = frames_elements()
    return 8.0 * E * (T + 1) + 16.0 * T * E / CHUNK


def make_video(seed: int, frames: int | None = None) -> np.ndarray:
    from cuda_multiddm_b200.media import synth_video
    spots = 4000 * SIDE * SIDE // (1024 * 1024)  # same spot density at every frame size
    return synth_video(seed, SIDE, SIDE, N_FRAMES if frames is None else frames, spots, spot_sigma=2.0,
                       amplitude=120.0, background=20.0, step_var=2.0, noise_sd=4.0, max_value=255)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(frames_per_launch: float):
    """DRAM bytes per lag launch of `frames_per_launch` frames, from the per-frame DRAM
    traffic in the committed ncu summary of the lag kernel (None if absent)."""
    p = ROOT / "profiles" / "lag_kernel_c2.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_frame:"):
            try:
                return float(line.split(":", 1)[1].split()[0]) * frames_per_launch
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi SM clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path("/tmp") / f"ddm_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for ln in self.path.read_text().splitlines():
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        try:
            self.path.unlink()
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline(seconds_hint: float = 20.0) -> dict:
    """The FP64 oracle (a port of the reference's path; the reference has no CPU path)
    timed on this host's cores, in steady state, on a bounded sample of frames."""
    from oracle import oracle as O
    taus, _ = workload()
    video = make_video(1002, frames=8)
    threads = os.cpu_count() or 1
    # one timed frame first, then as many as fit the hint
    t1 = O.bench_steady(video, SCALES, taus, 1, threads)
    n = max(1, min(64, int(seconds_hint / max(t1, 1e-3))))
    t = O.bench_steady(video, SCALES, taus, n, threads) if n > 1 else t1
    return {"value": n / t, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} steady-state frames of the 1024^2 x 4-scale x 64-tau workload, FP64 oracle "
                      f"(extract + R2C FFT at every scale + 64 lag pairs per frame), OpenMP {threads} threads"}


def job_throughput(times_ms, frames_per_rank: int, world: int, device=None):
    """Whole-job throughput of `world` ranks that each analysed frames_per_rank frames:
    every timing is reduced to its maximum over ranks (the job ends when the slowest rank
    does). Returns (value, e2e_value, max_ms, max_e2e_ms) for times_ms = [device, e2e]."""
    import torch
    t = torch.tensor(times_ms, dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total = frames_per_rank * world
    return total / (float(t[0]) / 1000.0), total / (float(t[1]) / 1000.0), float(t[0]), float(t[1])


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    base = cpu_baseline(seconds_hint=max(5.0, 2.0 * args.steps))
    line = {"metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * CHUNK / base["value"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "multiscale_1024_4scales_64tau", "frames": N_FRAMES, "side": SIDE,
                       "scales": SCALES, "taus": 64, "lambdas": 30, "chunk": CHUNK},
            "impl": "reference", "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference has no CPU implementation of this path; its GPU build cannot run this "
                    "configuration without reading past its accumulator allocation, so the reference arm "
                    "is the FP64 oracle port of its algorithm on the host cores"}
    print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    from cuda_multiddm_b200 import Engine, EngineConfig

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    taus, lambdas = workload()
    T = len(taus)
    video = make_video(1002 + rank)
    dev_video = torch.from_numpy(video).cuda()
    host_video = torch.from_numpy(video).pin_memory()
    cfg = EngineConfig(frame_width=SIDE, frame_height=SIDE, scales=SCALES, taus=taus, lambdas=lambdas,
                       tolerance=1.2, chunk_frames=CHUNK, estimator="unbiased", device=local,
                       lag_batch_frames=args.lag_batch)
    eng = Engine(cfg)
    stream = torch.cuda.ExternalStream(eng.info().stream)
    preroll = math.ceil(max(taus) / CHUNK) + 1
    cursor = [0]

    def next_chunk():
        i = cursor[0]
        cursor[0] = (i + CHUNK) % (N_FRAMES - N_FRAMES % CHUNK)
        return i

    def step_device():
        i = next_chunk()
        eng.submit(dev_video[i:i + CHUNK])

    for _ in range(preroll + args.warmup):
        step_device()
    eng.finalize()
    eng.synchronize()

    # ---- device-resident timed region --------------------------------------------
    eng.set_timing(True)
    eng.kernel_times()  # clear
    launches0 = eng.info().kernel_launches
    sampler = ClockSampler(local)
    sampler.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step_device()
    eng.finalize()
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    elapsed_ms = ev0.elapsed_time(ev1)
    ktimes = eng.kernel_times()
    launches = eng.info().kernel_launches - launches0
    if world > 1:
        dist.barrier()

    # ---- end to end from pinned host memory ---------------------------------------
    # Every step copies its chunk from pinned host memory and reads back the ISF of the
    # stream so far (ddm_finalize_async into one of two pinned buffers); the next chunk is
    # submitted while that result is on its way, and the region ends once the last one is in
    # host memory.
    eng.set_timing(False)
    isf_bufs = [eng.pinned_isf_buffer() for _ in range(2)]
    step_no = [0]

    def step_host():
        i = next_chunk()
        eng.submit(host_video[i:i + CHUNK].data_ptr(), CHUNK, False)
        eng.finalize_async(isf_bufs[step_no[0] % 2])
        step_no[0] += 1

    for _ in range(args.warmup):
        step_host()
    eng.wait_isf()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step_host()
    eng.wait_isf()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)

    # ---- max over ranks ---------------------------------------------------------------
    value, e2e_value, elapsed_ms, e2e_ms = job_throughput(
        [elapsed_ms, e2e_ms], args.steps * CHUNK, world, "cuda" if world > 1 else None)

    # Lag launches pair up to --lag-batch frames each (with batching, frames wait in the ring
    # for a full launch and the finalize at the end of the timed region pairs the rest), so
    # the algorithmic bytes of an average launch are the model's bytes per frame x the
    # frames per launch.
    lag_ms, lag_n = ktimes["lag"]
    lag_avg_s = lag_ms / 1000.0 / max(lag_n, 1)
    frames_per_launch = args.steps * CHUNK / max(lag_n, 1)
    bytes_per_launch = lag_bytes_per_frame(T) * frames_per_launch
    hbm_peak, peak_kind = measured_peaks()
    achieved = bytes_per_launch / lag_avg_s / 1e9
    # The model's bytes assume one partner read per (frame, tau); the kernel reads each
    # distinct partner frame of a launch once, so beside the model's fraction (above 1) the
    # DRAM traffic ncu measured per launch over the same live launch time is reported.
    traffic = profiled_traffic(frames_per_launch)
    dram_gbs = traffic / lag_avg_s / 1e9 if traffic else None

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "multiscale_1024_4scales_64tau" if SIDE == 1024 else
                           "small_512_4scales_64tau (profiling)", "frames": N_FRAMES, "side": SIDE,
                           "scales": SCALES, "taus": T, "tau_max": max(taus), "lambdas": len(lambdas),
                           "chunk": CHUNK, "lag_batch_frames": args.lag_batch or 32,
                           "estimator": "unbiased", "steady_state": True,
                           "l2": "inputs larger than L2 (ring of %d frames x %.1f MB)"
                                 % (eng.info().ring_slots, frames_elements() * 8 / 1e6),
                           "parallelism": f"replicas x{world} (independent streams, no collective)"},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": CHUNK * SIDE * SIDE,
                        "d2h_bytes_per_step": isf_bufs[0].nbytes},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                             "frac": achieved / hbm_peak, "traffic": traffic,
                             "traffic_gbs": dram_gbs, "traffic_frac": dram_gbs / hbm_peak if dram_gbs else None,
                             "kernel": "lag_kernel", "peak_kind": peak_kind,
                             "bytes_per_launch": bytes_per_launch, "frames_per_launch": frames_per_launch,
                             "avg_launch_ms": lag_avg_s * 1000.0},
                "kernels_ms": {k: {"total_ms": v[0], "launches": v[1]} for k, v in ktimes.items()},
                "gpu_launches": int(launches), "clocks": clocks}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_serving(args) -> None:
    """Serving workload (see cuda_multiddm_b200/serving_bench.py): p50/p99 chunk latency and
    analysed frames/s at each camera rate, the highest rate whose p99 stays under the chunk
    period, and each size's chunk latency alone through the plain path."""
    import torch

    from cuda_multiddm_b200 import serving_bench as SB

    torch.cuda.set_device(0)
    vids = SB.videos()
    # warm-up as long as a timed run (module loads; the pinned pool grows to the run's peak
    # number of streams, as it would on a server that has been up for a while)
    SB.run(camera_fps=240.0, periods=args.periods, vids=vids, seed=99)
    runs = [SB.run(camera_fps=f, periods=args.periods, vids=vids) for f in args.camera_fps]
    ok = [r["camera_fps"] for r in runs if r["p99_under_period"]]
    at30 = next((r for r in runs if r["camera_fps"] == 30.0), runs[0])
    line = {"metric": "serving: p99 chunk latency (30-frame chunks, mixed 256^2..1024^2 streams)",
            "value": at30["p99_latency_s"] * 1000.0, "unit": "ms", "higher_is_better": False, "n_gpus": 1,
            "data": "synthetic", "config": {"workload": "serving_mixed_streams", "arrivals_per_period": 8,
                                            "max_streams": 64, "chunk": 30},
            "runs": runs, "highest_camera_fps_with_p99_under_period": max(ok) if ok else None,
            "alone_chunk_latency_s": SB.alone_latency(vids)}
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--lag-batch", type=int, default=0,
                    help="frames paired per lag-kernel launch (1..64; 0 = the engine default, 32)")
    ap.add_argument("--workload", choices=["multiscale", "small", "serving"], default="multiscale",
                    help="small: 512^2 frames, scales 512..64, same taus and chunk (profiling only); "
                         "serving: many camera streams through one server (its own JSON line)")
    ap.add_argument("--camera-fps", type=float, nargs="+", default=[30.0, 120.0, 480.0],
                    help="serving: camera frame rates to run (30 fps = one 30-frame chunk per second)")
    ap.add_argument("--periods", type=float, default=20.0, help="serving: chunk periods of arrivals")
    args = ap.parse_args()
    if args.workload == "serving":
        run_serving(args)
        return
    if args.workload == "small":
        globals().update(SMALL)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
