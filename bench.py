"""Benchmark of the multi-scale DDM hot path on B200.

Workloads (seeded synthetic Brownian-particle video; the reference ships no data):

  c2 (default, the headline)  1000 frames of 1024x1024 uint8 (4000 Gaussian spots, sigma 2 px,
      amplitude 120 on background 20, steps N(0, 2 px^2) per axis per frame, i.e.
      D = 1 px^2/frame, Gaussian noise sd 4), scales {1024, 512, 256, 128}, 64 taus
      log-spaced 1..500, 30 lambdas log-spaced 2..512 px, tolerance 1.2, 30-frame chunks,
      unbiased estimator (tau_max > chunk)
  c1  200 frames of 256^2 uint8 (300 spots, steps N(0, 0.5 px^2)), one 256 tile, taus 1..20,
      10 lambdas log 4..128
  c3  600 frames of 2048^2 uint8 (16000 spots, D = 0.5), scales 2048..32 (5461 tiles per
      frame), 48 taus log 1..300, 40 lambdas log 2..1024
  c4  800 frames of 2048^2 uint16 holding 12-bit values (spots of amplitude 2000 on 300,
      Poisson shot noise, half the spots with D = 0.2 and half with D = 2.0), scales
      {2048, 1024, 512, 256}, 64 taus log 1..400, 30 lambdas log 2..1024, full 16-bit decode
  small  c2's taus and chunk on 512^2 frames (profiling captures only)
  serving  many camera streams through one server (its own JSON line)

One step = one chunk of 30 frames through the engine: extraction + 2-D R2C FFT of every
tile at every scale into the device ring, then |F(t) - F(t-tau)|^2 for every tau of the
30 new frames. The ring is pre-filled with ceil(tau_max / chunk) + 1 chunks first, so every
timed frame pairs at every lag (steady state). The steps cycle through the video. The
timed region ends with the azimuthal average (ISF ready).

  value    frames/s with the video resident in HBM (device pointers submitted)
  e2e      frames/s through the public API from pinned host memory: every step copies its
           30 frames host->device and reads the updated ISF (a live result) device->host,
           three results in flight (ddm_set_async_depth(4)); the region ends with the last
           result in host memory
  roofline the lag kernel against HBM: achieved = the compulsory DRAM bytes of its launches
           (each register frame and each distinct partner frame of a launch read once, each
           accumulator row read and written once; counted by the engine) / their CUDA-event
           time. model_frac gives the same launches against the survey's byte model
           8*E*(T+1) + 16*T*E/C per frame (one partner read per (frame, tau)), which the
           kernel beats by reusing partners, so it is above 1; traffic is ncu-measured DRAM
           bytes where a capture exists (traffic_source says which)

  python bench.py [--workload c1|c2|c3|c4|small|serving] [--gpus N --steps K --warmup W]
                  [--impl reference]
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

UNIT = "frames/s"
CHUNK = 30
ASYNC_DEPTH = 4  # e2e: live results in flight + 1 (ddm_set_async_depth)


def log_taus(lo: int, hi: int, n: int) -> list[int]:
    """n strictly increasing lags from lo to hi, log-spaced (cuda_multiddm_b200.media.log_taus;
    restated here so that the reference arm imports nothing of the product)."""
    out: list[int] = []
    for i in range(n):
        v = int(round(lo * (hi / lo) ** (i / (n - 1)))) if n > 1 else lo
        if out and v <= out[-1]:
            v = out[-1] + 1
        out.append(v)
    return out


def log_lambdas(lo: float, hi: float, n: int) -> list[float]:
    """n log-spaced wavelengths rounded to float32 (cuda_multiddm_b200.media.log_lambdas)."""
    return [float(np.float32(lo * (hi / lo) ** (i / (n - 1)))) if n > 1 else float(np.float32(lo))
            for i in range(n)]


# name -> workload. video: synth_video keyword arguments; spots scale with the frame area.
WORKLOADS = {
    "c1": dict(workload="plain_256_1scale_20tau", side=256, frames=200, scales=[256],
               taus=list(range(1, 21)), lambdas=log_lambdas(4, 128, 10), pixel_mode="byte0",
               video=dict(spots=300, step_var=0.5)),
    "c2": dict(workload="multiscale_1024_4scales_64tau", side=1024, frames=1000, scales=[1024, 512, 256, 128],
               taus=log_taus(1, 500, 64), lambdas=log_lambdas(2, 512, 30), pixel_mode="byte0",
               video=dict(spots=4000, step_var=2.0)),
    "c3": dict(workload="fine_2048_7scales_48tau", side=2048, frames=600,
               scales=[2048, 1024, 512, 256, 128, 64, 32], taus=log_taus(1, 300, 48),
               lambdas=log_lambdas(2, 1024, 40), pixel_mode="byte0", video=dict(spots=16000, step_var=1.0)),
    "c4": dict(workload="highbit_2048_u16_4scales_64tau", side=2048, frames=800, scales=[2048, 1024, 512, 256],
               taus=log_taus(1, 400, 64), lambdas=log_lambdas(2, 1024, 30), pixel_mode="u16",
               video=dict(spots=16000, amplitude=2000.0, background=300.0, noise_sd=-1.0, max_value=4095,
                          step_var=0.4, step_var_b=4.0)),
    "small": dict(workload="small_512_4scales_64tau (profiling)", side=512, frames=300, scales=[512, 256, 128, 64],
                  taus=log_taus(1, 500, 64), lambdas=log_lambdas(2, 512, 30), pixel_mode="byte0",
                  video=dict(spots=1000, step_var=2.0)),
}
WORKLOADS["multiscale"] = WORKLOADS["c2"]


def metric(w: dict) -> str:
    if w is WORKLOADS["c2"]:
        return "frames/s analysed (1024^2, 4 scales, 64 tau)"
    return f"frames/s analysed ({w['side']}^2, {len(w['scales'])} scales, {len(w['taus'])} tau)"


def frames_elements(w: dict) -> int:
    M = w["side"]
    return sum((M // s) ** 2 * s * (s // 2 + 1) for s in w["scales"])


def bytes_per_pixel(w: dict) -> int:
    return 2 if w["video"].get("max_value", 255) > 255 else 1


def model_bytes_per_frame(w: dict) -> float:
    """The survey's lag-kernel byte model: one F(t) read, one F(t - tau) read per tau, and the
    accumulators read and written once per 30-frame chunk."""
    E, T = frames_elements(w), len(w["taus"])
    return 8.0 * E * (T + 1) + 16.0 * T * E / CHUNK


def video_kwargs(w: dict) -> dict:
    kw = dict(spot_sigma=2.0, amplitude=120.0, background=20.0, noise_sd=4.0, max_value=255)
    kw.update(w["video"])
    return kw


def config_of(w: dict, world: int) -> dict:
    """The workload as both arms report it (identical keys and values)."""
    return {"workload": w["workload"], "frames": w["frames"], "side": w["side"], "scales": w["scales"],
            "taus": len(w["taus"]), "tau_max": max(w["taus"]), "lambdas": len(w["lambdas"]), "tolerance": 1.2,
            "chunk": CHUNK, "estimator": "unbiased", "pixel": "u16 (12-bit values)" if bytes_per_pixel(w) == 2
            else "u8", "steady_state": True,
            "l2": "inputs larger than L2: every step streams a ring of spectra far larger than 126 MB",
            "parallelism": f"replicas x{world} (independent streams, no collective)"}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(w: dict, frames: float):
    """ncu DRAM bytes of the lag kernel for `frames` analysed frames, from the per-frame
    figure in the committed capture of the headline workload (None for other workloads)."""
    if w is not WORKLOADS["c2"]:
        return None, None
    p = ROOT / "profiles" / "lag_kernel_c2.txt"
    if not p.exists():
        return None, None
    src, per_frame = None, None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_source:"):
            src = line.split(":", 1)[1].strip()
        if line.startswith("traffic_bytes_per_frame:"):
            try:
                per_frame = float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None, None
    return (per_frame * frames, src) if per_frame else (None, None)


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


# ------------------------------------------------------------------------------------------
# CPU side: the FP64 oracle (a port of the reference's algorithm; the reference has no CPU
# path). Its input comes from the oracle's own restatement of the generator, so this side
# never loads the product library.
# ------------------------------------------------------------------------------------------

def oracle_video(w: dict, seed: int):
    from oracle import oracle as O
    return O.synth_video(seed, w["side"], w["side"], w["frames"], **video_kwargs(w))


def oracle_seconds(video, w: dict, warm: int, timed: int, threads: int) -> float:
    from oracle import oracle as O
    pix = O.PIX_U16LE if w["pixel_mode"] == "u16" else O.PIX_BYTE0
    return O.bench_steady(video, w["scales"], w["taus"], timed, threads, warm_frames=warm, pixmode=pix)


def cpu_sample(w: dict, video, seconds: float, threads: int) -> tuple[int, float, float]:
    """(frames, seconds, seconds of one frame): a steady-state oracle sample of about
    `seconds` of timed work after one untimed frame."""
    t1 = oracle_seconds(video, w, 1, 1, threads)
    n = max(1, min(256, int(seconds / max(t1, 1e-4))))
    t = oracle_seconds(video, w, 1, n, threads) if n > 1 else t1
    return n, t, t1


def cpu_baseline(w: dict, seed: int) -> dict:
    threads = os.cpu_count() or 1
    video = oracle_video(w, seed)
    try:
        n, t, _ = cpu_sample(w, video, 20.0, threads)
    except MemoryError as exc:
        return {"value": None, "unit": UNIT, "cores": threads, "kind": "port", "sample": f"unavailable: {exc}"}
    return {"value": n / t, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} steady-state frames of the {w['workload']} workload after one untimed frame, FP64 "
                      f"oracle (extract + R2C FFT at every scale + {len(w['taus'])} lag pairs per frame), "
                      f"OpenMP {threads} threads"}


def run_reference(args, w: dict) -> None:
    """The reference arm: the FP64 oracle port of the reference's algorithm on the host cores
    (the reference has no CPU implementation of this path, and its CUDA build reads past its
    accumulator on multi-tile scales with several taus). Rank 0 alone runs. Each step is a
    sample of `f` frames of the workload (30, the chunk, when the whole run fits a few
    minutes; fewer for the larger workloads); W warm-up steps run untimed, then K steps are
    timed as one stretch, and ms_per_step is that stretch / K."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    video = oracle_video(w, 1002)
    t1 = oracle_seconds(video, w, 1, 1, threads)
    budget = 150.0  # seconds of oracle work for warm-up + timed steps
    f = max(1, min(CHUNK, int(budget / max(t1, 1e-4) / (args.steps + args.warmup))))
    secs = oracle_seconds(video, w, args.warmup * f, args.steps * f, threads)
    value = args.steps * f / secs
    sample = (f"each step: {f} steady-state frames of the {w['workload']} workload ({args.warmup} untimed "
              f"warm-up steps first), FP64 oracle (extract + R2C FFT at every scale + {len(w['taus'])} lag pairs "
              f"per frame), OpenMP {threads} threads")
    line = {"metric": metric(w), "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * secs / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(w, world), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "frames_per_step": f,
            "note": "the reference has no CPU implementation of this path; its GPU build cannot run this "
                    "configuration without reading past its accumulator allocation, so the reference arm "
                    "is the FP64 oracle port of its algorithm on the host cores"}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------
# GPU side
# ------------------------------------------------------------------------------------------

def make_video(w: dict, seed: int) -> np.ndarray:
    from cuda_multiddm_b200.media import synth_video
    return synth_video(seed, w["side"], w["side"], w["frames"], **video_kwargs(w))


def run_ours(args, w: dict) -> None:
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

    taus, lambdas, side, nfr = w["taus"], w["lambdas"], w["side"], w["frames"]
    T = len(taus)
    bpp = bytes_per_pixel(w)
    video = make_video(w, 1002 + rank)
    raw = video.view(np.uint8).reshape(nfr, side, side * bpp)
    dev_video = torch.from_numpy(raw).cuda()
    host_video = torch.from_numpy(raw).pin_memory()
    cfg = EngineConfig(frame_width=side, frame_height=side, scales=w["scales"], taus=taus, lambdas=lambdas,
                       tolerance=1.2, chunk_frames=CHUNK, estimator="unbiased", device=local,
                       lag_batch_frames=args.lag_batch, bytes_per_pixel=bpp, pixel_mode=w["pixel_mode"],
                       lag_geometry=args.lag_geometry, small_tile_dft=args.small_tile_dft,
                       fft_per_tile=args.fft_per_tile, fft_group_frames=args.fft_group)
    eng = Engine(cfg)
    stream = torch.cuda.ExternalStream(eng.info().stream)
    preroll = math.ceil(max(taus) / CHUNK) + 1
    cursor = [0]

    def next_chunk():
        i = cursor[0]
        cursor[0] = (i + CHUNK) % (nfr - nfr % CHUNK)
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
    eng.kernel_stats()  # clear
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
    kstats = eng.kernel_stats()
    launches = eng.info().kernel_launches - launches0
    if world > 1:
        dist.barrier()

    # ---- end to end from pinned host memory ---------------------------------------
    # Every step copies its chunk from pinned host memory and reads back the ISF of the
    # stream so far (ddm_finalize_async into one of ASYNC_DEPTH pinned buffers, ASYNC_DEPTH - 1
    # results in flight); the next chunks are submitted while earlier results are on their
    # way, and the region ends once the last one is in host memory.
    eng.set_timing(False)
    eng.set_async_depth(ASYNC_DEPTH)
    isf_bufs = [eng.pinned_isf_buffer() for _ in range(ASYNC_DEPTH)]
    step_no = [0]

    def step_host():
        i = next_chunk()
        eng.submit(host_video[i:i + CHUNK].data_ptr(), CHUNK, False)
        eng.finalize_async(isf_bufs[step_no[0] % ASYNC_DEPTH])
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

    # Roofline of the lag kernel: its compulsory bytes (counted by the engine per launch) over
    # its CUDA-event time on the engine's stream, against the measured copy bandwidth.
    lag_ms, lag_n, lag_bytes = kstats["lag"]
    frames_timed = args.steps * CHUNK
    lag_s = lag_ms / 1000.0
    hbm_peak, peak_kind = measured_peaks()
    achieved = lag_bytes / lag_s / 1e9
    model_gbs = model_bytes_per_frame(w) * frames_timed / lag_s / 1e9
    traffic_total, traffic_src = profiled_traffic(w, frames_timed)
    per_launch = max(lag_n, 1)

    if rank == 0:
        line = {"metric": metric(w), "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": config_of(w, world),
                "impl_config": {"lag_batch_frames": eng.info().lag_batch_frames,
                                "lag_geometry": args.lag_geometry, "small_tile_dft": bool(args.small_tile_dft),
                                "fft_per_tile": bool(args.fft_per_tile),
                                "fft_group_frames": eng.info().fft_group_frames,
                                "e2e_results_in_flight": ASYNC_DEPTH - 1,
                                "ring_slots": eng.info().ring_slots,
                                "frame_spectra_mb": frames_elements(w) * 8 / 1e6},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": CHUNK * side * side * bpp,
                        "d2h_bytes_per_step": isf_bufs[0].nbytes},
                "roofline": {"bound": "hbm", "kernel": "lag_pipe_kernel", "achieved": achieved, "peak": hbm_peak,
                             "unit": "GB/s", "frac": achieved / hbm_peak, "peak_kind": peak_kind,
                             "traffic": traffic_total / per_launch if traffic_total else None,
                             "traffic_source": traffic_src,
                             "bytes_per_launch": lag_bytes / per_launch, "launches": lag_n,
                             "avg_launch_ms": lag_ms / per_launch,
                             "frames_per_launch": frames_timed / per_launch,
                             "model_bytes_per_frame": model_bytes_per_frame(w),
                             "model_gbs": model_gbs, "model_frac": model_gbs / hbm_peak},
                "kernels_ms": {k: {"total_ms": v[0], "launches": v[1], "compulsory_bytes": v[2]}
                               for k, v in kstats.items()},
                "gpu_launches": int(launches), "clocks": clocks}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(w, 1002)
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


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


def file_pass(w: dict, movie: Path, n: int) -> float:
    """Seconds from the first frame read of `movie` to the ISF in host memory, through an
    engine opened beforehand (untimed), with the command line's loop: two pinned buffers, the
    next chunk read while the engine transforms and pairs the current one."""
    import ctypes as C

    from cuda_multiddm_b200 import Engine, EngineConfig
    from cuda_multiddm_b200._lib import MovieInfo, check, lib

    side = w["side"]
    cfg = EngineConfig(frame_width=side, frame_height=side, scales=w["scales"], taus=w["taus"],
                       lambdas=w["lambdas"], tolerance=1.2, chunk_frames=CHUNK, estimator="unbiased")
    with Engine(cfg) as eng:
        fb = side * side
        bufs = [lib().ddm_host_alloc(CHUNK * fb) for _ in range(2)]
        h, info = C.c_void_p(), MovieInfo()
        check(lib().ddm_movie_open(str(movie).encode(), 0, C.byref(h), C.byref(info)))
        try:
            eng.synchronize()
            t0 = time.perf_counter()
            sent, which = 0, 0
            k = min(CHUNK, n)
            check(lib().ddm_movie_read(h, bufs[which], k))
            while sent < n:
                eng.submit(bufs[which], k, False)
                sent += k
                which ^= 1
                if sent < n:
                    k = min(CHUNK, n - sent)
                    eng.wait_frames_copied(1)
                    check(lib().ddm_movie_read(h, bufs[which], k))
            eng.finalize()
            eng.isf()
            return time.perf_counter() - t0
        finally:
            lib().ddm_movie_close(h)
            for b in bufs:
                lib().ddm_host_free(b)


def run_file(args) -> None:
    """The headline configuration from a .movie file: the c2 video written as an IIDC .movie
    and the three parameter files, then (value) an engine opened beforehand reading the file
    with the command line's loop, timed from the first frame read to the ISF in host memory
    (best of --steps passes after one untimed pass), and (cli) the ddm program itself,
    `ddm -f video.movie -M -E unbiased -C 30` to the ISF text files, timed on the host clock
    around the whole process (CUDA context, allocation, file reads, ISF files) and by its own
    [Time elapsed] line; that whole-process time varies by a second or more between runs on a
    shared machine."""
    import re
    import shutil
    import tempfile

    from cuda_multiddm_b200 import media

    w = WORKLOADS["c2"]
    cli = Path(__file__).resolve().parent / "cuda_multiddm_b200" / "ddm"
    args.steps = min(args.steps, 5)
    d = Path(tempfile.mkdtemp(prefix="ddm_file_bench_"))

    def timed(cmd):
        t0 = time.perf_counter()
        r = subprocess.run(cmd, check=True, capture_output=True, text=True)
        wall = time.perf_counter() - t0
        g = {k: re.search(k + r":?\s+([0-9.]+) s", r.stdout) for k in ("Main", "Radial Average", "Total")}
        return {"wall_s": wall, **{k.lower().replace(" ", "_") + "_s": float(m.group(1)) if m else None
                                    for k, m in g.items()}}

    try:
        video = make_video(w, 1002)
        movie = d / "video.movie"
        media.write_movie(movie, video)
        ps, pt, pl = media.write_params(d, w["scales"], w["taus"], w["lambdas"])
        n = video.shape[0]

        def cmd(frames):
            return [str(cli), "-o", str(d / "out_"), "-N", str(frames), "-Q", str(pl), "-T", str(pt), "-S", str(ps),
                    "-f", str(movie), "-M", "-E", "unbiased", "-C", str(CHUNK), "-t", "20"]

        subprocess.run(cmd(n), check=True, capture_output=True, text=True)
        runs = [timed(cmd(n)) for _ in range(max(1, args.steps))]
        best = min(runs, key=lambda x: x["wall_s"])
        files = len(list(d.glob("out_*")))
        inproc = [file_pass(w, movie, n) for _ in range(max(1, args.steps) + 1)][1:]
        line = {"metric": "frames/s analysed from a .movie file (1024^2, 4 scales, 64 tau)",
                "value": n / min(inproc), "unit": "frames/s", "higher_is_better": True, "n_gpus": 1,
                "data": "synthetic", "config": config_of(w, 1), "frames": n,
                "movie_bytes": movie.stat().st_size, "in_process_s": inproc,
                "cli": {"isf_files": files, "runs": runs, "frames_per_s_whole_process": n / best["wall_s"],
                        "frames_per_s_cli_total": n / best["total_s"] if best["total_s"] else None},
                "note": "value: an open engine, from the first frame read from the file to the ISF in "
                        "host memory (the command line's loop: two pinned buffers, chunk k+1 read while "
                        "chunk k is processed); cli: the ddm program as a whole process (CUDA context, "
                        "allocation, file reads, ISF files) and by its own [Time elapsed] Total"}
        print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(d, ignore_errors=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--lag-batch", type=int, default=0,
                    help="frames paired per lag-kernel launch (1..64; 0 = the engine default, 32)")
    ap.add_argument("--lag-geometry", type=int, default=0, choices=[0, 1],
                    help="lag kernel: 0 one thread per element (4 consumer warps, 3 CTAs/SM), "
                         "1 two threads per element (8 consumer warps, 2 CTAs/SM)")
    ap.add_argument("--small-tile-dft", action="store_true",
                    help="split-BF16 tensor-core DFT for tiles of side 32..128 instead of the FP32 FFT")
    ap.add_argument("--fft-per-tile", action="store_true",
                    help="tiles of side 32..128 through the per-tile FFT kernel (default: two passes for every scale)")
    ap.add_argument("--fft-group", type=int, default=0,
                    help="frames per FFT launch (0 = the engine default: as many as 256 MB of spectra hold)")
    ap.add_argument("--workload", choices=["c1", "c2", "c3", "c4", "multiscale", "small", "serving", "c2file"],
                    default="c2",
                    help="c2 (default): the headline 1024^2 x 4-scale x 64-tau workload; c1, c3, c4: the other "
                         "configurations; small: 512^2 frames with c2's taus (profiling only); serving: many "
                         "camera streams through one server (its own JSON line); c2file: c2 through the ddm "
                         "command line from a .movie file to ISF files (--steps timed runs)")
    ap.add_argument("--camera-fps", type=float, nargs="+", default=[30.0, 120.0, 480.0],
                    help="serving: camera frame rates to run (30 fps = one 30-frame chunk per second)")
    ap.add_argument("--periods", type=float, default=20.0, help="serving: chunk periods of arrivals")
    args = ap.parse_args()
    if args.workload == "serving":
        run_serving(args)
        return
    if args.workload == "c2file":
        run_file(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, w)
    else:
        run_ours(args, w)


if __name__ == "__main__":
    main()
