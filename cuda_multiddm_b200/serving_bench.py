"""Serving benchmark (many camera streams on one GPU), run by `bench.py --workload serving`.

Workload: Poisson arrivals of seeded particle-video streams, 8 per chunk period on average,
at most 64 at once; each stream's frames are 256^2, 512^2 or 1024^2 uint8 (uniform), its
scales the frame side plus a random subset of the smaller powers of two down to 32, 20..100
taus log-spaced from 1 to 30..300 and 5..20 lambdas log-spaced from 2 px to its smallest
scale; 30-frame chunks from a camera of `camera_fps` frames/s (30 fps: one chunk per
second), 6..10 chunks per stream. A chunk is ready when its last frame is captured; its
latency is the time from then until its ISF is in host memory. Streams wait for admission
when the server's HBM budget is in use. Reported: p50/p99 chunk latency, analysed frames/s
of the whole run, and, for comparison, the chunk latency of one stream of each size run
alone through the plain engine path (submit from host, finalize, read the ISF).
"""
from __future__ import annotations

import statistics
import time

import numpy as np

from . import Engine, EngineConfig, Server, media

SIZES = (256, 512, 1024)
CHUNK = 30
ARRIVALS_PER_PERIOD = 8.0
MAX_STREAMS = 64


def stream_specs(seed: int, periods: float):
    rng = np.random.default_rng(seed)
    t, specs = 0.0, []
    while True:
        t += rng.exponential(1.0 / ARRIVALS_PER_PERIOD)
        if t > periods:
            return specs
        side = int(rng.choice(SIZES))
        smaller = [s for s in (512, 256, 128, 64, 32) if s < side]
        pick = sorted({s for s in smaller if rng.random() < 0.5}, reverse=True)
        scales = [side] + pick
        tau_max = int(rng.integers(30, 301))
        taus = media.log_taus(1, tau_max, int(rng.integers(20, min(100, tau_max) + 1)))
        lambdas = media.log_lambdas(2.0, float(min(scales)), int(rng.integers(5, 21)))
        specs.append(dict(t=t, side=side, scales=scales, taus=taus, lambdas=lambdas,
                          chunks=int(rng.integers(6, 11)), seed=int(rng.integers(1 << 30))))


def config(spec) -> EngineConfig:
    return EngineConfig(frame_width=spec["side"], frame_height=spec["side"], scales=spec["scales"], taus=spec["taus"],
                        lambdas=spec["lambdas"], chunk_frames=CHUNK, estimator="unbiased")


def videos(max_chunks: int = 10):
    """One seeded video per frame size, in page-locked host memory (a camera's DMA buffers):
    chunks are submitted from it without a copy."""
    import torch

    out = {}
    for side in SIZES:
        spots = max(50, 4000 * side * side // (1024 * 1024))
        v = media.synth_video(7000 + side, side, side, CHUNK * max_chunks, spots, step_var=2.0, noise_sd=4.0)
        out[side] = torch.from_numpy(v).pin_memory()
    return out


def percentile(v, p):
    return float(np.percentile(np.asarray(v), p)) if len(v) else float("nan")


def run(camera_fps: float = 30.0, periods: float = 20.0, seed: int = 5, vids=None, device: int = 0) -> dict:
    """Real-time drive of the server: arrivals, admission (on its own thread, so that opening
    a stream's engine never holds up the steps of the admitted ones), chunk submission at the
    camera rate, steps, result collection, removal after a stream's last chunk."""
    import queue
    import threading

    period = CHUNK / camera_fps
    specs = stream_specs(seed, periods)
    vids = vids or videos()
    lat, frames_done = [], 0
    host = {"submit": 0.0, "step": 0.0, "poll": 0.0}
    with Server(device=device, max_streams=MAX_STREAMS) as srv:
        t0 = srv.clock()
        to_admit, admitted = queue.Queue(), queue.Queue()
        freed = threading.Condition()
        busy_waits = [0]
        stop = threading.Event()

        def admission():
            while not stop.is_set():
                try:
                    spec = to_admit.get(timeout=0.01)
                except queue.Empty:
                    continue
                while not stop.is_set():
                    sid = srv.add_stream(config(spec))
                    if sid is not None:
                        admitted.put((sid, spec, srv.clock() - t0))
                        break
                    busy_waits[0] += 1
                    with freed:  # retry when a stream has left (or after a short while)
                        freed.wait(timeout=0.05)

        th = threading.Thread(target=admission, daemon=True)
        th.start()
        arrivals = list(specs)
        active, n_admitted = {}, 0
        try:
            while arrivals or n_admitted < len(specs) or active:
                now = srv.clock() - t0
                while arrivals and arrivals[0]["t"] * period <= now:
                    to_admit.put(arrivals.pop(0))
                while not admitted.empty():
                    sid, spec, t_adm = admitted.get()
                    n_admitted += 1
                    active[sid] = dict(spec=spec, start=t_adm, next=0, got=0, offset=(spec["seed"] % 4) * CHUNK)
                t_b = time.perf_counter()
                for sid, a in active.items():
                    sp = a["spec"]
                    v = vids[sp["side"]]
                    while a["next"] < sp["chunks"] and a["start"] + (a["next"] + 1) * period <= now:
                        f0 = (a["offset"] + a["next"] * CHUNK) % (v.shape[0] - CHUNK + 1)
                        srv.submit_pinned(sid, v[f0:f0 + CHUNK].data_ptr(), CHUNK)
                        a["next"] += 1
                t_c = time.perf_counter()
                issued = srv.step()
                t_d = time.perf_counter()
                host["submit"] += t_c - t_b
                host["step"] += t_d - t_c
                done = []
                for sid, a in active.items():
                    while (r := srv.poll(sid, copy=False)) is not None:
                        meta, _ = r
                        ready = t0 + a["start"] + (meta["chunk_index"] + 1) * period
                        lat.append(meta["done_s"] - ready)
                        frames_done += CHUNK
                        a["got"] += 1
                    if a["got"] == a["spec"]["chunks"]:
                        done.append(sid)
                host["poll"] += time.perf_counter() - t_d
                for sid in done:
                    srv.remove_stream(sid)
                    del active[sid]
                if done:
                    with freed:
                        freed.notify_all()
                if not issued:
                    time.sleep(0.0005)
        finally:
            stop.set()
            th.join()
        wall = srv.clock() - t0
        stats = srv.stats()
    return {"host_s": host, "server": {k: stats[k] for k in ("steps", "step_host_s", "gpu_s", "batched_launches")},
            "camera_fps": camera_fps, "chunk_period_s": period, "streams": len(specs), "chunks": len(lat),
            "p50_latency_s": percentile(lat, 50), "p99_latency_s": percentile(lat, 99),
            "max_latency_s": float(max(lat)) if lat else float("nan"),
            "frames_per_s": frames_done / wall, "wall_s": wall, "admission_waits": busy_waits[0],
            "p99_under_period": percentile(lat, 99) < period}


def alone_latency(vids, device: int = 0, chunks: int = 6) -> dict:
    """Per-chunk latency of one stream of each size alone through the plain engine path."""
    import torch

    out = {}
    for side in SIZES:
        spec = dict(side=side, scales=[s for s in (1024, 512, 256, 128) if s <= side][:4],
                    taus=media.log_taus(1, 100, 64), lambdas=media.log_lambdas(2.0, 128.0, 20))
        host = vids[side]
        cfg = config(spec)
        cfg.device = device
        ts = []
        with Engine(cfg) as eng:
            isf = np.zeros(eng.isf_size, np.float64)
            for k in range(chunks):
                t = time.perf_counter()
                eng.submit(host[k * CHUNK:(k + 1) * CHUNK].data_ptr(), CHUNK, False)
                eng.finalize()
                isf[:] = eng.isf()
                ts.append(time.perf_counter() - t)
        out[f"{side}"] = statistics.median(ts[1:])
    return out
