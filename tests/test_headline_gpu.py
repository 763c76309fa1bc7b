"""Parity of the benchmarked configuration itself: the headline workload (1000 frames of
1024^2 uint8 from the benchmark's generator, scales {1024, 512, 256, 128}, 64 taus
log-spaced 1..500, 30 lambdas log-spaced 2..512, 30-frame chunks, unbiased estimator) runs
through the C ABI exactly as the benchmark runs it -- 32-frame lag launches over a 591-slot
ring, a union of about 496 partner frames per launch, unfused entries for the larger taus,
the persistent grid walking every element block -- and again with 64-frame launches, and
both are compared with one FP64 oracle run; the 32-frame launches run in both lag-kernel
geometries (one thread per element, and two threads per element).

Tolerance: 1e-5 relative per ISF bin (FP32 FFT and lag arithmetic with compensated
accumulation, FP64 azimuthal reduction), with an absolute floor of 1e-9 of the largest
value of the scale's block for bins that are exactly zero in FP64 (lambdas longer than a
scale's tile give empty annuli). The worst relative error of every (scale, lambda, tau) bin
over the tiles is computed; with DDM_PARITY_REPORT set, it is written there as JSON.
"""
import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

from cuda_multiddm_b200 import Engine, EngineConfig
from oracle import oracle as O

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402

pytestmark = pytest.mark.gpu

RTOL = 1e-5


@pytest.fixture(scope="module")
def headline():
    w = bench.WORKLOADS["c2"]
    video = bench.make_video(w, 1002)
    want, _ = O.ddm_run(video, w["scales"], w["taus"], w["lambdas"], estimator=O.EST_UNBIASED, chunk=bench.CHUNK)
    return w, video, want


def per_bin_errors(got, want, scales, Q, T):
    """{scale: [Q][T] worst relative error over the tiles}, and the overall worst."""
    out, worst, off = {}, 0.0, 0
    M = scales[0]
    for s in scales:
        tiles = (M // s) ** 2
        g = got[off:off + tiles * Q * T].reshape(tiles, Q, T)
        wv = want[off:off + tiles * Q * T].reshape(tiles, Q, T)
        floor = 1e-9 * max(np.abs(wv).max(), 1e-300)
        assert np.all(np.abs(g - wv) <= RTOL * np.abs(wv) + floor), (s, float(np.abs(g - wv).max()))
        rel = (np.abs(g - wv) / np.maximum(np.abs(wv), floor)).max(axis=0)
        out[s] = rel
        worst = max(worst, float(rel.max()))
        off += tiles * Q * T
    assert off == got.size
    return out, worst


@pytest.mark.parametrize("lag_batch,ring,geometry", [(32, 591, 0), (64, 623, 0), (32, 591, 1)])
def test_headline_configuration_matches_oracle(headline, lag_batch, ring, geometry):
    w, video, want = headline
    side = w["side"]
    cfg = EngineConfig(frame_width=side, frame_height=side, scales=w["scales"], taus=w["taus"],
                       lambdas=w["lambdas"], tolerance=1.2, chunk_frames=bench.CHUNK, estimator="unbiased",
                       lag_batch_frames=lag_batch, lag_geometry=geometry)
    with Engine(cfg) as eng:
        info = eng.info()
        assert info.ring_slots == ring and info.lag_batch_frames == lag_batch
        for i in range(0, video.shape[0], bench.CHUNK):
            eng.submit(video[i:i + bench.CHUNK])
        eng.finalize()
        got = eng.isf()
    Q, T = len(w["lambdas"]), len(w["taus"])
    errs, worst = per_bin_errors(got, want, w["scales"], Q, T)
    assert worst <= RTOL
    path = os.environ.get("DDM_PARITY_REPORT")
    if path:
        rep = json.loads(Path(path).read_text()) if Path(path).exists() else {}
        rep[f"lag_batch_{lag_batch}_geometry_{geometry}"] = {
            "worst": worst,
            "worst_per_scale": {str(s): float(e.max()) for s, e in errs.items()},
            "taus": list(w["taus"]), "lambdas": list(w["lambdas"]),
            "per_scale_lambda_tau": {str(s): e.tolist() for s, e in errs.items()}}
        Path(path).write_text(json.dumps(rep))
