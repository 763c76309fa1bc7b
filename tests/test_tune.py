"""The autotuner (csrc/tune.cpp): shape keys (host only), and on the GPU the timing of the
candidates (lag blocking x lag-kernel geometry, then FFT launch groups), the JSON cache,
engines that take the cached values with lag_batch_frames = -1, and the CLI's -U flag."""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cuda_multiddm_b200 import DDMError, Engine, EngineConfig, autotune, media, tune_key

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "cuda_multiddm_b200" / "ddm"
CANDIDATES = {16, 24, 30, 32, 64}


def candidate_keys(chunk: int, best_j: int, best_g: int) -> set:
    """J/G/F/V keys the tuner times: every J with both geometries (64 with the first only) at
    the default FFT group and variant, then the winner's J/G with FFT groups of 4, 8 and 16
    frames and with the per-tile FFT variant."""
    js = CANDIDATES | {chunk}
    keys = {f"{j}/{g}/0/0" for j in js for g in ((0, 1) if j <= 32 else (0,))}
    return keys | {f"{best_j}/{best_g}/{f}/0" for f in (4, 8, 16)} | {f"{best_j}/{best_g}/0/1"}


def cfg(**kw):
    base = dict(frame_width=128, frame_height=128, scales=[128, 64], taus=list(range(1, 13)) + [20],
                lambdas=[3.0, 6.0, 12.0], chunk_frames=10, estimator="unbiased")
    base.update(kw)
    return EngineConfig(**base)


def test_shape_key_names_the_shape_and_ignores_order():
    k = tune_key(cfg())
    assert k.startswith("w128h128b1|s128,64|t13:20:") and k.endswith("|c10|e1")
    assert tune_key(cfg(scales=[64, 128], taus=[20] + list(range(12, 0, -1)))) == k  # sorted first
    assert tune_key(cfg(taus=list(range(1, 13)) + [21])) != k
    assert tune_key(cfg(taus=[1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 13, 20])) != k  # same count and largest
    assert tune_key(cfg(chunk_frames=30)) != k
    assert tune_key(cfg(frame_width=256)) != k
    assert tune_key(cfg(lambdas=[2.0])) == k  # lambdas do not change the lag work
    assert tune_key(cfg(small_tile_dft=True)) == k + "|dft"  # a precision choice, never tuned


@pytest.mark.gpu
def test_autotune_times_caches_and_is_used(tmp_path, monkeypatch):
    cache = tmp_path / "tune.json"
    first = autotune(cfg(), str(cache))
    assert not first["from_cache"] and first["lag_batch_frames"] in CANDIDATES | {10}
    assert first["frames_per_s"] > 0
    entry = json.loads(cache.read_text())[tune_key(cfg())]
    assert entry["lag_batch_frames"] == first["lag_batch_frames"]
    assert entry["lag_geometry"] == first["lag_geometry"] and entry["fft_group_frames"] == first["fft_group_frames"]
    fps = entry["candidates"]
    # the (J, geometry) winner of the first pass carried into the FFT-group pass
    j0, g0 = max(((int(k.split("/")[0]), int(k.split("/")[1])) for k in fps if k.endswith("/0/0")),
                 key=lambda jg: fps[f"{jg[0]}/{jg[1]}/0/0"])
    assert set(fps) == candidate_keys(10, j0, g0)
    assert entry["frames_per_s"] == pytest.approx(max(fps.values()), rel=1e-3)
    again = autotune(cfg(), str(cache))
    assert again["from_cache"] and again["lag_batch_frames"] == first["lag_batch_frames"]
    # a second shape goes in beside the first
    other = autotune(cfg(taus=[1, 2, 4, 8]), str(cache))
    assert set(json.loads(cache.read_text())) == {tune_key(cfg()), tune_key(cfg(taus=[1, 2, 4, 8]))}
    assert other["lag_batch_frames"] in CANDIDATES | {10}
    # lag_batch_frames = -1 takes the cached value, the same ISF as an explicit one
    frames = media.synth_video(51, 128, 128, 60, 30, step_var=1.0)
    monkeypatch.setenv("DDM_TUNE_CACHE", str(cache))
    with Engine(cfg(lag_batch_frames=-1)) as eng:
        inf = eng.info()
        assert inf.lag_batch_frames == first["lag_batch_frames"]
        assert inf.lag_geometry == first["lag_geometry"] and inf.fft_group_frames == first["fft_group_frames"]
        assert inf.fft_per_tile == first["fft_per_tile"]
        eng.submit(frames)
        eng.finalize()
        auto = eng.isf()
    with Engine(cfg(lag_batch_frames=first["lag_batch_frames"], lag_geometry=first["lag_geometry"],
                    fft_group_frames=first["fft_group_frames"], fft_per_tile=first["fft_per_tile"])) as eng:
        eng.submit(frames)
        eng.finalize()
        assert np.array_equal(eng.isf(), auto)
    # an unknown shape (or no cache) falls back to the default
    with Engine(cfg(lag_batch_frames=-1, chunk_frames=12)) as eng:
        assert eng.info().lag_batch_frames == 32
    monkeypatch.delenv("DDM_TUNE_CACHE")
    with Engine(cfg(lag_batch_frames=-1)) as eng:
        assert eng.info().lag_batch_frames == 32
    with pytest.raises(DDMError):
        autotune(cfg(estimator="compat", total_frames=40))


@pytest.mark.gpu
def test_cli_autotune_flag(tmp_path):
    ps, pt, pl = media.write_params(tmp_path, (128, 64), (1, 2, 4), (4.0, 8.0, 16.0))
    cache = tmp_path / "t.json"
    base = ["-N", "40", "-C", "10", "-Q", str(pl), "-T", str(pt), "-S", str(ps), "-B", "1", "-E", "unbiased"]
    r = subprocess.run([str(CLI), "-o", str(tmp_path / "a_"), *base, "-U", str(cache), "-v"], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "(timed)" in r.stderr and "lag_geometry" in r.stderr and len(json.loads(cache.read_text())) == 1
    r = subprocess.run([str(CLI), "-o", str(tmp_path / "b_"), *base, "-U", str(cache), "-v"], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0 and "(cached)" in r.stderr
    r = subprocess.run([str(CLI), "-o", str(tmp_path / "c_"), *base[:-2], "-U", str(cache)], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 1 and "-U tunes the unbiased estimator" in r.stderr
