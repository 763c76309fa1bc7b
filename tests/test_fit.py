"""The ISF fits that ddm_fit_isf runs on the GPU (the reference's
resources/python_tools/plot_averaged.py:57-141 analysis), against the oracle, which calls
the script's own solver (scipy.optimize.curve_fit, MINPACK Levenberg-Marquardt) with the
script's model and starting point.

CPU tests pin the oracle on curves of known parameters; GPU tests fit the engine's ISF on
the device and compare with the oracle on the same ISF values: parameters within 1e-3 of
their 1-sigma error (plus 1e-7 relative), errors within 1e-3 relative, the residual no larger
than scipy's; and the diffusion coefficient of Brownian synthetic video against its known
value.
"""
import numpy as np
import pytest

from cuda_multiddm_b200 import Engine, EngineConfig, media
from oracle import fit as OF


def test_oracle_recovers_known_curves():
    tau = np.array(media.log_taus(1, 200, 24), float)
    rng = np.random.default_rng(5)
    for F, A, B in ((0.05, 30.0, 2.0), (0.5, 2e3, 40.0), (0.01, 0.2, 1e-3)):
        y = OF.fit_func(tau, F, A, B)
        p, e = OF.fit_curve(tau, y)
        assert np.allclose(p, (F, A, B), rtol=1e-8), (p, (F, A, B))
        noisy = y * (1 + 1e-3 * rng.standard_normal(tau.size))
        p, e = OF.fit_curve(tau, noisy)
        assert np.all(np.abs(p - (F, A, B)) <= 6 * e)
    q = OF.q_vector([4.0, 8.0, 16.0])
    D, D_err = OF.diffusion(0.7 * q ** 2, q)
    assert abs(D - 0.7) < 1e-12 and D_err < 1e-12
    assert OF.SCIPY_VERSION


def _engine_isf_and_fits(frames, scales, taus, lambdas, fps=0.0, um=1.0, C=30, starts=("data",)):
    n, h, w = frames.shape
    cfg = EngineConfig(frame_width=w, frame_height=h, scales=scales, taus=taus, lambdas=lambdas, chunk_frames=C,
                       estimator="unbiased")
    with Engine(cfg) as eng:
        eng.submit(frames)
        eng.finalize()
        return eng.isf(), {st: eng.fit(fps=fps, um_per_px=um, start=st) for st in starts}


@pytest.mark.gpu
def test_device_fits_match_scipy_on_the_same_isf():
    frames = media.synth_video(71, 128, 128, 200, 100, step_var=1.0)
    scales, taus, lambdas = [128, 64], media.log_taus(1, 60, 16), [6.0, 9.0, 13.0, 19.0, 27.0]
    fps = 50.0  # lags in seconds with decay rates of a few per second: what the script's p0 suits
    isf, all_fits = _engine_isf_and_fits(frames, scales, taus, lambdas, fps=fps, um=0.5, starts=("data", "script"))
    tau_s = np.array([np.float32(t) / np.float32(fps) for t in taus], float)  # (float)tau / fps labels
    T, Q = len(taus), len(lambdas)
    for start, fits in all_fits.items():
        curves, off, tile_row = [], 0, 0
        for s in scales:
            tiles = (128 // s) ** 2
            blk = isf[off:off + tiles * Q * T].reshape(tiles, Q, T)
            for t in range(tiles):
                for q in range(Q):
                    curves.append((blk[t, q], fits["tile"][tile_row + t, q]))
            for q in range(Q):
                curves.append((blk[:, q].mean(axis=0), fits["scale"][scales.index(s), q]))
            off += tiles * Q * T
            tile_row += tiles
        compared = 0
        for y, got in curves:
            p, e = OF.fit_curve(tau_s, y, start=start)
            if start == "script" and not (np.all(np.isfinite(e)) and p[0] > 0):
                continue  # the fixed start stalls on this curve: nothing to compare
            compared += 1
            assert np.all(np.abs(got[:3] - p) <= 1e-3 * e + 1e-7 * np.abs(p)), (start, got[:3], p, e)
            assert np.allclose(got[3:], e, rtol=1e-3), (start, got[3:], e)
            rss = lambda pp: float(np.sum((OF.fit_func(tau_s, *pp) - y) ** 2))  # noqa: E731
            assert rss(got[:3]) <= rss(p) * (1 + 1e-9) + 1e-300
        assert compared >= len(curves) // 2, (start, compared)
    fits = all_fits["data"]
    q = OF.q_vector(lambdas, 0.5)
    for si in range(len(scales)):
        D, D_err = OF.diffusion(fits["scale"][si, :, 0], q)
        assert np.isclose(fits["scale_D"][si, 0], D, rtol=1e-9) and np.isclose(fits["scale_D"][si, 1], D_err, rtol=1e-6)


@pytest.mark.gpu
def test_brownian_video_gives_its_diffusion_coefficient():
    """Spots that step N(0, 1 px^2) per axis per frame diffuse with D = 0.5 px^2/frame. The
    annulus of lambda holds wave vectors from 2 pi / lambda to 1.2 times that, whose mean q^2 is
    about 1.21 (2 pi / lambda)^2, so the fits, which take q = 2 pi / lambda as the script does,
    give about 1.21 D (fps <= 0: lag in frames, 1 um per px)."""
    frames = media.synth_video(73, 128, 128, 400, 60, step_var=1.0, noise_sd=2.0)
    taus, lambdas = media.log_taus(1, 80, 20), [10.0, 13.0, 16.0, 20.0, 25.0]
    _, fits = _engine_isf_and_fits(frames, [128, 64], taus, lambdas)
    D = fits["data"]["scale_D"][0, 0]
    assert abs(D / (1.21 * 0.5) - 1) < 0.15, D
