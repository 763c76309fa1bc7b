"""The split-BF16 tensor-core DFT for tiles of side 32, 64 and 128 (small_tile_dft), through
the C ABI, against the FP64 oracle and beside the FP32 FFT path.

Tolerances: spectra within 2e-5 of the tile's largest FP64 magnitude (the hi/lo split keeps
16 significant bits of every operand; measured about 1e-6); ISF within 1e-3 relative per bin
of the FP64 oracle (the path's stated budget), while the FP32 path on the same frames stays
within 1e-5.
"""
import numpy as np
import pytest

from cuda_multiddm_b200 import Engine, EngineConfig, media
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def spectra_errors(frames, M, scales, pixel_mode="byte0"):
    bpp = 2 if frames.dtype == np.uint16 else 1
    raw = np.ascontiguousarray(frames).view(np.uint8).reshape(frames.shape[0], M, M * bpp)
    cfg = EngineConfig(frame_width=M, frame_height=M, scales=scales, taus=[1], lambdas=[2.0], chunk_frames=4,
                       bytes_per_pixel=bpp, pixel_mode=pixel_mode, small_tile_dft=True)
    with Engine(cfg) as eng:
        eng.submit(raw)
        specs = [eng.spectrum(f) for f in range(frames.shape[0])]
    worst = {}
    pix = O.PIX_U16LE if pixel_mode == "u16" else O.PIX_BYTE0
    for f, spec in enumerate(specs):
        off = 0
        for s in sorted(scales, reverse=True):
            side = M // s
            tiles = O.extract(raw[f], bpp, pix, 0, 0, M, s)
            n = s * (s // 2 + 1)
            for tile in range(side * side):
                ref = O.fft2_r2c(tiles[tile])
                got = spec[off + tile * n: off + (tile + 1) * n].reshape(s, s // 2 + 1)
                e = np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-300)
                worst[s] = max(worst.get(s, 0.0), float(e))
            off += side * side * n
    return worst


@pytest.mark.parametrize("M,scales", [(32, [32]), (128, [128, 64, 32]), (256, [256, 128, 64, 32, 16])])
def test_bf16_dft_spectra_match_fp64_fft(M, scales):
    rng = np.random.default_rng(M)
    frames = rng.integers(0, 256, size=(3, M, M), dtype=np.uint8)
    worst = spectra_errors(frames, M, scales)
    assert max(worst.values()) <= 2e-5, worst


def test_bf16_dft_spectra_u16_full_precision():
    frames = media.synth_video(21, 128, 128, 3, 40, amplitude=2000, background=300, noise_sd=-1, max_value=4095)
    worst = spectra_errors(frames, 128, [128, 64, 32], pixel_mode="u16")
    assert max(worst.values()) <= 2e-5, worst


def test_bf16_dft_isf_on_fine_scales_beside_fp32():
    """A smaller frame with the fine-scale configuration's scale ladder (down to 32-pixel tiles):
    ISF of the BF16 path within 1e-3 of the FP64 oracle, the FP32 path within 1e-5."""
    M, scales = 512, [512, 256, 128, 64, 32]
    frames = media.synth_video(33, M, M, 24, 250, step_var=1.0)
    taus = [1, 2, 3, 5, 8, 13]
    lambdas = media.log_lambdas(2, 512, 12)
    want, _ = O.ddm_run(frames, scales, taus, lambdas, estimator=O.EST_UNBIASED, chunk=8)
    got = {}
    for dft in (False, True):
        cfg = EngineConfig(frame_width=M, frame_height=M, scales=scales, taus=taus, lambdas=lambdas, chunk_frames=8,
                           estimator="unbiased", small_tile_dft=dft)
        with Engine(cfg) as eng:
            eng.submit(frames)
            eng.finalize()
            got[dft] = eng.isf()
    floor = 1e-9 * np.abs(want).max()
    for dft, rtol in ((False, 1e-5), (True, 1e-3)):
        err = np.abs(got[dft] - want) / np.maximum(np.abs(want), floor)
        assert np.all(np.abs(got[dft] - want) <= rtol * np.abs(want) + floor), (dft, float(err.max()))
    # the scales above 128 go through the FP32 FFT either way
    n_big = sum((M // s) ** 2 for s in (512, 256)) * len(lambdas) * len(taus)
    assert np.array_equal(got[True][:n_big], got[False][:n_big])
