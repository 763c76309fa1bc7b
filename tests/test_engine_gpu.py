"""GPU parity tests: the CUDA engine (through the C ABI) against the FP64 oracle.

Tolerance: ISF values agree with the FP64 oracle to 1e-5 relative per bin (FP32 FFT and
lag arithmetic; FP64 azimuthal reduction), with an absolute floor of 1e-9 of the largest
value of the (scale, tile) block for bins that are exactly zero in FP64.
"""
import numpy as np
import pytest

from cuda_multiddm_b200 import DDMError, Engine, EngineConfig, media
from cuda_multiddm_b200._lib import lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def assert_isf_close(got, want, scales, Q, T, rtol=RTOL):
    off = 0
    worst = 0.0
    ss = sorted(scales, reverse=True)
    for s in ss:
        size = (ss[0] // s) ** 2 * Q * T
        g, w = got[off:off + size], want[off:off + size]
        floor = 1e-9 * max(np.abs(w).max(), 1e-300)
        err = np.abs(g - w) / np.maximum(np.abs(w), floor)
        worst = max(worst, float(err.max()))
        assert np.all(np.abs(g - w) <= rtol * np.abs(w) + floor), (s, float(err.max()))
        off += size
    return worst


def engine_run(frames, scales, taus, lambdas, *, estimator, N=None, C=10, tol=1.2, multistream=True, G=0,
               x_off=0, y_off=0, pixel_mode="byte0", on_device=False, lag_batch=0):
    n, h, w = frames.shape[:3]
    bpp = 2 if frames.dtype == np.uint16 else 1
    raw = np.ascontiguousarray(frames).view(np.uint8).reshape(n, h, w * bpp)
    N = n if N is None else N
    cfg = EngineConfig(frame_width=w, frame_height=h, scales=scales, taus=taus, lambdas=lambdas, tolerance=tol,
                       chunk_frames=C, estimator=estimator, total_frames=N, multistream=multistream, dump_every=G,
                       bytes_per_pixel=bpp, pixel_mode=pixel_mode, x_offset=x_off, y_offset=y_off,
                       lag_batch_frames=lag_batch)
    with Engine(cfg) as eng:
        need = eng.info().frames_needed if estimator == "compat" else N
        if on_device:
            import torch
            t = torch.from_numpy(raw[:need].copy()).cuda()
            eng.submit(t)
            torch.cuda.synchronize()
        else:
            eng.submit(raw[:need])
        eng.finalize()
        return eng.isf(), eng.dumps(), eng.info()


@pytest.mark.parametrize("M,scales", [(256, [256, 128, 64, 32, 16, 8, 4, 2]), (2048, [2048, 1024])])
def test_spectra_match_fp64_fft(M, scales):
    rng = np.random.default_rng(M)
    frames = rng.integers(0, 256, size=(3, M, M), dtype=np.uint8)
    cfg = EngineConfig(frame_width=M, frame_height=M, scales=scales, taus=[1], lambdas=[2.0], chunk_frames=4)
    with Engine(cfg) as eng:
        eng.submit(frames)
        spec = eng.spectrum(1)
    off = 0
    for s in sorted(scales, reverse=True):
        tiles_side = M // s
        ref_tiles = O.extract(frames[1], 1, 0, 0, 0, M, s)
        for tile in [0, tiles_side * tiles_side - 1, (tiles_side * tiles_side) // 2]:
            ref = O.fft2_r2c(ref_tiles[tile])
            n = s * (s // 2 + 1)
            got = spec[off + tile * n: off + (tile + 1) * n].reshape(s, s // 2 + 1)
            scale = np.abs(ref).max()
            assert np.abs(got - ref).max() <= 2e-6 * scale, (s, tile)
            assert np.linalg.norm(got - ref) <= 1e-6 * np.linalg.norm(ref), (s, tile)
        off += tiles_side * tiles_side * s * (s // 2 + 1)


def _golden_cases():
    from cases import CASES
    return CASES


@pytest.mark.parametrize("case", _golden_cases(), ids=lambda c: c.name)
def test_compat_matches_oracle(case):
    frames = case.frames()
    if case.frame_offset:
        frames = frames[case.frame_offset:]
    kw = dict(estimator="compat", N=case.N, C=case.C, tol=case.tolerance, multistream=case.multistream,
              G=case.dump_every, x_off=case.x_off, y_off=case.y_off)
    isf, dumps, _ = engine_run(frames, case.scales, case.taus, case.lambdas, **kw)
    want, want_dumps = O.ddm_run(frames, case.scales, case.taus, case.lambdas, tol=case.tolerance, N=case.N,
                                 chunk=case.C, multistream=case.multistream, estimator=O.EST_COMPAT,
                                 dump_every=case.dump_every, x_off=case.x_off, y_off=case.y_off)
    Q, T = len(case.lambdas), len(case.taus)
    assert_isf_close(isf, want, case.scales, Q, T)
    assert len(dumps) == len(want_dumps)
    for d, wd in zip(dumps, want_dumps):
        assert_isf_close(d, wd, case.scales, Q, T)


def test_unbiased_multiscale_matches_oracle():
    frames = media.synth_video(77, 256, 256, 80, 150, step_var=1.0)
    scales = [256, 128, 64, 32]
    taus = [1, 2, 3, 5, 8, 13, 21, 34, 55]   # tau_max > chunk: only the unbiased path allows it
    lambdas = [2.0, 3.5, 6.0, 10.0, 17.0, 29.0, 50.0]
    isf, _, info = engine_run(frames, scales, taus, lambdas, estimator="unbiased", C=10)
    want, _ = O.ddm_run(frames, scales, taus, lambdas, estimator=O.EST_UNBIASED, chunk=10)
    assert_isf_close(isf, want, scales, len(lambdas), len(taus))
    # tau_max + one piece + one piece of FFT overlap + up to 31 frames held for a 32-frame launch
    assert info.ring_slots == 55 + 2 * 10 + 31


def test_u16_full_precision_matches_oracle():
    frames = media.synth_video(15, 64, 64, 24, 30, amplitude=2000, background=300, noise_sd=-1, max_value=4095)
    isf, _, _ = engine_run(frames, [64, 32], [1, 2, 4], [4.0, 8.0, 16.0], estimator="unbiased", C=8,
                           pixel_mode="u16")
    want, _ = O.ddm_run(frames, [64, 32], [1, 2, 4], [4.0, 8.0, 16.0], estimator=O.EST_UNBIASED, chunk=8,
                        pixmode=O.PIX_U16LE)
    assert_isf_close(isf, want, [64, 32], 3, 3)


def test_device_and_host_submission_identical():
    frames = media.synth_video(9, 160, 144, 30, 60)
    args = ([128, 64], [1, 2, 5, 11], [2.0, 5.0, 9.0, 20.0])
    kw = dict(estimator="unbiased", C=7, x_off=20, y_off=9)
    a, _, _ = engine_run(frames, *args, **kw)
    b, _, _ = engine_run(frames, *args, on_device=True, **kw)
    assert np.array_equal(a, b)


def test_two_pinned_buffers_refilled_after_wait_frames_copied():
    """A reader that alternates two pinned buffers, refilling each after
    ddm_wait_frames_copied(1) (the command line's file loop), gives the same ISF as
    submitting every chunk from its own buffer; `back` outside 0..7 is an argument error."""
    import torch
    frames = media.synth_video(19, 128, 128, 120, 60, step_var=1.0)
    kw = dict(frame_width=128, frame_height=128, scales=[128, 64], taus=[1, 2, 3, 7, 19, 40],
              lambdas=[3.0, 6.0, 12.0, 24.0], chunk_frames=20, estimator="unbiased")
    with Engine(EngineConfig(**kw)) as eng:
        for k in range(6):
            eng.submit(frames[20 * k:20 * k + 20].copy())
        eng.finalize()
        want = eng.isf()
    with Engine(EngineConfig(**kw)) as eng:
        bufs = [torch.empty((20, 128, 128), dtype=torch.uint8).pin_memory() for _ in range(2)]
        bufs[0].copy_(torch.from_numpy(frames[0:20]))
        for k in range(6):
            eng.submit(bufs[k % 2].data_ptr(), 20, False)
            if k < 5:
                eng.wait_frames_copied(1)
                bufs[(k + 1) % 2].copy_(torch.from_numpy(frames[20 * (k + 1):20 * (k + 2)]))
        eng.finalize()
        got = eng.isf()
        for bad in (-1, 8):
            with pytest.raises(DDMError):
                eng.wait_frames_copied(bad)
    assert np.array_equal(got, want)


def test_static_video_is_zero_and_intensity_scales_quadratically():
    static = np.repeat(media.synth_video(4, 64, 64, 1, 20, noise_sd=0.0), 12, axis=0)
    isf, _, _ = engine_run(static, [64, 32], [1, 3], [4.0, 8.0], estimator="unbiased", C=4)
    assert np.all(isf == 0.0)
    base = media.synth_video(5, 64, 64, 20, 20, amplitude=50, background=10, noise_sd=2.0, max_value=120)
    i1, _, _ = engine_run(base, [64], [1, 2, 3], [4.0, 8.0, 16.0], estimator="unbiased", C=5)
    i2, _, _ = engine_run((base.astype(np.uint16) * 2).astype(np.uint8), [64], [1, 2, 3], [4.0, 8.0, 16.0],
                          estimator="unbiased", C=5)
    np.testing.assert_allclose(i2, 4.0 * i1, rtol=1e-5)


def test_chunking_does_not_change_unbiased_result():
    frames = media.synth_video(21, 64, 64, 45, 30)
    args = ([64, 32], [1, 2, 4, 9, 17], [3.0, 6.0, 12.0])
    a, _, _ = engine_run(frames, *args, estimator="unbiased", C=5)
    b, _, _ = engine_run(frames, *args, estimator="unbiased", C=32)
    assert_isf_close(a, b, [64, 32], 3, 5, rtol=2e-6)


def test_full_lag_launches_match_oracle():
    """lag_batch_frames = 64 with 200 frames in 30-frame pieces: three full 64-frame lag
    launches (the two-lane kernel, windows that wrap its shared-memory ring and windows that
    do not) and an 8-frame launch at finalize; once against the oracle, once with a finalize
    after every piece (each flushes the held-back frames into smaller launches) against the
    first result."""
    frames = media.synth_video(41, 128, 128, 200, 80, step_var=1.0)
    scales, taus, lambdas = [128, 64], media.log_taus(1, 150, 24), [2.5, 5.0, 9.0, 17.0, 33.0]
    isf, _, info = engine_run(frames, scales, taus, lambdas, estimator="unbiased", C=30, lag_batch=64)
    want, _ = O.ddm_run(frames, scales, taus, lambdas, estimator=O.EST_UNBIASED, chunk=30)
    assert_isf_close(isf, want, scales, len(lambdas), len(taus))
    assert info.ring_slots == 150 + 2 * 30 + 63
    cfg = EngineConfig(frame_width=128, frame_height=128, scales=scales, taus=taus, lambdas=lambdas,
                       chunk_frames=30, estimator="unbiased", lag_batch_frames=64)
    with Engine(cfg) as eng:
        for c0 in range(0, 200, 30):
            eng.submit(frames[c0:c0 + 30])
            eng.finalize()
        live = eng.isf()
    assert_isf_close(live, isf, scales, len(lambdas), len(taus), rtol=2e-6)


def test_large_pair_table_two_ctas_per_sm_matches_oracle():
    """Taus 40 frames apart (48 of them, up to 1881) share no partner frames, so a 32-frame
    launch's union holds 1536 of them and its pair table needs over 8 KB: a lag CTA then takes
    more than 76.8 KB of shared memory, two fit on an SM instead of three, and the persistent
    grid (sized by the occupancy API) is two CTAs per SM walking the 518 element blocks of
    256^2 frames at scales 256 and 128. Early launches have partial windows (frames without
    all their partners yet), later ones full windows."""
    taus = [1 + 40 * i for i in range(48)]
    frames = media.synth_video(57, 256, 256, 1900, 200, step_var=1.0)
    scales, lambdas = [256, 128], [3.0, 8.0, 20.0, 60.0]
    # lower bound of a full 32-frame launch's shared memory (ring, barriers, accumulator ring,
    # flags, table with at least one run per group), against what three CTAs per SM allow
    J, T = 32, len(taus)
    union = len({w + j for w in (max(taus) - t for t in taus) for j in range(J)})
    groups = (union + 7) // 8
    table_ints = 5 + 64 + 3 * T + union + groups + 1 + groups
    smem = 64 * 1024 + 2 * 8 * 8 + 4 * 4 * 32 * 8 + 4 * (2 + table_ints)
    assert union == T * J and 3 * (smem + 1024) > 228 * 1024 and 2 * (smem + 1024) <= 228 * 1024
    isf, _, info = engine_run(frames, scales, taus, lambdas, estimator="unbiased", C=30)
    assert info.lag_batch_frames == 32
    want, _ = O.ddm_run(frames, scales, taus, lambdas, estimator=O.EST_UNBIASED, chunk=30)
    assert_isf_close(isf, want, scales, len(lambdas), len(taus))


def test_lag_batch_sizes_agree():
    """The same stream paired in launches of 1, 13, 30 and 64 frames gives the same ISF."""
    frames = media.synth_video(44, 64, 64, 90, 30, step_var=1.0)
    scales, taus, lambdas = [64, 32], [1, 2, 4, 8, 17, 33], [3.0, 6.0, 12.0]
    out = []
    for lb in (1, 13, 30, 64):
        cfg = EngineConfig(frame_width=64, frame_height=64, scales=scales, taus=taus, lambdas=lambdas,
                           chunk_frames=10, estimator="unbiased", lag_batch_frames=lb)
        with Engine(cfg) as eng:
            eng.submit(frames)
            eng.finalize()
            out.append(eng.isf())
    for o in out[1:]:
        assert_isf_close(o, out[0], scales, len(lambdas), len(taus), rtol=2e-6)


def test_fused_tau_runs_match_oracle():
    """Taus one frame apart are paired four entries per pass (one shared-memory load per
    partner for up to four register frames): 1..13 gives three fused runs and single
    entries around them. Launches of 4, 16, 30, 32 and 64 frames (the one- and two-lane
    kernels; the 120-frame stream in 10-frame pieces puts the runs' spans across the ring's
    wrap in some launches) against the oracle."""
    frames = media.synth_video(47, 64, 64, 120, 30, step_var=1.0)
    scales, taus, lambdas = [64, 32], list(range(1, 14)) + [20, 31], [3.0, 6.0, 12.0, 24.0]
    want, _ = O.ddm_run(frames, scales, taus, lambdas, estimator=O.EST_UNBIASED, chunk=10)
    for lb in (4, 16, 30, 32, 64):
        isf, _, _ = engine_run(frames, scales, taus, lambdas, estimator="unbiased", C=10, lag_batch=lb)
        assert_isf_close(isf, want, scales, len(lambdas), len(taus))


def test_fused_runs_over_many_element_blocks_match_oracle():
    """Fused tau runs with every CTA of the persistent lag grid walking several element blocks
    (512^2 frames, three scales: about 3,100 blocks of 128 elements for 444 CTAs, so the group
    counter runs on across blocks), in 32-frame and 64-frame (two-lane) launches."""
    frames = media.synth_video(49, 512, 512, 70, 1000, step_var=1.0)
    scales, taus, lambdas = [512, 256, 128], list(range(1, 14)) + [20, 31], [3.0, 6.0, 12.0, 24.0, 48.0]
    want, _ = O.ddm_run(frames, scales, taus, lambdas, estimator=O.EST_UNBIASED, chunk=10)
    for lb in (32, 64):
        isf, _, _ = engine_run(frames, scales, taus, lambdas, estimator="unbiased", C=10, lag_batch=lb)
        assert_isf_close(isf, want, scales, len(lambdas), len(taus))


def test_finalize_async_matches_finalize():
    """A live result per chunk through ddm_finalize_async, the next chunk submitted while the
    result is on its way, equals ddm_finalize + ddm_read_isf after every chunk bit for bit
    (pinned and pageable buffers); a short buffer is an argument error."""
    frames = media.synth_video(48, 128, 128, 90, 40, step_var=1.0)
    kw = dict(frame_width=128, frame_height=128, scales=[128, 64], taus=[1, 2, 3, 4, 7, 12, 25],
              lambdas=[3.0, 6.0, 12.0, 24.0], chunk_frames=15, estimator="unbiased")
    with Engine(EngineConfig(**kw)) as eng:
        want = []
        for c0 in range(0, 90, 15):
            eng.submit(frames[c0:c0 + 15])
            eng.finalize()
            want.append(eng.isf())
    for pinned in (True, False):
        with Engine(EngineConfig(**kw)) as eng:
            bufs = [eng.pinned_isf_buffer() if pinned else np.zeros(eng.isf_size) for _ in range(2)]
            got = []
            for k, c0 in enumerate(range(0, 90, 15)):
                eng.submit(frames[c0:c0 + 15])
                eng.finalize_async(bufs[k % 2])
                if k:  # finalize_async(k) waited for result k - 1
                    got.append(bufs[(k - 1) % 2].copy())
            eng.wait_isf()
            got.append(bufs[5 % 2].copy())
            eng.wait_isf()  # nothing pending: returns at once
            for g, w in zip(got, want):
                assert np.array_equal(g, w)
            with pytest.raises(ValueError):
                eng.finalize_async(np.zeros(eng.isf_size - 1))
            short = np.zeros(eng.isf_size)
            assert lib().ddm_finalize_async(eng._h, short.ctypes.data, eng.isf_size - 1) == 1  # DDM_ERR_INVALID_ARG


@pytest.mark.parametrize("depth", [3, 4, 8])
def test_finalize_async_depth_matches_finalize(depth):
    """With ddm_set_async_depth(d), d - 1 results stay in flight: finalize_async(k) returns
    once result k - d + 1 is in its buffer (the caller cycles d buffers), and every result
    equals ddm_finalize + ddm_read_isf after the same chunk bit for bit; the depth can change
    only with nothing in flight."""
    frames = media.synth_video(49, 128, 128, 150, 40, step_var=1.0)
    kw = dict(frame_width=128, frame_height=128, scales=[128, 64], taus=[1, 2, 3, 4, 7, 12, 25],
              lambdas=[3.0, 6.0, 12.0, 24.0], chunk_frames=15, estimator="unbiased")
    n = 150 // 15
    with Engine(EngineConfig(**kw)) as eng:
        want = []
        for c0 in range(0, 150, 15):
            eng.submit(frames[c0:c0 + 15])
            eng.finalize()
            want.append(eng.isf())
    with Engine(EngineConfig(**kw)) as eng:
        eng.set_async_depth(depth)
        bufs = [eng.pinned_isf_buffer() for _ in range(depth)]
        got = {}
        for k in range(n):
            eng.submit(frames[15 * k:15 * k + 15])
            eng.finalize_async(bufs[k % depth])
            if k - depth + 1 >= 0:
                got[k - depth + 1] = bufs[(k - depth + 1) % depth].copy()
            if k == 1:
                with pytest.raises(DDMError):  # results in flight
                    eng.set_async_depth(2)
        eng.wait_isf()
        for j in range(max(0, n - depth + 1), n):
            got[j] = bufs[j % depth].copy()
        assert sorted(got) == list(range(n))
        for j in range(n):
            assert np.array_equal(got[j], want[j]), j
        eng.set_async_depth(2)  # nothing in flight now
        for bad in (1, 9):
            with pytest.raises(DDMError):
                eng.set_async_depth(bad)


def test_compat_long_chunk_matches_oracle():
    """C = 100 with lag_batch_frames = 64: each reference iteration pairs 100 A-frames, run as
    a 64-frame launch and a 36-frame launch of the 64-frame kernel (the partial-window path);
    with the default, as launches of 32, 32, 32 and 4."""
    frames = media.synth_video(43, 64, 64, 200, 30, step_var=1.0)
    scales, taus, lambdas = [64, 32], [1, 2, 5, 13, 40, 99], [3.0, 6.0, 12.0, 24.0]
    want, _ = O.ddm_run(frames, scales, taus, lambdas, estimator=O.EST_COMPAT, chunk=100)
    for lb in (64, 0):
        isf, _, _ = engine_run(frames, scales, taus, lambdas, estimator="compat", C=100, lag_batch=lb)
        assert_isf_close(isf, want, scales, len(lambdas), len(taus))


def test_unaveraged_and_power_spectrum_match_oracle():
    """The -K and -A quantities through the C ABI: the per-wave-vector structure function
    before the azimuthal average (compat and unbiased) and |F / s^2|^2 of a frame."""
    frames = media.synth_video(47, 128, 128, 40, 60, step_var=1.0)
    scales, taus, lambdas = [128, 64, 32], [1, 3, 7], [3.0, 6.0, 12.0]
    for est, oest in (("unbiased", O.EST_UNBIASED), ("compat", O.EST_COMPAT)):
        cfg = EngineConfig(frame_width=128, frame_height=128, scales=scales, taus=taus, lambdas=lambdas,
                           chunk_frames=10, estimator=est, total_frames=40)
        with Engine(cfg) as eng:
            eng.submit(frames)
            eng.finalize()
            got = eng.unaveraged()
            power = eng.power_spectrum(39)
        _, want = O.ddm_run_unaveraged(frames, scales, taus, lambdas, chunk=10, estimator=oest)
        floor = 1e-9 * np.abs(want).max()
        assert np.all(np.abs(got - want) <= RTOL * np.abs(want) + floor), (est, float(np.abs(got - want).max()))
    off = 0
    for s in scales:
        px = O.extract(frames[39], 1, O.PIX_BYTE0, 0, 0, 128, s)
        for tile in range(px.shape[0]):
            want = (np.abs(O.fft2_r2c(px[tile])) / (s * s)).reshape(-1) ** 2
            n = want.size
            assert np.allclose(power[off:off + n], want, rtol=1e-5, atol=2e-6 * want.max()), (s, tile)
            off += n


def test_fine_scales_2048_matches_oracle():
    """The batched-fine-scales configuration's shape at a reduced frame count: 2048^2 frames,
    scales 2048 .. 32 (5461 tiles per frame), lambdas from 2 px to past the smallest tile."""
    frames = media.synth_video(1003, 2048, 2048, 16, 16000, step_var=1.0)
    scales = [2048, 1024, 512, 256, 128, 64, 32]
    taus, lambdas = [1, 2, 5, 11], media.log_lambdas(2, 512, 12)
    isf, _, _ = engine_run(frames, scales, taus, lambdas, estimator="unbiased", C=8)
    want, _ = O.ddm_run(frames, scales, taus, lambdas, estimator=O.EST_UNBIASED, chunk=8)
    assert_isf_close(isf, want, scales, len(lambdas), len(taus))


def test_high_bit_depth_2048_matches_oracle():
    """The high-bit-depth configuration's shape at a reduced frame count: 2048^2 uint16 holding
    12-bit values, Poisson shot noise, two populations (D = 0.2 and 2.0 px^2/frame), scales
    2048 .. 256, full 16-bit decoding."""
    frames = media.synth_video(1004, 2048, 2048, 12, 8000, amplitude=2000, background=300, step_var=0.4,
                               step_var_b=4.0, noise_sd=-1, max_value=4095)
    scales, taus, lambdas = [2048, 1024, 512, 256], [1, 3, 8], media.log_lambdas(2, 256, 10)
    isf, _, _ = engine_run(frames, scales, taus, lambdas, estimator="unbiased", C=6, pixel_mode="u16")
    want, _ = O.ddm_run(frames, scales, taus, lambdas, estimator=O.EST_UNBIASED, chunk=6, pixmode=O.PIX_U16LE)
    assert_isf_close(isf, want, scales, len(lambdas), len(taus))


def test_errors_are_status_codes():
    base = dict(frame_width=64, frame_height=64, taus=[1, 2], lambdas=[4.0], chunk_frames=4)
    with pytest.raises(DDMError) as e:
        Engine(EngineConfig(scales=[48], **base))
    assert "powers of two" in str(e.value)
    with pytest.raises(DDMError) as e:
        Engine(EngineConfig(scales=[128], **base))
    assert "smaller than actual image size" in str(e.value)
    with pytest.raises(DDMError) as e:
        Engine(EngineConfig(scales=[64], estimator="compat", total_frames=8, **{**base, "taus": [1, 9]}))
    assert "largest tau value" in str(e.value)
    with pytest.raises(DDMError) as e:
        Engine(EngineConfig(scales=[64], hbm_budget_bytes=1000, **base))
    assert e.value.status == 3
    with pytest.raises(DDMError) as e:
        Engine(EngineConfig(scales=[64], estimator="compat", total_frames=8,
                            **{**base, "lambdas": [100.0]}))
    assert "smallest scale" in str(e.value)
    # compat: frames beyond what the reference reads are refused; finalize without frames fails
    cfg = EngineConfig(scales=[64], estimator="compat", total_frames=8, **base)
    with Engine(cfg) as eng:
        with pytest.raises(DDMError) as e:
            eng.finalize()
        assert e.value.status == 5
        with pytest.raises(DDMError):
            eng.submit(np.zeros((9, 64, 64), np.uint8))


@pytest.mark.parametrize("per_tile", [False, True])
def test_kernel_launches_counted(per_tile):
    frames = media.synth_video(2, 64, 64, 8, 10)
    cfg = EngineConfig(frame_width=64, frame_height=64, scales=[64, 32], taus=[1, 2], lambdas=[4.0], chunk_frames=4,
                       estimator="unbiased", fft_per_tile=per_tile)
    with Engine(cfg) as eng:
        eng.submit(frames)
        eng.finalize()
        launches = eng.info().kernel_launches
    # per piece of 4 frames: a row-pass and a column-pass launch over both scales, or with
    # fft_per_tile one per-tile launch per scale (sides 32..128): two launches either way;
    # the 8 frames' lag pairs in one launch at finalize (launches take up to 32 frames); then
    # the two azimuthal stages
    assert launches == 2 * 2 + 1 + 2


def test_wait_timeout_is_reported_and_device_stays_usable():
    """The lag kernel's bounded waits: a pair table whose last window reaches a group of
    partner frames that is never copied (host-side fault injection) makes the pipeline waits
    run out after a short limit; the kernel returns a status instead of hanging, finalize
    reports DDM_ERR_CUDA, and the next engine on the device computes correct results."""
    from cuda_multiddm_b200._lib import FAULT_LAG_WAIT
    frames = media.synth_video(5, 64, 64, 20, 20, step_var=1.0)
    scales, taus, lambdas = [64, 32], [1, 2, 3, 5], [4.0, 8.0, 16.0]
    cfg = EngineConfig(frame_width=64, frame_height=64, scales=scales, taus=taus, lambdas=lambdas,
                       chunk_frames=10, estimator="unbiased")
    with Engine(cfg) as eng:
        eng.set_wait_limit(2_000_000)  # about 1 ms of SM clocks
        eng.inject_fault(FAULT_LAG_WAIT)
        eng.submit(frames)
        with pytest.raises(DDMError) as info:
            eng.finalize()
        assert info.value.status == 2 and "timed out" in str(info.value)
    with Engine(cfg) as eng:
        eng.submit(frames)
        eng.finalize()
        got = eng.isf()
    want, _ = O.ddm_run(frames, scales, taus, lambdas, estimator=O.EST_UNBIASED, chunk=10)
    assert_isf_close(got, want, scales, len(lambdas), len(taus))


@pytest.mark.parametrize("lag_batch", [16, 30, 32])
def test_wide_lag_geometry_matches_oracle(lag_batch):
    """The two-threads-per-element lag kernel (lag_geometry = 1) on a multi-scale, multi-tile
    case whose element blocks outnumber the persistent grid's CTAs, with fused tau runs, against
    the FP64 oracle; and against the one-thread-per-element kernel within FP32 rounding."""
    frames = media.synth_video(91, 512, 512, 70, 600, step_var=1.0)
    scales, taus = [512, 256, 128], [1, 2, 3, 4, 5, 6, 7, 8, 11, 17, 26, 40]
    lambdas = media.log_lambdas(2, 256, 9)
    want, _ = O.ddm_run(frames, scales, taus, lambdas, estimator=O.EST_UNBIASED, chunk=10)
    got = {}
    for geom in (0, 1):
        cfg = EngineConfig(frame_width=512, frame_height=512, scales=scales, taus=taus, lambdas=lambdas,
                           chunk_frames=10, estimator="unbiased", lag_batch_frames=lag_batch, lag_geometry=geom)
        with Engine(cfg) as eng:
            eng.submit(frames)
            eng.finalize()
            got[geom] = eng.isf()
        assert_isf_close(got[geom], want, scales, len(lambdas), len(taus))
    rel = np.abs(got[1] - got[0]) / np.maximum(np.abs(got[0]), 1e-9 * np.abs(got[0]).max())
    assert float(rel.max()) <= 2e-6


@pytest.mark.parametrize("pixel_mode", ["byte0", "u16"])
def test_per_tile_fft_equals_two_pass(pixel_mode):
    """Tiles of side 32..128 go through the two-pass FFT (default) or through one kernel that
    keeps each tile in shared memory between its passes (fft_per_tile): the same arithmetic,
    so the same spectra bit for bit; an ROI offset and several tiles per CTA included; and
    within 2e-6 of the FP64 FFT."""
    M = 256
    if pixel_mode == "u16":
        frames = media.synth_video(44, M + 8, M + 6, 3, 60, amplitude=2000, background=300, noise_sd=-1,
                                   max_value=4095)
    else:
        frames = np.random.default_rng(7).integers(0, 256, size=(3, M + 6, M + 8), dtype=np.uint8)
    n, h, w = frames.shape
    bpp = 2 if frames.dtype == np.uint16 else 1
    raw = np.ascontiguousarray(frames).view(np.uint8).reshape(n, h, w * bpp)
    scales = [256, 128, 64, 32, 16]
    spec = {}
    for per_tile in (False, True):
        cfg = EngineConfig(frame_width=w, frame_height=h, scales=scales, taus=[1], lambdas=[2.0], chunk_frames=4,
                           bytes_per_pixel=bpp, pixel_mode=pixel_mode, x_offset=3, y_offset=5,
                           fft_per_tile=per_tile)
        with Engine(cfg) as eng:
            assert eng.info().fft_per_tile == int(per_tile)
            eng.submit(raw)
            spec[per_tile] = [eng.spectrum(f) for f in range(n)]
    for f in range(n):
        assert np.array_equal(spec[False][f], spec[True][f])
    pix = O.PIX_U16LE if pixel_mode == "u16" else O.PIX_BYTE0
    off = 0
    for s in scales:
        tiles = O.extract(raw[1], bpp, pix, 3, 5, M, s)
        nel = s * (s // 2 + 1)
        for tile in (0, (M // s) ** 2 - 1):
            ref = O.fft2_r2c(tiles[tile])
            got = spec[True][1][off + tile * nel: off + (tile + 1) * nel].reshape(s, s // 2 + 1)
            assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max(), (s, tile)
        off += (M // s) ** 2 * nel
