"""CPU tests of the engine's host side: the C ABI exports, bit-exact masks, the reference
schedule, the ISF text format, .movie I/O and the synthetic generator."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from cuda_multiddm_b200 import media
from cuda_multiddm_b200._lib import LIB_PATH, SIGNATURES, lib
from oracle import oracle as O

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "ddm.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ddm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 25
    l = C.CDLL(str(LIB_PATH))
    missing = [n for n in names if not hasattr(l, n)]
    assert not missing, missing
    assert sorted(SIGNATURES) == names, "Python binding out of step with include/ddm.h"


@pytest.mark.parametrize("scale,tol,lambdas", [
    (2, 1.2, [1.0, 2.0]),
    (32, 1.2, [1.0, 2.0, 3.0, 4.0, 8.0, 16.0, 32.0, 64.0]),
    (64, 1.25, [2.0, 4.0, 8.0, 16.0, 32.0, 64.0]),
    (128, 1.05, [1.5, 2.0, 2.5, 3.3, 7.77, 12.0, 100.0, 1000.0]),
    (256, 1.37, [2.0, 3.0, 5.0, 9.0, 17.0, 33.0, 65.0, 129.0]),
    (512, 1.2, media.log_lambdas(2, 512, 30)),
])
def test_masks_bit_exact_to_oracle(scale, tol, lambdas):
    lam = np.asarray(lambdas, np.float32)
    m_ref, c_ref = O.masks(scale, lam, np.float32(tol))
    m = np.zeros((len(lam), scale, scale // 2 + 1), np.uint8)
    c = np.zeros(len(lam), np.int32)
    assert lib().ddm_build_masks(scale, lam.ctypes.data, len(lam), C.c_float(tol), m.ctypes.data,
                                 c.ctypes.data) == 0
    assert np.array_equal(c, c_ref)
    assert np.array_equal(m, m_ref)


def test_mask_boundaries_inclusive():
    # s = 64, lambda = 8: q = 8, q^2 = 64 -> (8, 0) has ratio exactly 1 (in);
    # tol 1.25: tol^2 = 1.5625 exactly; lambda = 16: q = 4, r^2 = 25 -> ratio 1.5625 (in)
    m, c = O.masks(64, [8.0, 16.0], np.float32(1.25))
    assert m[0, 0, 8] == 1 and m[0, 8, 0] == 1
    assert m[1, 0, 5] == 1 and m[1, 3, 4] == 1
    assert m[1, 0, 6] == 0


def _engine_schedule(N, C_, ms, taus, G=0):
    t = np.asarray(taus, np.int32)
    cap = N + C_ + 1
    A = np.zeros(cap, np.int32)
    B = np.zeros(cap * len(t), np.int32)
    ep = np.zeros(cap, np.int32)
    fr = np.zeros(1, np.int32)
    n = lib().ddm_compat_schedule(N, C_, int(ms), G, t.ctypes.data, len(t), cap, A.ctypes.data, B.ctypes.data,
                                  ep.ctypes.data, fr.ctypes.data)
    assert n >= 0
    return A[:n], B[:n * len(t)].reshape(n, len(t)), ep[:n], int(fr[0])


@pytest.mark.parametrize("N,C_,ms,G", [(40, 10, 1, 0), (40, 10, 0, 0), (29, 8, 1, 0), (29, 8, 0, 0), (10, 10, 1, 0),
                                       (15, 10, 1, 0), (7, 10, 1, 0), (36, 6, 1, 2), (36, 6, 0, 2), (19, 8, 0, 0),
                                       (200, 20, 1, 3), (61, 20, 1, 0)])
def test_schedule_matches_oracle(N, C_, ms, G):
    taus = sorted({1, 2, 3, C_ // 2, C_})
    A, B, ep, fr = _engine_schedule(N, C_, ms, taus, G)
    A2, B2, ep2, fr2 = O.compat_schedule(N, C_, bool(ms), taus, G)
    assert fr == fr2
    assert np.array_equal(A, A2) and np.array_equal(B, B2) and np.array_equal(ep, ep2)


def test_schedule_known_pairs():
    # multistream, N = 4 chunks of 10: interior pairs are (t, t+tau); the last chunk's
    # tail pairs with frame t + tau - 2C (the stale host buffer)
    A, B, _, fr = _engine_schedule(40, 10, 1, [1, 10])
    assert fr == 40
    assert list(A) == list(range(40))
    assert B[0].tolist() == [1, 10] and B[25].tolist() == [26, 35]
    assert B[39].tolist() == [20, 29] and B[31].tolist() == [32, 21]
    # single stream (-Z): chunk 1 is analysed twice, chunk 0 never
    A, B, _, _ = _engine_schedule(40, 10, 0, [1])
    assert A[:20].tolist() == list(range(10, 20)) * 2


def test_isf_text_format(tmp_path):
    isf = np.array([[1.0, 2.5e-7, 123456789.0], [0.0, 1 / 3, 4.0]])
    lam = np.array([2.0, 4.5], np.float32)
    taus = np.array([1, 2, 10], np.int32)
    p = tmp_path / "f"
    assert lib().ddm_write_isf_file(str(p).encode(), isf.ctypes.data, lam.ctypes.data, 2, taus.ctypes.data, 3,
                                    C.c_float(29.0)) == 0
    assert p.read_text() == "2 4.5 \n0.0344828 0.0689655 0.344828 \n1 2.5e-07 1.23457e+08 \n0 0.333333 4 \n"


def test_movie_roundtrip(tmp_path):
    fr = media.synth_video(5, 48, 32, 6, 10)
    p = tmp_path / "a.movie"
    media.write_movie(p, fr, frame_time_us=40000)
    h = C.c_void_p()
    from cuda_multiddm_b200._lib import MovieInfo
    info = MovieInfo()
    assert lib().ddm_movie_open(str(p).encode(), 2, C.byref(h), C.byref(info)) == 0
    assert (info.width, info.height, info.bytes_per_pixel) == (48, 32, 1)
    assert abs(info.fps - 25.0) < 1e-4
    out = np.zeros((4, 32, 48), np.uint8)
    assert lib().ddm_movie_read(h, out.ctypes.data, 4) == 0
    assert np.array_equal(out, fr[2:6])
    assert lib().ddm_movie_read(h, out.ctypes.data, 1) != 0  # past the end
    lib().ddm_movie_close(h)


def test_movie_u16_roundtrip(tmp_path):
    fr = media.synth_video(6, 16, 16, 3, 5, amplitude=2000, background=300, noise_sd=-1, max_value=4095)
    assert fr.dtype == np.uint16 and fr.max() <= 4095
    p = tmp_path / "b.movie"
    media.write_movie(p, fr)
    h = C.c_void_p()
    from cuda_multiddm_b200._lib import MovieInfo
    info = MovieInfo()
    assert lib().ddm_movie_open(str(p).encode(), 0, C.byref(h), C.byref(info)) == 0
    assert info.bytes_per_pixel == 2 and info.pixel_mode == 3
    out = np.zeros((3, 16, 16), np.uint16)
    assert lib().ddm_movie_read(h, out.ctypes.data, 3) == 0
    assert np.array_equal(out, fr)
    lib().ddm_movie_close(h)


def test_movie_reads_in_parallel_across_calls(tmp_path):
    """Frames are read with positioned reads from several threads: consecutive calls of 13 and
    27 frames return the file's frames in order, and a file cut inside a frame's data reports
    the record's offset."""
    fr = media.synth_video(7, 40, 24, 40, 10)
    p = tmp_path / "c.movie"
    media.write_movie(p, fr)
    from cuda_multiddm_b200._lib import MovieInfo
    h, info = C.c_void_p(), MovieInfo()
    assert lib().ddm_movie_open(str(p).encode(), 0, C.byref(h), C.byref(info)) == 0
    a = np.zeros((13, 24, 40), np.uint8)
    b = np.zeros((27, 24, 40), np.uint8)
    assert lib().ddm_movie_read(h, a.ctypes.data, 13) == 0
    assert lib().ddm_movie_read(h, b.ctypes.data, 27) == 0
    assert np.array_equal(np.concatenate([a, b]), fr)
    lib().ddm_movie_close(h)
    rec = 172 + 40 * 24
    q = tmp_path / "d.movie"
    q.write_bytes(p.read_bytes()[:10 * rec + 172 + 100])  # frame 10 cut inside its data
    assert lib().ddm_movie_open(str(q).encode(), 0, C.byref(h), C.byref(info)) == 0
    c = np.zeros((12, 24, 40), np.uint8)
    assert lib().ddm_movie_read(h, c.ctypes.data, 12) == 7  # DDM_ERR_IO
    assert f"Corrupted data at offset {10 * rec + 172}" in lib().ddm_last_error().decode()
    lib().ddm_movie_close(h)


def test_synth_deterministic_and_physical():
    a = media.synth_video(1001, 64, 64, 4, 20)
    b = media.synth_video(1001, 64, 64, 4, 20)
    c = media.synth_video(1002, 64, 64, 4, 20)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert a.dtype == np.uint8
    static = media.synth_video(3, 32, 32, 3, 5, step_var=0.0, noise_sd=0.0)
    assert np.array_equal(static[0], static[1]) and np.array_equal(static[1], static[2])


def test_log_lists():
    assert len(set(media.log_taus(1, 500, 64))) == 64 and media.log_taus(1, 500, 64)[-1] == 500
    assert len(set(media.log_taus(1, 300, 48))) == 48 and media.log_taus(1, 400, 64)[-1] == 400
    lam = media.log_lambdas(2, 512, 30)
    assert len(lam) == 30 and abs(lam[0] - 2) < 1e-6 and abs(lam[-1] - 512) < 1e-3


@pytest.mark.parametrize("idx", [4, 5])
def test_engine_masks_match_reference_hashes(idx):
    """The engine's own mask builder at s = 1024 and 2048 against the counts and FNV-1a hashes
    the reference's buildAzimuthMask produced (tests/golden/reference_outputs.json)."""
    import json
    from cases import MASK_CASES
    g = json.loads((ROOT / "tests" / "golden" / "reference_outputs.json").read_text())["masks"][idx]
    scale, tol, _ = MASK_CASES[idx]
    assert g["scale"] == scale
    lam = np.asarray(g["lambdas"], np.float32)
    m = np.zeros((len(lam), scale, scale // 2 + 1), np.uint8)
    c = np.zeros(len(lam), np.int32)
    assert lib().ddm_build_masks(scale, lam.ctypes.data, len(lam), C.c_float(tol), m.ctypes.data,
                                 c.ctypes.data) == 0
    assert c.tolist() == g["counts"]
    assert [str(O.fnv1a(m[q])) for q in range(len(lam))] == g["fnv"]


@pytest.mark.parametrize("kw", [
    dict(seed=3, width=96, height=64, frames=5, spots=40, step_var=2.0),
    dict(seed=9, width=64, height=64, frames=4, spots=30, amplitude=2000.0, background=300.0, noise_sd=-1.0,
         max_value=4095, step_var=0.4, step_var_b=4.0),
    dict(seed=1002, width=128, height=128, frames=3, spots=60, step_var=2.0),
])
def test_oracle_generator_bit_identical_to_product(kw):
    """The CPU arms make their input with the oracle's restatement of the generator (so they
    never load the product library); it must give the product generator's bytes exactly."""
    kw = dict(kw)
    args = (kw.pop("seed"), kw.pop("width"), kw.pop("height"), kw.pop("frames"), kw.pop("spots"))
    a = media.synth_video(*args, **kw)
    b = O.synth_video(*args, **kw)
    assert a.dtype == b.dtype and np.array_equal(a, b)
