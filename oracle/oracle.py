"""ctypes binding of the FP64 C oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Only the tests, the smoke check and the CPU-baseline leg of the benchmark use this module,
as the checker; the product never imports it. Build with `make -C oracle`.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path
from typing import Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_BIN = HERE / "_ref" / "ddm_ref"

EST_COMPAT, EST_UNBIASED = 0, 1
PIX_BYTE0, PIX_U16LE = 0, 1
LABEL_UNINIT = -1

_lib = None


def build() -> None:
    """Compile liboracle.so (and the reference program when its sources exist here)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle", "ref-if-present"], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        src = HERE / "ddm_oracle.c"
        if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
            subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
        l = C.CDLL(str(LIB_PATH))
        P = C.c_void_p
        l.orc_q_radius.restype = C.c_float
        l.orc_q_radius.argtypes = [C.c_int, C.c_float]
        l.orc_mask_build.restype = C.c_int
        l.orc_mask_build.argtypes = [C.c_int, P, C.c_int, C.c_float, P, P]
        l.orc_extract.restype = None
        l.orc_extract.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P]
        l.orc_fft2_r2c.restype = None
        l.orc_fft2_r2c.argtypes = [P, C.c_int, P]
        l.orc_compat_schedule.restype = C.c_int
        l.orc_compat_schedule.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_int, C.c_int, P, P, P, P]
        l.orc_ddm_run.restype = C.c_int
        l.orc_ddm_run.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_int,
                                  P, C.c_int, P, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                  P, P, C.c_int]
        l.orc_ddm_run_unaveraged.restype = C.c_int
        l.orc_ddm_run_unaveraged.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P,
                                             C.c_int, P, C.c_int, P, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int,
                                             C.c_int, P, P]
        l.orc_isf_size.restype = C.c_long
        l.orc_isf_size.argtypes = [P, C.c_int, C.c_int, C.c_int]
        l.orc_azimuthal.restype = None
        l.orc_azimuthal.argtypes = [P, C.c_int, C.c_int, C.c_int, P, C.c_int, C.c_float, P, P]
        l.orc_bench_steady.restype = C.c_double
        l.orc_bench_steady.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P, C.c_int, P, C.c_int,
                                       C.c_int, C.c_int, C.c_int]
        l.orc_fnv1a.restype = C.c_uint64
        l.orc_fnv1a.argtypes = [P, C.c_long]
        l.orc_synth_video.restype = C.c_int
        l.orc_synth_video.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                      C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, P]
        _lib = l
    return _lib


def _i32(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.int32))


def _f32(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.float32))


def q_radius(scale: int, lam: float) -> float:
    return float(lib().orc_q_radius(scale, lam))


def masks(scale: int, lambdas: Sequence[float], tol: float):
    """(mask[q, ky, kx] uint8, counts[q]) as buildAzimuthMask makes them."""
    lam = _f32(lambdas)
    m = np.zeros((len(lam), scale, scale // 2 + 1), np.uint8)
    cnt = np.zeros(len(lam), np.int32)
    lib().orc_mask_build(scale, lam.ctypes.data, len(lam), C.c_float(tol), m.ctypes.data, cnt.ctypes.data)
    return m, cnt


def fft2_r2c(tile: np.ndarray) -> np.ndarray:
    t = np.ascontiguousarray(tile, dtype=np.float64)
    s = t.shape[0]
    out = np.zeros((s, s // 2 + 1, 2), np.float64)
    lib().orc_fft2_r2c(t.ctypes.data, s, out.ctypes.data)
    return out[..., 0] + 1j * out[..., 1]


def extract(frame: np.ndarray, bpp: int, pixmode: int, x_off: int, y_off: int, main_scale: int,
            scale: int) -> np.ndarray:
    f = np.ascontiguousarray(frame, dtype=np.uint8)
    h = f.shape[0]
    w = f.shape[1] // bpp
    tiles = (main_scale // scale) ** 2
    out = np.zeros((tiles, scale, scale), np.float64)
    lib().orc_extract(f.ctypes.data, w, h, bpp, pixmode, x_off, y_off, main_scale, scale, out.ctypes.data)
    return out


def compat_schedule(N: int, C_: int, multistream: bool, taus: Sequence[int], dump_every: int = 0):
    """(A[calls], B[calls, T], epoch[calls], frames_read) of the reference's chunk loop."""
    t = _i32(taus)
    cap = N + C_ + 1
    A = np.zeros(cap, np.int32)
    B = np.zeros((cap, len(t)), np.int32)
    ep = np.zeros(cap, np.int32)
    fr = np.zeros(1, np.int32)
    n = lib().orc_compat_schedule(N, C_, int(multistream), dump_every, t.ctypes.data, len(t), cap, A.ctypes.data,
                                  B.ctypes.data, ep.ctypes.data, fr.ctypes.data)
    if n < 0:
        raise RuntimeError("orc_compat_schedule failed")
    return A[:n], B[:n], ep[:n], int(fr[0])


def isf_size(scales, n_lambda, n_tau) -> int:
    s = _i32(scales)
    return int(lib().orc_isf_size(s.ctypes.data, len(s), n_lambda, n_tau))


def ddm_run(frames: np.ndarray, scales, taus, lambdas, *, tol: float = 1.2, N: int | None = None, chunk: int = 30,
            multistream: bool = True, estimator: int = EST_COMPAT, dump_every: int = 0, x_off: int = 0,
            y_off: int = 0, pixmode: int = PIX_BYTE0, max_dumps: int = 16):
    """Whole path on uint8 frames [n, h, w] (1 byte per pixel) or uint16 frames [n, h, w]
    (2 bytes per pixel, little-endian). Returns (isf flat array, list of dump arrays)."""
    fr = np.ascontiguousarray(frames)
    n, h, w = fr.shape
    bpp = 2 if fr.dtype == np.uint16 else 1
    raw = fr.view(np.uint8).reshape(n, h, w * bpp)
    return ddm_run_bpp(raw, w, h, bpp, scales, taus, lambdas, tol=tol, N=N, chunk=chunk, multistream=multistream,
                       estimator=estimator, dump_every=dump_every, x_off=x_off, y_off=y_off, pixmode=pixmode,
                       max_dumps=max_dumps)


def ddm_run_bpp(frames_bytes: np.ndarray, w: int, h: int, bpp: int, scales, taus, lambdas, **kw):
    """As ddm_run, for raw multi-byte pixels [n, h, w*bpp] (explicit width and bpp)."""
    fr = np.ascontiguousarray(frames_bytes, dtype=np.uint8)
    s = _i32(scales)
    t = _i32(taus)
    l = _f32(lambdas)
    size = isf_size(s, len(l), len(t))
    isf = np.zeros(size, np.float64)
    max_dumps = kw.get("max_dumps", 16)
    dumps = np.zeros((max_dumps, size), np.float64)
    n = fr.shape[0]
    N = kw.get("N")
    N = n if N is None else N
    nd = lib().orc_ddm_run(fr.ctypes.data, n, w, h, bpp, kw.get("pixmode", PIX_BYTE0), kw.get("x_off", 0),
                           kw.get("y_off", 0), s.ctypes.data, len(s), t.ctypes.data, len(t), l.ctypes.data, len(l),
                           C.c_float(kw.get("tol", 1.2)), N, kw.get("chunk", 30), int(kw.get("multistream", True)),
                           kw.get("estimator", EST_COMPAT), kw.get("dump_every", 0), isf.ctypes.data,
                           dumps.ctypes.data, max_dumps)
    if nd < 0:
        raise RuntimeError(f"orc_ddm_run failed with {nd}")
    return isf, [dumps[i] for i in range(nd)]


def ddm_run_unaveraged(frames: np.ndarray, scales, taus, lambdas, *, tol: float = 1.2, chunk: int = 30,
                       estimator: int = EST_UNBIASED, multistream: bool = True):
    """uint8 frames [n, h, w] -> (isf, unaveraged [T, E]): the corrected -K output, 2 * mean
    |dF|^2 / s^4 per spectrum element (all scales concatenated, each [tile][ky][kx])."""
    fr = np.ascontiguousarray(frames, dtype=np.uint8)
    n, h, w = fr.shape
    s = _i32(scales)
    t = _i32(taus)
    l = _f32(lambdas)
    M = int(max(scales))
    E = sum((M // x) ** 2 * x * (x // 2 + 1) for x in scales)
    isf = np.zeros(isf_size(s, len(l), len(t)), np.float64)
    unav = np.zeros((len(t), E), np.float64)
    st = lib().orc_ddm_run_unaveraged(fr.ctypes.data, n, w, h, 1, PIX_BYTE0, 0, 0, s.ctypes.data, len(s),
                                      t.ctypes.data, len(t), l.ctypes.data, len(l), C.c_float(tol), n, chunk,
                                      int(multistream), estimator, isf.ctypes.data, unav.ctypes.data)
    if st < 0:
        raise RuntimeError(f"orc_ddm_run_unaveraged failed with {st}")
    return isf, unav


def azimuthal(acc: np.ndarray, scale: int, tiles: int, lambdas, tol: float, norm) -> np.ndarray:
    a = np.ascontiguousarray(acc, dtype=np.float64)
    T = a.shape[0]
    l = _f32(lambdas)
    nrm = np.ascontiguousarray(norm, dtype=np.float64)
    out = np.zeros((tiles, len(l), T), np.float64)
    lib().orc_azimuthal(a.ctypes.data, scale, tiles, T, l.ctypes.data, len(l), C.c_float(tol), nrm.ctypes.data,
                        out.ctypes.data)
    return out


def bench_steady(frames: np.ndarray, scales, taus, timed_frames: int, threads: int = 0, warm_frames: int = 0,
                 pixmode: int = PIX_BYTE0) -> float:
    """Seconds the FP64 path takes for `timed_frames` steady-state frames (after
    `warm_frames` untimed ones); uint8 or uint16 (little-endian) frames [n, h, w]."""
    fr = np.ascontiguousarray(frames)
    n, h, w = fr.shape
    bpp = 2 if fr.dtype == np.uint16 else 1
    raw = fr.view(np.uint8)
    s = _i32(scales)
    t = _i32(taus)
    r = float(lib().orc_bench_steady(raw.ctypes.data, n, w, h, bpp, pixmode, s.ctypes.data, len(s), t.ctypes.data,
                                     len(t), warm_frames, timed_frames, threads))
    if r < 0:
        raise MemoryError("orc_bench_steady: host allocation failed")
    return r


def fnv1a(data: np.ndarray) -> int:
    """64-bit FNV-1a over the bytes of `data` (C order)."""
    b = np.ascontiguousarray(data).view(np.uint8)
    return int(lib().orc_fnv1a(b.ctypes.data, b.size))


def synth_video(seed: int, width: int, height: int, frames: int, spots: int, *, spot_sigma: float = 2.0,
                amplitude: float = 120.0, background: float = 20.0, step_var: float = 0.5,
                step_var_b: float | None = None, noise_sd: float = 4.0, max_value: int = 255) -> np.ndarray:
    """The product generator's video (same arguments and defaults as
    cuda_multiddm_b200.media.synth_video), made by the oracle's own restatement."""
    dt = np.uint8 if max_value <= 255 else np.uint16
    out = np.zeros((frames, height, width), dt)
    st = lib().orc_synth_video(seed, width, height, frames, spots, spot_sigma, amplitude, background, step_var,
                               step_var if step_var_b is None else step_var_b, noise_sd, max_value,
                               out.ctypes.data)
    if st != 0:
        raise RuntimeError(f"orc_synth_video failed with {st}")
    return out
