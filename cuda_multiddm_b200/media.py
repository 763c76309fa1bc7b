"""Inputs for the engine: seeded synthetic particle video, camera .movie files, and the
lambda / tau / scale parameter files of the reference's CLI (src/main.cpp:246-313)."""
from __future__ import annotations

import struct
from pathlib import Path
from typing import Sequence

import numpy as np

from ._lib import check, lib

MOVIE_MAGIC = 0x496D6554  # 'TemI' (src/video_reader.cpp:47)
IIDC_HEADER = 172         # src/video_reader.cpp:55


def synth_video(seed: int, width: int, height: int, frames: int, spots: int, *, spot_sigma: float = 2.0,
                amplitude: float = 120.0, background: float = 20.0, step_var: float = 0.5,
                step_var_b: float | None = None, noise_sd: float = 4.0, max_value: int = 255) -> np.ndarray:
    """Brownian Gaussian spots (ddm_synth_video): uint8 [frames, h, w] if max_value <= 255,
    else uint16. noise_sd < 0 selects Poisson shot noise."""
    dtype = np.uint8 if max_value <= 255 else np.uint16
    out = np.empty((frames, height, width), dtype)
    check(lib().ddm_synth_video(seed, width, height, frames, spots, spot_sigma, amplitude, background, step_var,
                                step_var if step_var_b is None else step_var_b, noise_sd, max_value,
                                out.ctypes.data))
    return out


def write_movie(path: str | Path, frames: np.ndarray, *, frame_time_us: int = 1_000_000,
                pixel_mode: int | None = None) -> None:
    """IIDC .movie file (src/video_reader.hpp:48-114): per frame a 172-byte packed header
    (common block, then i_timestamp at byte 48 and i_size_x / i_size_y at 64 / 68) and the
    pixel bytes. uint16 frames are written little-endian (pixel mode 3)."""
    frames = np.ascontiguousarray(frames)
    n, h, w = frames.shape
    if pixel_mode is None:
        pixel_mode = 1 if frames.dtype == np.uint8 else 3
    bpp = 1 if pixel_mode == 1 else 2
    data_len = w * h * bpp
    with open(path, "wb") as f:
        for i in range(n):
            hdr = bytearray(IIDC_HEADER)
            struct.pack_into("<6I", hdr, 0, MOVIE_MAGIC, 1, 1, pixel_mode, IIDC_HEADER, data_len)
            struct.pack_into("<Q", hdr, 48, i * frame_time_us)
            struct.pack_into("<4I", hdr, 56, w, h, w, h)
            f.write(hdr)
            f.write(frames[i].astype("<u2" if bpp == 2 else np.uint8).tobytes())


def log_taus(lo: int, hi: int, n: int) -> list[int]:
    """n unique, strictly increasing lags from lo to hi: tau_i = max(round(lo*(hi/lo)^(i/(n-1))),
    tau_{i-1} + 1)."""
    out: list[int] = []
    for i in range(n):
        v = int(round(lo * (hi / lo) ** (i / (n - 1)))) if n > 1 else lo
        if out and v <= out[-1]:
            v = out[-1] + 1
        out.append(v)
    return out


def log_lambdas(lo: float, hi: float, n: int) -> list[float]:
    """n log-spaced wavelengths, rounded to float32 (what the CLI's float parse gives)."""
    return [float(np.float32(lo * (hi / lo) ** (i / (n - 1)))) if n > 1 else float(np.float32(lo))
            for i in range(n)]


def write_params(directory: str | Path, scales: Sequence[int], taus: Sequence[int], lambdas: Sequence[float]):
    """The three whitespace-separated parameter files; lambdas with 9 significant digits so
    every parser reads back the same float32. Returns (scale, tau, lambda) paths."""
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    ps, pt, pl = d / "scale.txt", d / "tau.txt", d / "lambda.txt"
    ps.write_text("".join(f"{int(s)}\n" for s in scales))
    pt.write_text("".join(f"{int(t)}\n" for t in taus))
    pl.write_text("".join(f"{float(x):.9g}\n" for x in lambdas))
    return ps, pt, pl


def read_isf_file(path: str | Path):
    """Parse one ISF text file: (lambdas, tau labels, isf[lambda, tau])."""
    lines = Path(path).read_text().split("\n")
    lam = np.array([float(x) for x in lines[0].split()])
    tau = np.array([float(x) for x in lines[1].split()])
    rows = [np.array([float(x) for x in ln.split()]) for ln in lines[2:2 + len(lam)]]
    return lam, tau, np.array(rows)


def sig_digit_tolerance(values: np.ndarray, digits: int = 6) -> np.ndarray:
    """Half a unit in the last printed digit of %g-formatted values."""
    v = np.abs(np.asarray(values, dtype=np.float64))
    with np.errstate(divide="ignore"):
        e = np.floor(np.log10(np.where(v > 0, v, 1.0)))
    return np.where(v > 0, 0.5 * 10.0 ** (e - (digits - 1)), 0.0)
