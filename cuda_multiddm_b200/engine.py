"""Python face of the engine: the reference's runDDM (src/DDM.cu:268-292) as a function,
and the streaming engine behind it as a class, both over the C ABI (include/ddm.h)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from ._lib import (EST_COMPAT, EST_UNBIASED, PIX_BYTE0, PIX_U16LE, Config, DDMError, Info, check, lib)

__all__ = ["Engine", "EngineConfig", "run_ddm", "isf_blocks"]


@dataclass
class EngineConfig:
    frame_width: int
    frame_height: int
    scales: Sequence[int]
    taus: Sequence[int]
    lambdas: Sequence[float]
    tolerance: float = 1.2
    chunk_frames: int = 30
    estimator: str = "unbiased"        # "compat" (reference schedule) or "unbiased"
    total_frames: int = 0
    multistream: bool = True
    dump_every: int = 0
    bytes_per_pixel: int = 1
    pixel_mode: str = "byte0"          # "byte0" (reference) or "u16"
    x_offset: int = 0
    y_offset: int = 0
    hbm_budget_bytes: int = 0
    device: int = 0
    stream: int | None = None          # a cudaStream_t as an integer, or None
    lag_batch_frames: int = 0          # frames per lag launch (1..64; 0 = 32 unbiased, min(chunk_frames, 32) compat;
                                       # -1 = the value autotune() cached for this shape in $DDM_TUNE_CACHE)
    small_tile_dft: bool = False       # split-BF16 tensor-core DFT for tiles of side 32..128
    lag_geometry: int = 0              # lag kernel: 0 one thread per element, 1 two threads per element
    fft_group_frames: int = 0          # frames per FFT launch (0 = as many as 256 MB of spectra hold)
    fft_per_tile: bool = False         # True: tiles of side 32..128 through the per-tile FFT kernel
    _keep: list = field(default_factory=list, repr=False)

    def to_c(self) -> Config:
        sc = (C.c_int * len(self.scales))(*[int(s) for s in self.scales])
        ta = (C.c_int * len(self.taus))(*[int(t) for t in self.taus])
        la = (C.c_float * len(self.lambdas))(*[float(x) for x in self.lambdas])
        self._keep = [sc, ta, la]
        est = {"compat": EST_COMPAT, "unbiased": EST_UNBIASED}[self.estimator]
        pix = {"byte0": PIX_BYTE0, "u16": PIX_U16LE}[self.pixel_mode]
        return Config(self.frame_width, self.frame_height, self.bytes_per_pixel, pix, self.x_offset,
                      self.y_offset, sc, len(self.scales), ta, len(self.taus), la, len(self.lambdas),
                      C.c_float(self.tolerance), self.chunk_frames, est, int(bool(self.multistream)),
                      self.total_frames, self.dump_every, self.hbm_budget_bytes, self.device,
                      C.c_void_p(self.stream) if self.stream else None, self.lag_batch_frames,
                      int(bool(self.small_tile_dft)), int(self.lag_geometry), int(self.fft_group_frames),
                      int(bool(self.fft_per_tile)))


def tune_key(cfg: EngineConfig) -> str:
    """The shape key the autotuner's cache files results under."""
    c = cfg.to_c()
    n = lib().ddm_tune_key(C.byref(c), None, 0)
    buf = C.create_string_buffer(n + 1)
    lib().ddm_tune_key(C.byref(c), buf, n + 1)
    return buf.value.decode()


def autotune(cfg: EngineConfig, cache: str | None = None) -> dict:
    """Time the lag blocking x lag-kernel geometry candidates, then the FFT launch groups, on
    cfg's shape (unbiased estimator) and return {"lag_batch_frames", "lag_geometry",
    "fft_group_frames", "frames_per_s", "from_cache"}; with `cache`, look the shape up there
    first and store the result afterwards (engines opened with lag_batch_frames = -1 and
    DDM_TUNE_CACHE set to that file use it)."""
    from ._lib import Tuning
    c = cfg.to_c()
    t = Tuning()
    check(lib().ddm_autotune(C.byref(c), cache.encode() if cache else None, C.byref(t)))
    return {"lag_batch_frames": t.lag_batch_frames, "lag_geometry": t.lag_geometry,
            "fft_group_frames": t.fft_group_frames, "fft_per_tile": t.fft_per_tile, "frames_per_s": t.frames_per_s,
            "from_cache": bool(t.from_cache)}


def isf_blocks(isf: np.ndarray, scales: Sequence[int], n_lambda: int, n_tau: int) -> dict:
    """Split a flat ISF result into {scale: array[tile, lambda, tau]} (scales descending)."""
    out, off = {}, 0
    ss = sorted(scales, reverse=True)
    for s in ss:
        tiles = (ss[0] // s) ** 2
        size = tiles * n_lambda * n_tau
        out[s] = isf[off:off + size].reshape(tiles, n_lambda, n_tau)
        off += size
    return out


class Engine:
    """One multi-scale DDM stream on one GPU (ddm_open .. ddm_close)."""

    def __init__(self, cfg: EngineConfig):
        self.cfg = cfg
        self._h = C.c_void_p()
        ccfg = cfg.to_c()
        check(lib().ddm_open(C.byref(ccfg), C.byref(self._h)))
        n_s, n_t, n_l = len(cfg.scales), len(cfg.taus), len(cfg.lambdas)
        s = np.zeros(n_s, np.int32)
        t = np.zeros(n_t, np.int32)
        l = np.zeros(n_l, np.float32)
        check(lib().ddm_get_params(self._h, s.ctypes.data, t.ctypes.data, l.ctypes.data))
        self.scales, self.taus, self.lambdas = s, t, l

    # -- lifecycle -------------------------------------------------------------------
    def close(self) -> None:
        if self._h:
            lib().ddm_close(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- streaming -------------------------------------------------------------------
    def submit(self, frames, count: int | None = None, on_device: bool | None = None) -> None:
        """Submit frames: a numpy array (host, frame-major), a torch tensor (host or CUDA),
        or a raw pointer with `count` and `on_device`."""
        if isinstance(frames, int):
            if count is None or on_device is None:
                raise ValueError("raw pointers need count and on_device")
            check(lib().ddm_submit_frames(self._h, C.c_void_p(frames), count, int(on_device)))
            return
        if hasattr(frames, "data_ptr"):  # torch tensor
            n = frames.shape[0] if count is None else count
            check(lib().ddm_submit_frames(self._h, C.c_void_p(frames.data_ptr()), n, int(frames.is_cuda)))
            return
        arr = np.ascontiguousarray(frames)
        n = arr.shape[0] if count is None else count
        check(lib().ddm_submit_frames(self._h, arr.ctypes.data, n, 0))

    def finalize(self) -> None:
        check(lib().ddm_finalize(self._h))

    def finalize_async(self, out: np.ndarray) -> None:
        """Queue finalize and an asynchronous copy of the ISF into `out` (float64, at least
        isf_size; pinned memory, e.g. pinned_isf_buffer(), overlaps the copy with later
        submits). `out` holds the result after wait_isf() or the next finalize_async()."""
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.size < self.isf_size:
            raise ValueError("finalize_async needs a contiguous float64 buffer of isf_size values")
        check(lib().ddm_finalize_async(self._h, out.ctypes.data, out.size))

    def wait_isf(self) -> None:
        check(lib().ddm_wait_isf(self._h))

    def wait_frames_copied(self, back: int = 1) -> None:
        """Block until the host frames of the submit call `back` calls before the last have
        been copied to the device (their buffer may be refilled)."""
        check(lib().ddm_wait_frames_copied(self._h, int(back)))

    def set_async_depth(self, depth: int) -> None:
        """Keep depth - 1 finalize_async results in flight (2..8; default 2): each call then
        returns once the result of depth - 1 calls before is in its buffer, so the caller
        cycles `depth` buffers. Only with no result in flight (after wait_isf)."""
        check(lib().ddm_set_async_depth(self._h, int(depth)))

    def pinned_isf_buffer(self) -> np.ndarray:
        """A page-locked float64 buffer of isf_size values (the array keeps its pinned
        tensor alive)."""
        import torch
        return torch.empty(self.isf_size, dtype=torch.float64).pin_memory().numpy()

    def synchronize(self) -> None:
        check(lib().ddm_synchronize(self._h))

    def set_wait_limit(self, cycles: int) -> None:
        """Limit of every lag-pipeline wait in SM clock cycles (0 = the default, ~0.2 s)."""
        check(lib().ddm_set_wait_limit(self._h, int(cycles)))

    def inject_fault(self, fault: int) -> None:
        """Test hook: make the next lag launch's waits run out (FAULT_LAG_WAIT)."""
        check(lib().ddm_inject_fault(self._h, int(fault)))

    def reset(self) -> None:
        check(lib().ddm_reset_accumulators(self._h))

    # -- results ---------------------------------------------------------------------
    @property
    def isf_size(self) -> int:
        return int(lib().ddm_isf_size(self._h))

    def isf(self) -> np.ndarray:
        out = np.zeros(self.isf_size, np.float64)
        check(lib().ddm_read_isf(self._h, out.ctypes.data, out.size))
        return out

    def isf_by_scale(self) -> dict:
        return isf_blocks(self.isf(), self.scales, len(self.lambdas), len(self.taus))

    def dumps(self) -> list[np.ndarray]:
        res = []
        for i in range(lib().ddm_dump_count(self._h)):
            out = np.zeros(self.isf_size, np.float64)
            check(lib().ddm_read_dump(self._h, i, out.ctypes.data, out.size))
            res.append(out)
        return res

    def pixel_counts(self) -> np.ndarray:
        out = np.zeros((len(self.scales), len(self.lambdas)), np.int32)
        check(lib().ddm_get_pixel_counts(self._h, out.ctypes.data))
        return out

    def mask(self, scale_index: int) -> np.ndarray:
        s = int(self.scales[scale_index])
        out = np.zeros((len(self.lambdas), s, s // 2 + 1), np.uint8)
        check(lib().ddm_get_mask(self._h, scale_index, out.ctypes.data, out.size))
        return out

    @property
    def frame_elements(self) -> int:
        return int(lib().ddm_frame_elements(self._h))

    def spectrum(self, frame: int) -> np.ndarray:
        out = np.zeros(2 * self.frame_elements, np.float32)
        check(lib().ddm_read_spectrum(self._h, frame, out.ctypes.data, out.size))
        return out.view(np.complex64)

    def accumulators(self) -> np.ndarray:
        out = np.zeros(len(self.taus) * self.frame_elements, np.float64)
        check(lib().ddm_read_accumulators(self._h, out.ctypes.data, out.size))
        return out.reshape(len(self.taus), self.frame_elements)

    def power_spectrum(self, frame: int) -> np.ndarray:
        """|F / s^2|^2 per element of a frame still in the ring (the -A output)."""
        out = np.zeros(self.frame_elements, np.float32)
        check(lib().ddm_read_power_spectrum(self._h, frame, out.ctypes.data, out.size))
        return out

    def unaveraged(self) -> np.ndarray:
        """[tau, element] structure function before the azimuthal average (the -K output),
        after finalize()."""
        out = np.zeros(len(self.taus) * self.frame_elements, np.float64)
        check(lib().ddm_read_unaveraged(self._h, out.ctypes.data, out.size))
        return out.reshape(len(self.taus), self.frame_elements)

    def fit(self, fps: float = 0.0, um_per_px: float = 1.0, start: str = "data") -> dict:
        """ISF fits after finalize(): {"tile": [tiles, lambda, 6], "scale": [scales, lambda, 6]
        with (F, A, B, sigma_F, sigma_A, sigma_B), "tile_D": [tiles, 2], "scale_D": [scales, 2]
        with (D, sigma_D)}. Lag times in seconds (tau / fps) or frames (fps <= 0). start: "data"
        (read off each curve) or "script" (the reference script's fixed p0)."""
        nt, S, Q = int(lib().ddm_tile_count(self._h)), len(self.scales), len(self.lambdas)
        tile, scale = np.zeros((nt, Q, 6)), np.zeros((S, Q, 6))
        tile_d, scale_d = np.zeros((nt, 2)), np.zeros((S, 2))
        st = {"data": 0, "script": 1}[start]
        check(lib().ddm_fit_isf(self._h, C.c_float(fps), C.c_double(um_per_px), st, tile.ctypes.data,
                                scale.ctypes.data, tile_d.ctypes.data, scale_d.ctypes.data))
        return {"tile": tile, "scale": scale, "tile_D": tile_d, "scale_D": scale_d}

    def set_timing(self, enabled: bool = True) -> None:
        check(lib().ddm_set_timing(self._h, int(enabled)))

    def kernel_times(self) -> dict:
        """{group: (device ms, launches)} since the last call; groups fft, lag, azimuth."""
        return {g: v[:2] for g, v in self.kernel_stats().items()}

    def kernel_stats(self) -> dict:
        """{group: (device ms, launches, compulsory DRAM bytes)} since the last call."""
        ms = np.zeros(3, np.float64)
        n = np.zeros(3, np.int64)
        b = np.zeros(3, np.float64)
        check(lib().ddm_kernel_stats(self._h, ms.ctypes.data, n.ctypes.data, b.ctypes.data))
        return {g: (float(ms[i]), int(n[i]), float(b[i])) for i, g in enumerate(("fft", "lag", "azimuth"))}

    def info(self) -> Info:
        inf = Info()
        check(lib().ddm_get_info(self._h, C.byref(inf)))
        return inf


def run_ddm(frames: np.ndarray, scales, taus, lambdas, *, tolerance: float = 1.2, chunk_frames: int = 30,
            estimator: str = "compat", total_frames: int | None = None, multistream: bool = True,
            x_offset: int = 0, y_offset: int = 0, pixel_mode: str = "byte0", dump_every: int = 0,
            device: int = 0):
    """The reference's runDDM on in-memory frames [n, h, w] (uint8) or [n, h, w*2]
    bytes / [n, h, w] uint16: returns (isf dict {scale: [tile, lambda, tau]}, dumps)."""
    frames = np.ascontiguousarray(frames)
    if frames.dtype == np.uint16:
        n, h, w = frames.shape
        bpp, raw = 2, frames.view(np.uint8).reshape(n, h, w * 2)
    else:
        n, h, w = frames.shape
        bpp, raw = 1, frames
    N = n if total_frames is None else total_frames
    cfg = EngineConfig(frame_width=w, frame_height=h, scales=scales, taus=taus, lambdas=lambdas,
                       tolerance=tolerance, chunk_frames=chunk_frames, estimator=estimator, total_frames=N,
                       multistream=multistream, dump_every=dump_every, bytes_per_pixel=bpp,
                       pixel_mode=pixel_mode if bpp == 2 else "byte0", x_offset=x_offset, y_offset=y_offset,
                       device=device)
    with Engine(cfg) as eng:
        need = eng.info().frames_needed if estimator == "compat" else N
        if need > raw.shape[0]:
            raise DDMError(5, f"the schedule reads {need} frames, {raw.shape[0]} given")
        eng.submit(raw[:need])
        eng.finalize()
        isf = eng.isf_by_scale()
        dumps = [isf_blocks(d, eng.scales, len(eng.lambdas), len(eng.taus)) for d in eng.dumps()]
    return isf, dumps
