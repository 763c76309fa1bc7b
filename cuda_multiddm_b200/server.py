"""Python face of the serving API (include/ddm.h, ddm_server_*): many DDM streams on one GPU
with admission by HBM footprint and continuous batching of their chunks."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import DDM_OK, ChunkResult, DDMError, ServerConfig, ServerStats, check, lib
from .engine import EngineConfig

DDM_ERR_BUSY = 8


class Server:
    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, max_streams: int = 0,
                 results_per_stream: int = 0):
        cfg = ServerConfig(device, hbm_budget_bytes, max_streams, results_per_stream)
        h = C.c_void_p()
        check(lib().ddm_server_open(C.byref(cfg), C.byref(h)))
        self._h = h
        self._isf: dict[int, np.ndarray] = {}  # per-stream result buffer
        self._cfgs: dict[int, EngineConfig] = {}
        self._res = ChunkResult()

    def close(self) -> None:
        if self._h:
            lib().ddm_server_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_stream(self, cfg: EngineConfig) -> int | None:
        """Stream id, or None when the server cannot admit it now (HBM budget or stream limit)."""
        c = cfg.to_c()
        sid = C.c_int()
        st = lib().ddm_server_add_stream(self._h, C.byref(c), C.byref(sid))
        if st == DDM_ERR_BUSY:
            return None
        check(st)
        M = max(cfg.scales)
        size = sum((M // s) ** 2 for s in cfg.scales) * len(cfg.lambdas) * len(cfg.taus)
        self._isf[sid.value] = np.zeros(size, np.float64)
        self._cfgs[sid.value] = cfg
        return sid.value

    def remove_stream(self, sid: int) -> None:
        check(lib().ddm_server_remove_stream(self._h, sid))
        self._isf.pop(sid, None)
        self._cfgs.pop(sid, None)

    def submit(self, sid: int, frames: np.ndarray) -> None:
        """Queue a chunk (copied)."""
        f = np.ascontiguousarray(frames)
        check(lib().ddm_server_submit(self._h, sid, f.ctypes.data, int(f.shape[0])))

    def submit_pinned(self, sid: int, ptr: int, count: int) -> None:
        """Queue a chunk from page-locked memory at `ptr` (e.g. a pinned torch tensor's
        data_ptr()) without copying; keep it unchanged until the chunk's result is polled."""
        check(lib().ddm_server_submit_pinned(self._h, sid, C.c_void_p(ptr), count))

    def step(self) -> int:
        n = C.c_int()
        check(lib().ddm_server_step(self._h, C.byref(n)))
        return n.value

    def poll(self, sid: int, copy: bool = True):
        """(ChunkResult fields as a dict, ISF array) of the stream's oldest finished chunk, or
        None. copy=False returns the stream's result buffer, overwritten by the next poll."""
        res, isf = self._res, self._isf[sid]
        st = lib().ddm_server_poll(self._h, sid, C.byref(res), isf.ctypes.data, isf.size)
        if st == 0:
            return None
        if st != 1:
            raise DDMError(st, lib().ddm_last_error().decode(errors="replace"))
        return {"chunk_index": res.chunk_index, "frames": res.frames, "submit_s": res.submit_s,
                "done_s": res.done_s, "latency_s": res.done_s - res.submit_s}, (isf.copy() if copy else isf)

    def wait(self) -> None:
        check(lib().ddm_server_wait(self._h))

    def clock(self) -> float:
        return float(lib().ddm_server_clock(self._h))

    def stats(self) -> dict:
        s = ServerStats()
        check(lib().ddm_server_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}


__all__ = ["Server", "DDM_ERR_BUSY", "DDM_OK"]
