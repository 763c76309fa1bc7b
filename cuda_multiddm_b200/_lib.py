"""ctypes binding of include/ddm.h (libddm_b200.so, built in-tree).

The library is loaded from this package directory only; a missing or stale build is an
error, never a silent fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libddm_b200.so"

DDM_OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory", 4: "invalid state",
          5: "frames missing", 6: "no suitable CUDA device", 7: "I/O error", 8: "busy"}

PIX_BYTE0, PIX_U16LE = 0, 1
FAULT_NONE, FAULT_LAG_WAIT = 0, 1
EST_COMPAT, EST_UNBIASED = 0, 1


class DDMError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class Config(C.Structure):
    _fields_ = [
        ("frame_width", C.c_int), ("frame_height", C.c_int), ("bytes_per_pixel", C.c_int),
        ("pixel_mode", C.c_int), ("x_offset", C.c_int), ("y_offset", C.c_int),
        ("scales", C.POINTER(C.c_int)), ("scale_count", C.c_int),
        ("taus", C.POINTER(C.c_int)), ("tau_count", C.c_int),
        ("lambdas", C.POINTER(C.c_float)), ("lambda_count", C.c_int),
        ("tolerance", C.c_float), ("chunk_frames", C.c_int), ("estimator", C.c_int),
        ("multistream", C.c_int), ("total_frames", C.c_int), ("dump_every", C.c_int),
        ("hbm_budget_bytes", C.c_size_t), ("device", C.c_int), ("stream", C.c_void_p),
        ("lag_batch_frames", C.c_int), ("small_tile_dft", C.c_int), ("lag_geometry", C.c_int),
        ("fft_group_frames", C.c_int), ("fft_per_tile", C.c_int),
    ]


class Info(C.Structure):
    _fields_ = [("frames_submitted", C.c_long), ("ring_slots", C.c_int), ("device_bytes", C.c_size_t),
                ("kernel_launches", C.c_long), ("stream", C.c_void_p), ("frames_needed", C.c_long),
                ("lag_batch_frames", C.c_int), ("lag_geometry", C.c_int), ("fft_group_frames", C.c_int),
                ("fft_per_tile", C.c_int)]


class Tuning(C.Structure):
    _fields_ = [("lag_batch_frames", C.c_int), ("frames_per_s", C.c_double), ("from_cache", C.c_int),
                ("lag_geometry", C.c_int), ("fft_group_frames", C.c_int),
                ("fft_per_tile", C.c_int)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget_bytes", C.c_size_t), ("max_streams", C.c_int),
                ("results_per_stream", C.c_int)]


class ChunkResult(C.Structure):
    _fields_ = [("chunk_index", C.c_long), ("frames", C.c_long), ("submit_s", C.c_double), ("done_s", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("streams", C.c_int), ("device_bytes", C.c_size_t), ("budget_bytes", C.c_size_t),
                ("batched_launches", C.c_long), ("chunks_pending", C.c_long), ("steps", C.c_long),
                ("step_host_s", C.c_double), ("gpu_s", C.c_double)]


class MovieInfo(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("bytes_per_pixel", C.c_int), ("fps", C.c_float),
                ("camera_type", C.c_int), ("pixel_mode", C.c_int)]


# name -> (restype, argtypes); every symbol include/ddm.h declares
SIGNATURES = {
    "ddm_open": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "ddm_close": (C.c_int, [C.c_void_p]),
    "ddm_submit_frames": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "ddm_finalize": (C.c_int, [C.c_void_p]),
    "ddm_isf_size": (C.c_long, [C.c_void_p]),
    "ddm_read_isf": (C.c_int, [C.c_void_p, C.c_void_p, C.c_long]),
    "ddm_finalize_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_long]),
    "ddm_autotune": (C.c_int, [C.POINTER(Config), C.c_char_p, C.POINTER(Tuning)]),
    "ddm_tune_key": (C.c_long, [C.POINTER(Config), C.c_char_p, C.c_long]),
    "ddm_wait_isf": (C.c_int, [C.c_void_p]),
    "ddm_set_async_depth": (C.c_int, [C.c_void_p, C.c_int]),
    "ddm_wait_frames_copied": (C.c_int, [C.c_void_p, C.c_int]),
    "ddm_dump_count": (C.c_int, [C.c_void_p]),
    "ddm_read_dump": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_long]),
    "ddm_reset_accumulators": (C.c_int, [C.c_void_p]),
    "ddm_synchronize": (C.c_int, [C.c_void_p]),
    "ddm_get_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ddm_get_pixel_counts": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ddm_get_mask": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_long]),
    "ddm_frame_elements": (C.c_long, [C.c_void_p]),
    "ddm_read_spectrum": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_long]),
    "ddm_read_accumulators": (C.c_int, [C.c_void_p, C.c_void_p, C.c_long]),
    "ddm_read_power_spectrum": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_long]),
    "ddm_read_unaveraged": (C.c_int, [C.c_void_p, C.c_void_p, C.c_long]),
    "ddm_tile_count": (C.c_long, [C.c_void_p]),
    "ddm_server_open": (C.c_int, [C.POINTER(ServerConfig), C.POINTER(C.c_void_p)]),
    "ddm_server_close": (C.c_int, [C.c_void_p]),
    "ddm_server_add_stream": (C.c_int, [C.c_void_p, C.POINTER(Config), C.POINTER(C.c_int)]),
    "ddm_server_remove_stream": (C.c_int, [C.c_void_p, C.c_int]),
    "ddm_server_submit": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "ddm_server_submit_pinned": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "ddm_server_step": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "ddm_server_poll": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(ChunkResult), C.c_void_p, C.c_long]),
    "ddm_server_wait": (C.c_int, [C.c_void_p]),
    "ddm_server_clock": (C.c_double, [C.c_void_p]),
    "ddm_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
    "ddm_fit_isf": (C.c_int, [C.c_void_p, C.c_float, C.c_double, C.c_int, C.c_void_p, C.c_void_p,
                              C.c_void_p, C.c_void_p]),
    "ddm_get_info": (C.c_int, [C.c_void_p, C.POINTER(Info)]),
    "ddm_set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "ddm_kernel_times": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "ddm_kernel_stats": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ddm_build_masks": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_float, C.c_void_p, C.c_void_p]),
    "ddm_compat_schedule": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ddm_lag_accumulate_static": (C.c_int, [C.c_void_p, C.c_int, C.c_longlong, C.c_void_p, C.c_void_p, C.c_int,
                                            C.c_void_p, C.c_int, C.c_void_p]),
    "ddm_set_wait_limit": (C.c_int, [C.c_void_p, C.c_longlong]),
    "ddm_inject_fault": (C.c_int, [C.c_void_p, C.c_int]),
    "ddm_host_alloc": (C.c_void_p, [C.c_size_t]),
    "ddm_host_free": (None, [C.c_void_p]),
    "ddm_last_error": (C.c_char_p, []),
    "ddm_status_string": (C.c_char_p, [C.c_int]),
    "ddm_write_isf_file": (C.c_int, [C.c_char_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_float]),
    "ddm_synth_video": (C.c_int, [C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                  C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_void_p]),
    "ddm_movie_open": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(MovieInfo)]),
    "ddm_movie_read": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "ddm_movie_close": (C.c_int, [C.c_void_p]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded engine library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m cuda_multiddm_b200.build`")
        l = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def check(status: int) -> None:
    if status != DDM_OK:
        raise DDMError(status, lib().ddm_last_error().decode(errors="replace"))
