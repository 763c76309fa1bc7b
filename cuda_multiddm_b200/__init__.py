"""Multi-scale DDM engine for NVIDIA B200 (sm_100a).

The computation lives in libddm_b200.so (C ABI: include/ddm.h), built in-tree by
`python -m cuda_multiddm_b200.build`; this package is a thin Python face over it.
"""
from ._lib import DDMError, lib  # noqa: F401
from .engine import Engine, EngineConfig, autotune, isf_blocks, run_ddm, tune_key  # noqa: F401
from .server import Server  # noqa: F401
from .media import (log_lambdas, log_taus, read_isf_file, synth_video, write_movie,  # noqa: F401
                    write_params)

__all__ = ["DDMError", "Engine", "EngineConfig", "Server", "run_ddm", "isf_blocks", "autotune", "tune_key", "synth_video", "write_movie",
           "write_params", "read_isf_file", "log_taus", "log_lambdas", "lib"]
