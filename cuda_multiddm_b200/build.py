"""Build the engine library (libddm_b200.so) and the ddm CLI in-tree, for sm_100a.

    python -m cuda_multiddm_b200.build          # incremental
    python -m cuda_multiddm_b200.build --force  # rebuild everything

nvcc cross-compiles without a GPU, so this runs on any machine with CUDA 12.9.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libddm_b200.so"
CLI = PKG / "ddm"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off",
              f"-I{ROOT / 'include'}", f"-I{CSRC}"]

SOURCES = ["engine.cu", "server.cu", "noalloc.cu", "host.cpp", "synth.cpp", "movie.cpp", "tune.cpp"]


def _nvcc() -> str:
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        raise RuntimeError("nvcc not found")
    return nvcc


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:4])} ...")


def build(force: bool = False, verbose: bool = False) -> Path:
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.hpp")) + [ROOT / "include" / "ddm.h"]
    objs = []
    for src in SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s, *headers]):
            cmd = [nvcc, *NVCC_FLAGS, "-c", str(s), "-o", str(o)]
            if src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if verbose else []
            else:
                cmd = [nvcc, *NVCC_FLAGS, "-x", "c++", "-c", str(s), "-o", str(o)]
            _run(cmd)
    if force or _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-Xcompiler", "-fopenmp", "-o", str(LIB), *map(str, objs), "-lgomp"])
    cli_src = CSRC / "ddm_cli.cpp"
    if force or _stale(CLI, [cli_src, LIB, ROOT / "include" / "ddm.h"]):
        _run(["g++", "-O2", "-std=c++17", f"-I{ROOT / 'include'}", str(cli_src), "-o", str(CLI),
              f"-L{PKG}", "-lddm_b200", "-Wl,-rpath,$ORIGIN"])
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="print ptxas register/smem usage")
    a = ap.parse_args()
    if a.verbose:
        nvcc = _nvcc()
        res = subprocess.run([nvcc, *NVCC_FLAGS, "-Xptxas", "-v", "-c", str(CSRC / "engine.cu"), "-o", os.devnull],
                             capture_output=True, text=True)
        sys.stderr.write(res.stderr)
    print(build(force=a.force))


if __name__ == "__main__":
    main()
