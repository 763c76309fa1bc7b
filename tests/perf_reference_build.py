"""Times the reference program (zhangyuyi99/cuda_multiDDM compiled from its sources for
sm_100a by oracle/Makefile, oracle/_ref/ddm_ref) and this repository's ddm CLI on the same
GPU, with the same flags, in the reference's own benchmark mode (-B: synthetic frames, no
file input), and prints one JSON line per configuration. Run on a GPU host from the
repository root:

    python tests/perf_reference_build.py

Only configurations whose scales are single-tile are run: the reference's final analysis
reads its accumulator at n*(tile*T + tau*tiles) (src/DDM.cu:122 with
src/azimuthal_average.cu:324), which for the last scale with several tiles and T > 1 reads
past the end of the allocation, so the multi-scale benchmark configuration cannot be run on
the reference safely. Both programs print "[Time elapsed] ... (x frame / second)" covering
set-up, the chunk loop and the azimuthal analysis; that figure is compared.
"""
from __future__ import annotations

import json
import re
import subprocess
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from cuda_multiddm_b200.media import log_lambdas, log_taus, write_params  # noqa: E402

REF = ROOT / "oracle" / "_ref" / "ddm_ref"
OURS = ROOT / "cuda_multiddm_b200" / "ddm"

CONFIGS = [
    # name, scales, taus, lambdas, N, C (reference needs C >= tau_max)
    ("single_256_tau20", [256], list(range(1, 21)), log_lambdas(4, 128, 10), 200, 20),
    ("single_1024_tau64_log500", [1024], log_taus(1, 500, 64), log_lambdas(2, 512, 30), 1000, 500),
]


def fps_of(stdout: str) -> float | None:
    m = re.search(r"\(([0-9.eE+-]+) frame / second\)", stdout)
    return float(m.group(1)) if m else None


def run(binary: Path, args: list[str], runs: int = 2) -> dict:
    best = None
    for _ in range(runs):
        res = subprocess.run([str(binary), *args], capture_output=True, text=True, timeout=1800)
        if res.returncode != 0:
            return {"rc": res.returncode, "stderr": res.stderr[-400:]}
        f = fps_of(res.stdout)
        best = f if best is None or (f is not None and f > best) else best
    return {"rc": 0, "frames_per_s": best}


def main() -> None:
    for name, scales, taus, lambdas, N, C in CONFIGS:
        with tempfile.TemporaryDirectory() as tmp:
            ps, pt, pl = write_params(tmp, scales, taus, lambdas)
            common = ["-N", str(N), "-Q", str(pl), "-T", str(pt), "-S", str(ps), "-B", "1"]
            ref = run(REF, ["-o", f"{tmp}/ref_", "-C", str(C), *common])
            ours = run(OURS, ["-o", f"{tmp}/ours_", "-C", str(C), *common])
            ours_u = run(OURS, ["-o", f"{tmp}/oursu_", "-C", "30", "-E", "unbiased", *common])
        line = {"config": name, "scales": scales, "taus": len(taus), "tau_max": max(taus), "N": N,
                "reference_chunk": C, "reference": ref, "ours_same_flags": ours,
                "ours_unbiased_chunk30": ours_u}
        if ref.get("frames_per_s") and ours.get("frames_per_s"):
            line["speedup_same_flags"] = ours["frames_per_s"] / ref["frames_per_s"]
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
