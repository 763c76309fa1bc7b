"""Times the reference program (zhangyuyi99/cuda_multiDDM compiled from its sources for
sm_100a by oracle/Makefile, oracle/_ref/ddm_ref) and this repository's ddm CLI on the same
GPU, with the same flags, in the reference's own benchmark mode (-B: synthetic frames, no
file input), and prints one JSON line per configuration. Run on a GPU host from the
repository root:

    python oracle/perf_reference_build.py

Only configurations whose scales are single-tile are run: the reference's final analysis
reads its accumulator at n*(tile*T + tau*tiles) (src/DDM.cu:122 with
src/azimuthal_average.cu:324), which for the last scale with several tiles and T > 1 reads
past the end of the allocation, so the multi-scale benchmark configuration cannot be run on
the reference safely. Both programs print "[Time elapsed] ... (x frame / second)" covering
set-up, the chunk loop and the azimuthal analysis. With a few hundred frames that figure is
dominated by fixed costs (CUDA context, gigabyte-sized allocations), so each program also
runs at two frame counts and the marginal throughput (extra frames / extra total time) is
reported: the steady-state analysed frames/s.
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
    # name, scales, taus, lambdas, (N small, N large), C (the reference needs C >= tau_max)
    ("single_256_tau20", [256], list(range(1, 21)), log_lambdas(4, 128, 10), (2000, 20000), 20),
    ("single_1024_tau64_log500", [1024], log_taus(1, 500, 64), log_lambdas(2, 512, 30), (2000, 20000), 500),
]


def total_seconds(stdout: str) -> float | None:
    m = re.search(r"Total\s+([0-9.eE+-]+) s", stdout)
    return float(m.group(1)) if m else None


def run(binary: Path, args: list[str], n_small: int, n_large: int) -> dict:
    """Best-of-two total time at each frame count; returns both and the marginal rate."""
    out = {}
    for n in (n_small, n_large):
        best = None
        for _ in range(2):
            res = subprocess.run([str(binary), "-N", str(n), *args], capture_output=True, text=True, timeout=1800)
            if res.returncode != 0:
                return {"rc": res.returncode, "N": n, "stderr": res.stderr[-400:]}
            t = total_seconds(res.stdout)
            best = t if best is None or (t is not None and t < best) else best
        out[n] = best
    return {"rc": 0, "total_s": {str(k): v for k, v in out.items()},
            "frames_per_s_at_large_N": n_large / out[n_large],
            "marginal_frames_per_s": (n_large - n_small) / (out[n_large] - out[n_small])}


def main() -> None:
    for name, scales, taus, lambdas, (n1, n2), C in CONFIGS:
        with tempfile.TemporaryDirectory() as tmp:
            ps, pt, pl = write_params(tmp, scales, taus, lambdas)
            common = ["-Q", str(pl), "-T", str(pt), "-S", str(ps), "-B", "1"]
            ref = run(REF, ["-o", f"{tmp}/ref_", "-C", str(C), *common], n1, n2)
            ours = run(OURS, ["-o", f"{tmp}/ours_", "-C", str(C), *common], n1, n2)
            ours_u = run(OURS, ["-o", f"{tmp}/oursu_", "-C", "30", "-E", "unbiased", *common], n1, n2)
        line = {"config": name, "scales": scales, "taus": len(taus), "tau_max": max(taus), "N": [n1, n2],
                "reference_chunk": C, "reference": ref, "ours_same_flags": ours,
                "ours_unbiased_chunk30": ours_u}
        if ref.get("rc") == 0 and ours.get("rc") == 0:
            line["marginal_speedup_same_flags"] = ours["marginal_frames_per_s"] / ref["marginal_frames_per_s"]
            line["speedup_at_large_N_same_flags"] = ours["frames_per_s_at_large_N"] / ref["frames_per_s_at_large_N"]
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
