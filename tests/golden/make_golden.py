"""Generate the golden fixtures from the reference program itself.

Runs on a GPU host, from the repository root, after `make -C oracle ref` has built
oracle/_ref/ddm_ref and oracle/_ref/ref_harness from the reference's sources:

    python tests/golden/make_golden.py [OUTDIR]

For each case in cases.py it writes the synthetic video as an IIDC .movie file plus the
lambda / tau / scale files, runs the reference CLI on it, and stores every ISF text file it
writes; it also records buildAzimuthMask counts and mask hashes, and analyseFFTDevice
outputs, from ref_harness. Output: OUTDIR/reference_outputs.json (default
tests/golden/_out), copied by hand into tests/golden/.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))

from cases import CASES, MASK_CASES, REDUCE_CASES, frames_digest  # noqa: E402

from cuda_multiddm_b200.media import write_movie, write_params  # noqa: E402

REF = ROOT / "oracle" / "_ref" / "ddm_ref"
HARNESS = ROOT / "oracle" / "_ref" / "ref_harness"


def run_case(case, work: Path) -> dict:
    frames = case.frames()
    d = work / case.name
    d.mkdir(parents=True)
    movie = d / "in.movie"
    write_movie(movie, frames, frame_time_us=case.frame_time_us)
    ps, pt, pl = write_params(d, case.scales, case.taus, case.lambdas)
    out_prefix = d / "out" / "isf_"
    out_prefix.parent.mkdir()
    cmd = [str(REF), "-o", str(out_prefix), "-Q", str(pl), "-T", str(pt), "-S", str(ps), "-M", "-f", str(movie),
           *case.cli_args()]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    files = {p.name: p.read_text() for p in sorted(out_prefix.parent.iterdir())}
    return {"name": case.name, "cmd_args": case.cli_args(), "returncode": res.returncode,
            "stdout_tail": res.stdout[-2000:], "stderr_tail": res.stderr[-2000:],
            "frames_sha256": frames_digest(frames), "files": files}


def run_masks() -> list:
    out = []
    for scale, tol, lambdas in MASK_CASES:
        args = [str(HARNESS), "mask", str(scale), repr(float(tol))] + [f"{x:.9g}" for x in lambdas]
        res = subprocess.run(args, capture_output=True, text=True, timeout=600)
        lines = res.stdout.split("\n")
        counts = [int(x) for x in lines[0].split()[1:]]
        hashes = [int(ln.split()[2]) for ln in lines[1:] if ln.startswith("fnv")]
        out.append({"scale": scale, "tolerance": tol, "lambdas": [float(f"{x:.9g}") for x in lambdas],
                    "counts": counts, "fnv": [str(h) for h in hashes], "returncode": res.returncode})
    return out


def run_reduce() -> list:
    out = []
    for scale, taus, tol, frames, seed, lambdas in REDUCE_CASES:
        args = [str(HARNESS), "reduce", str(scale), str(taus), repr(float(tol)), str(frames), str(seed)] + \
               [f"{x:.9g}" for x in lambdas]
        res = subprocess.run(args, capture_output=True, text=True, timeout=600)
        vals = [[int(ln.split()[1]), int(ln.split()[2]), float(ln.split()[3])]
                for ln in res.stdout.split("\n") if ln.startswith("isf")]
        out.append({"scale": scale, "taus": taus, "tolerance": tol, "frames": frames, "seed": seed,
                    "lambdas": lambdas, "isf": vals, "returncode": res.returncode})
    return out


def main() -> None:
    outdir = Path(sys.argv[1]) if len(sys.argv) > 1 else ROOT / "tests" / "golden" / "_out"
    outdir.mkdir(parents=True, exist_ok=True)
    result = {"reference": "zhangyuyi99/cuda_multiDDM src/, built by oracle/Makefile for sm_100a",
              "cases": [], "masks": run_masks(), "reduce": run_reduce()}
    with tempfile.TemporaryDirectory() as tmp:
        for case in CASES:
            result["cases"].append(run_case(case, Path(tmp)))
    (outdir / "reference_outputs.json").write_text(json.dumps(result, indent=1))
    bad = [c["name"] for c in result["cases"] if c["returncode"] != 0]
    print(f"wrote {outdir / 'reference_outputs.json'}; failed cases: {bad}")
    sys.exit(1 if bad else 0)


if __name__ == "__main__":
    os.chdir(ROOT)
    main()
