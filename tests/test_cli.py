"""The ddm CLI as a drop-in for the reference's ./ddm: same files, same text layout, same
checks and messages. GPU tests run it on the golden cases' .movie files and compare every
output file with the reference program's; CPU tests cover the argument checks that fail
before any device work."""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cases import CASES
from cuda_multiddm_b200.media import sig_digit_tolerance, write_movie, write_params

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "cuda_multiddm_b200" / "ddm"
GOLDEN = ROOT / "tests" / "golden" / "reference_outputs.json"


def run_cli(args, cwd=None):
    return subprocess.run([str(CLI), *args], capture_output=True, text=True, timeout=600, cwd=cwd)


def params(tmp_path, scales=(64,), taus=(1, 2), lambdas=(4.0, 8.0)):
    return write_params(tmp_path, scales, taus, lambdas)


def test_requires_input(tmp_path):
    ps, pt, pl = params(tmp_path)
    r = run_cli(["-o", str(tmp_path / "o"), "-N", "10", "-Q", str(pl), "-T", str(pt), "-S", str(ps)])
    assert r.returncode == 1 and "[Error] Must specify input." in r.stderr
    assert r.stdout.startswith("DDM Start")


@pytest.mark.parametrize("scales,taus,lambdas,msg", [
    ((48,), (1,), (4.0,), "scales must be powers of two (> 0)"),
    ((64, 64), (1,), (4.0,), "scales should be descending order"),
    ((64,), (2, 2), (4.0,), "Tau vector should be ascending order"),
    ((64,), (-1, 2), (4.0,), "Tau values should be positive"),
    ((64,), (1,), (4.0, 4.0), "q-vector vector should be ascending order"),
    ((64,), (1,), (100.0,), "The largest q-vector should be smaller than the smallest scale."),
])
def test_reference_parameter_checks(tmp_path, scales, taus, lambdas, msg):
    ps, pt, pl = params(tmp_path, scales, taus, lambdas)
    r = run_cli(["-o", str(tmp_path / "o"), "-N", "10", "-Q", str(pl), "-T", str(pt), "-S", str(ps), "-B", "1"])
    assert r.returncode == 1
    assert f"[Error] {msg}" in r.stderr


def test_missing_parameter_file(tmp_path):
    r = run_cli(["-o", "x", "-N", "10", "-Q", str(tmp_path / "nope"), "-T", "a", "-S", "b", "-B", "1"])
    assert r.returncode == 1 and "[Error] cannot open lambda-file." in r.stderr


def test_tolerance_warning_and_tau_chunk_check(tmp_path):
    ps, pt, pl = params(tmp_path, (64,), (1, 40), (4.0,))
    r = run_cli(["-o", str(tmp_path / "o"), "-N", "10", "-Q", str(pl), "-T", str(pt), "-S", str(ps), "-B", "1",
                 "-t", "0", "-C", "30"])
    assert "[Warning] mask_tolerance is likely undesired value" in r.stderr
    assert r.returncode == 1
    assert "[Error] the largest tau value must be smaller than number frames in a chunk" in r.stderr


def _golden():
    if not GOLDEN.exists():
        pytest.skip("reference fixtures not generated")
    return {c["name"]: c for c in json.loads(GOLDEN.read_text())["cases"]}


def parse(text):
    lines = text.split("\n")
    lam = lines[0].split()
    vals = np.array([[float(x) for x in ln.split()] for ln in lines[2:2 + len(lam)]])
    return lines[:2], vals


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: c.name)
def test_cli_output_files_match_reference(case, tmp_path):
    g = _golden()[case.name]
    frames = case.frames()
    movie = tmp_path / "in.movie"
    write_movie(movie, frames, frame_time_us=case.frame_time_us)
    ps, pt, pl = write_params(tmp_path, case.scales, case.taus, case.lambdas)
    out = tmp_path / "out"
    out.mkdir()
    r = run_cli(["-o", str(out / "isf_"), "-Q", str(pl), "-T", str(pt), "-S", str(ps), "-M", "-f", str(movie),
                 *case.cli_args()])
    assert r.returncode == 0, r.stderr
    assert "[Time elapsed]" in r.stdout and r.stdout.rstrip().endswith("DDM End")
    produced = {p.name: p.read_text() for p in out.iterdir()}
    assert sorted(produced) == sorted(g["files"])
    for name, text in g["files"].items():
        h_ref, v_ref = parse(text)
        h_got, v_got = parse(produced[name])
        assert h_got == h_ref, name
        tol = 1e-5 * np.abs(v_ref) + sig_digit_tolerance(v_ref) + sig_digit_tolerance(v_got)
        assert np.all(np.abs(v_got - v_ref) <= tol), name


@pytest.mark.gpu
def test_cli_benchmark_mode_runs(tmp_path):
    ps, pt, pl = params(tmp_path, (128, 64), (1, 2, 4), (4.0, 8.0, 16.0))
    r = run_cli(["-o", str(tmp_path / "b_"), "-N", "40", "-C", "10", "-Q", str(pl), "-T", str(pt), "-S", str(ps),
                 "-B", "1"])
    assert r.returncode == 0, r.stderr
    assert len(list(tmp_path.glob("b_*"))) == 1 + 4
