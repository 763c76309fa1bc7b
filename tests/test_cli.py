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


def _read_rows(path):
    lines = path.read_text().split("\n")
    assert lines[-1] == ""  # every line ends with a newline
    return lines[:-1]


@pytest.mark.gpu
def test_cli_debug_outputs_K_and_A(tmp_path):
    """-K and -A with their corrected contents: -K files hold, per tau, 2 mean|dF|^2 / s^4 of
    every wave vector (checked against the FP64 oracle, and its annulus means against the ISF
    file); -A files hold |F/s^2|^2 of every frame and tile of each chunk (against the oracle's
    FFT)."""
    from cuda_multiddm_b200.media import synth_video
    from oracle import oracle as O

    scales, taus, lambdas, C, N = [64, 32], [1, 2, 4], [4.0, 8.0], 10, 30
    frames = synth_video(61, 64, 64, N, 25, step_var=1.0)
    movie = tmp_path / "in.movie"
    write_movie(movie, frames, frame_time_us=1_000_000)
    ps, pt, pl = write_params(tmp_path, scales, taus, lambdas)
    out = tmp_path / "out"
    out.mkdir()
    r = run_cli(["-o", str(out / "d_"), "-N", str(N), "-C", str(C), "-Q", str(pl), "-T", str(pt), "-S", str(ps),
                 "-M", "-f", str(movie), "-K", "1", "-A", "-E", "unbiased", "-D", "0.5"])
    assert r.returncode == 0, r.stderr

    # -D: the fit file's layout (values are checked against scipy in test_fit.py)
    fit = (out / "d_fit").read_text().splitlines()
    assert fit[0].startswith("# I(tau) = A (1 - exp(-F tau)) + B; tau in s")
    kinds = [ln.split()[0] for ln in fit[1:]]
    assert kinds.count("scale") == 2 and kinds.count("tile") == 1 + 4
    assert kinds.count("curve") == (2 + 1 + 4) * len(lambdas)
    assert all(np.isfinite(float(ln.split()[5])) for ln in fit[1:] if ln.startswith("curve"))

    want_isf, want_unav = O.ddm_run_unaveraged(frames, scales, taus, lambdas, chunk=C)
    off = 0
    for s in scales:
        n = s * (s // 2 + 1)
        m, cnt = O.masks(s, lambdas, 1.2)
        for tile in range((64 // s) ** 2):
            rows = _read_rows(out / f"d_{s}-{tile}-nonAve")
            assert rows[0] == "".join(f"{x:g} " for x in lambdas)
            assert len(rows) == 2 + len(taus)
            got = np.array([[float(v) for v in row.split()] for row in rows[2:]])
            assert got.shape == (len(taus), n)
            want = want_unav[:, off:off + n]
            tol = 1e-5 * np.abs(want) + sig_digit_tolerance(want) + 1e-9 * np.abs(want).max()
            assert np.all(np.abs(got - want) <= tol), (s, tile)
            isf = parse((out / f"d_{s}-{tile}").read_text())[1]  # [q][tau]
            for q in range(len(lambdas)):
                if cnt[q]:
                    mean = got[:, m[q].reshape(-1).astype(bool)].mean(axis=1)
                    assert np.allclose(mean, isf[q], rtol=2e-5, atol=1e-9 * np.abs(isf).max())
            off += n

    for k in range(N // C):
        for si, s in enumerate(scales):
            rows = _read_rows(out / f"d__fft_chunk_{k}-{s}")
            tiles = (64 // s) ** 2
            assert len(rows) == C * tiles
            for f in (0, C - 1):
                tiles_px = O.extract(frames[k * C + f], 1, O.PIX_BYTE0, 0, 0, 64, s)
                for tile in range(tiles):
                    want = np.abs(O.fft2_r2c(tiles_px[tile]) / (s * s)).reshape(-1) ** 2
                    got = np.array([float(v) for v in rows[f * tiles + tile].split()])
                    assert np.allclose(got, want, rtol=1e-4, atol=1e-6 * want.max())


@pytest.mark.gpu
def test_cli_tensor_core_dft_flag(tmp_path):
    """-X sends the tiles of side 32..128 through the split-BF16 tensor-core DFT: every ISF
    file agrees with the FP32 run's within the path's 1e-3 budget (plus half a unit of the
    6th printed digit), and the larger scale's files, still from the FP32 FFT, are identical."""
    from cuda_multiddm_b200 import media
    from cuda_multiddm_b200.media import read_isf_file
    frames = media.synth_video(19, 256, 256, 40, 120, step_var=1.0)
    movie = tmp_path / "v.movie"
    write_movie(movie, frames)
    ps, pt, pl = write_params(tmp_path, (256, 128, 64), (1, 2, 3, 5, 8), (4.0, 8.0, 16.0, 32.0))
    base = ["-N", "40", "-C", "10", "-Q", str(pl), "-T", str(pt), "-S", str(ps), "-M", "-f", str(movie),
            "-E", "unbiased"]
    for tag, extra in (("a_", []), ("b_", ["-X"])):
        r = run_cli(["-o", str(tmp_path / tag), *base, *extra])
        assert r.returncode == 0, r.stderr
    n = 0
    for fa in sorted(tmp_path.glob("a_*")):
        fb = tmp_path / fa.name.replace("a_", "b_", 1)
        _, _, ia = read_isf_file(fa)
        _, _, ib = read_isf_file(fb)
        if fa.name.startswith("a_256"):
            assert fa.read_text() == fb.read_text()
        tol = 1e-3 * np.abs(ia) + sig_digit_tolerance(ia) + sig_digit_tolerance(ib)
        assert np.all(np.abs(ia - ib) <= tol), fa.name
        n += 1
    assert n == 1 + 4 + 16
