"""Pins the FP64 oracle against outputs of the reference program itself.

tests/golden/reference_outputs.json was produced by tests/golden/make_golden.py on a B200,
running zhangyuyi99/cuda_multiDDM compiled from its own sources (oracle/Makefile). The
reference computes in FP32 (cuFFT, float accumulators, float partial sums) and prints six
significant digits, so ISF values are compared at 1e-5 relative plus half a unit in the
sixth printed digit. Masks are compared bit for bit (pixel counts and a hash of every mask).
"""
import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from cases import CASES, MASK_CASES, REDUCE_CASES, frames_digest, harness_acc
from cuda_multiddm_b200._lib import lib
from cuda_multiddm_b200.media import sig_digit_tolerance
from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_outputs.json"
REF_RTOL = 1e-5


def golden():
    if not GOLDEN.exists():
        pytest.skip("reference fixtures not generated")
    return json.loads(GOLDEN.read_text())


def parse(text):
    lines = text.split("\n")
    lam = [float(x) for x in lines[0].split()]
    tau = [float(x) for x in lines[1].split()]
    isf = np.array([[float(x) for x in ln.split()] for ln in lines[2:2 + len(lam)]])
    return lines, lam, tau, isf


def oracle_blocks(case):
    frames = case.frames()
    if case.frame_offset:
        frames = frames[case.frame_offset:]
    isf, dumps = O.ddm_run(frames, case.scales, case.taus, case.lambdas, tol=case.tolerance, N=case.N,
                           chunk=case.C, multistream=case.multistream, estimator=O.EST_COMPAT,
                           dump_every=case.dump_every, x_off=case.x_off, y_off=case.y_off)
    return isf, dumps


def split(isf, scales, Q, T):
    out, off = {}, 0
    for s in scales:
        tiles = (scales[0] // s) ** 2
        for tile in range(tiles):
            out[(s, tile)] = isf[off:off + Q * T].reshape(Q, T)
            off += Q * T
    return out


def expected_header(case, fps_int):
    lam = np.asarray(case.lambdas, np.float32)
    taus = np.asarray(case.taus, np.int32)
    dummy = np.zeros(len(lam) * len(taus))
    import tempfile
    with tempfile.NamedTemporaryFile() as f:
        assert lib().ddm_write_isf_file(f.name.encode(), dummy.ctypes.data, lam.ctypes.data, len(lam),
                                        taus.ctypes.data, len(taus), C.c_float(fps_int)) == 0
        return Path(f.name).read_text().split("\n")[:2]


@pytest.mark.parametrize("case", CASES, ids=lambda c: c.name)
def test_oracle_matches_reference_program(case):
    g = {c["name"]: c for c in golden()["cases"]}[case.name]
    assert g["returncode"] == 0
    assert frames_digest(case.frames()) == g["frames_sha256"], "synthetic input differs from the fixture's"
    isf, dumps = oracle_blocks(case)
    Q, T = len(case.lambdas), len(case.taus)
    fps = 1.0 if case.index_fps else 1e6 / np.float32(case.frame_time_us)
    header = expected_header(case, float(int(np.float32(fps))))
    worst = 0.0
    blocks = [("isf_", isf)] + [(f"isf__t{i}_", d) for i, d in enumerate(dumps)]
    seen = 0
    for prefix, arr in blocks:
        for (s, tile), want in split(arr, case.scales, Q, T).items():
            name = f"{prefix}{s}-{tile}"
            assert name in g["files"], name
            lines, lam, tau, ref = parse(g["files"][name])
            assert lines[:2] == header, (name, lines[:2], header)
            tol = REF_RTOL * np.abs(ref) + sig_digit_tolerance(ref)
            err = np.abs(want - ref)
            assert np.all(err <= tol), (name, float((err / np.maximum(np.abs(ref), 1e-30)).max()))
            nz = np.abs(ref) > 0
            if nz.any():
                worst = max(worst, float((err[nz] / np.abs(ref[nz])).max()))
            seen += 1
    assert seen == len(g["files"]), "the reference wrote files the oracle does not produce"
    print(f"{case.name}: worst relative difference {worst:.2e}")


@pytest.mark.parametrize("idx", range(len(MASK_CASES)))
def test_masks_match_reference_build_azimuth_mask(idx):
    g = golden()["masks"][idx]
    scale, tol, lambdas = MASK_CASES[idx]
    assert g["returncode"] == 0 and g["scale"] == scale
    m, counts = O.masks(scale, np.asarray(g["lambdas"], np.float32), np.float32(tol))
    assert counts.tolist() == g["counts"]
    for q in range(len(counts)):
        # FNV-1a over the mask bytes, as ref_harness prints it
        assert str(O.fnv1a(m[q])) == g["fnv"][q], (scale, q)


@pytest.mark.parametrize("idx", range(len(REDUCE_CASES)))
def test_azimuthal_matches_reference_analyse_fft_device(idx):
    g = golden()["reduce"][idx]
    scale, taus, tol, frames, seed, lambdas = REDUCE_CASES[idx]
    acc = harness_acc(scale, taus, seed).astype(np.float64)
    out = O.azimuthal(acc, scale, 1, np.asarray(lambdas, np.float32), np.float32(tol),
                      np.full(taus, float(frames)))
    for q, t, v in g["isf"]:
        want = out[0, q, t]
        assert abs(want - v) <= 2e-6 * abs(v) + 1e-12, (q, t, want, v)


def test_unaveraged_annulus_means_are_the_isf():
    """The corrected -K quantity (2 mean|dF|^2 / s^4 per wave vector) averages over each
    annulus mask to the ISF bin: the property that defines the format."""
    from cuda_multiddm_b200 import media

    frames = media.synth_video(9, 64, 64, 25, 20, step_var=1.0)
    scales, taus, lambdas = [64, 32], [1, 2, 5], [3.0, 6.0, 12.0]
    for est in (O.EST_UNBIASED, O.EST_COMPAT):
        isf, unav = O.ddm_run_unaveraged(frames, scales, taus, lambdas, chunk=10, estimator=est)
        off = isf_off = 0
        for s in scales:
            n = s * (s // 2 + 1)
            m, cnt = O.masks(s, lambdas, 1.2)
            for tile in range((64 // s) ** 2):
                block = isf[isf_off:isf_off + len(lambdas) * len(taus)].reshape(len(lambdas), len(taus))
                for q in range(len(lambdas)):
                    if cnt[q]:
                        mean = unav[:, off:off + n][:, m[q].reshape(-1).astype(bool)].mean(axis=1)
                        np.testing.assert_allclose(mean, block[q], rtol=1e-12, atol=1e-300)
                off += n
                isf_off += len(lambdas) * len(taus)
