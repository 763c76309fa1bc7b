"""ddm_lag_accumulate_static -- the lag kernel on caller-owned device memory, for callers
that cannot let the library allocate device memory (acquisition loops that reserve all
their memory up front, applications whose own pool allocator owns every device buffer).

The test plays such a caller: it owns the spectra ring and the accumulators (allocated
here, by the test, through torch), calls the entry point twice in a row through the C ABI,
and checks the result against the engine's own accumulators for the same frames (the
existing ddm_submit_frames path), at the tolerance the other GPU tests use (1e-5 relative).
It is collected last so that a run stopping at the first failure has run every other test;
it passes alone in a fresh process too, since its first call performs the per-device set-up.
"""
import ctypes as C

import numpy as np
import pytest

from cuda_multiddm_b200 import Engine, EngineConfig, media
from cuda_multiddm_b200._lib import lib

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def test_static_lag_matches_engine_on_two_calls():
    import torch

    scales, taus, lambdas, F = [64, 32], [1, 2, 3, 5, 9], [4.0, 8.0], 8
    frames = media.synth_video(31, 64, 64, 2 * F, 25, step_var=1.0)
    cfg = EngineConfig(frame_width=64, frame_height=64, scales=scales, taus=taus, lambdas=lambdas,
                       chunk_frames=F, estimator="unbiased")
    with Engine(cfg) as eng:
        assert eng.info().ring_slots >= 2 * F  # every frame's spectrum is still in the ring
        eng.submit(frames)
        want = eng.accumulators()
        spectra = np.stack([eng.spectrum(f) for f in range(2 * F)])  # [frames][E] complex64
    E = spectra.shape[1]
    T = len(taus)

    torch.cuda.set_device(0)
    ring = torch.from_numpy(spectra.view(np.float32).copy()).cuda()  # float2 [frames][E]
    acc = torch.zeros((T, E, 2), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        n0 = call * F  # the engine pairs the new frames n0 + j with the frames tau earlier
        a = np.arange(n0, n0 + F, dtype=np.int32)
        b = np.array([[n0 + j - t if n0 + j - t >= 0 else -1 for j in range(F)] for t in taus], np.int32)
        st = lib().ddm_lag_accumulate_static(C.c_void_p(ring.data_ptr()), 2 * F, E, C.c_void_p(acc.data_ptr()),
                                             a.ctypes.data, F, b.ctypes.data, T, C.c_void_p(stream))
        assert st == 0, lib().ddm_last_error().decode()
    torch.cuda.synchronize()
    got = acc[..., 0].double().cpu().numpy() - acc[..., 1].double().cpu().numpy()
    floor = 1e-9 * np.abs(want).max()
    assert np.all(np.abs(got - want) <= RTOL * np.abs(want) + floor), float(np.abs(got - want).max())


def test_static_lag_refuses_requests_beyond_its_table():
    import torch

    ring = torch.zeros((4, 64, 2), dtype=torch.float32, device="cuda")
    acc = torch.zeros((200, 64, 2), dtype=torch.float32, device="cuda")
    a = np.zeros(4, np.int32)
    b = np.zeros((200, 4), np.int32)
    st = lib().ddm_lag_accumulate_static(C.c_void_p(ring.data_ptr()), 4, 64, C.c_void_p(acc.data_ptr()),
                                         a.ctypes.data, 4, b.ctypes.data, 200, None)
    assert st == 1 and b"tau_count must be 1..128" in lib().ddm_last_error()


def _numpy_lag(ring_c: np.ndarray, a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """float64 sum over j of |ring[a[j]] - ring[b[t, j]]|^2, skipping -1 slots."""
    r = ring_c.astype(np.complex128)
    out = np.zeros((b.shape[0], r.shape[1]))
    for t in range(b.shape[0]):
        for j in range(a.shape[0]):
            if a[j] >= 0 and b[t, j] >= 0:
                out[t] += np.abs(r[a[j]] - r[b[t, j]]) ** 2
    return out


def _call_static(ring, slots, E, acc, a, b):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    st = lib().ddm_lag_accumulate_static(C.c_void_p(ring.data_ptr()), slots, E, C.c_void_p(acc.data_ptr()),
                                         a.ctypes.data, a.shape[0], b.ctypes.data, b.shape[0], C.c_void_p(stream))
    assert st == 0, lib().ddm_last_error().decode()


@pytest.mark.parametrize("F,T,pattern", [(5, 7, "permuted"), (32, 128, "shifted"), (32, 128, "disjoint")])
def test_static_lag_matches_numpy(F, T, pattern):
    """Fewer frames than the kernel instance holds (F = 5 runs the 8-frame kernel), -1 slots,
    ring slots out of frame order, and the stated limits (32 frames, 128 rows), as rows that
    share their partners (shifted) and rows that share nothing (disjoint)."""
    import torch

    rng = np.random.default_rng(F * 1000 + T)
    slots, E = 300, 2048 + 64
    ring_c = (rng.standard_normal((slots, E)) + 1j * rng.standard_normal((slots, E))).astype(np.complex64)
    perm = rng.permutation(slots).astype(np.int32)  # frame label f lives in ring slot perm[f]
    if pattern == "shifted":
        labels_a = np.arange(200, 200 + F)
        taus = np.arange(1, T + 1)
        b = np.array([[perm[l - t] for l in labels_a] for t in taus], np.int32)
        a = perm[labels_a].astype(np.int32)
    else:
        a = perm[rng.choice(slots, F, replace=False)].astype(np.int32)
        b = rng.integers(0, slots, size=(T, F)).astype(np.int32)
    if pattern == "permuted":
        a[1] = -1
        b[2, :] = -1
        b[4, 3] = -1
    ring = torch.from_numpy(ring_c.view(np.float32).copy()).cuda()
    acc = torch.zeros((T, E, 2), dtype=torch.float32, device="cuda")
    want = np.zeros((T, E))
    for _ in range(2):  # two calls in a row accumulate
        _call_static(ring, slots, E, acc, a, b)
        want += _numpy_lag(ring_c, a, b)
    torch.cuda.synchronize()
    got = acc[..., 0].double().cpu().numpy() - acc[..., 1].double().cpu().numpy()
    floor = 1e-9 * np.abs(want).max()
    err = np.abs(got - want) / np.maximum(np.abs(want), floor)
    assert np.all(np.abs(got - want) <= RTOL * np.abs(want) + floor), float(err.max())


def test_static_lag_refuses_slots_below_minus_one():
    import torch

    ring = torch.zeros((4, 64, 2), dtype=torch.float32, device="cuda")
    acc = torch.zeros((2, 64, 2), dtype=torch.float32, device="cuda")
    a = np.zeros(4, np.int32)
    b = np.zeros((2, 4), np.int32)
    b[1, 2] = -2
    st = lib().ddm_lag_accumulate_static(C.c_void_p(ring.data_ptr()), 4, 64, C.c_void_p(acc.data_ptr()),
                                         a.ctypes.data, 4, b.ctypes.data, 2, None)
    assert st == 1 and b"b_slots entry outside -1..ring_slots-1" in lib().ddm_last_error()
