"""Serving: many streams through one server (continuous batching, one lag launch per step
over all streams) give, chunk for chunk, the same ISF as each stream run alone through its
own engine; admission follows the HBM budget."""
import numpy as np
import pytest

from cuda_multiddm_b200 import Engine, EngineConfig, Server, media

pytestmark = pytest.mark.gpu

STREAMS = [  # (seed, side, scales, taus, lambdas)
    (1, 64, [64, 32], [1, 2, 3, 5, 8], [4.0, 8.0, 16.0]),
    (2, 128, [128, 64, 32], [1, 2, 4, 8, 16, 25], [3.0, 6.0, 12.0, 24.0]),
    (3, 256, [256, 128], [1, 3, 9, 27], [5.0, 10.0, 20.0, 40.0, 80.0]),
    (4, 128, [128], list(range(1, 21)), [4.0, 8.0]),
]
C, CHUNKS = 10, 5


def _cfg(side, scales, taus, lambdas):
    return EngineConfig(frame_width=side, frame_height=side, scales=scales, taus=taus, lambdas=lambdas,
                        chunk_frames=C, estimator="unbiased")


def _alone(frames, cfg):
    out = []
    with Engine(cfg) as eng:
        for k in range(CHUNKS):
            eng.submit(frames[k * C:(k + 1) * C])
            eng.finalize()
            out.append(eng.isf())
    return out


def test_each_stream_same_alone_and_in_the_mix():
    videos = [media.synth_video(seed, side, side, C * CHUNKS, side * side // 200, step_var=1.0)
              for seed, side, *_ in STREAMS]
    want = [_alone(v, _cfg(*s[1:])) for v, s in zip(videos, STREAMS)]
    got = [[] for _ in STREAMS]
    with Server() as srv:
        ids = [srv.add_stream(_cfg(*s[1:])) for s in STREAMS]
        assert all(i is not None for i in ids)
        # streams join at different times and submit at different rates
        for k in range(CHUNKS + 2):
            for j, sid in enumerate(ids):
                c = k - (j % 3)
                if 0 <= c < CHUNKS:
                    srv.submit(sid, videos[j][c * C:(c + 1) * C])
            srv.step()
            for j, sid in enumerate(ids):
                while (r := srv.poll(sid)) is not None:
                    got[j].append(r)
        while any(len(g) < CHUNKS for g in got):
            srv.step()
            srv.wait()
            for j, sid in enumerate(ids):
                while (r := srv.poll(sid)) is not None:
                    got[j].append(r)
        stats = srv.stats()
    assert stats["batched_launches"] >= 1
    for j in range(len(STREAMS)):
        assert [m["chunk_index"] for m, _ in got[j]] == list(range(CHUNKS))
        for k, (meta, isf) in enumerate(got[j]):
            assert meta["frames"] == (k + 1) * C and meta["done_s"] >= meta["submit_s"]
            np.testing.assert_array_equal(isf, want[j][k])


def test_admission_follows_the_hbm_budget():
    cfg = _cfg(256, [256, 128], [1, 2, 4], [4.0, 8.0])
    alone = _cfg(256, [256, 128], [1, 2, 4], [4.0, 8.0])
    alone.lag_batch_frames = C  # a served stream pairs each chunk at once
    with Engine(alone) as eng:
        one = eng.info().device_bytes
    with Server(hbm_budget_bytes=int(2.5 * one)) as srv:
        a, b = srv.add_stream(cfg), srv.add_stream(cfg)
        assert a is not None and b is not None
        assert srv.add_stream(cfg) is None          # a third does not fit now
        srv.remove_stream(a)
        c = srv.add_stream(cfg)                      # it does once a stream has left
        assert c is not None
        assert srv.stats()["streams"] == 2
