"""Parity cases run through the reference program (zhangyuyi99/cuda_multiDDM, built from
its sources by oracle/Makefile) to make the golden fixtures in this directory, and through
the oracle and the engine by the tests.

Every case is safe for the reference by construction: its final analysis indexes the
accumulator as n*(tile*T + tau*tiles) (src/DDM.cu:122 with src/azimuthal_average.cu:324)
while the data sits at n*(tau*tiles + tile). That reads the right bins only for tile 0, a
single-tile scale or T = 1, and for the last scale with several tiles and T > 1 it reads
past the end of the accumulator allocation. So multi-tile scales appear only with T = 1.
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Case:
    name: str
    seed: int
    width: int
    height: int
    frames_in_file: int
    scales: list
    taus: list
    lambdas: list
    N: int
    C: int
    tol_percent: int = 20
    multistream: bool = True
    dump_every: int = 0
    x_off: int = 0
    y_off: int = 0
    frame_offset: int = 0
    frame_time_us: int = 1_000_000
    index_fps: bool = False
    u16: bool = False
    spots: int = 40
    gen: dict = field(default_factory=dict)

    @property
    def tolerance(self) -> float:
        return float(np.float32(1.0 + self.tol_percent / 100.0))  # src/main.cpp:195-200

    def frames(self) -> np.ndarray:
        from cuda_multiddm_b200.media import synth_video
        kw = dict(spot_sigma=2.0, amplitude=120.0, background=20.0, step_var=0.5, noise_sd=4.0, max_value=255)
        kw.update(self.gen)
        return synth_video(self.seed, self.width, self.height, self.frames_in_file, self.spots, **kw)

    def cli_args(self) -> list:
        a = ["-N", str(self.N), "-C", str(self.C), "-t", str(self.tol_percent)]
        if not self.multistream:
            a.append("-Z")
        if self.dump_every:
            a += ["-G", str(self.dump_every)]
        if self.x_off:
            a += ["-x", str(self.x_off)]
        if self.y_off:
            a += ["-y", str(self.y_off)]
        if self.frame_offset:
            a += ["-s", str(self.frame_offset)]
        if self.index_fps:
            a.append("-I")
        return a


def frames_digest(frames: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(frames).tobytes()).hexdigest()


CASES = [
    # the plain single-scale workload: 200 frames 256^2, one 256 tile, tau 1..20, 10 lambdas 4..128
    Case("c1_plain", 1001, 256, 256, 200, [256], list(range(1, 21)),
         [4.0, 5.87, 8.62, 12.7, 18.6, 27.3, 40.1, 58.8, 86.3, 126.7], N=200, C=20, spots=300),
    # four scales, every tile (T = 1), ROI offset inside a larger frame, 25% tolerance
    Case("t1_multiscale_roi", 1010, 320, 288, 40, [256, 128, 64, 32], [3], [2.5, 4.0, 7.0, 12.0, 20.0, 31.0],
         N=40, C=10, tol_percent=25, x_off=16, y_off=8, spots=200),
    # leftover frames (N = 3*8 + 5) and a 30 fps clock (tau labels tau/30)
    Case("leftover", 1011, 128, 128, 29, [128], [1, 2, 3, 5, 8], [4.0, 8.0, 16.0, 32.0], N=29, C=8,
         frame_time_us=33333),
    # single-stream schedule (-Z): chunk 0 never analysed, chunk 1 twice
    Case("single_stream", 1012, 128, 128, 32, [128], [1, 2, 4, 7], [3.0, 6.0, 12.0, 24.0], N=32, C=8,
         multistream=False),
    # N = C: the tail pairs with real frames past N, read from the file
    Case("one_chunk_lookahead", 1013, 128, 128, 20, [128], [1, 2, 3, 4, 5, 6], [4.0, 8.0, 16.0], N=10, C=10),
    # -G 2 rolling snapshots
    Case("rolling_dump", 1014, 128, 128, 36, [128], [1, 2, 3], [4.0, 8.0, 16.0], N=36, C=6, dump_every=2),
    # 16-bit little-endian movie: the reference reads only the first (low) byte of each pixel
    Case("u16_byte0", 1015, 64, 64, 16, [64], [1, 2], [4.0, 8.0], N=16, C=4, u16=True,
         gen=dict(amplitude=2000.0, background=300.0, noise_sd=-1.0, max_value=4095)),
    # -s frame offset and -I frame-index labels
    Case("frame_offset", 1016, 128, 128, 30, [128], [1, 3], [4.0, 8.0, 16.0], N=24, C=8, frame_offset=5,
         index_fps=True, frame_time_us=40000),
    # -Z with leftover, ROI 64 inside 128
    Case("single_stream_leftover", 1017, 128, 128, 24, [64], [1, 2, 4, 8], [2.0, 4.0, 8.0, 16.0], N=19, C=8,
         multistream=False, x_off=30, y_off=50),
]

# buildAzimuthMask cases: (scale, tolerance as the CLI makes it, lambdas)
MASK_CASES = [
    (32, 1.2, [1.0, 2.0, 3.0, 4.0, 8.0, 16.0, 32.0]),
    (64, 1.25, [2.0, 4.0, 8.0, 16.0, 32.0, 64.0]),        # q^2 and tol^2 land exactly on the bounds
    (128, 1.05, [1.5, 2.0, 2.5, 3.3, 7.77, 12.0, 100.0]),
    (256, 1.37, [2.0, 3.0, 5.0, 9.0, 17.0, 33.0, 65.0, 129.0]),
    (1024, 1.2, [2.0 * (256.0 ** (i / 29)) for i in range(30)]),
    (2048, 1.2, [2.0 * (256.0 ** (i / 39)) for i in range(40)]),
]

# analyseFFTDevice cases: (scale, taus, tolerance, frames, seed, lambdas)
REDUCE_CASES = [
    (64, 3, 1.2, 50, 7, [2.0, 4.0, 8.0, 16.0]),
    (128, 2, 1.3, 1000, 11, [2.5, 5.0, 10.0, 20.0, 40.0]),
]


def harness_acc(scale: int, taus: int, seed: int) -> np.ndarray:
    """The accumulator ref_harness builds for `reduce` (LCG documented there), as float32."""
    n = scale * (scale // 2 + 1)
    out = np.empty(n * taus, np.float64)
    x = seed & 0xFFFFFFFFFFFFFFFF
    for i in range(out.size):
        out[i] = (x >> 40) / 16777216.0 * 1000.0
        x = (x * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
    return out.astype(np.float32).reshape(taus, n)
