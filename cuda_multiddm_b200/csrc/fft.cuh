// 2-D R2C FFT of every tile of every scale (replaces parseBufferScalePow2 + cufftExecR2C,
// src/DDM_kernel.cuh:43-78 and src/DDM.cu:171-192).
//
// Two passes, each one launch over all scales of a group of frames:
//   fft_rows_kernel  reads the u8/u16 pixels of two tile rows, packs them as the real and
//                    imaginary parts of one complex row, transforms it and splits the
//                    result into the two half-spectrum rows X[y][kx], kx in [0, s/2]
//                    (written to the frame's ring slot);
//   fft_cols_kernel  transforms every column kx of every tile along y, in place.
// Frames are processed in small groups so the row pass's output is still in L2 when the
// column pass reads it back.
//
// The 1-D transform is a Stockham autosort FFT (the formulation of Govindaraju, Lloyd,
// Dotsenko, Smith & Manferdelli, "High performance discrete Fourier transforms on
// graphics processors", SC 2008): passes of radix 16 and one closing pass of radix 2, 4
// or 8, each thread holding 16 values in registers per pass, natural order in and out.
// A team of L/16 threads (1 for L < 16) owns one transform; a CTA of kFftThreads threads
// runs 256/team transforms side by side in shared memory. Element i of a transform sits
// at i + i/16 (one float2 of padding per 16) so the strided stores of a pass hit distinct
// banks; transforms are kFftPad(L) elements apart.
//
// Twiddles e^{-2 pi i m / M} (M = largest scale) come from a table computed in FP64 on the
// host and rounded to FP32; the radix-16 kernels use the exact values of cos/sin(k pi/8).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ddm {

constexpr int kFftThreads = 256;
constexpr int kFftMaxLog2 = 12;  // largest transform: 4096

__host__ __device__ constexpr int fft_team(int L) { return L >= 16 ? L / 16 : 1; }
__host__ __device__ constexpr int fft_per_cta(int L) {
    return kFftThreads / fft_team(L) < 1 ? 1 : kFftThreads / fft_team(L);
}
__host__ __device__ constexpr int kFftPad(int L) { return L + L / 16 + 1; }
__device__ __forceinline__ int fpad(int i) { return i + (i >> 4); }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }  // a * (-i)

// 4-point forward DFT of (a, b, c, d), natural order out
__device__ __forceinline__ void dft4(float2 &a, float2 &b, float2 &c, float2 &d) {
    const float2 s0 = cadd(a, c), d0 = csub(a, c), s1 = cadd(b, d), d1 = mul_mi(csub(b, d));
    a = cadd(s0, s1);
    c = csub(s0, s1);
    b = cadd(d0, d1);
    d = csub(d0, d1);
}

// e^{-2 pi i m / 16} for m = 0..9 (exact cos/sin of multiples of pi/8)
__device__ __forceinline__ float2 w16(int m) {
    constexpr float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f, r2 = 0.70710678118654752440f;
    switch (m) {
        case 0: return make_float2(1.f, 0.f);
        case 1: return make_float2(c1, -s1);
        case 2: return make_float2(r2, -r2);
        case 3: return make_float2(s1, -c1);
        case 4: return make_float2(0.f, -1.f);
        case 6: return make_float2(-r2, -r2);
        default: return make_float2(-c1, s1);  // m = 9
    }
}

// In-register forward DFT of length R (2, 4, 8 or 16) of v[0..R), natural order in and out.
template <int R>
__device__ __forceinline__ void dft_reg(float2 *v) {
    if constexpr (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        dft4(v[0], v[1], v[2], v[3]);
    } else if constexpr (R == 8) {
        // X[k1 + 2 k2] = sum_n2 w4^{n2 k2} w8^{n2 k1} sum_n1 x[4 n1 + n2] (-1)^{n1 k1};
        // y[2 n2 + k1] holds the inner sums, then the twiddles w8^{n2 k1}
        float2 y[8];
#pragma unroll
        for (int n2 = 0; n2 < 4; n2++) {
            y[2 * n2] = cadd(v[n2], v[n2 + 4]);
            y[2 * n2 + 1] = csub(v[n2], v[n2 + 4]);
        }
        constexpr float r2 = 0.70710678118654752440f;
        y[3] = cmulf(y[3], make_float2(r2, -r2));
        y[5] = mul_mi(y[5]);
        y[7] = cmulf(y[7], make_float2(-r2, -r2));
        dft4(y[0], y[2], y[4], y[6]);
        dft4(y[1], y[3], y[5], y[7]);
        // the dft4 over n2 leaves X[k1 + 2 k2] in y[2 k2 + k1]: natural order
#pragma unroll
        for (int k = 0; k < 8; k++) v[k] = y[k];
    } else {
        // R == 16: X[k1 + 4 k2] = sum_n2 w4^{n2 k2} w16^{n2 k1} sum_n1 x[4 n1 + n2] w4^{n1 k1}
        float2 y[16];
#pragma unroll
        for (int n2 = 0; n2 < 4; n2++) {
            float2 a = v[n2], b = v[n2 + 4], c = v[n2 + 8], d = v[n2 + 12];
            dft4(a, b, c, d);
            y[4 * n2 + 0] = a;
            y[4 * n2 + 1] = n2 ? cmulf(b, w16(n2)) : b;
            y[4 * n2 + 2] = n2 ? cmulf(c, w16(2 * n2)) : c;
            y[4 * n2 + 3] = n2 ? cmulf(d, w16(3 * n2)) : d;
        }
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++) {
            float2 a = y[k1], b = y[4 + k1], c = y[8 + k1], d = y[12 + k1];
            dft4(a, b, c, d);
            v[k1] = a;
            v[k1 + 4] = b;
            v[k1 + 8] = c;
            v[k1 + 12] = d;
        }
    }
}

template <int R>
__host__ __device__ constexpr int ilog2c() { return R <= 1 ? 0 : 1 + ilog2c<R / 2>(); }

// One Stockham pass of radix R over a transform of length L at buf (padded layout), by
// thread t of a team of `team`; every thread handles 16/R groups (R = L for L < 16).
template <int R>
__device__ __forceinline__ void stockham_pass(float2 *buf, int L, int Ns, int t, int team,
                                              const float2 *__restrict__ tw, int log2M, bool active) {
    constexpr int G = R >= 16 ? 1 : 16 / R;
    float2 v[G * R];
    const int stride = L / R;
    int ngroups = stride / team;  // groups per thread (1 for radix 16)
    if (ngroups > G) ngroups = G;
    if (active) {
#pragma unroll
        for (int g = 0; g < G; g++) {
            if (g < ngroups) {
                const int j = t + g * team;
                const int jm = j & (Ns - 1);
#pragma unroll
                for (int r = 0; r < R; r++) {
                    float2 x = buf[fpad(j + r * stride)];
                    if (r > 0 && Ns > 1) {
                        // e^{-2 pi i (j mod Ns) r / (Ns R)} = tw[(j mod Ns) r M / (Ns R)]
                        const int m = (jm * r) << (log2M - (__ffs(Ns) - 1) - ilog2c<R>());
                        x = cmulf(x, __ldg(tw + m));
                    }
                    v[g * R + r] = x;
                }
            }
        }
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int g = 0; g < G; g++) {
            if (g < ngroups) {
                dft_reg<R>(v + g * R);
                const int j = t + g * team;
                const int idx = (j & ~(Ns - 1)) * R + (j & (Ns - 1));
#pragma unroll
                for (int r = 0; r < R; r++) buf[fpad(idx + r * Ns)] = v[g * R + r];
            }
        }
    }
    __syncthreads();
}

// Full forward transform of length L (= 2^log2L <= 2^kFftMaxLog2) of the team's buffer.
__device__ void fft_team_transform(float2 *buf, int log2L, int t, int team, const float2 *__restrict__ tw,
                                   int log2M, bool active) {
    const int L = 1 << log2L;
    if (L < 16) {
        if (L == 2) stockham_pass<2>(buf, L, 1, t, team, tw, log2M, active);
        else if (L == 4) stockham_pass<4>(buf, L, 1, t, team, tw, log2M, active);
        else if (L == 8) stockham_pass<8>(buf, L, 1, t, team, tw, log2M, active);
        return;
    }
    int Ns = 1, left = log2L;
    for (; left >= 4; left -= 4, Ns <<= 4) stockham_pass<16>(buf, L, Ns, t, team, tw, log2M, active);
    if (left == 1) stockham_pass<2>(buf, L, Ns, t, team, tw, log2M, active);
    else if (left == 2) stockham_pass<4>(buf, L, Ns, t, team, tw, log2M, active);
    else if (left == 3) stockham_pass<8>(buf, L, Ns, t, team, tw, log2M, active);
}

// Per-scale launch geometry shared by both passes (ctas_per_frame over row pairs or columns).
struct FftScale {
    int s, log2s, tiles_side;
    int ctas_per_frame;
    int cta_begin;        // first CTA (blockIdx.x) of this scale
    long long n, off;     // elements per tile, offset of the scale in a frame
};

struct FftArgs {
    int S;
    FftScale sc[16];
    // source pixels (rows pass)
    const uint8_t *src;
    long long frame_stride, row_pitch;
    int bpp, pixmode, x_off, y_off;
    // ring
    float2 *ring;
    long long E;
    long long first_label;
    int R;
    const float2 *tw;
    int log2M;
};

__device__ __forceinline__ int fft_find_scale(const FftArgs &a) {
    int si = 0;
    while (si + 1 < a.S && static_cast<int>(blockIdx.x) >= a.sc[si + 1].cta_begin) si++;
    return si;
}

__device__ __forceinline__ float fft_pixel(const uint8_t *p, int pixmode) {
    if (pixmode == 1) return static_cast<float>(static_cast<unsigned>(p[0]) | (static_cast<unsigned>(p[1]) << 8));
    return static_cast<float>(p[0]);
}

// grid (sum of ctas_per_frame, frames). CTA = fft_per_cta(s) consecutive row pairs of the
// flattened (tile, pair) index of one frame at one scale.
__global__ void __launch_bounds__(kFftThreads) fft_rows_kernel(FftArgs a) {
    extern __shared__ float2 fsm[];
    const FftScale &sc = a.sc[fft_find_scale(a)];
    const int s = sc.s, L = s, team = fft_team(L), nT = fft_per_cta(L), TS = kFftPad(L);
    const int pairs_per_tile = s / 2;
    const int total_pairs = sc.tiles_side * sc.tiles_side * pairs_per_tile;
    const int g0 = (blockIdx.x - sc.cta_begin) * nT;
    const int f = blockIdx.y;
    const uint8_t *fsrc = a.src + f * a.frame_stride;
    // load: element (c, i) = (pixel(row 2p, i), pixel(row 2p+1, i)) of pair g0 + c
    for (int q = threadIdx.x; q < nT * L; q += kFftThreads) {
        const int c = q >> sc.log2s, i = q & (L - 1);
        const int g = g0 + c;
        float2 z = make_float2(0.f, 0.f);
        if (g < total_pairs) {
            const int tile = g / pairs_per_tile, py = 2 * (g - tile * pairs_per_tile);
            const int ty = tile / sc.tiles_side, tx = tile - ty * sc.tiles_side;
            const long long Y = static_cast<long long>(ty) * s + py + a.y_off;
            const long long X = static_cast<long long>(tx) * s + i + a.x_off;
            const uint8_t *p0 = fsrc + Y * a.row_pitch + X * a.bpp;
            z = make_float2(fft_pixel(p0, a.pixmode), fft_pixel(p0 + a.row_pitch, a.pixmode));
        }
        fsm[c * TS + fpad(i)] = z;
    }
    __syncthreads();
    const int c_me = threadIdx.x / team, t = threadIdx.x - c_me * team;
    fft_team_transform(fsm + c_me * TS, sc.log2s, t, team, a.tw, a.log2M, c_me < nT);
    // split Z = X0 + i X1 into the two real rows' half spectra
    const int nx = s / 2 + 1;
    const long long slot = (a.first_label + f) % a.R;
    float2 *out = a.ring + slot * a.E + sc.off;
    for (int q = threadIdx.x; q < nT * nx; q += kFftThreads) {
        const int c = q / nx, k = q - c * nx;
        const int g = g0 + c;
        if (g >= total_pairs) continue;
        const float2 *z = fsm + c * TS;
        const float2 zk = z[fpad(k & (L - 1))], zm = z[fpad((L - k) & (L - 1))];
        const int tile = g / pairs_per_tile, py = 2 * (g - tile * pairs_per_tile);
        float2 *o = out + tile * sc.n + static_cast<long long>(py) * nx + k;
        o[0] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        o[nx] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    }
}

// grid (sum of ctas_per_frame, frames). CTA = fft_per_cta(s) consecutive columns of the
// flattened (tile, kx) index of one frame at one scale, transformed along y in place.
__global__ void __launch_bounds__(kFftThreads) fft_cols_kernel(FftArgs a) {
    extern __shared__ float2 fsm[];
    const FftScale &sc = a.sc[fft_find_scale(a)];
    const int s = sc.s, L = s, team = fft_team(L), nT = fft_per_cta(L), TS = kFftPad(L);
    const int nx = s / 2 + 1;
    const int total_cols = sc.tiles_side * sc.tiles_side * nx;
    const int g0 = (blockIdx.x - sc.cta_begin) * nT;
    const long long slot = (a.first_label + blockIdx.y) % a.R;
    float2 *base = a.ring + slot * a.E + sc.off;
    for (int q = threadIdx.x; q < nT * L; q += kFftThreads) {
        const int y = q / nT, c = q - y * nT;
        const int g = g0 + c;
        float2 v = make_float2(0.f, 0.f);
        if (g < total_cols) {
            const int tile = g / nx, col = g - tile * nx;
            v = base[tile * sc.n + static_cast<long long>(y) * nx + col];
        }
        fsm[c * TS + fpad(y)] = v;
    }
    __syncthreads();
    const int c_me = threadIdx.x / team, t = threadIdx.x - c_me * team;
    fft_team_transform(fsm + c_me * TS, sc.log2s, t, team, a.tw, a.log2M, c_me < nT);
    for (int q = threadIdx.x; q < nT * L; q += kFftThreads) {
        const int y = q / nT, c = q - y * nT;
        const int g = g0 + c;
        if (g >= total_cols) continue;
        const int tile = g / nx, col = g - tile * nx;
        base[tile * sc.n + static_cast<long long>(y) * nx + col] = fsm[c * TS + fpad(y)];
    }
}

inline size_t fft_smem_bytes(int L) { return sizeof(float2) * static_cast<size_t>(fft_per_cta(L)) * kFftPad(L); }

}  // namespace ddm
