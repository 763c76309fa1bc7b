// Device kernels of the DDM engine (sm_100a).
//
//   fft_rows_kernel    tile extraction + u8/u16 -> f32 + row pass of the 2-D R2C FFT
//                      (replaces parseBufferScalePow2 + the first half of cufftExecR2C,
//                      src/DDM_kernel.cuh:43-78, src/DDM.cu:188-192)
//   fft_cols_kernel    column pass, in place in the ring slot
//   lag_pipe_kernel    (lag.cuh) |F(a) - F(b)|^2 accumulation for a block of frames
//                      against every tau (replaces processFFT, src/DDM_kernel.cuh:85-101)
//   azimuth_kernel     masked azimuthal average of every (scale, tile, tau) row over the
//                      annulus index lists, FP64 (replaces maskReduce + host sums,
//                      src/azimuthal_average.cu:292-346)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ddm {

constexpr int kMaxScales = 16;
constexpr int kFftThreads = 256;
constexpr int kAzThreads = 256;
constexpr int kMaxJ = 32;  // frames held in registers by one lag-kernel thread

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ unsigned bitrev(unsigned k, int log2n) {
    return log2n == 0 ? 0u : (__brev(k) >> (32 - log2n));
}

// `count` forward DIF radix-2 transforms of length L (= 2^log2L) in shared memory,
// natural-order input, bit-reversed output. Element m of transform c sits at
// x[m * mstride + c * cstride]. kInterleaved: consecutive threads walk transforms
// first (column layout, cstride 1), else butterflies first (row layout, mstride 1).
// tw[m] = e^{-2 pi i m / tw_n}, m < tw_n / 2.
template <bool kInterleaved>
__device__ void fft_dif_smem(float2 *x, int count, int log2L, int mstride, int cstride,
                             const float2 *__restrict__ tw, int log2tw) {
    const int half = 1 << (log2L - 1);
    const int total = count * half;
    for (int lh = log2L - 1; lh >= 0; lh--) {
        const int h = 1 << lh;
        const int tw_shift = log2tw - lh - 1;  // twiddle index j * tw_n / (2h)
        for (int b = threadIdx.x; b < total; b += blockDim.x) {
            int c, bf;
            if (kInterleaved) {
                c = b % count;
                bf = b / count;
            } else {
                c = b >> (log2L - 1);
                bf = b & (half - 1);
            }
            const int j = bf & (h - 1);
            const int i0 = ((bf - j) << 1) + j;
            float2 *xc = x + c * cstride;
            const float2 u = xc[i0 * mstride], v = xc[(i0 + h) * mstride];
            const float2 w = tw[j << tw_shift];
            xc[i0 * mstride] = make_float2(u.x + v.x, u.y + v.y);
            xc[(i0 + h) * mstride] = cmul(make_float2(u.x - v.x, u.y - v.y), w);
        }
        __syncthreads();
    }
}

struct RowArgs {
    const uint8_t *src;
    long long frame_stride;  // bytes between frames
    long long row_pitch;     // bytes between rows
    int bpp, pixmode, x_off, y_off;
    int s, log2s, tiles_side, pairs_per_cta, ctas_per_tile;
    long long n, off, E;     // elements per tile, scale offset, elements per frame
    long long first_label;
    int R;
    float2 *ring;
    const float2 *tw;
    int log2tw;
};

__device__ __forceinline__ float load_pixel(const uint8_t *p, int pixmode) {
    if (pixmode == 1) return static_cast<float>(static_cast<unsigned>(p[0]) | (static_cast<unsigned>(p[1]) << 8));
    return static_cast<float>(p[0]);
}

// grid (tiles * ctas_per_tile, frames); each CTA transforms pairs_per_cta row pairs of
// one tile: rows y, y+1 go in as the real and imaginary parts of one complex FFT.
__global__ void __launch_bounds__(kFftThreads) fft_rows_kernel(RowArgs a) {
    extern __shared__ float2 sm[];
    const int f = blockIdx.y;
    const int tile = blockIdx.x / a.ctas_per_tile, g = blockIdx.x % a.ctas_per_tile;
    const int ty = tile / a.tiles_side, tx = tile % a.tiles_side;
    const int s = a.s, P = a.pairs_per_cta;
    const int y_base = g * P * 2;
    const uint8_t *fsrc = a.src + f * a.frame_stride;
    for (int i = threadIdx.x; i < P * s; i += blockDim.x) {
        const int p = i >> a.log2s, x = i & (s - 1);
        const long long Y = (long long)ty * s + y_base + 2 * p + a.y_off;
        const long long X = (long long)tx * s + x + a.x_off;
        const uint8_t *p0 = fsrc + Y * a.row_pitch + X * a.bpp;
        sm[i] = make_float2(load_pixel(p0, a.pixmode), load_pixel(p0 + a.row_pitch, a.pixmode));
    }
    __syncthreads();
    fft_dif_smem<false>(sm, P, a.log2s, 1, s, a.tw, a.log2tw);
    const int nx = s / 2 + 1;
    const long long slot = (a.first_label + f) % a.R;
    float2 *out = a.ring + slot * a.E + a.off + (long long)tile * a.n;
    for (int i = threadIdx.x; i < P * nx; i += blockDim.x) {
        const int p = i / nx, k = i - p * nx;
        const float2 *z = sm + p * s;
        const float2 zk = z[bitrev(k & (s - 1), a.log2s)];
        const float2 zm = z[bitrev((s - k) & (s - 1), a.log2s)];
        const int y = y_base + 2 * p;
        out[(long long)y * nx + k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        out[(long long)(y + 1) * nx + k] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    }
}

struct ColArgs {
    int s, log2s, P, groups_per_tile;
    long long n, off, E;
    long long first_label;
    int R;
    float2 *ring;
    const float2 *tw;
    int log2tw;
};

// grid (tiles * groups_per_tile, frames); each CTA transforms P adjacent columns of one
// tile along y, in place.
__global__ void __launch_bounds__(kFftThreads) fft_cols_kernel(ColArgs a) {
    extern __shared__ float2 sm[];
    const int f = blockIdx.y;
    const int tile = blockIdx.x / a.groups_per_tile, grp = blockIdx.x % a.groups_per_tile;
    const int s = a.s, P = a.P, nx = s / 2 + 1;
    const int c0 = grp * P;
    const int ncols = min(P, nx - c0);
    const long long slot = (a.first_label + f) % a.R;
    float2 *base = a.ring + slot * a.E + a.off + (long long)tile * a.n + c0;
    for (int i = threadIdx.x; i < s * P; i += blockDim.x) {
        const int y = i / P, p = i - y * P;
        sm[i] = p < ncols ? base[(long long)y * nx + p] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    fft_dif_smem<true>(sm, P, a.log2s, P, 1, a.tw, a.log2tw);
    for (int i = threadIdx.x; i < s * P; i += blockDim.x) {
        const int ky = i / P, p = i - ky * P;
        if (p < ncols) base[(long long)ky * nx + p] = sm[bitrev(ky, a.log2s) * P + p];
    }
}

struct ScaleDesc {
    int s, tiles;
    long long n, off;     // elements per tile, offset of the scale in a frame
    long long isf_off;    // offset of the scale's block in the ISF output
    int q_base;           // index of (scale, q = 0) in q_ptr / counts
    double inv_s4;
};

struct AzArgs {
    int S, T, Q;
    ScaleDesc sc[kMaxScales];
    int block_prefix[kMaxScales + 1];  // first block of each scale
    const float2 *acc;
    long long E;
    const int *q_ptr;   // [S*(Q+1)] absolute offsets into idx
    const int *idx;     // element indices within a tile, per (scale, q)
    const int *counts;  // [S*Q]
    const double *norm; // [T]
    double *isf;
};

// One CTA per (scale, tile, tau); warp w reduces q = w, w + 8, ... in FP64.
__global__ void __launch_bounds__(kAzThreads) azimuth_kernel(AzArgs a) {
    int si = 0;
    while (si + 1 < a.S && (int)blockIdx.x >= a.block_prefix[si + 1]) si++;
    const ScaleDesc &sc = a.sc[si];
    const int rem = blockIdx.x - a.block_prefix[si];
    const int tile = rem / a.T, t = rem - tile * a.T;
    const float2 *row = a.acc + (long long)t * a.E + sc.off + (long long)tile * sc.n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double nrm = a.norm[t];
    for (int q = warp; q < a.Q; q += kAzThreads / 32) {
        const int beg = a.q_ptr[si * (a.Q + 1) + q], end = a.q_ptr[si * (a.Q + 1) + q + 1];
        double sum = 0.0;
        for (int i = beg + lane; i < end; i += 32) {
            const float2 v = row[a.idx[i]];
            sum += (double)v.x - (double)v.y;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
        if (lane == 0) {
            const int P = a.counts[sc.q_base + q];
            const double v = (P != 0 && nrm != 0.0) ? 2.0 * sum * sc.inv_s4 / (double)P / nrm : 0.0;
            a.isf[sc.isf_off + ((long long)tile * a.Q + q) * a.T + t] = v;
        }
    }
}

}  // namespace ddm
