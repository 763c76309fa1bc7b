// Device kernels of the DDM engine (sm_100a).
//
//   fft_rows_kernel,   (fft.cuh) tile extraction + 2-D R2C FFT per scale (replaces
//   fft_cols_kernel    parseBufferScalePow2 + cufftExecR2C, src/DDM_kernel.cuh:43-78)
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
constexpr int kAzThreads = 256;
constexpr int kMaxJ = 32;  // frames held in registers by one lag-kernel thread

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
