// Device kernels of the DDM engine (sm_100a).
//
//   fft_rows_kernel,   (fft.cuh) tile extraction + 2-D R2C FFT per scale (replaces
//   fft_cols_kernel    parseBufferScalePow2 + cufftExecR2C, src/DDM_kernel.cuh:43-78)
//   lag_pipe_kernel    (lag.cuh) |F(a) - F(b)|^2 accumulation for a block of frames
//                      against every tau (replaces processFFT, src/DDM_kernel.cuh:85-101)
//   azimuth_partial_kernel, azimuth_final_kernel
//                      masked azimuthal average of every (scale, tile, lambda, tau) bin over
//                      the annulus index lists, FP64, in two deterministic stages (replaces
//                      maskReduce + the host sums, src/azimuthal_average.cu:292-346)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ddm {

constexpr int kMaxScales = 16;
constexpr int kAzThreads = 256;
constexpr int kMaxJ = 64;          // register frames per element of one lag-kernel launch
constexpr int kPieceFrames = 32;   // frames per ingest piece (FFT group, staging) at most

struct ScaleDesc {
    int s, tiles;
    long long n, off;     // elements per tile, offset of the scale in a frame
    long long isf_off;    // offset of the scale's block in the ISF output
    int q_base;           // index of (scale, q = 0) in counts / chunk_first / chunk_count
    double inv_s4;
    // azimuthal work: the scale's annulus index lists cut into chunks of <= kAzChunk entries
    int nchunks;          // chunks of all q of this scale
    int chunk_off;        // first chunk of the scale in chunk_beg / chunk_end
    long long item_base;  // first (chunk, tile, tau) item of the scale; items are ordered (tile, tau, chunk)
};

constexpr int kAzChunk = 1024;   // annulus indices summed by one warp
constexpr int kAzWarps = kAzThreads / 32;

struct AzArgs {
    int S, T, Q;
    ScaleDesc sc[kMaxScales];
    const float2 *acc;
    long long E;
    const int *idx;          // element indices within a tile, CSR per (scale, q)
    const int *chunk_beg;    // [chunks] absolute offsets into idx
    const int *chunk_end;
    const int *chunk_first;  // [S*Q] first chunk of (scale, q), relative to the scale
    const int *chunk_count;  // [S*Q]
    const int *counts;       // [S*Q] annulus pixel counts
    const double *norm;      // [T]
    double *partial;         // [items] stage-1 sums
    double *isf;
    long long items, bins;
};

__device__ __forceinline__ int az_scale_of(const AzArgs &a, long long item) {
    int si = 0;
    while (si + 1 < a.S && item >= a.sc[si + 1].item_base) si++;
    return si;
}

// Stage 1: one warp per (scale, tile, tau, chunk) item sums the accumulator values
// (sum - compensation, in FP64) at the chunk's annulus indices into partial[item].
__global__ void __launch_bounds__(kAzThreads) azimuth_partial_kernel(AzArgs a) {
    const long long item = static_cast<long long>(blockIdx.x) * kAzWarps + (threadIdx.x >> 5);
    if (item >= a.items) return;
    const int lane = threadIdx.x & 31;
    const int si = az_scale_of(a, item);
    const ScaleDesc &sc = a.sc[si];
    const long long rel = item - sc.item_base;
    const long long row_id = rel / sc.nchunks;   // tile * T + tau
    const int c = static_cast<int>(rel - row_id * sc.nchunks);
    const int tile = static_cast<int>(row_id / a.T), t = static_cast<int>(row_id - static_cast<long long>(tile) * a.T);
    const float2 *row = a.acc + static_cast<long long>(t) * a.E + sc.off + static_cast<long long>(tile) * sc.n;
    const int beg = a.chunk_beg[sc.chunk_off + c], end = a.chunk_end[sc.chunk_off + c];
    double sum = 0.0;
    for (int i = beg + lane; i < end; i += 32) {
        const float2 v = row[a.idx[i]];
        sum += static_cast<double>(v.x) - static_cast<double>(v.y);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
    if (lane == 0) a.partial[item] = sum;
}

// Stage 2: one thread per (scale, tile, q, tau) bin adds its chunks' partials in order and
// normalises: ISF = 2 * sum / s^4 / pixel_count / norm[tau] (0 for an empty annulus).
__global__ void __launch_bounds__(kAzThreads) azimuth_final_kernel(AzArgs a) {
    const long long bin = static_cast<long long>(blockIdx.x) * kAzThreads + threadIdx.x;
    if (bin >= a.bins) return;
    int si = 0;
    while (si + 1 < a.S && bin >= a.sc[si + 1].isf_off) si++;
    const ScaleDesc &sc = a.sc[si];
    const long long rel = bin - sc.isf_off;  // ((tile * Q + q) * T + t)
    const int t = static_cast<int>(rel % a.T);
    const long long tq = rel / a.T;
    const int q = static_cast<int>(tq % a.Q);
    const int tile = static_cast<int>(tq / a.Q);
    const int first = a.chunk_first[sc.q_base + q], cnt = a.chunk_count[sc.q_base + q];
    const double *p = a.partial + sc.item_base + (static_cast<long long>(tile) * a.T + t) * sc.nchunks + first;
    double sum = 0.0;
    for (int c = 0; c < cnt; c++) sum += p[c];
    const int P = a.counts[sc.q_base + q];
    const double nrm = a.norm[t];
    a.isf[bin] = (P != 0 && nrm != 0.0) ? 2.0 * sum * sc.inv_s4 / static_cast<double>(P) / nrm : 0.0;
}

}  // namespace ddm
