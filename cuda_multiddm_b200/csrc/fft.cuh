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
// runs 256/team transforms side by side in shared memory, thread tid working on transform
// tid % (256/team) (transforms fastest: a half-warp then spans 16 transforms, or all of a
// CTA's transforms and 16/that many team members, which with the transform stride below
// keeps every pass and staging access free of bank conflicts at every length -- with teams
// fastest the lengths 32..128 took two wavefronts per access). Element i of a transform
// sits at i + i/16 (one float2 of padding per 16); transforms are kFftPad(L) elements apart.
//
// Every transform length is a template parameter (one instance per log2 L, chosen per scale
// at run time), so all index arithmetic folds to constants. Twiddles come from per-length
// tables computed in FP64 on the host and rounded to FP32 (a pass loads the entries of the
// powers of two of r and forms the others as products, at most three roundings each: 4
// loads instead of 15 per radix-16 group, measured 6 % faster per pass); the radix-16
// kernels use the exact values of cos/sin(k pi/8).
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

namespace ddm {

constexpr int kFftThreads = 256;
constexpr int kFftMaxLog2 = 12;  // largest transform: 4096

__host__ __device__ constexpr int fft_team(int L) { return L >= 16 ? L / 16 : 1; }
__host__ __device__ constexpr int fft_per_cta(int L) {
    return kFftThreads / fft_team(L) < 1 ? 1 : kFftThreads / fft_team(L);
}
// Distance (in float2) between the transforms of a CTA: at least L + L/16 (padded length),
// rounded up so that the column pass's transposed accesses -- NT transforms x 16/NT rows per
// half-warp for NT < 16, 16 transforms for NT >= 16 -- hit 16 distinct 8-byte bank pairs:
// stride = 16/NT (mod 16) when NT < 16, odd otherwise.
__host__ __device__ constexpr int kFftPadTarget(int L) {
    return fft_per_cta(L) < 16 ? 16 / fft_per_cta(L) : 1;
}
__host__ __device__ constexpr int kFftPad(int L) {
    return (L + L / 16 + 1) + ((kFftPadTarget(L) < 16 && fft_per_cta(L) < 16)
                                   ? ((kFftPadTarget(L) - (L + L / 16 + 1) % 16) + 16) % 16
                                   : ((L + L / 16 + 1) % 2 == 0 ? 1 : 0));
}
__device__ __forceinline__ int fpad(int i) { return i + (i >> 4); }

// Butterfly adds and subtractions as one packed FP32x2 instruction each (sm_100a FADD2 / FFMA2
// through the compiler's builtins). Both round exactly as the two scalar operations would: a
// sum is one rounding either way, and b * (-1) + a is exact before its single rounding, i.e.
// a - b. The spectra are therefore the same bit for bit.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
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

// One Stockham pass of radix R over a transform of length L = 2^LOG2L held in buf (padded
// layout) by thread t of its team, with NS the product of the earlier passes' radices.
// Every thread handles G = STRIDE/TEAM groups of R values (1 group for radix 16).
// tw is the table of length L: tw[m] = e^{-2 pi i m / L}.
template <int LOG2L, int R, int NS>
__device__ __forceinline__ void stockham_pass(float2 *buf, int t, const float2 *__restrict__ tw) {
    constexpr int L = 1 << LOG2L;
    constexpr int TEAM = L >= 16 ? L / 16 : 1;
    constexpr int STRIDE = L / R;
    constexpr int G = STRIDE / TEAM < 1 ? 1 : STRIDE / TEAM;
    constexpr int SHIFT = LOG2L - ilog2c<NS>() - ilog2c<R>();  // e^{-2 pi i jm r / (NS R)} = tw[(jm r) << SHIFT]
    float2 v[G * R];
#pragma unroll
    for (int g = 0; g < G; g++) {
        const int j = t + g * TEAM;
        const int jm = j & (NS - 1);
        // twiddles w^(jm r), r < R: the table entries of the powers of two of r, the others
        // as products of those (at most three roundings each)
        float2 wp[R];
        if constexpr (NS > 1) {
#pragma unroll
            for (int b = 1; b < R; b <<= 1) wp[b] = __ldg(tw + ((jm * b) << SHIFT));
#pragma unroll
            for (int r = 3; r < R; r++)
                if (r & (r - 1)) wp[r] = cmulf(wp[r & (r - 1)], wp[r & -r]);
        }
#pragma unroll
        for (int r = 0; r < R; r++) {
            float2 x = buf[fpad(j + r * STRIDE)];
            if (NS > 1 && r > 0) x = cmulf(x, wp[r]);
            v[g * R + r] = x;
        }
    }
    __syncthreads();
#pragma unroll
    for (int g = 0; g < G; g++) {
        dft_reg<R>(v + g * R);
        const int j = t + g * TEAM;
        const int idx = (j & ~(NS - 1)) * R + (j & (NS - 1));
#pragma unroll
        for (int r = 0; r < R; r++) buf[fpad(idx + r * NS)] = v[g * R + r];
    }
    __syncthreads();
}

// The same pass with its inputs read by load(i) and its outputs written by store(i, v) (element
// i of the transform) instead of the shared-memory buffer, and no barriers: for a first pass
// that reads global memory or a last pass that writes it, the caller orders the rest.
template <int LOG2L, int R, int NS, class Load, class Store>
__device__ __forceinline__ void stockham_pass_io(int t, const float2 *__restrict__ tw, Load load, Store store) {
    constexpr int L = 1 << LOG2L;
    constexpr int TEAM = L >= 16 ? L / 16 : 1;
    constexpr int STRIDE = L / R;
    constexpr int G = STRIDE / TEAM < 1 ? 1 : STRIDE / TEAM;
    constexpr int SHIFT = LOG2L - ilog2c<NS>() - ilog2c<R>();
    float2 v[G * R];
#pragma unroll
    for (int g = 0; g < G; g++) {
        const int j = t + g * TEAM;
        const int jm = j & (NS - 1);
        float2 wp[R];
        if constexpr (NS > 1) {
#pragma unroll
            for (int b = 1; b < R; b <<= 1) wp[b] = __ldg(tw + ((jm * b) << SHIFT));
#pragma unroll
            for (int r = 3; r < R; r++)
                if (r & (r - 1)) wp[r] = cmulf(wp[r & (r - 1)], wp[r & -r]);
        }
#pragma unroll
        for (int r = 0; r < R; r++) {
            float2 x = load(j + r * STRIDE);
            if (NS > 1 && r > 0) x = cmulf(x, wp[r]);
            v[g * R + r] = x;
        }
    }
#pragma unroll
    for (int g = 0; g < G; g++) {
        dft_reg<R>(v + g * R);
        const int j = t + g * TEAM;
        const int idx = (j & ~(NS - 1)) * R + (j & (NS - 1));
#pragma unroll
        for (int r = 0; r < R; r++) store(idx + r * NS, v[g * R + r]);
    }
}

// Forward transform of length 2^LOG2L whose input is read by load(i) and whose output is
// written by store(i, v) in global memory: the first pass loads its inputs into registers
// straight from global memory and the last pass stores straight to it; the passes between
// run in place in the shared-memory buffer as fft_transform's do. The same passes and
// arithmetic as fft_transform (same results bit for bit), with one shared-memory round trip
// of the transform's data fewer at each end.
template <int LOG2L, int NS = 1, class Load, class Store>
__device__ __forceinline__ void fft_transform_io(float2 *buf, int t, const float2 *__restrict__ tw, Load load,
                                                 Store store) {
    constexpr int L = 1 << LOG2L;
    constexpr int left = LOG2L - ilog2c<NS>();
    constexpr int R = L < 16 ? L : (left >= 4 ? 16 : (1 << left));
    constexpr bool first = NS == 1, last = NS * R == L;
    auto sload = [buf](int i) { return buf[fpad(i)]; };
    auto sstore = [buf](int i, float2 v) { buf[fpad(i)] = v; };
    if constexpr (first && last) {  // one pass (team of one thread): global to global
        stockham_pass_io<LOG2L, R, NS>(t, tw, load, store);
    } else if constexpr (first) {
        stockham_pass_io<LOG2L, R, NS>(t, tw, load, sstore);
        __syncthreads();
        fft_transform_io<LOG2L, NS * R>(buf, t, tw, load, store);
    } else if constexpr (last) {  // after a barrier: the previous pass's stores are visible
        stockham_pass_io<LOG2L, R, NS>(t, tw, sload, store);
    } else {
        stockham_pass<LOG2L, R, NS>(buf, t, tw);  // in place, ends with a barrier
        fft_transform_io<LOG2L, NS * R>(buf, t, tw, load, store);
    }
}

// Forward transform of length 2^LOG2L: radix-16 passes, then one pass of radix 2, 4 or 8.
template <int LOG2L, int NS = 1>
__device__ __forceinline__ void fft_transform(float2 *buf, int t, const float2 *__restrict__ tw) {
    constexpr int L = 1 << LOG2L;
    if constexpr (L < 16) {
        stockham_pass<LOG2L, L, 1>(buf, t, tw);
    } else {
        constexpr int left = LOG2L - ilog2c<NS>();
        if constexpr (left >= 4) {
            stockham_pass<LOG2L, 16, NS>(buf, t, tw);
            fft_transform<LOG2L, NS * 16>(buf, t, tw);
        } else if constexpr (left == 3) {
            stockham_pass<LOG2L, 8, NS>(buf, t, tw);
        } else if constexpr (left == 2) {
            stockham_pass<LOG2L, 4, NS>(buf, t, tw);
        } else if constexpr (left == 1) {
            stockham_pass<LOG2L, 2, NS>(buf, t, tw);
        }
    }
}

// Per-scale launch geometry shared by both passes (ctas_per_frame over row pairs or columns).
struct FftScale {
    int s, log2s, tiles_side, log2side;
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
    int vec4;  // 1: bpp == 1 and every row start is 4-byte aligned (vectorised pixel loads)
    // ring
    float2 *ring;
    long long E;
    long long first_label;
    int R;
    const float2 *tw;  // tables of length 2, 4, ..., M back to back: the one of length L at tw + L - 2
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

// Loads NT consecutive row pairs (g0, g0 + 1, ...) of the flattened (tile, pair) index of one
// frame into the transform slots of fsm, rows 2p and 2p+1 of a tile packed as the real and
// imaginary parts (zeros past total_pairs).
template <int LOG2L>
__device__ __forceinline__ void fft_load_pairs(const FftArgs &a, const FftScale &sc, float2 *fsm, int g0,
                                               int total_pairs, const uint8_t *fsrc) {
    constexpr int L = 1 << LOG2L, NT = fft_per_cta(L), TS = kFftPad(L);
    constexpr int ITER = NT * L / kFftThreads;
    if constexpr (L >= 4) {
        if (a.vec4) {  // one byte per pixel, 4-byte aligned rows: 4 pixels of each row per load
#pragma unroll
            for (int it = 0; it < ITER / 4; it++) {
                const int q = threadIdx.x + it * kFftThreads;
                const int c = q >> (LOG2L - 2), i = (q & (L / 4 - 1)) * 4;
                const int g = g0 + c;
                uchar4 r0 = make_uchar4(0, 0, 0, 0), r1 = r0;
                if (g < total_pairs) {
                    const int tile = g >> (LOG2L - 1);
                    const int py = 2 * (g & (L / 2 - 1));
                    const int ty = tile >> sc.log2side, tx = tile & (sc.tiles_side - 1);
                    const long long Y = (static_cast<long long>(ty) << LOG2L) + py + a.y_off;
                    const long long X = (static_cast<long long>(tx) << LOG2L) + i + a.x_off;
                    const uint8_t *p0 = fsrc + Y * a.row_pitch + X;
                    r0 = *reinterpret_cast<const uchar4 *>(p0);
                    r1 = *reinterpret_cast<const uchar4 *>(p0 + a.row_pitch);
                }
                float2 *d = fsm + c * TS + fpad(i);  // i .. i+3 share one 16-element pad block
                // In order d[0..3], the one-float2 pad per 16 elements already spreads a
                // half-warp's stores over 16 bank pairs -- except at L = 32, where two
                // transforms share a half-warp; there thread t = 4a + b stores value (k + a) mod 4.
                const float2 v[4] = {make_float2(r0.x, r1.x), make_float2(r0.y, r1.y), make_float2(r0.z, r1.z),
                                     make_float2(r0.w, r1.w)};
                const int a4 = L == 32 ? (threadIdx.x >> 2) & 3 : 0;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const int m = (k + a4) & 3;
                    d[m] = m == 0 ? v[0] : m == 1 ? v[1] : m == 2 ? v[2] : v[3];
                }
            }
            return;
        }
    }
#pragma unroll
    for (int it = 0; it < ITER; it++) {
        const int q = threadIdx.x + it * kFftThreads;
        const int c = q >> LOG2L, i = q & (L - 1);
        const int g = g0 + c;
        float2 z = make_float2(0.f, 0.f);
        if (g < total_pairs) {
            const int tile = g >> (LOG2L - 1 > 0 ? LOG2L - 1 : 0);
            const int py = 2 * (g & (L / 2 - 1));
            const int ty = tile >> sc.log2side, tx = tile & (sc.tiles_side - 1);
            const long long Y = (static_cast<long long>(ty) << LOG2L) + py + a.y_off;
            const long long X = (static_cast<long long>(tx) << LOG2L) + i + a.x_off;
            const uint8_t *p0 = fsrc + Y * a.row_pitch + X * a.bpp;
            z = make_float2(fft_pixel(p0, a.pixmode), fft_pixel(p0 + a.row_pitch, a.pixmode));
        }
        fsm[c * TS + fpad(i)] = z;
    }
}

// Row pass at scale 2^LOG2L: the CTA transforms NT consecutive row pairs of the flattened
// (tile, pair) index of frame blockIdx.y, rows 2p and 2p+1 packed as real and imaginary parts.
template <int LOG2L>
__device__ __forceinline__ void fft_rows_body(const FftArgs &a, const FftScale &sc, float2 *fsm) {
    constexpr int L = 1 << LOG2L, TEAM = fft_team(L), NT = fft_per_cta(L), TS = kFftPad(L);
    constexpr int NX = L / 2 + 1;
    const int total_pairs = (1 << (2 * sc.log2side)) * (L / 2);
    const int g0 = (blockIdx.x - sc.cta_begin) * NT;
    fft_load_pairs<LOG2L>(a, sc, fsm, g0, total_pairs, a.src + blockIdx.y * a.frame_stride);
    __syncthreads();
    const int c_me = threadIdx.x & (NT - 1), t = threadIdx.x / NT;  // transforms fastest (no bank conflicts)
    fft_transform<LOG2L>(fsm + c_me * TS, t, a.tw + (L - 2));  // ends with a CTA barrier
    // split Z = X0 + i X1 into the two real rows' half spectra, teams fastest again so that
    // a team's consecutive threads store consecutive elements of one output row
    const int c_out = threadIdx.x / TEAM, t_out = threadIdx.x & (TEAM - 1);
    const float2 *buf = fsm + c_out * TS;
    const int g = g0 + c_out;
    if (g >= total_pairs) return;
    const int tile = g >> (LOG2L - 1 > 0 ? LOG2L - 1 : 0);
    const int py = 2 * (g & (L / 2 - 1));
    const long long slot = (a.first_label + blockIdx.y) % a.R;
    float2 *o = a.ring + slot * a.E + sc.off + tile * sc.n + static_cast<long long>(py) * NX;
#pragma unroll
    for (int m = 0; m < (NX + TEAM - 1) / TEAM; m++) {
        const int k = t_out + m * TEAM;
        if (k < NX) {
            const float2 zk = buf[fpad(k & (L - 1))], zm = buf[fpad((L - k) & (L - 1))];
            o[k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
            o[NX + k] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
        }
    }
}

// Column pass at scale 2^LOG2L: NT consecutive columns of the flattened (tile, kx) index of
// frame blockIdx.y, transformed along y in place.
template <int LOG2L>
__device__ __forceinline__ void fft_cols_body(const FftArgs &a, const FftScale &sc, float2 *fsm) {
    constexpr int L = 1 << LOG2L, NT = fft_per_cta(L), TS = kFftPad(L);
    constexpr int NX = L / 2 + 1;
    const int total_cols = (1 << (2 * sc.log2side)) * NX;
    const int g0 = (blockIdx.x - sc.cta_begin) * NT;
    const long long slot = (a.first_label + blockIdx.y) % a.R;
    float2 *base = a.ring + slot * a.E + sc.off;
    // transforms fastest (no bank conflicts in the shared-memory passes); a half-warp's global
    // accesses cover NT consecutive columns (of one row of a tile) times 16/NT rows
    const int c_me = threadIdx.x & (NT - 1), t = threadIdx.x / NT;
    const int g = g0 + c_me;
    const bool valid = g < total_cols;  // threads past the last column still take every barrier
    const int tile = valid ? g / NX : 0, col = valid ? g - tile * NX : 0;
    float2 *colp = base + tile * sc.n + col;
    fft_transform_io<LOG2L>(
        fsm + c_me * TS, t, a.tw + (L - 2),
        [&](int y) { return valid ? colp[static_cast<long long>(y) * NX] : make_float2(0.f, 0.f); },
        [&](int y, float2 v) {
            if (valid) colp[static_cast<long long>(y) * NX] = v;
        });
}

// Both passes of the tiles of side 32, 64 and 128 in one kernel, the tile held in shared
// memory between them (one HBM write of each half spectrum, no intermediate round trip).
// A CTA owns kFftTileTiles(L) consecutive tiles of frame blockIdx.y: 1 at 128 (its 64 row pairs
// in two rounds of 32 transforms), 2 at 64, 8 at 32 (one round). Row rounds load row pairs
// into the transform slots, transform them and split each into two half-spectrum rows of the
// tile buffer Yt[tile][y][kx] (rows NXP float2 apart); column rounds transform NT columns of Yt
// along y, the first pass reading Yt and the last writing the ring slot directly.
__host__ __device__ constexpr int kFftTileTiles(int L) {
    return fft_per_cta(L) / (L / 2) > 1 ? fft_per_cta(L) / (L / 2) : 1;
}
__host__ __device__ constexpr int kFftTileNxp(int L) { return L / 2 + 2; }
inline size_t fft_tile_smem_bytes(int L) {
    return sizeof(float2) * (static_cast<size_t>(fft_per_cta(L)) * kFftPad(L) +
                             static_cast<size_t>(kFftTileTiles(L)) * L * kFftTileNxp(L));
}

template <int LOG2L>
__device__ __forceinline__ void fft_tile_body(const FftArgs &a, const FftScale &sc, float2 *fsm) {
    constexpr int L = 1 << LOG2L, TEAM = fft_team(L), NT = fft_per_cta(L), TS = kFftPad(L);
    constexpr int NX = L / 2 + 1, NXP = kFftTileNxp(L), TPC = kFftTileTiles(L);
    float2 *yt = fsm + NT * TS;  // [TPC][L][NXP]
    const int tiles = 1 << (2 * sc.log2side);
    const int tile0 = (blockIdx.x - sc.cta_begin) * TPC;
    const int ntl = tiles - tile0 < TPC ? tiles - tile0 : TPC;  // tiles of this CTA
    const int pairs = ntl * (L / 2);
    const int c_me = threadIdx.x & (NT - 1), t = threadIdx.x / NT;
    const int c_out = threadIdx.x / TEAM, t_out = threadIdx.x & (TEAM - 1);
    // ---- rows: pairs of the CTA's tiles, NT per round
    for (int r0 = 0; r0 < pairs; r0 += NT) {
        fft_load_pairs<LOG2L>(a, sc, fsm, tile0 * (L / 2) + r0, tile0 * (L / 2) + pairs,
                              a.src + blockIdx.y * a.frame_stride);
        __syncthreads();
        fft_transform<LOG2L>(fsm + c_me * TS, t, a.tw + (L - 2));  // ends with a CTA barrier
        const int g = r0 + c_out;  // pair of the CTA's tiles
        if (g < pairs) {
            const float2 *buf = fsm + c_out * TS;
            const int tl = g >> (LOG2L - 1), py = 2 * (g & (L / 2 - 1));
            float2 *o = yt + (tl * L + py) * NXP;
#pragma unroll
            for (int m = 0; m < (NX + TEAM - 1) / TEAM; m++) {
                const int k = t_out + m * TEAM;
                if (k < NX) {
                    const float2 zk = buf[fpad(k & (L - 1))], zm = buf[fpad((L - k) & (L - 1))];
                    o[k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
                    o[NXP + k] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
                }
            }
        }
        __syncthreads();  // the slots are reloaded next round; Yt is read by the columns
    }
    // ---- columns: (tile, kx) of the CTA's tiles, NT per round
    const long long slot = (a.first_label + blockIdx.y) % a.R;
    float2 *base = a.ring + slot * a.E + sc.off;
    const int cols = ntl * NX;
    for (int c0 = 0; c0 < cols; c0 += NT) {
        // the first pass reads its column of Yt straight into registers, the last writes the
        // half spectrum's column straight to the ring slot (fft_transform_io)
        const int g = c0 + c_me;
        const bool valid = g < cols;  // threads past the last column still take every barrier
        const int tl = valid ? g / NX : 0, col = valid ? g - tl * NX : 0;
        const float2 *ycol = yt + tl * L * NXP + col;
        float2 *ocol = base + (tile0 + tl) * sc.n + col;
        fft_transform_io<LOG2L>(
            fsm + c_me * TS, t, a.tw + (L - 2),
            [&](int y) { return valid ? ycol[y * NXP] : make_float2(0.f, 0.f); },
            [&](int y, float2 v) {
                if (valid) ocol[static_cast<long long>(y) * NX] = v;
            });
        __syncthreads();  // the next round's first pass rewrites the transform slots
    }
}

// One instance per tile side (32, 64, 128), so that each gets the registers its own body
// needs; grid (tiles / kFftTileTiles(L), frames) of the scale a.sc[0].
// (side 128 holds 103 KB of shared memory, so two CTAs per SM at most; the others three)
template <int LOG2L>
__global__ void __launch_bounds__(kFftThreads, LOG2L == 7 ? 2 : 3) fft_tile_kernel(FftArgs a) {
    extern __shared__ float2 fsm[];
    fft_tile_body<LOG2L>(a, a.sc[0], fsm);
}

#define DDM_FFT_DISPATCH(BODY)                      \
    switch (sc.log2s) {                             \
        case 1: BODY<1>(a, sc, fsm); break;         \
        case 2: BODY<2>(a, sc, fsm); break;         \
        case 3: BODY<3>(a, sc, fsm); break;         \
        case 4: BODY<4>(a, sc, fsm); break;         \
        case 5: BODY<5>(a, sc, fsm); break;         \
        case 6: BODY<6>(a, sc, fsm); break;         \
        case 7: BODY<7>(a, sc, fsm); break;         \
        case 8: BODY<8>(a, sc, fsm); break;         \
        case 9: BODY<9>(a, sc, fsm); break;         \
        case 10: BODY<10>(a, sc, fsm); break;       \
        case 11: BODY<11>(a, sc, fsm); break;       \
        default: BODY<12>(a, sc, fsm); break;       \
    }

// grid (sum of ctas_per_frame, frames)
__global__ void __launch_bounds__(kFftThreads, 4) fft_rows_kernel(FftArgs a) {
    extern __shared__ float2 fsm[];
    const FftScale &sc = a.sc[fft_find_scale(a)];
    DDM_FFT_DISPATCH(fft_rows_body)
}

__global__ void __launch_bounds__(kFftThreads, 4) fft_cols_kernel(FftArgs a) {
    extern __shared__ float2 fsm[];
    const FftScale &sc = a.sc[fft_find_scale(a)];
    DDM_FFT_DISPATCH(fft_cols_body)
}
#undef DDM_FFT_DISPATCH

inline size_t fft_smem_bytes(int L) { return sizeof(float2) * static_cast<size_t>(fft_per_cta(L)) * kFftPad(L); }

// Twiddle tables for lengths 2, 4, ..., M back to back (length L at offset L - 2), from FP64
// math rounded to FP32: entry m of the length-L table is e^{-2 pi i m / L}.
inline std::vector<float2> fft_twiddle_tables(int M) {
    std::vector<float2> tw;
    const double two_pi = 6.283185307179586476925286766559;
    for (int L = 2; L <= M; L <<= 1)
        for (int m = 0; m < L; m++) {
            const double ang = two_pi * m / L;
            tw.push_back(make_float2(static_cast<float>(std::cos(ang)), static_cast<float>(-std::sin(ang))));
        }
    return tw;
}

}  // namespace ddm
