// Split-BF16 tensor-core DFT of the small tiles (s = 32, 64, 128): the optional
// alternative to the FP32 Stockham FFT (csrc/fft.cuh) for those scales, replacing the
// reference's batched cuFFT R2C (src/DDM.cu:189-192, plans :648-677) there.
//
// The 2-D R2C DFT of an s x s real tile X, as two GEMMs on the 5th-generation tensor
// cores (tcgen05.mma, kind::f16 with BF16 operands and FP32 accumulators in TMEM):
//
//   row step     Yr[y][kx] = sum_x X[y][x] cos(2 pi kx x / s)
//                Yi[y][kx] = -sum_x X[y][x] sin(2 pi kx x / s)         kx in [0, s/2]
//   column step  Zr[ky][kx] = sum_y cos(2 pi ky y / s) Yr[y][kx] + sin(2 pi ky y / s) Yi[y][kx]
//                Zi[ky][kx] = sum_y cos(2 pi ky y / s) Yi[y][kx] - sin(2 pi ky y / s) Yr[y][kx]
//
// i.e. Z = F X F^T restricted to kx <= s/2, with F = cos - i sin (unnormalised, e^{-i}).
// Precision: every FP32 value v that enters a product is split as v = hi + lo, both BF16
// (hi = bf16(v), lo = bf16(v - hi), together 16 significant bits), and a product a * b is
// formed as hi*hi + hi*lo + lo*hi (the lo*lo term, below 2^-16 relative, is dropped), all
// accumulated in FP32. The cos/sin tables are split on the host from FP64 values. u8 pixels
// (and the BYTE0 mode's first bytes) are exact in BF16; full 16-bit pixels are exact as
// hi + lo. The spectra are within about 1e-5 of the tile maximum of the FP64 transform.
//
// Work per CTA (persistent; one CTA per SM, 128 threads): a batch is 128 rows of tiles
// (128 / s tiles), the M of one MMA. Per batch:
//   1. pixels -> BF16 (hi [, lo]) into shared memory as the A operand (rows (tile, y), K = x)
//   2. thread 0 issues the row-step MMAs (B = the first N1 rows of the cos / sin tables,
//      N1 = s/2 + 1 rounded up to 16) into TMEM, commit -> mbarrier
//   3. all threads read their TMEM lane (one row (tile, y)), split Yr, Yi into hi / lo and
//      store them as the column step's B operands (rows kx, K = y) over the A operand's space
//   4. thread 0 issues the column-step MMAs per tile (A = the cos / sin tables padded to 128
//      rows, M = ky), commit -> mbarrier
//   5. thread ky < s reads row ky of Zr, Zi and writes the half-spectrum row to the ring slot.
// Operands use the tensor cores' K-major layout without swizzle: 8 x 8 core matrices of 128
// bytes, element (r, k) at ((r / 8) * (K / 8) + k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// so the stride between K-adjacent core matrices (LBO) is 128 B and between 8-row groups
// (SBO) K * 16 B. Every mbarrier wait is bounded and reports through the status word; the
// TMEM allocation is released by the allocating warp before the CTA exits.
#pragma once

#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "fft.cuh"
#include "lag.cuh"

namespace ddm {

constexpr int kDftThreads = 128;
constexpr int kDftMinLog2 = 5, kDftMaxLog2 = 7;  // s = 32, 64, 128
constexpr uint32_t kDftTmemCols = 256;

__host__ __device__ constexpr int dft_n1(int s) { return ((s / 2 + 1) + 15) / 16 * 16; }
// bytes of one K-major BF16 operand of `rows` rows and K = s
__host__ __device__ constexpr uint32_t dft_operand_bytes(int rows, int s) { return static_cast<uint32_t>(rows) * s * 2; }
// the cos/sin tables: [part hi, lo][C, S][128 rows][s] -> 4 operands of 128 rows
__host__ __device__ constexpr uint32_t dft_table_bytes(int s) { return 4 * dft_operand_bytes(128, s); }
// per batch: A (pixels hi, lo) or, over the same space, per tile the column step's B operands
// [Yr hi, Yr lo, Yi hi, Yi lo][N1 rows][s]
__host__ __device__ constexpr uint32_t dft_region_bytes(int s) {
    return (2 * dft_operand_bytes(128, s) > (128 / s) * 4 * dft_operand_bytes(dft_n1(s), s))
               ? 2 * dft_operand_bytes(128, s)
               : (128 / s) * 4 * dft_operand_bytes(dft_n1(s), s);
}
// dynamic shared memory: 1 KB alignment slack, tables, region, mbarrier + TMEM address; at
// least 77 KB, so that at most two CTAs share an SM and their TMEM allocations (256 columns
// each) never exceed the SM's 512 columns
__host__ __device__ constexpr uint32_t dft_smem_used(int s) { return 1024 + dft_table_bytes(s) + dft_region_bytes(s) + 64; }
__host__ __device__ constexpr uint32_t dft_smem_bytes(int s) { return dft_smem_used(s) > 77u * 1024 ? dft_smem_used(s) : 77u * 1024; }

static_assert(dft_smem_bytes(128) <= 227 * 1024, "s = 128 DFT does not fit shared memory");
static_assert(3 * dft_smem_bytes(32) > 228 * 1024 && 3 * dft_smem_bytes(64) > 228 * 1024,
              "three DFT CTAs on one SM would need more TMEM columns than it has");
static_assert(2 * dft_n1(128) <= static_cast<int>(kDftTmemCols), "row-step accumulators exceed the TMEM allocation");
static_assert((128 / 64) * 2 * dft_n1(64) <= static_cast<int>(kDftTmemCols), "s = 64 accumulators exceed TMEM");
static_assert((128 / 32) * 2 * dft_n1(32) <= static_cast<int>(kDftTmemCols), "s = 32 accumulators exceed TMEM");

__host__ __device__ constexpr uint32_t dft_core_offset(int r, int k, int s) {
    return static_cast<uint32_t>(((r >> 3) * (s >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// ---- tcgen05 wrappers ---------------------------------------------------------------------

// Shared-memory matrix descriptor (tcgen05): start address, LBO, SBO (all >> 4), version 1,
// no swizzle.
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((saddr & 0x3FFFFu) >> 4) | (static_cast<uint64_t>((lbo & 0x3FFFFu) >> 4) << 16) |
           (static_cast<uint64_t>((sbo & 0x3FFFFu) >> 4) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16: FP32 D, BF16 A and B, both K-major, M x N, optional
// negation of B.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N, bool neg_b) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((neg_b ? 1u : 0u) << 14) | (static_cast<uint32_t>(N >> 3) << 17) |
           (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive 32-bit TMEM columns of this thread's lane. The load and its wait are one
// asm statement, so no use of the registers can be scheduled before the wait.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

struct DftArgs {
    const uint8_t *src;
    long long frame_stride, row_pitch;
    int bpp, pixmode, x_off, y_off;
    float2 *ring;
    long long E;
    long long first_label;
    int R;
    int nframes;
    FftScale sc;
    const uint4 *tables;  // dft_table_bytes(s) bytes, already in the shared-memory layout
    int *status;
    int vec16;            // 1: one byte per pixel and every tile row 16-byte aligned (16-pixel loads)
};

// the column step's output of a batch, staged as [tile][ky][kx] over the operand region
static_assert(128 * (128 / 2 + 1) * 8 <= dft_region_bytes(128) && 2 * 64 * (64 / 2 + 1) * 8 <= dft_region_bytes(64) &&
                  4 * 32 * (32 / 2 + 1) * 8 <= dft_region_bytes(32),
              "a batch's half spectra must fit the operand region");

// bounded wait on the CTA's mbarrier; false after kWaitCycles
__device__ __forceinline__ bool dft_wait(uint64_t *bar, uint32_t parity) { return mbar_wait_bounded(bar, parity); }

template <int LOG2S>
__global__ void __launch_bounds__(kDftThreads, 1) dft_bf16_kernel(DftArgs a) {
    constexpr int S = 1 << LOG2S;
    constexpr int N1 = dft_n1(S);
    constexpr int TPB = 128 / S;                       // tiles per batch
    constexpr uint32_t OP128 = dft_operand_bytes(128, S);
    constexpr uint32_t OPN1 = dft_operand_bytes(N1, S);
    constexpr uint32_t SBO = S * 16, LBO = 128;
    constexpr int KSTEPS = S / 16;
    constexpr int NX = S / 2 + 1;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u);
    unsigned char *tab = smem;                          // [hi, lo][C, S] x OP128
    unsigned char *reg = smem + dft_table_bytes(S);     // A (pixels) / B (row spectra)
    uint64_t *bar = reinterpret_cast<uint64_t *>(reg + dft_region_bytes(S));
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(bar + 2);

    const int tid = threadIdx.x, warp = tid >> 5;
    // tables: plain 16-byte loads, once per CTA
    for (uint32_t i = tid; i < dft_table_bytes(S) / 16; i += kDftThreads)
        reinterpret_cast<uint4 *>(tab)[i] = a.tables[i];
    if (tid == 0) {
        mbar_init(bar, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(kDftTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;  // this warp's TMEM lanes

    const FftScale &sc = a.sc;
    const int tiles = 1 << (2 * sc.log2side);
    const int batches = (tiles + TPB - 1) / TPB;
    const long long items = static_cast<long long>(batches) * a.nframes;
    const bool two_part_a = a.pixmode == 1;  // full 16-bit pixels: hi + lo
    const uint32_t tab_addr = smem_addr(tab), reg_addr = smem_addr(reg);
    uint32_t phase = 0;

    for (long long item = blockIdx.x; item < items && !*abort_flag; item += gridDim.x) {
        const int f = static_cast<int>(item / batches);
        const int b = static_cast<int>(item - static_cast<long long>(f) * batches);
        // ---- 1. pixels of row `tid` = (tile tl, y) -> A operand (hi, lo) --------------------
        {
            const int tl = tid / S, y = tid & (S - 1);
            const int tile = b * TPB + tl;
            const uint8_t *fsrc = a.src + static_cast<long long>(f) * a.frame_stride;
            const bool valid = tile < tiles;
            const int ty = tile >> sc.log2side, tx = tile & (sc.tiles_side - 1);
            const long long Y = (static_cast<long long>(ty) << LOG2S) + y + a.y_off;
            const long long X0 = (static_cast<long long>(tx) << LOG2S) + a.x_off;
            const uint8_t *row = fsrc + Y * a.row_pitch + X0 * a.bpp;
            if (a.vec16) {  // bytes: exact in BF16, no lo part; 16 pixels per load
#pragma unroll 2
                for (int k16 = 0; k16 < S / 16; k16++) {
                    uint4 u = make_uint4(0u, 0u, 0u, 0u);
                    if (valid) u = *reinterpret_cast<const uint4 *>(row + k16 * 16);
                    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        __align__(16) __nv_bfloat16 hi[8];
#pragma unroll
                        for (int i = 0; i < 8; i++)
                            hi[i] = __float2bfloat16_rn(static_cast<float>((w[h * 2 + i / 4] >> (8 * (i & 3))) & 0xFFu));
                        *reinterpret_cast<uint4 *>(reg + dft_core_offset(tid, k16 * 16 + h * 8, S)) =
                            *reinterpret_cast<const uint4 *>(hi);
                    }
                }
            } else {
#pragma unroll 2
                for (int kg = 0; kg < S / 8; kg++) {
                    __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        float v = 0.f;
                        if (valid) v = fft_pixel(row + (kg * 8 + i) * a.bpp, a.pixmode);
                        hi[i] = __float2bfloat16_rn(v);
                        lo[i] = __float2bfloat16_rn(v - __bfloat162float(hi[i]));
                    }
                    const uint32_t off = dft_core_offset(tid, kg * 8, S);
                    *reinterpret_cast<uint4 *>(reg + off) = *reinterpret_cast<const uint4 *>(hi);
                    if (two_part_a) *reinterpret_cast<uint4 *>(reg + OP128 + off) = *reinterpret_cast<const uint4 *>(lo);
                }
            }
        }
        fence_proxy_async_smem();
        __syncthreads();
        // ---- 2. row step: D[c][row][kx], c = 0 cos (cols 0..N1), 1 sin (cols N1..2 N1) -------
        if (tid == 0) {
            tc_fence_after();
            constexpr uint32_t idesc = umma_idesc_bf16(128, N1, false);
            for (int c = 0; c < 2; c++) {
                const uint32_t d = tmem + static_cast<uint32_t>(c * N1);
                int first = 1;
                for (int ks = 0; ks < KSTEPS; ks++) {
                    // (A part, table part): hi*hi, hi*lo, and lo*hi for 16-bit pixels
                    for (int p = 0; p < (two_part_a ? 3 : 2); p++) {
                        const int ap = p == 2 ? 1 : 0, tp = p == 1 ? 1 : 0;
                        const uint64_t ad = umma_smem_desc(reg_addr + ap * OP128 + ks * 256, LBO, SBO);
                        const uint64_t bd = umma_smem_desc(tab_addr + (tp * 2 + c) * OP128 + ks * 256, LBO, SBO);
                        umma_bf16(d, ad, bd, idesc, first ? 0u : 1u);
                        first = 0;
                    }
                }
            }
            umma_commit(bar);
        }
        if (!dft_wait(bar, phase & 1)) *abort_flag = 1;
        phase++;
        tc_fence_after();
        if (*abort_flag) break;
        // ---- 3. TMEM row (tile tl, y) -> column-step B operands of tile tl ------------------
        {
            const int tl = tid / S, y = tid & (S - 1);
            unsigned char *bt = reg + tl * 4 * OPN1;  // [Yr hi, Yr lo, Yi hi, Yi lo]
#pragma unroll 1
            for (int k0 = 0; k0 < N1; k0 += 16) {
                float re[16], im[16];
                tmem_ld16(tmem + lane_base + k0, re);
                tmem_ld16(tmem + lane_base + N1 + k0, im);
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const uint32_t off = dft_core_offset(k0 + i, y, S);
                    const float yr = re[i], yi = -im[i];
                    const __nv_bfloat16 rh = __float2bfloat16_rn(yr), ih = __float2bfloat16_rn(yi);
                    *reinterpret_cast<__nv_bfloat16 *>(bt + off) = rh;
                    *reinterpret_cast<__nv_bfloat16 *>(bt + OPN1 + off) = __float2bfloat16_rn(yr - __bfloat162float(rh));
                    *reinterpret_cast<__nv_bfloat16 *>(bt + 2 * OPN1 + off) = ih;
                    *reinterpret_cast<__nv_bfloat16 *>(bt + 3 * OPN1 + off) = __float2bfloat16_rn(yi - __bfloat162float(ih));
                }
            }
        }
        tc_fence_before();
        fence_proxy_async_smem();
        __syncthreads();
        // ---- 4. column step per tile: Zr at cols t*2N1, Zi at t*2N1 + N1 --------------------
        if (tid == 0) {
            tc_fence_after();
            constexpr uint32_t idesc = umma_idesc_bf16(128, N1, false);
            constexpr uint32_t idesc_neg = umma_idesc_bf16(128, N1, true);
            for (int tl = 0; tl < TPB; tl++) {
                const uint32_t bt = reg_addr + tl * 4 * OPN1;
                for (int z = 0; z < 2; z++) {  // 0: Zr = C.Yr + S.Yi, 1: Zi = C.Yi - S.Yr
                    const uint32_t d = tmem + static_cast<uint32_t>(tl * 2 * N1 + z * N1);
                    int first = 1;
                    for (int term = 0; term < 2; term++) {  // table C or S
                        const int yb = (z == 0) ? (term == 0 ? 0 : 2) : (term == 0 ? 2 : 0);  // Yr or Yi
                        const uint32_t id = (z == 1 && term == 1) ? idesc_neg : idesc;
                        for (int ks = 0; ks < KSTEPS; ks++) {
                            for (int p = 0; p < 3; p++) {  // table hi * Y hi, table hi * Y lo, table lo * Y hi
                                const int tp = p == 2 ? 1 : 0, yp = p == 1 ? 1 : 0;
                                const uint64_t ad = umma_smem_desc(tab_addr + (tp * 2 + term) * OP128 + ks * 256, LBO, SBO);
                                const uint64_t bd = umma_smem_desc(bt + (yb + yp) * OPN1 + ks * 256, LBO, SBO);
                                umma_bf16(d, ad, bd, id, first ? 0u : 1u);
                                first = 0;
                            }
                        }
                    }
                }
            }
            umma_commit(bar);
        }
        if (!dft_wait(bar, phase & 1)) *abort_flag = 1;
        phase++;
        tc_fence_after();
        if (*abort_flag) break;
        // ---- 5. rows ky < s of Zr, Zi -> staged [tile][ky][kx] over the operand region (the
        // column step has finished reading it), then one coalesced copy of the batch's tiles,
        // which are consecutive in the ring slot ------------------------------------------------
        {
            float2 *stage = reinterpret_cast<float2 *>(reg);
            for (int tl = 0; tl < TPB; tl++) {
                // every warp takes part in the TMEM loads (sync.aligned); lanes ky >= s hold the
                // padding rows of the tables and stage nothing
                float2 *o = stage + (tl * S + tid) * NX;
#pragma unroll 1
                for (int k0 = 0; k0 < N1; k0 += 16) {
                    float zr[16], zi[16];
                    tmem_ld16(tmem + lane_base + tl * 2 * N1 + k0, zr);
                    tmem_ld16(tmem + lane_base + tl * 2 * N1 + N1 + k0, zi);
                    if (tid < S) {
#pragma unroll
                        for (int i = 0; i < 16; i++)
                            if (k0 + i < NX) o[k0 + i] = make_float2(zr[i], zi[i]);
                    }
                }
            }
            __syncthreads();
            const long long slot = (a.first_label + f) % a.R;
            const int ntl = tiles - b * TPB < TPB ? tiles - b * TPB : TPB;
            // sc.n = S * NX is even and every tile starts on a 16-byte boundary of the ring slot
            uint4 *dst = reinterpret_cast<uint4 *>(a.ring + slot * a.E + sc.off + static_cast<long long>(b * TPB) * sc.n);
            const uint4 *src = reinterpret_cast<const uint4 *>(stage);
            const int n16 = ntl * S * NX / 2;
            for (int i = tid; i < n16; i += kDftThreads) dst[i] = src[i];
        }
        tc_fence_before();
        __syncthreads();
    }
    __syncthreads();
    if (*abort_flag && tid == 0) atomicExch(a.status, 2);
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kDftTmemCols) : "memory");
    }
}

// Host: the cos / sin tables of one s split into BF16 hi / lo, in the kernel's shared-memory
// layout: [part hi, lo][table C, S][128 rows (ky or kx; rows >= s are zero)][K = s].
inline uint16_t bf16_bits_rn(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return static_cast<uint16_t>((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
}
inline float bf16_value(uint16_t b) {
    const uint32_t u = static_cast<uint32_t>(b) << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline std::vector<uint16_t> dft_tables(int s) {
    std::vector<uint16_t> t(dft_table_bytes(s) / 2, 0);
    const double two_pi = 6.283185307179586476925286766559;
    for (int c = 0; c < 2; c++)
        for (int r = 0; r < s; r++)
            for (int k = 0; k < s; k++) {
                const long long m = (static_cast<long long>(r) * k) % s;  // exact argument reduction
                const double ang = two_pi * static_cast<double>(m) / s;
                const double v = c == 0 ? std::cos(ang) : std::sin(ang);
                const uint16_t hi = bf16_bits_rn(static_cast<float>(v));
                const uint16_t lo = bf16_bits_rn(static_cast<float>(v - static_cast<double>(bf16_value(hi))));
                const size_t off = dft_core_offset(r, k, s) / 2;
                t[(0 * 2 + c) * (dft_operand_bytes(128, s) / 2) + off] = hi;
                t[(1 * 2 + c) * (dft_operand_bytes(128, s) / 2) + off] = lo;
            }
    return t;
}

}  // namespace ddm
