// Lag kernel: accumulates |F(x) - F(y)|^2 for a block of J "register" frames x against
// the partner frame y of every tau, per spectrum element (replaces processFFT,
// src/DDM_kernel.cuh:85-101, which the reference launches once per (scale, tau, frame)).
//
// Work decomposition. One CTA owns a block of kLagBlock consecutive elements of the
// flattened frame vector (all scales and tiles concatenated, so the kernel needs no
// geometry). Its threads keep the J register frames of their element in registers. The
// partner of (register frame j, tau entry e) is window position ub_e + j of a sorted list
// of distinct partner frames (the "union"), which the host builds per launch: windows of
// consecutive taus overlap, so a chunk of 30 frames against 64 log-spaced taus up to 500
// needs about 480 distinct partner frames instead of 30 * 64 = 1920 frame reads.
//
// Data movement (sm_100a). Partner frames stream through a ring of kLagSlots shared-memory
// slots, one slot = the CTA's element block of one frame (1 KB), grouped by kLagGroup. The
// ring in HBM is addressed through 2-D tensor maps ([slots][elements], boxes of 1..8 slots
// x kLagBlock elements), so a run of consecutive frames arrives with one
// cp.async.bulk.tensor.2d (no multicast) that completes on the group's "full" mbarrier. A
// dedicated producer warp refills a group once every consumer warp has arrived on its
// "empty" mbarrier, i.e. has moved past the last window that reads it.
// The ring is a power of two of slots, so a window position becomes a shared-memory address
// with one add and one mask. The |dF|^2 arithmetic uses packed FP32x2 instructions.
// Accumulators (FP32 sum + Kahan compensation, 8 B) are loaded three entries ahead with
// plain coalesced loads and written back once per entry.
//
// Every mbarrier wait is bounded (kWaitCycles clock cycles); a wait that runs out
// sets *status to 1, and the CTA waits (bounded again) for its own copies in flight before
// returning, so a broken schedule ends the kernel instead of hanging the GPU.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace ddm {

constexpr int kLagBlock = 128;                     // elements per CTA, one per consumer thread
constexpr int kLagConsumerWarps = kLagBlock / 32;
constexpr int kLagThreads = kLagBlock + 32;        // consumers + one producer warp
constexpr int kLagSlotsLog2 = 6;
constexpr int kLagSlots = 1 << kLagSlotsLog2;      // shared-memory frame slots (> 32 frames)
constexpr uint32_t kLagSlotBytes = kLagBlock * 8;  // one frame of the CTA's elements
constexpr uint32_t kLagRingBytes = kLagSlots * kLagSlotBytes;
constexpr uint32_t kLagRingMask = kLagRingBytes - kLagSlotBytes;  // slot bits of a ring offset
constexpr int kLagSmemMax = 220 * 1024;
// Register-frame counts the kernel is instantiated for (a launch uses the smallest >= nreg).
constexpr int kLagJs[] = {4, 8, 16, 20, 24, 30, 32};
constexpr int kNumLagJs = sizeof(kLagJs) / sizeof(kLagJs[0]);

// Union entries are copied in groups of kLagGroup consecutive entries; a group's ring
// slots arrive as runs of 1, 2, 4 or 8 consecutive slots (one 2-D TMA box each).
constexpr int kLagGroupLog2 = 3;
constexpr int kLagGroup = 1 << kLagGroupLog2;
constexpr int kLagGroupSlotsLog2 = kLagSlotsLog2 - kLagGroupLog2;
constexpr int kLagGroupSlots = 1 << kLagGroupSlotsLog2;
constexpr int kLagRunKinds = 4;  // box heights 1, 2, 4, 8

// A run: ring slot in bits 0..19, log2(rows) in bits 20..21, position in its group in 22..24.
__host__ __device__ constexpr int lag_run(int rel, int slot, int log2rows) {
    return slot | (log2rows << 20) | (rel << 22);
}
__host__ __device__ constexpr int lag_run_slot(int run) { return run & 0xFFFFF; }
__host__ __device__ constexpr int lag_run_log2rows(int run) { return (run >> 20) & 3; }
__host__ __device__ constexpr int lag_run_rel(int run) { return (run >> 22) & 7; }

// Lag table layout (ints): header, register frames, then ntau accumulator indices, ntau
// union starts, ntau full-window flags, nunion ring slots, ngroups+1 run offsets, nruns runs.
constexpr int kTabNreg = 0, kTabNtau = 1, kTabNunion = 2, kTabNgroups = 3, kTabNruns = 4, kTabReg = 5;
constexpr int kTabEntries = kTabReg + 32;
__host__ __device__ constexpr int lag_table_ints(int ntau, int nunion, int ngroups, int nruns) {
    return kTabEntries + 3 * ntau + nunion + ngroups + 1 + nruns;
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false if the phase did not complete within kWaitCycles SM clocks (about
// 0.2 s at 2 GHz, four orders of magnitude above any legitimate copy latency).
constexpr long long kWaitCycles = 400000000LL;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > kWaitCycles) return false;
    return true;
}

// Packed FP32x2 helpers (sm_100a): one instruction for both halves of a complex value.
__device__ __forceinline__ unsigned long long f2_sub(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

__device__ __forceinline__ unsigned long long f2_fma_sq(unsigned long long d, unsigned long long acc) {
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %1, %2;" : "=l"(r) : "l"(d), "l"(acc));
    return r;
}

__device__ __forceinline__ float f2_hsum(unsigned long long v) {
    return __uint_as_float(static_cast<unsigned>(v)) + __uint_as_float(static_cast<unsigned>(v >> 32));
}

// 2-D TMA copy of a box of `rows` consecutive ring slots x kLagBlock elements (the box
// shape is fixed by the tensor map) into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// Tensor maps of the ring viewed as a 2-D array [slots][elements] of 8-byte values, with
// boxes of kLagBlock elements x 1, 2, 4 or 8 slots.
struct LagMaps {
    CUtensorMap box[kLagRunKinds];
};

// Warp-specialised pipeline over groups of kLagGroup union entries. Warps
// 0..kLagConsumerWarps-1 consume (one spectrum element per thread); the last warp produces
// (its lane 0 issues the copies). Group g occupies shared-memory slots
// [(g % groups) * kLagGroup, +kLagGroup); its consecutive ring slots arrive as a few 2-D
// boxes (runs) that all complete on full[g % groups]; empty[g % groups] completes when every
// consumer warp has moved past the group. Neither side ever waits for the whole CTA.
template <int J>
__global__ void __launch_bounds__(kLagThreads, 3)
    lag_pipe_kernel(const float2 *__restrict__ ring, float2 *__restrict__ acc, long long E,
                    const int *__restrict__ table, int *__restrict__ status, const __grid_constant__ LagMaps maps) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // ring slots must start on 1 KB boundaries (TMA destinations): align the base at run time
    unsigned char *smem = smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + kLagRingBytes);
    uint64_t *empty = full + kLagGroupSlots;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(empty + kLagGroupSlots);
    int *tab = const_cast<int *>(reinterpret_cast<volatile int *>(abort_flag + 1));

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int ntab = lag_table_ints(table[kTabNtau], table[kTabNunion], table[kTabNgroups], table[kTabNruns]);
    for (int i = tid; i < ntab; i += kLagThreads) tab[i] = table[i];
    if (tid == 0) {
        for (int i = 0; i < kLagGroupSlots; i++) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], kLagConsumerWarps);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();

    const int nreg = tab[kTabNreg], ntau = tab[kTabNtau], nu = tab[kTabNunion];
    const int ngroups = tab[kTabNgroups];
    const int *ent_acc = tab + kTabEntries;
    const int *ent_ub = ent_acc + ntau;
    const int *ent_full = ent_ub + ntau;
    const int *uslot = ent_full + ntau;
    const int *gptr = uslot + nu;
    const int *runs = gptr + ngroups + 1;
    const long long e0 = static_cast<long long>(blockIdx.x) * kLagBlock;

    if (warp == kLagConsumerWarps) {
        // ---------------- producer: group g is fill g / kLagGroupSlots of group slot g % kLagGroupSlots
        if (lane == 0) {
            for (int g = 0; g < ngroups; g++) {
                const int gs = g & (kLagGroupSlots - 1), fill = g >> kLagGroupSlotsLog2;
                if (fill > 0 && !mbar_wait_bounded(&empty[gs], (fill - 1) & 1)) {
                    *abort_flag = 1;
                    break;
                }
                if (*abort_flag) break;
                const int r0 = gptr[g], r1 = gptr[g + 1];
                if (r0 == r1) {  // no frame in the group: complete the phase without data
                    mbar_arrive(&full[gs]);
                    continue;
                }
                uint32_t bytes = 0;
                for (int r = r0; r < r1; r++) bytes += kLagSlotBytes << lag_run_log2rows(runs[r]);
                mbar_expect_tx(&full[gs], bytes);
                for (int r = r0; r < r1; r++) {
                    const int run = runs[r];
                    tma_load_2d(smem + (gs * kLagGroup + lag_run_rel(run)) * kLagSlotBytes,
                                &maps.box[lag_run_log2rows(run)], static_cast<int>(e0), lag_run_slot(run), &full[gs]);
                }
            }
        }
    } else {
        // ---------------- consumers
        const long long k = e0 + tid;
        const bool valid = k < E;
        const uint32_t toff = static_cast<uint32_t>(tid) * sizeof(float2);
        const unsigned long long *ring64 = reinterpret_cast<const unsigned long long *>(ring);
        unsigned long long r[J];
#pragma unroll
        for (int j = 0; j < J; j++) {
            const int s = j < nreg ? tab[kTabReg + j] : -1;
            r[j] = (valid && s >= 0) ? __ldg(ring64 + static_cast<long long>(s) * E + k) : 0ull;
        }
        const float2 zero = make_float2(0.f, 0.f);
        float2 a0 = (valid && ntau > 0) ? acc[static_cast<long long>(ent_acc[0]) * E + k] : zero;
        float2 a1 = (valid && ntau > 1) ? acc[static_cast<long long>(ent_acc[1]) * E + k] : zero;
        float2 a2 = (valid && ntau > 2) ? acc[static_cast<long long>(ent_acc[2]) * E + k] : zero;
        int waited = 0, released = 0;  // in groups
        for (int e = 0; e < ntau; e++) {
            const float2 a3 = (valid && e + 3 < ntau) ? acc[static_cast<long long>(ent_acc[e + 3]) * E + k] : zero;
            const int ub = ent_ub[e];
            // Wait for every group this window reaches that no earlier window reached; groups
            // without frames included (they complete by the producer's bare arrival), so a
            // consumer never releases a group the producer has not issued yet.
            const int glast = (ub + nreg - 1) >> kLagGroupLog2;
            bool ok = true;
            for (int g = waited; g <= glast; g++) {
                if (!mbar_wait_bounded(&full[g & (kLagGroupSlots - 1)], (g >> kLagGroupSlotsLog2) & 1)) {
                    ok = false;
                    break;
                }
            }
            if (glast + 1 > waited) waited = glast + 1;
            if (!ok) *abort_flag = 1;
            if (*abort_flag) break;
            const uint32_t o = static_cast<uint32_t>(ub) * kLagSlotBytes;
            // four independent packed accumulators (j mod 4) keep the FMA pipeline full
            unsigned long long acc2[4] = {0ull, 0ull, 0ull, 0ull};
            const int s0 = ub & (kLagSlots - 1);
            if (ent_full[e] && s0 + J <= kLagSlots) {
                // whole window present and contiguous in the ring: fixed offsets from one base
                const unsigned char *w = smem + s0 * kLagSlotBytes + toff;
#pragma unroll
                for (int j = 0; j < J; j++) {
                    const unsigned long long b = *reinterpret_cast<const unsigned long long *>(w + j * kLagSlotBytes);
                    acc2[j & 3] = f2_fma_sq(f2_sub(r[j], b), acc2[j & 3]);
                }
            } else if (ent_full[e]) {  // nreg == J, every register frame and partner present
#pragma unroll
                for (int j = 0; j < J; j++) {
                    const uint32_t off = ((o + j * kLagSlotBytes) & kLagRingMask) | toff;
                    const unsigned long long b = *reinterpret_cast<const unsigned long long *>(smem + off);
                    acc2[j & 3] = f2_fma_sq(f2_sub(r[j], b), acc2[j & 3]);
                }
            } else {
#pragma unroll
                for (int j = 0; j < J; j++) {
                    if (j < nreg && tab[kTabReg + j] >= 0 && uslot[ub + j] >= 0) {
                        const uint32_t off = ((o + j * kLagSlotBytes) & kLagRingMask) | toff;
                        const unsigned long long b = *reinterpret_cast<const unsigned long long *>(smem + off);
                        acc2[j & 3] = f2_fma_sq(f2_sub(r[j], b), acc2[j & 3]);
                    }
                }
            }
            const float sum = (f2_hsum(acc2[0]) + f2_hsum(acc2[1])) + (f2_hsum(acc2[2]) + f2_hsum(acc2[3]));
            // Kahan step: a.x running sum, a.y compensation (true value a.x - a.y)
            const float y = sum - a0.y;
            const float t = a0.x + y;
            a0.y = (t - a0.x) - y;
            a0.x = t;
            if (valid) acc[static_cast<long long>(ent_acc[e]) * E + k] = a0;
            a0 = a1;
            a1 = a2;
            a2 = a3;
            // release the groups no later window reads (all their entries lie below the next window)
            const int next_g = (e + 1 < ntau ? ent_ub[e + 1] : nu) >> kLagGroupLog2;
            __syncwarp();
            if (lane == 0)
                for (; released < next_g; released++) mbar_arrive(&empty[released & (kLagGroupSlots - 1)]);
        }
    }
    __syncthreads();
    if (*abort_flag) {
        if (tid == 0) {
            atomicExch(status, 1);
            // drain: wait (bounded) until every copy this CTA issued has landed
            for (int gs = 0; gs < kLagGroupSlots; gs++) {
                for (int g = gs; g < ngroups; g += kLagGroupSlots) {
                    if (!mbar_try_wait(&full[gs], (g >> kLagGroupSlotsLog2) & 1)) {
                        mbar_wait_bounded(&full[gs], (g >> kLagGroupSlotsLog2) & 1);
                        break;
                    }
                }
            }
        }
        __syncthreads();
    }
}

inline size_t lag_smem_bytes(int table_ints) {
    return 1024 + kLagRingBytes + 2 * sizeof(uint64_t) * kLagGroupSlots + sizeof(int) * (1 + table_ints);
}

}  // namespace ddm
