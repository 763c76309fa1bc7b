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
// slots, one slot = the CTA's element block of one frame (2 KB), each filled by a single
// 1-D bulk copy (cp.async.bulk, the TMA's linear mode; no multicast) that completes on the
// slot's mbarrier. Thread 0 is the producer; after every tau entry the CTA synchronises,
// which frees every union index below the next entry's window, and thread 0 refills those
// slots kLagSlots ahead. Accumulators (FP32 sum + Kahan compensation, 8 B) are loaded two
// entries ahead with plain coalesced loads and written back once per entry.
//
// Every mbarrier wait is bounded (about one second of clock cycles); a wait that runs out
// sets *status to 1, and the CTA waits (bounded again) for its own copies in flight before
// returning, so a broken schedule ends the kernel instead of hanging the GPU.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ddm {

constexpr int kLagBlock = 256;    // elements per CTA (= threads)
constexpr int kLagSlots = 48;     // shared-memory frame slots (> kMaxJ)
constexpr int kLagSmemMax = 220 * 1024;
// Register-frame counts the kernel is instantiated for (a launch uses the smallest >= nreg).
constexpr int kLagJs[] = {4, 8, 16, 20, 24, 30, 32};
constexpr int kNumLagJs = sizeof(kLagJs) / sizeof(kLagJs[0]);

// Lag table layout (ints): header, register frames, tau entries, union slots.
constexpr int kTabNreg = 0, kTabNtau = 1, kTabNunion = 2, kTabReg = 3;
constexpr int kTabEntries = kTabReg + 32;  // then ntau acc indices, ntau union starts,
                                           // ntau full-window flags, nunion ring slots

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

// Bounded wait: false if the phase did not complete within ~1 s of SM clocks.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > 2000000000LL) return false;
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

template <int J>
__global__ void __launch_bounds__(kLagBlock, 2)
    lag_pipe_kernel(const float2 *__restrict__ ring, float2 *__restrict__ acc, long long E,
                    const int *__restrict__ table, int *__restrict__ status) {
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned long long *slots = reinterpret_cast<unsigned long long *>(smem);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + sizeof(float2) * kLagSlots * kLagBlock);
    int *abort_flag = reinterpret_cast<int *>(full + kLagSlots);
    int *tab = abort_flag + 1;

    const int tid = threadIdx.x;
    const int ntab = kTabEntries + 3 * table[kTabNtau] + table[kTabNunion];
    for (int i = tid; i < ntab; i += kLagBlock) tab[i] = table[i];
    if (tid == 0) {
        for (int i = 0; i < kLagSlots; i++) mbar_init(&full[i], 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();

    const int nreg = tab[kTabNreg], ntau = tab[kTabNtau], nu = tab[kTabNunion];
    const int *ent_acc = tab + kTabEntries;
    const int *ent_ub = ent_acc + ntau;
    const int *ent_full = ent_ub + ntau;
    const int *uslot = ent_full + ntau;
    const long long e0 = static_cast<long long>(blockIdx.x) * kLagBlock;
    const long long k = e0 + tid;
    const bool valid = k < E;
    const uint32_t bytes = static_cast<uint32_t>(
        sizeof(float2) * (E - e0 < kLagBlock ? E - e0 : static_cast<long long>(kLagBlock)));

    // Producer state lives in thread 0 only. Union index u is the (u / kLagSlots)-th use of
    // slot u % kLagSlots, and every use completes exactly one phase of the slot's barrier:
    // a copy's transaction bytes, or a bare arrival when there is no frame to copy.
    int issued = 0;
    auto issue_upto = [&](int limit) {
        for (; issued < nu && issued < limit; issued++) {
            const int s = uslot[issued];
            uint64_t *bar = &full[issued % kLagSlots];
            if (s < 0) {  // no such frame: nothing to copy, nobody waits; keep the phase count
                mbar_arrive(bar);
                continue;
            }
            mbar_expect_tx(bar, bytes);
            bulk_load(slots + (issued % kLagSlots) * kLagBlock, ring + static_cast<long long>(s) * E + e0, bytes,
                      bar);
        }
    };
    if (tid == 0) issue_upto(kLagSlots);

    const unsigned long long *ring64 = reinterpret_cast<const unsigned long long *>(ring);
    unsigned long long r[J];
#pragma unroll
    for (int j = 0; j < J; j++) {
        const int s = j < nreg ? tab[kTabReg + j] : -1;
        r[j] = (valid && s >= 0) ? __ldg(ring64 + static_cast<long long>(s) * E + k) : 0ull;
    }
    const float2 zero = make_float2(0.f, 0.f);
    float2 a_cur = (valid && ntau > 0) ? acc[static_cast<long long>(ent_acc[0]) * E + k] : zero;
    float2 a_nxt = (valid && ntau > 1) ? acc[static_cast<long long>(ent_acc[1]) * E + k] : zero;

    int waited = 0;  // union indices below this have been waited for by this thread
    bool ok = true;
    for (int e = 0; e < ntau; e++) {
        const float2 a_far = (valid && e + 2 < ntau) ? acc[static_cast<long long>(ent_acc[e + 2]) * E + k] : zero;
        const int ub = ent_ub[e];
        // Wait once for each partner frame that enters the window with this entry.
        const int wend = ub + nreg;
        for (int u = waited > ub ? waited : ub; u < wend; u++) {
            if (uslot[u] >= 0 && !mbar_wait_bounded(&full[u % kLagSlots], (u / kLagSlots) & 1)) {
                ok = false;
                break;
            }
        }
        waited = wend;
        float sum = 0.f;
        if (ok) {
            const int s0 = ub % kLagSlots;
            const int wrap = kLagSlots - s0;  // j >= wrap wraps to the start of the ring
            const unsigned long long *lo = slots + s0 * kLagBlock + tid;
            const unsigned long long *hi = lo - kLagSlots * kLagBlock;
            if (ent_full[e]) {  // nreg == J, every register frame and partner present
                unsigned long long acc2 = 0ull;
#pragma unroll
                for (int j = 0; j < J; j++) {
                    const unsigned long long b = (j < wrap ? lo : hi)[j * kLagBlock];
                    acc2 = f2_fma_sq(f2_sub(r[j], b), acc2);
                }
                sum = f2_hsum(acc2);
            } else {
                unsigned long long acc2 = 0ull;
#pragma unroll
                for (int j = 0; j < J; j++) {
                    if (j < nreg && tab[kTabReg + j] >= 0 && uslot[ub + j] >= 0) {
                        const unsigned long long b = (j < wrap ? lo : hi)[j * kLagBlock];
                        acc2 = f2_fma_sq(f2_sub(r[j], b), acc2);
                    }
                }
                sum = f2_hsum(acc2);
            }
        }
        if (!ok) atomicExch(abort_flag, 1);
        // Kahan step: a.x running sum, a.y compensation (true value a.x - a.y)
        const float y = sum - a_cur.y;
        const float t = a_cur.x + y;
        a_cur.y = (t - a_cur.x) - y;
        a_cur.x = t;
        if (valid && ok) acc[static_cast<long long>(ent_acc[e]) * E + k] = a_cur;
        a_cur = a_nxt;
        a_nxt = a_far;
        __syncthreads();  // every thread is done with union indices below the next window
        if (*abort_flag) break;
        if (tid == 0) {
            fence_proxy_async_smem();
            issue_upto((e + 1 < ntau ? ent_ub[e + 1] : nu) + kLagSlots);
        }
    }
    if (*abort_flag) {
        if (tid == 0) {
            atomicExch(status, 1);
            // drain: wait (bounded) for the copies this CTA issued into its own shared memory
            for (int u = issued - 1; u >= 0 && u >= issued - kLagSlots; u--)
                if (uslot[u] >= 0) mbar_wait_bounded(&full[u % kLagSlots], (u / kLagSlots) & 1);
        }
        __syncthreads();
    }
}

inline size_t lag_smem_bytes(int table_ints) {
    return sizeof(float2) * kLagSlots * kLagBlock + sizeof(uint64_t) * kLagSlots + sizeof(int) * (1 + table_ints);
}

}  // namespace ddm
