// Lag kernel: accumulates |F(x) - F(y)|^2 for a block of J "register" frames x against
// the partner frame y of every tau, per spectrum element (replaces processFFT,
// src/DDM_kernel.cuh:85-101, which the reference launches once per (scale, tau, frame)).
//
// Work decomposition. One CTA owns a block of consecutive elements of the flattened frame
// vector (all scales and tiles concatenated, so the kernel needs no geometry). Its threads
// keep the J register frames of their element in registers. The partner of (register
// frame j, tau entry e) is window position ub_e + j of a sorted list of distinct partner
// frames (the "union"), which the host builds per launch: windows of consecutive taus
// overlap, so a chunk of 30 frames against 64 log-spaced taus up to 500 needs 484 distinct
// partner frames instead of 30 * 64 = 1920 frame reads, and 64 frames need 563.
//
// Data movement (sm_100a). Partner frames stream through a ring of shared-memory slots,
// one slot = the CTA's element block of one frame, grouped by kLagGroup. The ring in HBM is
// addressed through 2-D tensor maps ([slots][elements], boxes of 1..8 slots x the CTA's
// elements), so a run of consecutive frames arrives with one cp.async.bulk.tensor.2d (no
// multicast) that completes on the group's "full" mbarrier. A dedicated producer warp
// refills a group once every consumer warp has arrived on its "empty" mbarrier. Consumers
// wait once per window for every group it reaches, then release the groups no later window
// reads. The |dF|^2 arithmetic is a packed FP32x2 add (FADD2) and two scalar FMAs per pair.
// Accumulators (FP32 sum + Kahan compensation, 8 B) are prefetched kLagAccSlots entries ahead
// by each consumer thread with cp.async into a private shared-memory ring and written back
// once per entry with plain coalesced stores. (Prefetching into registers instead did not
// work: the loop rotates the prefetched values from register to register every entry, and
// each such move waits for its load, so the loads were exposed one entry after their issue.)
//
// Fused runs. With the register frames in registers and the partners in shared memory, the
// kernel is bound by its shared-memory loads (one 8-byte load per pair) as much as by HBM:
// without any arithmetic the ring alone streams at the copy bandwidth. Taus one frame apart
// (1, 2, 3, ... in a log-spaced list) have windows one union entry apart, so four such
// entries are paired in one pass over the span of their windows: each partner value is
// loaded once and paired with up to four register frames (35 loads for 128 pairs instead
// of 128), one accumulator per entry.
//
// Persistent grid. An engine's launch has kLagCtasPerSm CTAs per SM (or fewer, one per
// element block), and CTA c walks element blocks c, c + gridDim.x, ...: the table, the
// barriers and the pipeline are set up once, the producer runs into the next block's groups
// while the consumers finish the current one (the group counter runs on across blocks, and
// the consumers release every group of a block at its end), and as the CTAs retire the SMs
// pass to the next piece's FFT on the other stream instead of to further lag blocks.
//
// Every mbarrier wait of the pipeline is bounded (wait_cycles clock cycles, a launch
// argument, kWaitCycles by default); a wait that runs out sets *status to 1, and the CTA
// waits for its own copies in flight (bounded by kWaitCycles, whatever the launch's limit,
// so no CTA exits while a copy into its shared memory may still land) before returning: a
// broken schedule ends the kernel instead of hanging the GPU.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace ddm {

constexpr int kLagConsumerWarps = 4;
constexpr int kLagThreads = kLagConsumerWarps * 32 + 32;  // consumers + one producer warp
constexpr int kLagCtasPerSm = 3;  // registers (128 a thread) and shared memory (~70 KB a CTA) both allow 3
// Geometries of the kernel (template parameter GEO): 0 "narrow", the layout above -- one
// consumer thread per element holding all J <= 32 register frames, four consumer warps, three
// CTAs per SM; 1 "wide" -- two lanes per element holding J/2 frames each (a warp's partner
// load then reads 16 elements, one shared-memory wavefront for 32 pairs), eight consumer warps
// over the same 128-element block, two CTAs per SM (16 consumer warps per SM instead of 12).
constexpr int kLagGeoms = 2;
__host__ __device__ constexpr int lag_cwarps(int G) { return G ? 8 : kLagConsumerWarps; }
__host__ __device__ constexpr int lag_threads(int G) { return (lag_cwarps(G) + 1) * 32; }
__host__ __device__ constexpr int lag_ctas_per_sm(int G) { return G ? 2 : kLagCtasPerSm; }
constexpr int kLagSmemMax = 220 * 1024;
// Register-frame counts the kernel is instantiated for (a launch uses the smallest >= nreg).
constexpr int kLagJs[] = {4, 8, 16, 20, 24, 30, 32, 64};
constexpr int kNumLagJs = sizeof(kLagJs) / sizeof(kLagJs[0]);
constexpr int kLagMaxJ = 64;

// Union entries are copied in groups of kLagGroup consecutive entries; a group's ring
// slots arrive as runs of 1, 2, 4 or 8 consecutive slots (one 2-D TMA box each).
constexpr int kLagGroupLog2 = 3;
constexpr int kLagGroup = 1 << kLagGroupLog2;
constexpr int kLagRunKinds = 4;  // box heights 1, 2, 4, 8
// Consecutive tau entries whose windows start one union entry apart (taus one frame apart)
// are paired kLagFuse at a time: each partner value is read from shared memory once and
// paired with up to kLagFuse register frames (entry e + r pairs window position q with
// register frame q - r). Table flag bits per entry: 1 = full window, 2 = first of a run.
constexpr int kLagFuse = 4;
constexpr int kLagFullFlag = 1, kLagRunFlag = 2;
// Accumulator prefetch depth in entries: each consumer thread copies its element's accumulator
// of entry e + kLagAccSlots into a private shared-memory slot with cp.async while it works on
// entry e (kLagAccSlots x 8 B per consumer thread; a fused run consumes kLagFuse at once).
constexpr int kLagAccSlots = 4;
static_assert(kLagAccSlots >= kLagFuse && (kLagAccSlots & (kLagAccSlots - 1)) == 0, "accumulator ring");

// Geometry of the kernel instantiated for J register frames per element. Up to 32 frames one
// consumer thread owns an element and holds all J frames in registers; for 64 frames two
// lanes of a warp (l and l + 16) share an element, each holding 32 frames, and add their
// pair sums with one shuffle per tau, so the register budget (128 per thread) and three CTAs
// per SM stay those of 32 frames while the partner reuse is that of 64. A CTA's element
// block is therefore 128 or 64 elements and a ring slot 1 KB or 512 B. The ring must hold a
// window plus its alignment, ceil((J - 1) / kLagGroup) + 1 groups, with room to read ahead:
// 64 slots (8 groups) up to 32 frames, 128 slots (16 groups) for 64; both are 64 KB.
__host__ __device__ constexpr int lag_lanes(int J, int G = 0) { return (J > 32 || G) ? 2 : 1; }
__host__ __device__ constexpr int lag_cta_elems(int J, int G = 0) { return lag_cwarps(G) * 32 / lag_lanes(J, G); }
__host__ __device__ constexpr uint32_t lag_slot_bytes(int J, int G = 0) { return lag_cta_elems(J, G) * 8u; }
// tensor-map box width index (LagMaps::box[w]): 128-element blocks 0, 64-element blocks 1
__host__ __device__ constexpr int lag_map_index(int J, int G = 0) { return lag_cta_elems(J, G) == 128 ? 0 : 1; }
__host__ __device__ constexpr int lag_ring_slots(int J) { return J > 32 ? 128 : 64; }
__host__ __device__ constexpr int lag_group_slots(int J) { return lag_ring_slots(J) / kLagGroup; }

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
constexpr int kTabEntries = kTabReg + kLagMaxJ;
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

// Device status word values (0 = fine): a pipeline wait that ran out, the tensor-core DFT's
// wait that ran out (csrc/dft_bf16.cuh), a lag kernel whose shared memory was not 1 KB aligned.
constexpr int kLagStatusWait = 1, kLagStatusDftWait = 2, kLagStatusMisaligned = 3;
inline const char *device_status_text(int st) {
    return st == kLagStatusMisaligned ? "the lag kernel's shared memory was not 1 KB aligned"
           : st == kLagStatusDftWait  ? "a tensor-core DFT wait timed out"
                                      : "a lag-kernel pipeline wait timed out";
}

// Bounded wait: false if the phase did not complete within kWaitCycles SM clocks (about
// 0.2 s at 2 GHz, four orders of magnitude above any legitimate copy latency).
constexpr long long kWaitCycles = 400000000LL;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, long long limit = kWaitCycles) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}

// Per-thread asynchronous 8-byte copy global -> shared (cp.async, the generic proxy) and its
// group bookkeeping: the accumulator prefetch ring of the consumers.
__device__ __forceinline__ void cp_async_8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// |dF|^2 accumulation: the difference as one packed FP32x2 add (sm_100a FADD2, through the
// compiler's builtin), the squares as two scalar FMAs (measured 11 % faster per launch than a
// packed FFMA2 on the same chain). With the register frames stored negated, d = b + (-r) is
// exactly -(r - b), so |d|^2 is the pair's |dF|^2 bit for bit.
__device__ __forceinline__ float2 f2_diff_sq_acc(float2 b, float2 neg_r, float2 acc) {
    const float2 d = __fadd2_rn(b, neg_r);
    return make_float2(fmaf(d.x, d.x, acc.x), fmaf(d.y, d.y, acc.y));
}

// 2-D TMA copy of a box of `rows` consecutive ring slots x a CTA's elements (the box
// shape is fixed by the tensor map) into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// Tensor maps of the ring viewed as a 2-D array [slots][elements] of 8-byte values, with
// boxes of 128 (box[0][*]) or 64 (box[1][*]) elements x 1, 2, 4 or 8 slots.
struct LagMaps {
    CUtensorMap box[2][kLagRunKinds];
};

// Warp-specialised pipeline over groups of kLagGroup union entries. A run of kLagFuse
// entries (table flag kLagRunFlag) is one pass over the span of its windows. Warps
// 0..kLagConsumerWarps-1 consume; the last warp produces (its lane 0 issues the copies).
// Running group G (group g of the CTA's n-th element block, G = n * ngroups + g) occupies
// shared-memory slots [(G % kGS) * kLagGroup, +kLagGroup) with kGS = lag_group_slots(J); its
// consecutive ring slots arrive as a few 2-D boxes (runs) that all complete on full[G % kGS];
// empty[G % kGS] completes when every consumer warp has moved past the group. Union entry u
// of the n-th element block therefore sits in shared-memory slot
// (n * ngroups * kLagGroup + u) % lag_ring_slots(J). Neither side
// ever waits for the whole CTA. The CTA handles element blocks block_begin, + block_step, ...
// below block_end; `maps` may live in kernel parameter space or global memory.
template <int J, int GEO = 0>
__device__ __forceinline__ void lag_pipe_body(const float2 *__restrict__ ring, float2 *__restrict__ acc, long long E,
                                              const int *__restrict__ table, int *__restrict__ status,
                                              const LagMaps &maps, int block_begin, int block_end, int block_step,
                                              long long wait_cycles) {
    constexpr int kLanes = lag_lanes(J, GEO);
    constexpr int kJT = J / kLanes;  // register frames per thread
    constexpr int kElems = lag_cta_elems(J, GEO);
    constexpr int kCW = lag_cwarps(GEO);  // consumer warps; warp kCW produces
    constexpr int kThreads = lag_threads(GEO);
    constexpr uint32_t kSlotBytes = lag_slot_bytes(J, GEO);
    constexpr int kMap = lag_map_index(J, GEO);  // tensor-map box width of this geometry
    constexpr int kSlots = lag_ring_slots(J);
    constexpr int kGS = lag_group_slots(J);
    constexpr uint32_t kRingBytes = kSlots * kSlotBytes;
    static_assert(J % kLanes == 0 && (kSlots & (kSlots - 1)) == 0 && (kGS & (kGS - 1)) == 0, "lag geometry");
    // Ring slots are TMA destinations and start on 1 KB boundaries: the dynamic shared memory of
    // a kernel without static shared memory starts on one, so the ring sits at the array's
    // (link-time constant) address, which every slot address then folds in as an immediate. A
    // base that is not so aligned is reported (status 3) before anything is copied.
    extern __shared__ __align__(1024) unsigned char smem[];
    if (smem_addr(smem) & 1023u) {
        if (threadIdx.x == 0) atomicExch(status, kLagStatusMisaligned);
        return;
    }
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + kRingBytes);
    uint64_t *empty = full + kGS;
    // accumulator prefetch ring: entry e's value of consumer thread t in accring[(e % kLagAccSlots) * kCT + t]
    constexpr int kCT = kCW * 32;
    float2 *accring = reinterpret_cast<float2 *>(empty + kGS);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(accring + kLagAccSlots * kCT);
    volatile int *issued = abort_flag + 1;  // groups the producer has issued (running count)
    int *tab = const_cast<int *>(reinterpret_cast<volatile int *>(abort_flag + 2));

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int ntab = lag_table_ints(table[kTabNtau], table[kTabNunion], table[kTabNgroups], table[kTabNruns]);
    for (int i = tid; i < ntab; i += kThreads) tab[i] = table[i];
    if (tid == 0) {
        for (int i = 0; i < kGS; i++) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], kCW);
        }
        *abort_flag = 0;
        *issued = 0;
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

    if (warp == kCW) {
        // ---------------- producer: running group G is fill G / kGS of group slot G % kGS
        if (lane == 0 && ngroups > 0) {
            // group g of the CTA's element block `block`
            long long e0 = static_cast<long long>(block_begin) * kElems;
            for (int G = 0, g = 0, block = block_begin; block < block_end; G++) {
                const int gs = G & (kGS - 1), fill = G / kGS;
                if (fill > 0 && !mbar_wait_bounded(&empty[gs], (fill - 1) & 1, wait_cycles)) {
                    *abort_flag = 1;
                    break;
                }
                if (*abort_flag) break;
                const int r0 = gptr[g], r1 = gptr[g + 1];
                *issued = G + 1;
                if (r0 == r1) {  // no frame in the group: complete the phase without data
                    mbar_arrive(&full[gs]);
                } else {
                    uint32_t bytes = 0;
                    for (int r = r0; r < r1; r++) bytes += kSlotBytes << lag_run_log2rows(runs[r]);
                    mbar_expect_tx(&full[gs], bytes);
                    for (int r = r0; r < r1; r++) {
                        const int run = runs[r];
                        tma_load_2d(smem + (gs * kLagGroup + lag_run_rel(run)) * kSlotBytes,
                                    &maps.box[kMap][lag_run_log2rows(run)], static_cast<int>(e0),
                                    lag_run_slot(run), &full[gs]);
                    }
                }
                if (++g == ngroups) {
                    g = 0;
                    block += block_step;
                    e0 = static_cast<long long>(block) * kElems;
                }
            }
        }
    } else {
        // ---------------- consumers. With two lanes per element, lanes l and l + 16 of a warp
        // share element l: each half-warp then reads 16 consecutive elements (128 B, every
        // bank once) of one slot, so a 64-bit shared load stays at two wavefronts.
        const int h = kLanes == 2 ? (lane >> 4) : 0;
        const int m = kLanes == 2 ? warp * 16 + (lane & 15) : tid;  // element within the CTA's block
        int Gbase = 0;
        for (int block = block_begin; block < block_end && !*abort_flag; block += block_step, Gbase += ngroups) {
            const long long k = static_cast<long long>(block) * kElems + m;
            const bool valid = k < E;
            const uint32_t toff = static_cast<uint32_t>(m) * sizeof(float2);
            const int j0 = h * kJT;  // first register frame of this thread
            float2 nr[kJT];          // register frames j0 .. j0 + kJT - 1, negated
#pragma unroll
            for (int i = 0; i < kJT; i++) {
                const int s = j0 + i < nreg ? tab[kTabReg + j0 + i] : -1;
                const float2 v = (valid && s >= 0) ? __ldg(ring + static_cast<long long>(s) * E + k) : make_float2(0.f, 0.f);
                nr[i] = make_float2(-v.x, -v.y);
            }
            const float2 zero = make_float2(0.f, 0.f);
            // Accumulator prefetch: one cp.async group per entry, committed in entry order (empty
            // past the last entry or for an element past E); before entry e is finished, the
            // groups of entries 0 .. e + kLagAccSlots - 1 are committed. The copies land in shared
            // memory without holding a register, so the wait before the Kahan step (wait_group)
            // finds them there kLagAccSlots entries after their issue.
            float2 *my_acc = accring + tid;
            auto prefetch_acc = [&](int ee) {
                if (valid && ee < ntau)
                    cp_async_8(my_acc + (ee & (kLagAccSlots - 1)) * kCT, acc + static_cast<long long>(ent_acc[ee]) * E + k);
                cp_async_commit();
            };
#pragma unroll
            for (int ee = 0; ee < kLagAccSlots; ee++) prefetch_acc(ee);
            int waited = 0, released = 0;  // in groups; warp-uniform
            for (int e = 0; e < ntau;) {
                const int flags = ent_full[e];
                const int nrun = (flags & kLagRunFlag) ? kLagFuse : 1;  // entries handled in this pass
                const int ub = ent_ub[e];
                // Wait for every group this window (or run of windows) reaches that no earlier
                // window reached; groups without frames included (they complete by the producer's
                // bare arrival), so a consumer never releases a group the producer has not issued
                // yet. One wait per window keeps its shared-memory loads free to issue back to back.
                const int glast = (ub + nrun - 1 + nreg - 1) >> kLagGroupLog2;
                bool ok = true;
                for (; waited <= glast; waited++) {
                    const int G = Gbase + waited;
                    if (!mbar_wait_bounded(&full[G & (kGS - 1)], (G / kGS) & 1, wait_cycles)) {
                        ok = false;
                        break;
                    }
                }
                // A warp leaves on its own failed wait only (no shared flag read per entry): the
                // others then run out of bounded waits in turn, the producer on the empty barriers
                // this warp no longer arrives on, the consumers on the groups it no longer issues.
                if (!ok) {
                    *abort_flag = 1;
                    break;
                }
                const int s0 = (Gbase * kLagGroup + ub) & (kSlots - 1);  // group G sits in group slot G % kGS
                // byte offset of this thread's first partner: slot (s0 + j0) of the ring, element m
                const uint32_t o = static_cast<uint32_t>((s0 + j0) & (kSlots - 1)) * kSlotBytes + toff;
                if (nrun == kLagFuse) {
                    static_assert(kLagFuse == 4, "the run consumes the four prefetched accumulators");
                    // entries e .. e + 3, windows ub .. ub + 3: position q of the run's span (one
                    // shared-memory load) pairs with register frame q - r of entry e + r; one
                    // packed accumulator per entry
                    float2 c[kLagFuse] = {zero, zero, zero, zero};
                    if (s0 + J + kLagFuse - 1 <= kSlots) {
                        const unsigned char *w = smem + o;
#pragma unroll
                        for (int q = 0; q < kJT + kLagFuse - 1; q++) {
                            const float2 b = *reinterpret_cast<const float2 *>(w + q * kSlotBytes);
#pragma unroll
                            for (int r = 0; r < kLagFuse; r++)
                                if (q - r >= 0 && q - r < kJT) c[r] = f2_diff_sq_acc(b, nr[q - r], c[r]);
                        }
                    } else {
#pragma unroll
                        for (int q = 0; q < kJT + kLagFuse - 1; q++) {
                            const uint32_t off = (o + q * kSlotBytes) & (kRingBytes - 1);
                            const float2 b = *reinterpret_cast<const float2 *>(smem + off);
#pragma unroll
                            for (int r = 0; r < kLagFuse; r++)
                                if (q - r >= 0 && q - r < kJT) c[r] = f2_diff_sq_acc(b, nr[q - r], c[r]);
                        }
                    }
                    float sum[kLagFuse];
#pragma unroll
                    for (int r = 0; r < kLagFuse; r++) {
                        sum[r] = c[r].x + c[r].y;
                        if (kLanes == 2) sum[r] += __shfl_xor_sync(0xffffffffu, sum[r], 16);
                    }
                    cp_async_wait<kLagAccSlots - kLagFuse>();  // entries e .. e + 3 landed
                    float2 ar[kLagFuse];
#pragma unroll
                    for (int r = 0; r < kLagFuse; r++) ar[r] = my_acc[((e + r) & (kLagAccSlots - 1)) * kCT];
#pragma unroll
                    for (int r = 0; r < kLagFuse; r++) {
                        const float y = sum[r] - ar[r].y;
                        const float t = ar[r].x + y;
                        ar[r].y = (t - ar[r].x) - y;
                        ar[r].x = t;
                        if (valid && h == 0) acc[static_cast<long long>(ent_acc[e + r]) * E + k] = ar[r];
                    }
#pragma unroll
                    for (int r = 0; r < kLagFuse; r++) prefetch_acc(e + kLagAccSlots + r);
                } else {
                    // one window; four independent packed accumulators (i mod 4) keep the FMA pipeline full
                    float2 acc2[4] = {zero, zero, zero, zero};
                    if ((flags & kLagFullFlag) && s0 + J <= kSlots) {
                        // whole window present and contiguous in the ring: fixed offsets from one base
                        const unsigned char *w = smem + o;
#pragma unroll
                        for (int i = 0; i < kJT; i++)
                            acc2[i & 3] = f2_diff_sq_acc(*reinterpret_cast<const float2 *>(w + i * kSlotBytes), nr[i], acc2[i & 3]);
                    } else if (flags & kLagFullFlag) {  // nreg == J, every register frame and partner present
#pragma unroll
                        for (int i = 0; i < kJT; i++) {
                            const uint32_t off = (o + i * kSlotBytes) & (kRingBytes - 1);  // toff < kSlotBytes survives the mask
                            acc2[i & 3] = f2_diff_sq_acc(*reinterpret_cast<const float2 *>(smem + off), nr[i], acc2[i & 3]);
                        }
                    } else {
#pragma unroll
                        for (int i = 0; i < kJT; i++) {
                            const int j = j0 + i;
                            if (j < nreg && tab[kTabReg + j] >= 0 && uslot[ub + j] >= 0) {
                                const uint32_t off = (o + i * kSlotBytes) & (kRingBytes - 1);
                                acc2[i & 3] = f2_diff_sq_acc(*reinterpret_cast<const float2 *>(smem + off), nr[i], acc2[i & 3]);
                            }
                        }
                    }
                    float sum = ((acc2[0].x + acc2[0].y) + (acc2[1].x + acc2[1].y)) +
                                ((acc2[2].x + acc2[2].y) + (acc2[3].x + acc2[3].y));
                    if (kLanes == 2) sum += __shfl_xor_sync(0xffffffffu, sum, 16);  // same value in both lanes
                    // Kahan step: a.x running sum, a.y compensation (true value a.x - a.y)
                    cp_async_wait<kLagAccSlots - 1>();  // entry e landed
                    float2 a0 = my_acc[(e & (kLagAccSlots - 1)) * kCT];
                    const float y = sum - a0.y;
                    const float t = a0.x + y;
                    a0.y = (t - a0.x) - y;
                    a0.x = t;
                    if (valid && h == 0) acc[static_cast<long long>(ent_acc[e]) * E + k] = a0;
                    prefetch_acc(e + kLagAccSlots);
                }
                e += nrun;
                // release the groups no later window reads (all their entries lie below the next
                // window); after the last window every group of the block, the partial last one too
                const int rel = e < ntau ? ent_ub[e] >> kLagGroupLog2 : ngroups;
                if (rel > released) {
                    __syncwarp();
                    if (lane == 0)
                        for (int g = released; g < rel; g++) mbar_arrive(&empty[(Gbase + g) & (kGS - 1)]);
                    released = rel;
                }
            }
            if (*abort_flag) break;
            // groups no window reached (none in tables of the host's builder): wait and release
            for (; waited < ngroups; waited++) {
                const int G = Gbase + waited;
                if (!mbar_wait_bounded(&full[G & (kGS - 1)], (G / kGS) & 1, wait_cycles)) {
                    *abort_flag = 1;
                    break;
                }
            }
            if (*abort_flag) break;
            if (released < ngroups) {
                __syncwarp();
                if (lane == 0)
                    for (int g = released; g < ngroups; g++) mbar_arrive(&empty[(Gbase + g) & (kGS - 1)]);
            }
        }
        cp_async_wait<0>();  // a warp that left early may still have accumulator copies in flight
    }
    __syncthreads();
    if (*abort_flag) {
        if (tid == 0) {
            atomicExch(status, kLagStatusWait);
            // drain: wait (bounded) until every copy this CTA issued has landed; a group slot
            // holds at most one fill in flight, its latest
            const int n = *issued;
            for (int G = n > kGS ? n - kGS : 0; G < n; G++) mbar_wait_bounded(&full[G & (kGS - 1)], (G / kGS) & 1);
        }
        __syncthreads();
    }
}

// One engine's launch: CTA b handles element blocks b, b + gridDim.x, ... below nblocks.
template <int J, int GEO = 0>
__global__ void __launch_bounds__(lag_threads(GEO), lag_ctas_per_sm(GEO))
    lag_pipe_kernel(const float2 *__restrict__ ring, float2 *__restrict__ acc, long long E,
                    const int *__restrict__ table, int *__restrict__ status, const __grid_constant__ LagMaps maps,
                    int nblocks, long long wait_cycles) {
    lag_pipe_body<J, GEO>(ring, acc, E, table, status, maps, static_cast<int>(blockIdx.x), nblocks,
                        static_cast<int>(gridDim.x), wait_cycles);
}

// The lag work of several engines (served streams) in one launch: item i owns CTAs
// [cta_begin, next item's cta_begin) and runs its own ring, accumulators, table and tensor
// maps (64-byte aligned, in global memory) exactly as its own launch would.
struct LagBatchItem {
    const float2 *ring;
    float2 *acc;
    long long E;
    const int *table;
    int *status;
    const LagMaps *maps;
    int cta_begin;
    int pad;
};

template <int J>
__global__ void __launch_bounds__(kLagThreads, kLagCtasPerSm)
    lag_batch_kernel(const LagBatchItem *__restrict__ items, int n) {
    int lo = 0, hi = n - 1;  // the last item whose first CTA is at or before this one
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].cta_begin <= static_cast<int>(blockIdx.x)) lo = mid;
        else hi = mid - 1;
    }
    const LagBatchItem &it = items[lo];
    const int b = static_cast<int>(blockIdx.x) - it.cta_begin;
    lag_pipe_body<J>(it.ring, it.acc, it.E, it.table, it.status, *it.maps, b, b + 1, 1, kWaitCycles);
}

// Dynamic shared memory of a launch of lag_pipe_kernel<J> with a table of table_ints ints
// (ring, barriers, accumulator prefetch ring, abort flag, issued-group count, table).
inline size_t lag_smem_bytes(int J, int table_ints, int G = 0) {
    return static_cast<size_t>(lag_ring_slots(J)) * lag_slot_bytes(J, G) + 2 * sizeof(uint64_t) * lag_group_slots(J) +
           sizeof(float2) * kLagAccSlots * lag_cwarps(G) * 32 + sizeof(int) * (2 + table_ints);
}

}  // namespace ddm
