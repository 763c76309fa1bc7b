// ddm_lag_accumulate_static: the lag kernel on caller-owned device buffers, allocating
// nothing on the device.
//
// Who needs it. Some callers cannot let a library call cudaMalloc: real-time camera
// acquisition loops that reserve all their device memory at start-up and must not stall
// mid-stream (cudaMalloc can synchronise the device and take unbounded time), and host
// applications whose own pool allocator hands out every device buffer. The engine
// (ddm_open) allocates its ring, accumulators and per-launch pair tables itself; this entry
// point runs the same lag kernel on a ring and accumulators the caller provides, and keeps
// the kernel's only other device memory -- its pair table and a status word -- in the
// file-scope array below.
//
// The array: kStaticTableInts + kStaticStatusInts ints (about 37 KB), held by every GPU
// that loads the library until the process exits. It is shared by all calls: each call
// overwrites the table and clears the status word before its launch, and two calls whose
// kernels overlap on a GPU would race on it. Calls are therefore serialised inside this
// process (a per-process lock) and each call returns only after its kernel has finished.
//
// Cost. Rows of b_slots that are shifts of one frame sequence share their partner frames in
// the kernel's window list (see lay_out_windows), so the usual causal pattern runs at the
// engine's speed. Rows that share nothing each stream their own partner frames: up to
// tau_count times the partner traffic of the engine's launch for the same pairs.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ddm.h"
#include "errors.hpp"
#include "lag.cuh"
#include "lag_host.hpp"

namespace {

using namespace ddm;

constexpr int kStaticMaxFrames = 32;   // register frames per call
constexpr int kStaticMaxTaus = 128;    // accumulator rows per call
constexpr int kStaticTableInts = 9216; // >= lag_table_capacity(128, 128 * 32)
constexpr int kStaticStatusInts = 64;  // status word (+ padding)

static_assert(lag_table_ints(kStaticMaxTaus, kStaticMaxTaus * kStaticMaxFrames,
                             (kStaticMaxTaus * kStaticMaxFrames + kLagGroup - 1) / kLagGroup,
                             kStaticMaxTaus * kStaticMaxFrames) <= kStaticTableInts,
              "static lag table too small for the stated maximum");

__device__ __align__(256) int g_static_scratch[kStaticTableInts + kStaticStatusInts];

std::mutex g_lock;

// With the device current: the array's device address in the current context and the
// shared-memory limit of the kernel instance about to run. Both are looked up on every call
// (neither allocates once the module is loaded), so a context made after cudaDeviceReset, or
// a caller's own context made current with cuCtxSetCurrent, gets its own copy's address
// instead of an address cached from an earlier context.
// Also the CTAs of that instance one SM holds with `smem` bytes of shared memory each (the
// persistent grid's size per SM; a large pair table can leave room for fewer than the
// engine's kLagCtasPerSm).
template <int J>
int setup_call(size_t smem, int **base, int *ctas_per_sm) {
    cudaError_t err = cudaGetSymbolAddress(reinterpret_cast<void **>(base), g_static_scratch);
    if (err != cudaSuccess)
        return fail(DDM_ERR_CUDA, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(err));
    err = cudaFuncSetAttribute(lag_pipe_kernel<J>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax);
    if (err == cudaSuccess)
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, lag_pipe_kernel<J>, kLagThreads, smem);
    if (err != cudaSuccess)
        return fail(DDM_ERR_CUDA, std::string("lag kernel set-up failed: ") + cudaGetErrorString(err));
    return DDM_OK;
}

// Window starts for the caller's rows. Row t must see positions [w_t, w_t + F) of one
// position list equal to its b_slots row. Rows that are shifts of one frame sequence (the
// usual b[t][j] = a[j] - tau_t pattern) share most positions, so each row is laid over the
// tail of the list where it matches and only its new positions are appended: the union the
// kernel streams then holds each partner frame once, and rows one frame apart form the
// kernel's fused runs. Rows are tried in the caller's order and reversed (window starts must
// ascend; the accumulator row travels with each entry) and the shorter list is kept.
void lay_out_windows(const int *b, int T, int F, bool reversed, std::vector<int> *ent_acc, std::vector<int> *ent_w,
                     std::vector<int> *pos) {
    ent_acc->clear();
    ent_w->clear();
    pos->clear();
    int prev = -1;
    for (int i = 0; i < T; i++) {
        const int t = reversed ? T - 1 - i : i;
        const int *row = b + static_cast<size_t>(t) * F;
        const int n = static_cast<int>(pos->size());
        int w = n;  // disjoint by default
        for (int c = std::max(prev + 1, n - F + 1); c < n; c++) {
            bool match = true;
            for (int j = 0; j < F && c + j < n && match; j++) match = (*pos)[c + j] == row[j];
            if (match) {
                w = c;
                break;
            }
        }
        for (int j = n - w; j < F; j++) pos->push_back(row[j]);
        ent_acc->push_back(t);
        ent_w->push_back(w);
        prev = w;
    }
}

}  // namespace

extern "C" int ddm_lag_accumulate_static(const void *ring, int ring_slots, long long elements, void *acc,
                                         const int *a_slots, int frame_count, const int *b_slots, int tau_count,
                                         void *stream) {
    clear_error();
    if (!ring || !acc || !a_slots || !b_slots)
        return fail(DDM_ERR_INVALID_ARG, "ddm_lag_accumulate_static: null pointer");
    if (frame_count < 1 || frame_count > kStaticMaxFrames)
        return fail(DDM_ERR_INVALID_ARG, "ddm_lag_accumulate_static: frame_count must be 1.." +
                                             std::to_string(kStaticMaxFrames));
    if (tau_count < 1 || tau_count > kStaticMaxTaus)
        return fail(DDM_ERR_INVALID_ARG, "ddm_lag_accumulate_static: tau_count must be 1.." +
                                             std::to_string(kStaticMaxTaus) +
                                             " (the static pair table holds at most that many rows)");
    if (elements <= 0 || elements % 2 != 0)
        return fail(DDM_ERR_INVALID_ARG, "ddm_lag_accumulate_static: elements must be positive and even");
    if (ring_slots < 1 || ring_slots > 0xFFFFF)
        return fail(DDM_ERR_INVALID_ARG, "ddm_lag_accumulate_static: ring_slots must be 1..1048575");
    if (reinterpret_cast<uintptr_t>(ring) % 16 != 0 || reinterpret_cast<uintptr_t>(acc) % 8 != 0)
        return fail(DDM_ERR_INVALID_ARG,
                    "ddm_lag_accumulate_static: ring must be 16-byte aligned and acc 8-byte aligned");
    for (int j = 0; j < frame_count; j++)
        if (a_slots[j] < -1 || a_slots[j] >= ring_slots)
            return fail(DDM_ERR_INVALID_ARG, "ddm_lag_accumulate_static: a_slots entry outside -1..ring_slots-1");
    for (int i = 0; i < tau_count * frame_count; i++)
        if (b_slots[i] < -1 || b_slots[i] >= ring_slots)
            return fail(DDM_ERR_INVALID_ARG, "ddm_lag_accumulate_static: b_slots entry outside -1..ring_slots-1");

    const int F = frame_count;
    std::vector<int> ent_acc, ent_w, pos, acc2, w2, pos2;
    lay_out_windows(b_slots, tau_count, F, false, &ent_acc, &ent_w, &pos);
    lay_out_windows(b_slots, tau_count, F, true, &acc2, &w2, &pos2);
    if (pos2.size() < pos.size()) {
        ent_acc.swap(acc2);
        ent_w.swap(w2);
        pos.swap(pos2);
    }
    const int J = lag_pick_j(F);
    std::vector<int> table;
    std::string err = build_lag_table(F, a_slots, ent_acc, ent_w, pos, J, &table);
    if (!err.empty()) return fail(DDM_ERR_INVALID_ARG, "ddm_lag_accumulate_static: " + err);
    if (static_cast<int>(table.size()) > kStaticTableInts)
        return fail(DDM_ERR_INVALID_ARG, "ddm_lag_accumulate_static: pair table exceeds the static maximum");
    LagMaps maps;
    err = make_lag_maps(ring, elements, ring_slots, &maps);
    if (!err.empty()) return fail(DDM_ERR_INVALID_ARG, "ddm_lag_accumulate_static: " + err);

    std::lock_guard<std::mutex> guard(g_lock);
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        return fail(DDM_ERR_NO_DEVICE, "ddm_lag_accumulate_static: no current CUDA device");
    const size_t smem = lag_smem_bytes(J, static_cast<int>(table.size()));
    int *base = nullptr, per_sm = 0;
    int st = DDM_OK;
    switch (J) {
#define LAG_CASE(JJ) \
    case JJ: st = setup_call<JJ>(smem, &base, &per_sm); break;
        LAG_CASE(4) LAG_CASE(8) LAG_CASE(16) LAG_CASE(20) LAG_CASE(24) LAG_CASE(30) LAG_CASE(32)
#undef LAG_CASE
        default: return fail(DDM_ERR_STATE, "ddm_lag_accumulate_static: no kernel for this frame count");
    }
    if (st) return st;
    int *d_table = base;
    int *d_status = base + kStaticTableInts;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t ce = cudaMemcpyAsync(d_table, table.data(), sizeof(int) * table.size(), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(d_status, 0, sizeof(int), s);
    if (ce != cudaSuccess) {
        cudaStreamSynchronize(s);  // a queued table copy may still read `table`
        return fail(DDM_ERR_CUDA, std::string("ddm_lag_accumulate_static: ") + cudaGetErrorString(ce));
    }
    // persistent grid as the engine's: the CTAs the SMs hold at once walk the element blocks
    const unsigned blocks = static_cast<unsigned>((elements + lag_cta_elems(J) - 1) / lag_cta_elems(J));
    const unsigned grid =
        std::min<unsigned>(blocks, static_cast<unsigned>(std::max(1, std::min(per_sm, kLagCtasPerSm)) * sms));
    const float2 *r = static_cast<const float2 *>(ring);
    float2 *a = static_cast<float2 *>(acc);
    switch (J) {
#define LAG_CASE(JJ) \
    case JJ:                                                                                              \
        lag_pipe_kernel<JJ><<<grid, kLagThreads, smem, s>>>(r, a, elements, d_table, d_status, maps,              \
                                                            static_cast<int>(blocks), kWaitCycles);               \
        break;
        LAG_CASE(4) LAG_CASE(8) LAG_CASE(16) LAG_CASE(20) LAG_CASE(24) LAG_CASE(30) LAG_CASE(32)
#undef LAG_CASE
        default: break;
    }
    // From here on every return waits for the stream first, still under the lock, so no call
    // returns while its kernel may still read the shared table.
    ce = cudaGetLastError();
    int status = 0;
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
    const cudaError_t se = cudaStreamSynchronize(s);
    if (ce == cudaSuccess) ce = se;
    if (ce != cudaSuccess) return fail(DDM_ERR_CUDA, std::string("ddm_lag_accumulate_static: ") + cudaGetErrorString(ce));
    if (status != 0)
        return fail(DDM_ERR_CUDA, std::string("ddm_lag_accumulate_static: ") + device_status_text(status) +
                                      "; accumulators incomplete");
    return DDM_OK;
}
