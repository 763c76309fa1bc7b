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
#include <cuda.h>
#include <cuda_runtime.h>

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
constexpr int kMaxDevices = 64;

static_assert(lag_table_ints(kStaticMaxTaus, kStaticMaxTaus * kStaticMaxFrames,
                             (kStaticMaxTaus * kStaticMaxFrames + kLagGroup - 1) / kLagGroup,
                             kStaticMaxTaus * kStaticMaxFrames) <= kStaticTableInts,
              "static lag table too small for the stated maximum");

__device__ __align__(256) int g_static_scratch[kStaticTableInts + kStaticStatusInts];

struct DeviceScratch {
    bool ready = false;
    int *base = nullptr;  // device address of g_static_scratch on this device
};
DeviceScratch g_dev[kMaxDevices];
std::mutex g_lock;

// Once per device, with that device current: the array's device address and the kernel's
// shared-memory limit. Runs on the first call on each device.
int setup_device(int dev) {
    DeviceScratch &d = g_dev[dev];
    if (d.ready) return DDM_OK;
    cudaError_t err = cudaGetSymbolAddress(reinterpret_cast<void **>(&d.base), g_static_scratch);
    if (err != cudaSuccess)
        return fail(DDM_ERR_CUDA, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(err));
    const int attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if (cudaFuncSetAttribute(lag_pipe_kernel<4>, static_cast<cudaFuncAttribute>(attr), kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<8>, static_cast<cudaFuncAttribute>(attr), kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<16>, static_cast<cudaFuncAttribute>(attr), kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<20>, static_cast<cudaFuncAttribute>(attr), kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<24>, static_cast<cudaFuncAttribute>(attr), kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<30>, static_cast<cudaFuncAttribute>(attr), kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<32>, static_cast<cudaFuncAttribute>(attr), kLagSmemMax) != cudaSuccess)
        return fail(DDM_ERR_CUDA, "cudaFuncSetAttribute failed");
    d.ready = true;
    return DDM_OK;
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
    for (int j = 0; j < frame_count; j++)
        if (a_slots[j] >= ring_slots) return fail(DDM_ERR_INVALID_ARG, "a_slots entry outside the ring");
    for (int i = 0; i < tau_count * frame_count; i++)
        if (b_slots[i] >= ring_slots) return fail(DDM_ERR_INVALID_ARG, "b_slots entry outside the ring");

    // Entry t pairs register frame j with window position t*F + j: the table's windows are
    // the caller's rows of b_slots, laid end to end.
    const int F = frame_count;
    std::vector<int> ent_acc(tau_count), ent_w(tau_count), pos(static_cast<size_t>(tau_count) * F);
    for (int t = 0; t < tau_count; t++) {
        ent_acc[t] = t;
        ent_w[t] = t * F;
        for (int j = 0; j < F; j++) pos[static_cast<size_t>(t) * F + j] = b_slots[static_cast<size_t>(t) * F + j];
    }
    const int J = lag_pick_j(F);
    std::vector<int> table;
    std::string err = build_lag_table(F, a_slots, ent_acc, ent_w, pos, J, &table);
    if (!err.empty()) return fail(DDM_ERR_INVALID_ARG, "ddm_lag_accumulate_static: " + err);
    if (static_cast<int>(table.size()) > kStaticTableInts)
        return fail(DDM_ERR_INVALID_ARG, "ddm_lag_accumulate_static: pair table exceeds the static maximum");
    LagMaps maps;
    err = make_lag_maps(ring, elements, ring_slots, &maps);
    if (!err.empty()) return fail(DDM_ERR_CUDA, "ddm_lag_accumulate_static: " + err);

    std::lock_guard<std::mutex> guard(g_lock);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(DDM_ERR_NO_DEVICE, "ddm_lag_accumulate_static: no current CUDA device");
    int st = setup_device(dev);
    if (st) return st;
    int *d_table = g_dev[dev].base;
    int *d_status = g_dev[dev].base + kStaticTableInts;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t ce = cudaMemcpyAsync(d_table, table.data(), sizeof(int) * table.size(), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(d_status, 0, sizeof(int), s);
    if (ce != cudaSuccess) return fail(DDM_ERR_CUDA, std::string("ddm_lag_accumulate_static: ") + cudaGetErrorString(ce));
    const unsigned blocks = static_cast<unsigned>((elements + lag_cta_elems(J) - 1) / lag_cta_elems(J));
    const size_t smem = lag_smem_bytes(J, static_cast<int>(table.size()));
    const float2 *r = static_cast<const float2 *>(ring);
    float2 *a = static_cast<float2 *>(acc);
    switch (J) {
#define LAG_CASE(JJ) \
    case JJ:                                                                                              \
        lag_pipe_kernel<JJ><<<blocks, kLagThreads, smem, s>>>(r, a, elements, d_table, d_status, maps,            \
                                                              static_cast<int>(blocks));                          \
        break;
        LAG_CASE(4) LAG_CASE(8) LAG_CASE(16) LAG_CASE(20) LAG_CASE(24) LAG_CASE(30) LAG_CASE(32)
#undef LAG_CASE
        default: return fail(DDM_ERR_STATE, "ddm_lag_accumulate_static: no kernel for this frame count");
    }
    ce = cudaGetLastError();
    if (ce != cudaSuccess) return fail(DDM_ERR_CUDA, std::string("ddm_lag_accumulate_static: ") + cudaGetErrorString(ce));
    int status = 0;
    ce = cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return fail(DDM_ERR_CUDA, std::string("ddm_lag_accumulate_static: ") + cudaGetErrorString(ce));
    if (status != 0) return fail(DDM_ERR_CUDA, "ddm_lag_accumulate_static: a pipeline wait timed out; accumulators incomplete");
    return DDM_OK;
}
