// Engine internals shared with the serving layer (server.cu): deferred lag launches, which
// a server gathers from many engines into one batched launch, and asynchronous finalize.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/ddm.h"
#include "lag.cuh"

namespace ddm {

// Private streams an engine takes from the stream pool (FFT, host copies, results, uploads)
// when given a stream to queue on, as a server's engines are.
constexpr int kEngineStreams = 4;

struct DeferredLag {  // one lag launch an engine would have issued
    int J;
    const int *table;  // device copy of its table (the engine's table ring)
    unsigned blocks;
    size_t smem;
};

struct LagTarget {  // what a lag launch of this engine reads and writes
    const float2 *ring;
    float2 *acc;
    long long E;
    int *status;
    const LagMaps *maps;  // host copy of the ring's tensor maps
};

// With deferral on, lag launches are queued (tables already uploaded on the engine's stream)
// for the caller to issue, on the engine's stream, after the work queued before them.
void engine_defer_lag(ddm_engine *e, bool on);
std::vector<DeferredLag> engine_take_deferred(ddm_engine *e);
LagTarget engine_lag_target(const ddm_engine *e);
// Validation and sizing of ddm_open only: the device bytes checked against the HBM budget.
int engine_plan_bytes(const ddm_config *cfg, size_t *need);
// ddm_close without synchronising: device memory is freed in stream order on the engine's
// stream; the caller makes sure none of the engine's queued copies still reads its host
// buffers (they return to the pinned pool at once).
void engine_close_async(ddm_engine *e);
// ddm_finalize without the device-status read and its synchronisation.
int engine_finalize_async(ddm_engine *e);
cudaStream_t engine_stream(const ddm_engine *e);
const double *engine_isf_device(const ddm_engine *e);
const int *engine_status_device(const ddm_engine *e);

}  // namespace ddm
