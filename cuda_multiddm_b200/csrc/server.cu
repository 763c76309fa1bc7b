// Serving many DDM streams on one GPU: admission by HBM footprint, per-stream device state
// (FFT ring, accumulators) kept resident, and continuous batching: every step takes the
// next pending chunk of every stream that has one, runs each stream's FFT, then ONE lag
// launch (per register-frame count) over all those streams' lag work, then each stream's
// azimuthal average and the copy of its ISF to host memory. Steps do not wait for the GPU:
// a stream's result is ready when a host callback queued behind its copy has run, so
// chunks that arrive while earlier ones are on the GPU are taken by the next step.
// (The reference analyses one video per process: src/DDM.cu:268-892.)
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ddm.h"
#include "engine_internal.hpp"
#include "errors.hpp"
#include "lag.cuh"
#include "pinned_pool.hpp"
#include "stream_pool.hpp"

using namespace ddm;

namespace {

constexpr int kItemRing = 4;  // batch descriptor buffers in flight
constexpr size_t kPinnedArenaBytes = 2ull << 30;  // page-locked at server open for the pinned pool's misses

using Clock = std::chrono::steady_clock;

struct PinnedBuf {
    void *p = nullptr;
    size_t bytes = 0;
    bool owned = true;  // false: the caller's page-locked buffer (ddm_server_submit_pinned)
};

struct Slot {  // one chunk on its way through the GPU, and its result
    double *isf_h = nullptr;  // pinned
    int *status_h = nullptr;  // pinned
    PinnedBuf frames;         // the chunk's frames (held until the result is in)
    long chunk_index = 0;
    long frames_done = 0;
    double submit_s = 0.0;
    std::atomic<double> done_s{0.0};
    std::atomic<int> state{0};  // 0 free, 1 on the GPU, 2 result ready
    const ddm_server *server = nullptr;
};

struct PendingChunk {
    PinnedBuf frames;
    int count;
    double submit_s;
};

struct Stream {
    ddm_engine *eng = nullptr;
    cudaEvent_t gone = nullptr;  // removal: recorded after the stream's last queued work
    size_t bytes = 0;
    size_t frame_bytes = 0;
    long isf_size = 0;
    long chunks_submitted = 0, chunks_issued = 0, frames_issued = 0;
    LagMaps *maps_d = nullptr;
    LagMaps *maps_h = nullptr;  // pinned source of the maps_d upload
    std::deque<PendingChunk> pending;
    std::vector<std::unique_ptr<Slot>> slots;
    std::deque<Slot *> order;  // slots in flight or ready, in chunk order
    std::vector<PinnedBuf> free_bufs;
};

void CUDART_CB on_result(void *arg) {  // runs on a CUDA driver thread: no CUDA calls here
    Slot *s = static_cast<Slot *>(arg);
    s->done_s.store(ddm_server_clock(s->server));
    s->state.store(2);
}

}  // namespace

struct ddm_server {
    int device = 0;
    cudaStream_t stream = nullptr;
    size_t budget = 0, used = 0, reserved = 0;
    int opening = 0;  // streams being admitted outside the lock
    int max_streams = 64, results_per_stream = 4;
    Clock::time_point t0 = Clock::now();
    int next_id = 1;
    std::map<int, Stream> streams;
    std::list<Stream> closing;  // removed, waiting for their queued work before release
    mutable std::mutex lock;
    // batched lag descriptors
    LagBatchItem *items_h = nullptr, *items_d = nullptr;
    int items_cap = 0, items_next = 0;
    cudaEvent_t items_ev[kItemRing] = {};
    bool items_used[kItemRing] = {};
    long launches = 0;
    long steps = 0;
    double step_host_s = 0.0, gpu_s = 0.0;
    std::deque<std::pair<cudaEvent_t, cudaEvent_t>> step_ev;  // steps whose GPU time is not yet counted
    std::vector<cudaEvent_t> spare_ev;
};

namespace {

// Adds the GPU time of finished steps to gpu_s and recycles their events.
void collect_step_times(ddm_server *s) {
    while (!s->step_ev.empty() && cudaEventQuery(s->step_ev.front().second) == cudaSuccess) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, s->step_ev.front().first, s->step_ev.front().second) == cudaSuccess)
            s->gpu_s += ms / 1000.0;
        s->spare_ev.push_back(s->step_ev.front().first);
        s->spare_ev.push_back(s->step_ev.front().second);
        s->step_ev.pop_front();
    }
}

void release_stream(Stream &st);

void reap(ddm_server *s, bool wait) {
    for (auto it = s->closing.begin(); it != s->closing.end();) {
        Stream &st = *it;
        if (wait || !st.gone || cudaEventQuery(st.gone) == cudaSuccess) {
            if (wait && st.gone) cudaEventSynchronize(st.gone);
            s->used -= st.bytes;
            release_stream(st);
            it = s->closing.erase(it);
        } else {
            ++it;
        }
    }
}

cudaEvent_t take_event(ddm_server *s) {
    if (!s->spare_ev.empty()) {
        cudaEvent_t ev = s->spare_ev.back();
        s->spare_ev.pop_back();
        return ev;
    }
    cudaEvent_t ev = nullptr;
    if (cudaEventCreate(&ev) != cudaSuccess) return nullptr;
    return ev;
}

#define CUDA_TRY(expr)                                                                            \
    do {                                                                                          \
        cudaError_t err__ = (expr);                                                               \
        if (err__ != cudaSuccess) return fail(DDM_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(err__)); \
    } while (0)

void drop(PinnedBuf &b) {
    if (b.owned) pinned_release(b.p);
    b = PinnedBuf();
}

int pinned(PinnedBuf *b, size_t bytes) {
    if (b->owned && b->bytes >= bytes && b->p) return DDM_OK;
    drop(*b);
    b->p = pinned_alloc(bytes);
    if (!b->p) return fail(DDM_ERR_OUT_OF_MEMORY, "pinned host buffer");
    b->bytes = bytes;
    b->owned = true;
    return DDM_OK;
}

// Releases a stream whose queued work has all run (its removal event has completed).
void release_stream(Stream &st) {
    engine_close_async(st.eng);
    cudaFreeAsync(st.maps_d, nullptr);
    pinned_release(st.maps_h);
    for (auto &sl : st.slots) {
        pinned_release(sl->isf_h);
        pinned_release(sl->status_h);
        drop(sl->frames);
    }
    for (auto &pc : st.pending) drop(pc.frames);
    for (auto &b : st.free_bufs) drop(b);
    if (st.gone) cudaEventDestroy(st.gone);
    st = Stream();
}

int ensure_items(ddm_server *s, int n) {
    if (n <= s->items_cap) return DDM_OK;
    CUDA_TRY(cudaStreamSynchronize(s->stream));  // no batch descriptors in flight
    if (s->items_h) cudaFreeHost(s->items_h);
    cudaFree(s->items_d);
    s->items_h = nullptr;
    s->items_d = nullptr;
    const int cap = std::max(n, 64);
    if (cudaMallocHost(reinterpret_cast<void **>(&s->items_h), sizeof(LagBatchItem) * cap * kItemRing) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void **>(&s->items_d), sizeof(LagBatchItem) * cap * kItemRing) != cudaSuccess)
        return fail(DDM_ERR_OUT_OF_MEMORY, "batch descriptor buffers");
    s->items_cap = cap;
    std::fill(s->items_used, s->items_used + kItemRing, false);
    return DDM_OK;
}

// One launch of lag_batch_kernel<J> over `work` (engine, its deferred launches of this J).
int launch_batch(ddm_server *s, int J, const std::vector<std::pair<Stream *, DeferredLag>> &work) {
    if (work.empty()) return DDM_OK;
    int st = ensure_items(s, static_cast<int>(work.size()));
    if (st) return st;
    const int ring = s->items_next;
    s->items_next = (s->items_next + 1) % kItemRing;
    if (s->items_used[ring]) CUDA_TRY(cudaEventSynchronize(s->items_ev[ring]));
    LagBatchItem *h = s->items_h + static_cast<size_t>(ring) * s->items_cap;
    LagBatchItem *d = s->items_d + static_cast<size_t>(ring) * s->items_cap;
    int cta = 0;
    size_t smem = 0;
    for (size_t i = 0; i < work.size(); i++) {
        const LagTarget t = engine_lag_target(work[i].first->eng);
        h[i] = LagBatchItem{t.ring, t.acc, t.E, work[i].second.table, t.status, work[i].first->maps_d, cta, 0};
        cta += static_cast<int>(work[i].second.blocks);
        smem = std::max(smem, work[i].second.smem);
    }
    const int n = static_cast<int>(work.size());
    CUDA_TRY(cudaMemcpyAsync(d, h, sizeof(LagBatchItem) * n, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaEventRecord(s->items_ev[ring], s->stream));
    s->items_used[ring] = true;
    switch (J) {
#define BATCH_CASE(JJ) \
    case JJ: lag_batch_kernel<JJ><<<cta, kLagThreads, smem, s->stream>>>(d, n); break;
        BATCH_CASE(4) BATCH_CASE(8) BATCH_CASE(16) BATCH_CASE(20) BATCH_CASE(24) BATCH_CASE(30) BATCH_CASE(32)
        BATCH_CASE(64)
#undef BATCH_CASE
        default: return fail(DDM_ERR_STATE, "internal: no batched lag kernel for this frame count");
    }
    CUDA_TRY(cudaGetLastError());
    s->launches++;
    return DDM_OK;
}

}  // namespace

extern "C" double ddm_server_clock(const ddm_server *s) {
    if (!s) return 0.0;
    return std::chrono::duration<double>(Clock::now() - s->t0).count();
}

extern "C" int ddm_server_open(const ddm_server_config *cfg, ddm_server **out) {
    clear_error();
    if (!cfg || !out) return fail(DDM_ERR_INVALID_ARG, "ddm_server_open: null argument");
    *out = nullptr;
    if (cfg->max_streams < 0 || cfg->results_per_stream < 0)
        return fail(DDM_ERR_INVALID_ARG, "ddm_server_open: negative limit");
    std::unique_ptr<ddm_server> s(new ddm_server);
    s->device = cfg->device;
    if (cudaSetDevice(s->device) != cudaSuccess) return fail(DDM_ERR_NO_DEVICE, "cudaSetDevice failed");
    size_t free_b = 0, total_b = 0;
    CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    s->budget = cfg->hbm_budget_bytes ? cfg->hbm_budget_bytes : (free_b > (2ull << 30) ? free_b - (2ull << 30) : 0);
    if (cfg->max_streams) s->max_streams = cfg->max_streams;
    if (cfg->results_per_stream) s->results_per_stream = cfg->results_per_stream;
    CUDA_TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    // Keep freed stream memory in the device pool, so streams that leave make room for the
    // next ones without a trip through the driver, and map the whole budget into the pool
    // now: growing the pool while streams run holds up their work (measured: a p99 chunk
    // latency of about 1 s on a cold pool against 12 ms on a warm one).
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        void *warm = nullptr;
        if (s->budget && cudaMallocAsync(&warm, s->budget, s->stream) == cudaSuccess) {
            cudaFreeAsync(warm, s->stream);
            cudaStreamSynchronize(s->stream);
        }
        cudaGetLastError();  // a budget the pool cannot map at once is not an error
    }
    // the private streams of every slot's engine, made now while the device is idle (made
    // while streams run, each took tens of milliseconds and held up the steps' launches)
    StreamPool::get().reserve(s->device, kEngineStreams * s->max_streams);
    // and page-locked memory for the streams' chunk and result buffers (a miss of the pinned
    // pool otherwise pins memory while the admitted streams run); not an error if refused
    if (!PinnedPool::get().reserve_arena(kPinnedArenaBytes)) cudaGetLastError();
    for (int i = 0; i < kItemRing; i++) CUDA_TRY(cudaEventCreateWithFlags(&s->items_ev[i], cudaEventDisableTiming));
    const int attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
#define BATCH_ATTR(JJ) \
    CUDA_TRY(cudaFuncSetAttribute(lag_batch_kernel<JJ>, static_cast<cudaFuncAttribute>(attr), kLagSmemMax));
    BATCH_ATTR(4) BATCH_ATTR(8) BATCH_ATTR(16) BATCH_ATTR(20) BATCH_ATTR(24) BATCH_ATTR(30) BATCH_ATTR(32) BATCH_ATTR(64)
#undef BATCH_ATTR
    *out = s.release();
    return DDM_OK;
}

extern "C" int ddm_server_close(ddm_server *s) {
    if (!s) return DDM_OK;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    for (auto &pr : s->step_ev) {
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    for (cudaEvent_t ev : s->spare_ev) cudaEventDestroy(ev);
    reap(s, true);
    for (auto &kv : s->streams) release_stream(kv.second);
    s->streams.clear();
    cudaStreamSynchronize(s->stream);  // the stream-ordered frees
    cudaMemPool_t pool;  // hand the warm pool back to the device
    if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
        uint64_t none = 0;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &none);
        cudaMemPoolTrimTo(pool, 0);
    }
    if (s->items_h) cudaFreeHost(s->items_h);
    cudaFree(s->items_d);
    for (cudaEvent_t ev : s->items_ev)
        if (ev) cudaEventDestroy(ev);
    cudaStreamDestroy(s->stream);
    delete s;
    return DDM_OK;
}

extern "C" int ddm_server_add_stream(ddm_server *s, const ddm_config *cfg, int *stream_id) {
    clear_error();
    if (!s || !cfg || !stream_id) return fail(DDM_ERR_INVALID_ARG, "ddm_server_add_stream: null argument");
    if (cfg->estimator != DDM_EST_UNBIASED)
        return fail(DDM_ERR_INVALID_ARG, "served streams use the unbiased estimator (open-ended, a result per chunk)");
    ddm_config c = *cfg;
    c.device = s->device;
    c.stream = s->stream;      // all engines queue on the server's stream
    c.lag_batch_frames = std::min(cfg->chunk_frames > 0 ? cfg->chunk_frames : 1, 32);  // pair every chunk at once
    c.dump_every = 0;
    c.hbm_budget_bytes = 0;
    size_t need = 0;
    int r = engine_plan_bytes(&c, &need);
    if (r) return r;
    // admission: reserve the stream's bytes under the lock, build its engine without it (steps
    // of the admitted streams go on meanwhile), then insert it
    {
        std::lock_guard<std::mutex> g(s->lock);
        reap(s, false);
        if (static_cast<int>(s->streams.size()) + s->opening >= s->max_streams)
            return fail(DDM_ERR_BUSY, "all stream slots are taken");
        if (s->used + s->reserved + need > s->budget)
            return fail(DDM_ERR_BUSY, "not admitted now: the stream needs " + std::to_string(need) +
                                          " device bytes, " + std::to_string(s->budget - s->used - s->reserved) +
                                          " of the budget are free");
        s->reserved += need;
        s->opening++;
    }
    Stream st;
    auto unreserve = [&]() {
        std::lock_guard<std::mutex> g(s->lock);
        s->reserved -= need;
        s->opening--;
    };
    r = ddm_open(&c, &st.eng);
    if (r) {
        unreserve();
        return r == DDM_ERR_OUT_OF_MEMORY ? fail(DDM_ERR_BUSY, std::string("not admitted now: ") + ddm_last_error()) : r;
    }
    engine_defer_lag(st.eng, true);
    ddm_info info;
    ddm_get_info(st.eng, &info);
    st.bytes = info.device_bytes;
    st.frame_bytes = static_cast<size_t>(cfg->frame_width) * cfg->frame_height * cfg->bytes_per_pixel;
    st.isf_size = ddm_isf_size(st.eng);
    const LagTarget t = engine_lag_target(st.eng);
    // the tensor maps go up from page-locked memory: a copy from pageable memory may wait for
    // the shared stream to drain, holding up this call and the steps' launches meanwhile
    st.maps_h = static_cast<LagMaps *>(pinned_alloc(sizeof(LagMaps)));
    bool ok = st.maps_h != nullptr;
    if (ok) *st.maps_h = *t.maps;
    ok = ok && cudaMallocAsync(reinterpret_cast<void **>(&st.maps_d), sizeof(LagMaps), s->stream) == cudaSuccess &&
         cudaMemcpyAsync(st.maps_d, st.maps_h, sizeof(LagMaps), cudaMemcpyHostToDevice, s->stream) == cudaSuccess;
    for (int i = 0; ok && i < s->results_per_stream; i++) {
        auto sl = std::make_unique<Slot>();
        sl->server = s;
        sl->isf_h = static_cast<double *>(pinned_alloc(sizeof(double) * std::max<long>(st.isf_size, 1)));
        sl->status_h = static_cast<int *>(pinned_alloc(sizeof(int)));
        ok = sl->isf_h && sl->status_h;
        st.slots.push_back(std::move(sl));
    }
    std::lock_guard<std::mutex> g(s->lock);
    s->reserved -= need;
    s->opening--;
    if (!ok) {
        cudaStreamSynchronize(s->stream);
        release_stream(st);
        return fail(DDM_ERR_OUT_OF_MEMORY, "server stream buffers");
    }
    s->used += st.bytes;
    const int id = s->next_id++;
    s->streams.emplace(id, std::move(st));
    *stream_id = id;
    return DDM_OK;
}

extern "C" int ddm_server_remove_stream(ddm_server *s, int stream_id) {
    clear_error();
    if (!s) return fail(DDM_ERR_INVALID_ARG, "null server");
    std::lock_guard<std::mutex> g(s->lock);
    auto it = s->streams.find(stream_id);
    if (it == s->streams.end()) return fail(DDM_ERR_INVALID_ARG, "unknown stream");
    // released once the server's stream has run everything queued for it (result callbacks
    // included), without waiting here
    Stream st = std::move(it->second);
    s->streams.erase(it);
    if (cudaEventCreateWithFlags(&st.gone, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventRecord(st.gone, s->stream) != cudaSuccess) {
        if (st.gone) cudaEventDestroy(st.gone);
        st.gone = nullptr;
        CUDA_TRY(cudaStreamSynchronize(s->stream));
    }
    s->closing.push_back(std::move(st));
    reap(s, false);
    return DDM_OK;
}

namespace {

int submit_chunk(ddm_server *s, int stream_id, const void *frames, int count, bool copy) {
    clear_error();
    if (!s || !frames || count <= 0) return fail(DDM_ERR_INVALID_ARG, "ddm_server_submit: bad argument");
    std::lock_guard<std::mutex> g(s->lock);
    auto it = s->streams.find(stream_id);
    if (it == s->streams.end()) return fail(DDM_ERR_INVALID_ARG, "unknown stream");
    Stream &st = it->second;
    PendingChunk pc;
    if (copy) {
        if (!st.free_bufs.empty()) {
            pc.frames = st.free_bufs.back();
            st.free_bufs.pop_back();
        }
        int r = pinned(&pc.frames, st.frame_bytes * count);
        if (r) return r;
        std::memcpy(pc.frames.p, frames, st.frame_bytes * count);
    } else {
        pc.frames.p = const_cast<void *>(frames);
        pc.frames.bytes = st.frame_bytes * count;
        pc.frames.owned = false;
    }
    pc.count = count;
    pc.submit_s = ddm_server_clock(s);
    st.pending.push_back(pc);
    st.chunks_submitted++;
    return DDM_OK;
}

}  // namespace

extern "C" int ddm_server_submit(ddm_server *s, int stream_id, const void *frames, int count) {
    return submit_chunk(s, stream_id, frames, count, true);
}

extern "C" int ddm_server_submit_pinned(ddm_server *s, int stream_id, const void *frames, int count) {
    return submit_chunk(s, stream_id, frames, count, false);
}

extern "C" int ddm_server_step(ddm_server *s, int *chunks_issued) {
    clear_error();
    if (!s) return fail(DDM_ERR_INVALID_ARG, "null server");
    std::lock_guard<std::mutex> g(s->lock);
    if (chunks_issued) *chunks_issued = 0;
    const auto t_start = Clock::now();
    reap(s, false);
    collect_step_times(s);
    cudaEvent_t ev0 = nullptr;
    bool any = false;
    for (auto &kv : s->streams) any = any || !kv.second.pending.empty();
    if (any && (ev0 = take_event(s))) CUDA_TRY(cudaEventRecord(ev0, s->stream));
    std::vector<std::pair<Stream *, Slot *>> taken;
    std::map<int, std::vector<std::pair<Stream *, DeferredLag>>> by_j;
    // 1. each stream's next chunk: H2D copy and FFT (the engine's own stream pair), lag work deferred
    for (auto &kv : s->streams) {
        Stream &st = kv.second;
        if (st.pending.empty()) continue;
        Slot *slot = nullptr;
        for (auto &sl : st.slots)
            if (sl->state.load() == 0) {
                slot = sl.get();
                break;
            }
        if (!slot) continue;  // the caller has not collected earlier results yet
        PendingChunk pc = st.pending.front();
        st.pending.pop_front();
        int r = ddm_submit_frames(st.eng, pc.frames.p, pc.count, 0);
        if (r) return r;
        slot->frames = pc.frames;
        slot->chunk_index = st.chunks_issued++;
        st.frames_issued += pc.count;
        slot->frames_done = st.frames_issued;
        slot->submit_s = pc.submit_s;
        slot->state.store(1);
        st.order.push_back(slot);
        taken.emplace_back(&st, slot);
        for (const DeferredLag &d : engine_take_deferred(st.eng)) by_j[d.J].emplace_back(&st, d);
    }
    // 2. one lag launch per register-frame count over every taken stream
    for (auto &kv : by_j) {
        int r = launch_batch(s, kv.first, kv.second);
        if (r) return r;
    }
    // 3. per stream: azimuthal average, ISF and status to host, completion callback
    for (auto &ts : taken) {
        Stream &st = *ts.first;
        Slot *slot = ts.second;
        int r = engine_finalize_async(st.eng);
        if (r) return r;
        CUDA_TRY(cudaMemcpyAsync(slot->isf_h, engine_isf_device(st.eng), sizeof(double) * st.isf_size,
                                 cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaMemcpyAsync(slot->status_h, engine_status_device(st.eng), sizeof(int), cudaMemcpyDeviceToHost,
                                 s->stream));
        CUDA_TRY(cudaLaunchHostFunc(s->stream, on_result, slot));
    }
    if (ev0) {
        cudaEvent_t ev1 = take_event(s);
        if (ev1) {
            CUDA_TRY(cudaEventRecord(ev1, s->stream));
            s->step_ev.emplace_back(ev0, ev1);
        } else {
            s->spare_ev.push_back(ev0);
        }
    }
    if (!taken.empty()) {
        s->steps++;
        s->step_host_s += std::chrono::duration<double>(Clock::now() - t_start).count();
    }
    if (chunks_issued) *chunks_issued = static_cast<int>(taken.size());
    return DDM_OK;
}

extern "C" int ddm_server_poll(ddm_server *s, int stream_id, ddm_chunk_result *res, double *isf, long capacity) {
    clear_error();
    if (!s) return fail(DDM_ERR_INVALID_ARG, "null server");
    std::lock_guard<std::mutex> g(s->lock);
    auto it = s->streams.find(stream_id);
    if (it == s->streams.end()) return fail(DDM_ERR_INVALID_ARG, "unknown stream");
    Stream &st = it->second;
    if (st.order.empty() || st.order.front()->state.load() != 2) return 0;
    Slot *slot = st.order.front();
    if (*slot->status_h != 0)
        return fail(DDM_ERR_CUDA, std::string(device_status_text(*slot->status_h)) + "; results are incomplete");
    if (isf) {
        if (capacity < st.isf_size) return fail(DDM_ERR_INVALID_ARG, "ddm_server_poll: ISF buffer too small");
        std::memcpy(isf, slot->isf_h, sizeof(double) * st.isf_size);
    }
    if (res) {
        res->chunk_index = slot->chunk_index;
        res->frames = slot->frames_done;
        res->submit_s = slot->submit_s;
        res->done_s = slot->done_s.load();
    }
    st.order.pop_front();
    if (slot->frames.owned) st.free_bufs.push_back(slot->frames);
    slot->frames = PinnedBuf();
    slot->state.store(0);
    return 1;
}

extern "C" int ddm_server_wait(ddm_server *s) {
    clear_error();
    if (!s) return fail(DDM_ERR_INVALID_ARG, "null server");
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return DDM_OK;
}

extern "C" int ddm_server_get_stats(const ddm_server *s, ddm_server_stats *info) {
    if (!s || !info) return fail(DDM_ERR_INVALID_ARG, "bad argument");
    std::lock_guard<std::mutex> g(s->lock);
    info->streams = static_cast<int>(s->streams.size());
    info->device_bytes = s->used;
    info->budget_bytes = s->budget;
    info->batched_launches = s->launches;
    long pending = 0;
    for (const auto &kv : s->streams) pending += static_cast<long>(kv.second.pending.size());
    info->chunks_pending = pending;
    info->steps = s->steps;
    info->step_host_s = s->step_host_s;
    collect_step_times(const_cast<ddm_server *>(s));
    info->gpu_s = s->gpu_s;
    return DDM_OK;
}
