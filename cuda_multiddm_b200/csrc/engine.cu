// The DDM engine behind include/ddm.h: device buffers, the frame ring, scheduling of
// the lag pairs (reference schedule or unbiased), -G snapshots and the C ABI.
//
// Device layout (one engine):
//   ring   float2 [R][E]   spectra of the last R frames; frame label f lives in slot f % R.
//                          A frame is the concatenation over scales (descending) of
//                          [tile][ky][kx], kx in [0, s/2]; E = sum_s tiles_s * s * (s/2+1).
//   acc    float2 [T][E]   per (tau, element): FP32 running sum of |dF|^2 and its Kahan
//                          compensation (true value = sum - comp), unnormalised.
//   stage  uint8  [J][M][M*bpp]   ROI of host-submitted frames (one piece at a time).
//   tables int    [kTables][tab_stride]  lag-kernel pair tables, a ring of slots.
//   masks  int    CSR of annulus element indices per (scale, q); counts [S][Q].
//   isf    double [sum_s tiles_s * Q * T].
#include <algorithm>
#include <cstdlib>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/ddm.h"
#include "errors.hpp"
#include "host.hpp"
#include "dft_bf16.cuh"
#include "fft.cuh"
#include "fit.cuh"
#include "kernels.cuh"
#include "lag.cuh"
#include "engine_internal.hpp"
#include "lag_host.hpp"
#include "pinned_pool.hpp"
#include "stream_pool.hpp"
#include "tune.hpp"

namespace ddm {

namespace {
thread_local std::string g_last_error;
}

int fail(int status, const std::string &message) {
    g_last_error = message;
    return status;
}
void clear_error() { g_last_error.clear(); }
const char *last_error() { return g_last_error.c_str(); }

}  // namespace ddm

using namespace ddm;

namespace {

constexpr int kTables = 64;  // lag tables in flight
constexpr int kAsyncMax = 8;  // ddm_finalize_async result slots (ddm_set_async_depth)
constexpr int kSubmitEvents = 8;  // submit calls ddm_wait_frames_copied can look back over

struct Launch {  // one lag-kernel launch: register frames, tau windows (ascending), position slots
    int nreg = 0;
    int reg[kMaxJ];
    std::vector<int> ent_acc, ent_w, pos;
};

int log2i(long long v) {
    int l = 0;
    while ((1LL << l) < v) l++;
    return l;
}

}  // namespace

struct ddm_engine {
    // configuration (sorted copies)
    int w = 0, h = 0, bpp = 1, pixmode = 0, x_off = 0, y_off = 0;
    std::vector<int> scales, taus;
    std::vector<float> lambdas;
    float tol = 1.2f;
    int C = 30, estimator = DDM_EST_UNBIASED, multistream = 1, N = 0, G = 0, device = 0;
    int M = 0, S = 0, T = 0, Q = 0, tau_max = 0;
    int sms = 0;  // SMs of the device (persistent lag grid)
    // resident CTAs per SM of a lag kernel instance (key J * kLagGeoms + G) at a launch's
    // dynamic shared-memory size: the persistent grid is that many CTAs per SM
    std::vector<std::tuple<int, size_t, int>> lag_resident;
    long long E = 0;
    std::vector<ScaleDesc> sd;
    long long isf_size = 0;

    // device state
    cudaStream_t stream = nullptr;      // lag, azimuth, accumulator work ("main")
    bool own_stream = false;
    // The FFT of a piece runs on its own stream, so it overlaps the lag kernel of the piece
    // before (the FFT is compute/L2-bound, the lag kernel HBM-bound). ev_fft orders each lag
    // after the FFT of its frames; ev_guard[piece & 1], recorded on the main stream when a
    // piece's FFT is issued, holds back the next piece's FFT until every lag issued before
    // this one has finished, so an FFT never overwrites ring slots a running lag still reads
    // (the ring carries one extra piece of slots for that).
    cudaStream_t fft_stream = nullptr;
    cudaEvent_t ev_fft = nullptr, ev_guard[2] = {nullptr, nullptr};
    // Host-submitted frames: their copies into the staging buffer run on copy_stream, one FFT
    // group at a time, so the copy of group g + 1 overlaps the FFT of group g; ev_copy orders
    // each group's FFT after its copies, ev_stage holds the next piece's copies until the
    // FFTs reading the staging buffer are done.
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_copy = nullptr, ev_stage = nullptr;
    bool stage_busy = false;
    long long pieces = 0;
    int R = 0, jmax = 32;
    float2 *ring = nullptr, *acc = nullptr, *tw = nullptr;
    // split-BF16 tensor-core DFT of the tiles of side 32, 64, 128 (ddm_config.small_tile_dft):
    // its cos/sin tables per log2 s - 5, in the kernel's shared-memory layout
    bool small_dft = false;
    int lag_geom = 0;  // lag-kernel geometry for launches of up to 32 frames (ddm_config.lag_geometry)
    int fft_group = 0;  // frames per FFT launch (ddm_config.fft_group_frames; 0 = the 256 MB rule)
    int fft_per_tile = 0;  // 1: tiles of side 32..128 through the per-tile kernel (ddm_config.fft_per_tile)
    uint4 *dft_tab[kDftMaxLog2 - kDftMinLog2 + 1] = {nullptr, nullptr, nullptr};
    uint8_t *stage = nullptr;
    int *tables_d = nullptr, *tables_h = nullptr;
    cudaEvent_t tab_ev[kTables] = {};    // table slot i uploaded (its pinned host copy is free again)
    cudaEvent_t tab_free[kTables] = {};  // the launch that read device table slot i is done
    // Small uploads (lag tables, norms) run on upload_stream as soon as they are built, and the
    // engine's stream waits for them: queued in stream order, a few KB could sit behind the
    // next chunk's frame copies on the copy engine when the stream reached them.
    cudaStream_t upload_stream = nullptr;
    bool tab_used[kTables] = {};
    int tab_stride = 0, tab_next = 0;
    int *idx_d = nullptr, *counts_d = nullptr;                  // annulus CSR indices, pixel counts
    int *chunk_beg_d = nullptr, *chunk_end_d = nullptr;          // azimuthal chunks of the CSR
    int *chunk_first_d = nullptr, *chunk_count_d = nullptr;      // per (scale, q)
    double *partial_d = nullptr;                                 // stage-1 azimuthal sums
    long long az_items = 0;
    double *norm_d = nullptr, *isf_d = nullptr;  // norm_d: two halves of T, alternating like norm_h
    // norm uploads alternate between two pinned halves, so a finalize never waits for the
    // previous one's upload (which runs after that finalize's lag work)
    double *norm_h = nullptr;                // pinned sources of the norm upload, 2 x T
    cudaEvent_t norm_ev[2] = {nullptr, nullptr};    // the upload from half i has read it
    cudaEvent_t norm_free[2] = {nullptr, nullptr};  // the azimuthal average that read device half i is done
    int norm_slot = 0;
    // ddm_finalize_async results alternate between two slots: the status word copied with
    // the result, the event after both copies, and whether it has been waited for
    int *async_status_h = nullptr;           // pinned, kAsyncMax ints
    cudaEvent_t async_ev[kAsyncMax] = {};
    bool async_pending[kAsyncMax] = {};
    int async_slot = 0;                      // slot of the next result
    int async_depth = 2;                     // result slots in use (ddm_set_async_depth)
    // copy stream: the host frames of each of the last kSubmitEvents submit calls have been read
    cudaEvent_t submit_ev[kSubmitEvents] = {};
    long long submit_calls = 0;
    // their copies run on result_stream, so the next chunk's lag work does not queue behind
    // them; ev_isf_ready orders a copy after its azimuthal average, ev_isf_read holds the
    // next azimuthal average (which rewrites isf_d) until the copy has read it
    cudaStream_t result_stream = nullptr;
    cudaEvent_t ev_isf_ready = nullptr, ev_isf_read = nullptr;
    double *fit_d = nullptr;                // ISF fitting: means, tau, q, curve fits, D (first fit call)
    int *status_d = nullptr;                // set by kernels whose bounded waits ran out
    long long wait_cycles = kWaitCycles;    // limit of every lag-pipeline wait (ddm_set_wait_limit)
    int inject = DDM_FAULT_NONE;            // one-shot fault for the next lag launch (ddm_inject_fault)
    LagMaps maps;                           // 2-D tensor maps of the ring for the lag kernel
    bool defer_lag = false;                 // served: lag launches are collected, not issued
    std::vector<DeferredLag> deferred;
    size_t device_bytes = 0;
    std::vector<int> counts_h;             // [S][Q]
    std::vector<std::vector<int>> q_ptr_s, idx_s;  // per scale CSR (host copy)

    // stream state
    long long submitted = 0;               // frame labels 0 .. submitted-1 are in (or passed) the ring
    // Unbiased estimator: frames lag_next .. submitted-1 are in the ring but not paired yet.
    // Lag launches take up to lag_batch frames (ddm_config.lag_batch_frames; the partner
    // frames a launch streams are shared by all its register frames). By default it equals
    // the ingest piece and every piece is paired at once; a larger batch holds frames back
    // for fuller launches, and flush_lag pairs the rest before any result is read. Compat
    // iterations are cut into launches of lag_batch A-frames.
    long long lag_next = 0;
    int lag_batch = 32;
    long long launches = 0;
    std::vector<double> pair_count;        // unbiased: pairs per tau since the last purge
    std::vector<CompatIteration> its;      // compat schedule
    size_t next_it = 0;
    int frames_read = 0;
    bool finalized = false;
    std::vector<std::vector<double>> dumps;
    std::vector<double> host_norm;

    // kernel timing (ddm_set_timing): event pairs and launch counts per kernel group
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> tev[3];
    std::vector<cudaEvent_t> tev_pool;  // read-out timing events, reused (creating them per
                                        // range made a small workload's steps host-bound)
    long tlaunch[3] = {0, 0, 0};
    // compulsory DRAM bytes of the kernels launched since the last ddm_kernel_stats: what
    // each kernel must move at least (its inputs read once, its outputs written once)
    double tbytes[3] = {0.0, 0.0, 0.0};
    double az_bytes = 0.0;  // per azimuthal average: every masked accumulator element, all taus
};

namespace {

#define CUDA_TRY(expr)                                                                     \
    do {                                                                                   \
        cudaError_t err__ = (expr);                                                        \
        if (err__ != cudaSuccess)                                                          \
            return fail(err__ == cudaErrorMemoryAllocation ? DDM_ERR_OUT_OF_MEMORY : DDM_ERR_CUDA, \
                        std::string(#expr) + ": " + cudaGetErrorString(err__));           \
    } while (0)

template <typename Tp>
int dev_alloc(ddm_engine *e, Tp **p, size_t count) {
    size_t bytes = sizeof(Tp) * std::max<size_t>(count, 1);
    // stream-ordered from the device's memory pool (no device-wide synchronisation when
    // engines come and go), on the engine's private FFT stream, complete before it is used
    cudaError_t err = cudaMallocAsync(reinterpret_cast<void **>(p), bytes, e->fft_stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->fft_stream);
    if (err != cudaSuccess)
        return fail(DDM_ERR_OUT_OF_MEMORY, std::string("cudaMalloc of ") + std::to_string(bytes) +
                                               " bytes failed: " + cudaGetErrorString(err));
    e->device_bytes += bytes;
    return DDM_OK;
}

// Releases everything; device memory is freed in stream order after the engine's queued
// work, host buffers go back to the pinned pool (callers make sure no copy still reads them).
void free_all(ddm_engine *e) {
    if (e->upload_stream) cudaStreamSynchronize(e->upload_stream);  // uploads read pinned buffers freed below
    if (e->stream && e->ev_isf_read) cudaStreamWaitEvent(e->stream, e->ev_isf_read, 0);  // a result copy reads isf_d
    void *dev[] = {e->ring, e->acc, e->tw, e->stage, e->tables_d, e->chunk_beg_d, e->chunk_end_d,
                   e->chunk_first_d, e->chunk_count_d, e->partial_d, e->idx_d, e->counts_d, e->norm_d,
                   e->isf_d, e->fit_d, e->status_d, e->dft_tab[0], e->dft_tab[1], e->dft_tab[2]};
    cudaStream_t fs = e->stream ? e->stream : e->fft_stream;
    for (void *p : dev)
        if (p) cudaFreeAsync(p, fs);
    pinned_release(e->norm_h);
    pinned_release(e->async_status_h);
    for (int i = 0; i < 2; i++) {
        if (e->norm_ev[i]) cudaEventDestroy(e->norm_ev[i]);
        if (e->norm_free[i]) cudaEventDestroy(e->norm_free[i]);
    }
    for (int i = 0; i < kAsyncMax; i++)
        if (e->async_ev[i]) cudaEventDestroy(e->async_ev[i]);
    for (int i = 0; i < kSubmitEvents; i++)
        if (e->submit_ev[i]) cudaEventDestroy(e->submit_ev[i]);
    pinned_release(e->tables_h);
    for (int i = 0; i < kTables; i++) {
        if (e->tab_ev[i]) cudaEventDestroy(e->tab_ev[i]);
        if (e->tab_free[i]) cudaEventDestroy(e->tab_free[i]);
    }
    for (int g = 0; g < 3; g++)
        for (auto &pr : e->tev[g]) {
            cudaEventDestroy(pr.first);
            cudaEventDestroy(pr.second);
        }
    for (cudaEvent_t ev : e->tev_pool) cudaEventDestroy(ev);
    if (e->ev_fft) cudaEventDestroy(e->ev_fft);
    if (e->ev_copy) cudaEventDestroy(e->ev_copy);
    if (e->ev_stage) cudaEventDestroy(e->ev_stage);
    stream_release(e->device, e->copy_stream);
    if (e->ev_isf_ready) cudaEventDestroy(e->ev_isf_ready);
    if (e->ev_isf_read) cudaEventDestroy(e->ev_isf_read);
    stream_release(e->device, e->result_stream);
    stream_release(e->device, e->upload_stream);
    for (cudaEvent_t ev : e->ev_guard)
        if (ev) cudaEventDestroy(ev);
    stream_release(e->device, e->fft_stream);
    if (e->own_stream) stream_release(e->device, e->stream);
}

// Brackets a group of launches with events when timing is on (group 0 FFT, 1 lag, 2 azimuth).
// A timing event from the engine's pool (created when the pool is empty; nullptr on failure).
inline cudaEvent_t timing_event(ddm_engine *e) {
    if (!e->tev_pool.empty()) {
        cudaEvent_t ev = e->tev_pool.back();
        e->tev_pool.pop_back();
        return ev;
    }
    cudaEvent_t ev = nullptr;
    return cudaEventCreate(&ev) == cudaSuccess ? ev : nullptr;
}

struct TimedRange {
    ddm_engine *e;
    int group;
    cudaStream_t stream;
    cudaEvent_t start = nullptr;
    TimedRange(ddm_engine *e_, int g) : e(e_), group(g), stream(g == 0 ? e_->fft_stream : e_->stream) {
        if (e->timing && (start = timing_event(e))) cudaEventRecord(start, stream);
    }
    ~TimedRange() {  // a range left on an error path gives its event back
        if (start) e->tev_pool.push_back(start);
    }
    TimedRange(const TimedRange &) = delete;
    TimedRange &operator=(const TimedRange &) = delete;
    void end(long launches) {
        e->tlaunch[group] += launches;
        if (!start) return;
        if (cudaEvent_t stop = timing_event(e)) {
            cudaEventRecord(stop, stream);
            e->tev[group].push_back({start, stop});
        } else {
            e->tev_pool.push_back(start);
        }
        start = nullptr;
    }
};

// ---------------------------------------------------------------------------------
// FFT of a piece of frames into ring slots (first_label + f) % R
// ---------------------------------------------------------------------------------

// `before_group(f0, nf)` runs before each group's kernels are queued (the host path queues the
// group's copies there).
int launch_fft(ddm_engine *e, const uint8_t *src, long long frame_stride, long long row_pitch,
               int x_off, int y_off, int nframes, long long first_label,
               const std::function<int(int, int)> &before_group = nullptr) {
    TimedRange tr(e, 0);
    FftArgs rows, cols;
    std::memset(&rows, 0, sizeof(rows));
    rows.S = e->S;
    rows.src = src;
    rows.frame_stride = frame_stride;
    rows.row_pitch = row_pitch;
    rows.bpp = e->bpp;
    rows.pixmode = e->pixmode;
    rows.x_off = x_off;
    rows.y_off = y_off;
    rows.vec4 = (e->bpp == 1 && x_off % 4 == 0 && row_pitch % 4 == 0 && frame_stride % 4 == 0 &&
                 reinterpret_cast<uintptr_t>(src) % 4 == 0)
                    ? 1
                    : 0;
    rows.ring = e->ring;
    rows.E = e->E;
    rows.R = e->R;
    rows.tw = e->tw;
    cols = rows;
    std::vector<FftScale> tile_scales;  // scales of side 32..128 through the per-tile kernel
    int row_ctas = 0, col_ctas = 0, nfft = 0;
    size_t smem = 0;
    std::vector<FftScale> dft_scales;  // scales for the tensor-core DFT
    for (int si = 0; si < e->S; si++) {
        const ScaleDesc &d = e->sd[si];
        const int s = d.s, per = fft_per_cta(s), side = e->M / s;
        FftScale fs;
        fs.s = s;
        fs.log2s = log2i(s);
        fs.tiles_side = side;
        fs.log2side = log2i(side);
        fs.n = d.n;
        fs.off = d.off;
        if (e->small_dft && fs.log2s >= kDftMinLog2 && fs.log2s <= kDftMaxLog2) {
            dft_scales.push_back(fs);
            continue;
        }
        if (e->fft_per_tile && fs.log2s >= 5 && fs.log2s <= 7) {
            fs.cta_begin = 0;
            fs.ctas_per_frame = (d.tiles + kFftTileTiles(s) - 1) / kFftTileTiles(s);
            tile_scales.push_back(fs);
            continue;
        }
        fs.cta_begin = row_ctas;
        fs.ctas_per_frame = static_cast<int>((static_cast<long long>(d.tiles) * (s / 2) + per - 1) / per);
        rows.sc[nfft] = fs;
        row_ctas += fs.ctas_per_frame;
        fs.cta_begin = col_ctas;
        fs.ctas_per_frame = static_cast<int>((static_cast<long long>(d.tiles) * (s / 2 + 1) + per - 1) / per);
        cols.sc[nfft] = fs;
        col_ctas += fs.ctas_per_frame;
        nfft++;
        smem = std::max(smem, fft_smem_bytes(s));
    }
    rows.S = cols.S = nfft;
    // Frames go through both passes in groups of up to 256 MB of spectra (15 frames of the
    // 1024^2 x 4-scale shape): fewer, larger launches were measured faster than groups small
    // enough for the row pass's output to stay in L2 (frames/s at 34 / 64 / 100 / 256 MB:
    // 0.98 / 1 / 1.015 / 1.025), and two or more groups per piece keep the host copies of a
    // group overlapping the FFT of the one before (one group per piece: -6 % end to end).
    const long long frame_bytes = e->E * static_cast<long long>(sizeof(float2));
    const int group = e->fft_group > 0 ? std::min(e->fft_group, nframes)
                                       : static_cast<int>(std::max<long long>(
                                             1, std::min<long long>(nframes, (256LL << 20) / frame_bytes)));
    for (int f0 = 0; f0 < nframes; f0 += group) {
        const int nf = std::min(group, nframes - f0);
        if (before_group) {
            int st = before_group(f0, nf);
            if (st) return st;
        }
        rows.src = src + f0 * frame_stride;
        rows.first_label = cols.first_label = first_label + f0;
        for (const FftScale &fs : tile_scales) {
            FftArgs t = rows;
            t.S = 1;
            t.sc[0] = fs;
            const dim3 grid(fs.ctas_per_frame, nf);
            const size_t ts = fft_tile_smem_bytes(fs.s);
            switch (fs.log2s) {
                case 5: fft_tile_kernel<5><<<grid, kFftThreads, ts, e->fft_stream>>>(t); break;
                case 6: fft_tile_kernel<6><<<grid, kFftThreads, ts, e->fft_stream>>>(t); break;
                default: fft_tile_kernel<7><<<grid, kFftThreads, ts, e->fft_stream>>>(t); break;
            }
            CUDA_TRY(cudaGetLastError());
            e->launches += 1;
            tr.e->tlaunch[0] += 1;
        }
        if (nfft > 0) {
            fft_rows_kernel<<<dim3(row_ctas, nf), kFftThreads, smem, e->fft_stream>>>(rows);
            CUDA_TRY(cudaGetLastError());
            fft_cols_kernel<<<dim3(col_ctas, nf), kFftThreads, smem, e->fft_stream>>>(cols);
            CUDA_TRY(cudaGetLastError());
            e->launches += 2;
            tr.e->tlaunch[0] += 2;
        }
        for (const FftScale &fs : dft_scales) {
            DftArgs d;
            d.src = rows.src;
            d.frame_stride = frame_stride;
            d.row_pitch = row_pitch;
            d.bpp = e->bpp;
            d.pixmode = e->pixmode;
            d.x_off = x_off;
            d.y_off = y_off;
            d.ring = e->ring;
            d.E = e->E;
            d.first_label = first_label + f0;
            d.R = e->R;
            d.nframes = nf;
            d.sc = fs;
            d.tables = e->dft_tab[fs.log2s - kDftMinLog2];
            d.status = e->status_d;
            d.vec16 = (e->bpp == 1 && x_off % 16 == 0 && row_pitch % 16 == 0 && frame_stride % 16 == 0 &&
                       reinterpret_cast<uintptr_t>(rows.src) % 16 == 0)
                          ? 1
                          : 0;
            const long long tiles = 1LL << (2 * fs.log2side), tpb = 128 / fs.s;
            const long long items = (tiles + tpb - 1) / tpb * nf;
            const unsigned grid = static_cast<unsigned>(std::min<long long>(items, e->sms));
            switch (fs.log2s) {
                case 5: dft_bf16_kernel<5><<<grid, kDftThreads, dft_smem_bytes(32), e->fft_stream>>>(d); break;
                case 6: dft_bf16_kernel<6><<<grid, kDftThreads, dft_smem_bytes(64), e->fft_stream>>>(d); break;
                default: dft_bf16_kernel<7><<<grid, kDftThreads, dft_smem_bytes(128), e->fft_stream>>>(d); break;
            }
            CUDA_TRY(cudaGetLastError());
            e->launches += 1;
            tr.e->tlaunch[0] += 1;
        }
        // the ROI's pixels read once and the frame's spectra written once
        e->tbytes[0] += static_cast<double>(nf) *
                        (static_cast<double>(e->M) * e->M * e->bpp + static_cast<double>(frame_bytes));
    }
    tr.end(0);
    return DDM_OK;
}

// ---------------------------------------------------------------------------------
// Lag launches
// ---------------------------------------------------------------------------------

// CTAs of `kernel` that fit on one SM with `smem` bytes of dynamic shared memory each (the
// register and shared-memory budgets of the instance), cached per engine.
template <class K>
int lag_resident_ctas(ddm_engine *e, int key, size_t smem, K kernel, int threads) {
    for (const auto &r : e->lag_resident)
        if (std::get<0>(r) == key && std::get<1>(r) == smem) return std::get<2>(r);
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess || n < 1) n = 1;
    if (e->lag_resident.size() > 64) e->lag_resident.clear();
    e->lag_resident.emplace_back(key, smem, n);
    return n;
}

int launch_lag(ddm_engine *e, const Launch &L) {
    if (L.nreg <= 0 || L.ent_acc.empty()) return DDM_OK;
    const int J = lag_pick_j(L.nreg);
    if (J == 0) return fail(DDM_ERR_STATE, "internal: no lag kernel for this frame count");
    std::vector<int> table;
    std::string err = build_lag_table(L.nreg, L.reg, L.ent_acc, L.ent_w, L.pos, J, &table);
    if (!err.empty()) return fail(DDM_ERR_STATE, "internal: " + err);
    const int ntab = static_cast<int>(table.size());
    if (ntab > e->tab_stride) return fail(DDM_ERR_STATE, "internal: lag table overflow");
    if (e->inject == DDM_FAULT_LAG_WAIT) {
        // Test of the error path: the last entry's window is moved to start at the end of
        // the partner list, so it reaches groups the producer never issues and the
        // consumers' waits run out. Every entry becomes a single full window (no fused
        // runs, no per-slot checks), so every shared-memory offset stays masked to the ring
        // and the kernel reads nothing outside its table.
        int *ent_ub = table.data() + kTabEntries + L.ent_acc.size();
        int *ent_full = ent_ub + L.ent_acc.size();
        for (size_t i = 0; i < L.ent_acc.size(); i++) ent_full[i] = kLagFullFlag;
        ent_ub[L.ent_acc.size() - 1] = table[kTabNgroups] * kLagGroup;
        e->inject = DDM_FAULT_NONE;
    }
    const int ts = e->tab_next;
    e->tab_next = (e->tab_next + 1) % kTables;
    if (e->tab_used[ts]) CUDA_TRY(cudaEventSynchronize(e->tab_ev[ts]));
    int *th = e->tables_h + static_cast<size_t>(ts) * e->tab_stride;
    std::copy(table.begin(), table.end(), th);
    int *td = e->tables_d + static_cast<size_t>(ts) * e->tab_stride;
    if (e->defer_lag) {  // a server launches the lag work on the engine's stream later: upload in its order
        CUDA_TRY(cudaMemcpyAsync(td, th, sizeof(int) * ntab, cudaMemcpyHostToDevice, e->stream));
        CUDA_TRY(cudaEventRecord(e->tab_ev[ts], e->stream));
    } else {  // ahead of the stream, once the launch that last read the device slot is done
        CUDA_TRY(cudaStreamWaitEvent(e->upload_stream, e->tab_free[ts], 0));
        CUDA_TRY(cudaMemcpyAsync(td, th, sizeof(int) * ntab, cudaMemcpyHostToDevice, e->upload_stream));
        CUDA_TRY(cudaEventRecord(e->tab_ev[ts], e->upload_stream));
        CUDA_TRY(cudaStreamWaitEvent(e->stream, e->tab_ev[ts], 0));
    }
    e->tab_used[ts] = true;

    const int G = J <= 32 ? e->lag_geom : 0;
    const unsigned blocks = static_cast<unsigned>((e->E + lag_cta_elems(J, G) - 1) / lag_cta_elems(J, G));
    const size_t smem = lag_smem_bytes(J, ntab, G);
    if (e->defer_lag) {  // a server issues it with other engines' work in one launch
        e->deferred.push_back(DeferredLag{J, td, blocks, smem});
        return DDM_OK;
    }
    TimedRange tr(e, 1);
    // persistent grid: every resident CTA walks element blocks blockIdx.x, + gridDim.x, ...
    // (as many CTAs as fit on the SMs at once: lag_ctas_per_sm(G) per SM unless a large pair
    // table leaves room for fewer)
    switch (J * kLagGeoms + G) {
#define LAG_CASE(JJ, GG)                                                                                     \
    case JJ * kLagGeoms + GG: {                                                                              \
        const int per_sm = lag_resident_ctas(e, JJ * kLagGeoms + GG, smem, lag_pipe_kernel<JJ, GG>,         \
                                             lag_threads(GG));                                               \
        const unsigned grid = std::min<unsigned>(blocks, static_cast<unsigned>(per_sm * e->sms));          \
        lag_pipe_kernel<JJ, GG><<<grid, lag_threads(GG), smem, e->stream>>>(e->ring, e->acc, e->E, td,      \
                                                                           e->status_d, e->maps,             \
                                                                           static_cast<int>(blocks),         \
                                                                           e->wait_cycles);                  \
        break;                                                                                               \
    }
        LAG_CASE(4, 0) LAG_CASE(8, 0) LAG_CASE(16, 0) LAG_CASE(20, 0) LAG_CASE(24, 0) LAG_CASE(30, 0)
        LAG_CASE(32, 0) LAG_CASE(64, 0)
        LAG_CASE(4, 1) LAG_CASE(8, 1) LAG_CASE(16, 1) LAG_CASE(20, 1) LAG_CASE(24, 1) LAG_CASE(30, 1)
        LAG_CASE(32, 1)
#undef LAG_CASE
        default: return fail(DDM_ERR_STATE, "internal: no lag kernel for this frame count");
    }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(e->tab_free[ts], e->stream));
    tr.end(1);
    e->launches++;
    {
        // every register frame and every distinct partner frame of the launch read once, every
        // accumulator row read and written once
        int frames = 0;
        for (int j = 0; j < L.nreg; j++) frames += L.reg[j] >= 0;
        const int *uslot = table.data() + kTabEntries + 3 * table[kTabNtau];
        for (int u = 0; u < table[kTabNunion]; u++) frames += uslot[u] >= 0;
        e->tbytes[1] += 8.0 * static_cast<double>(e->E) * (frames + 2.0 * table[kTabNtau]);
    }
    return DDM_OK;
}

// Device status word set by kernels whose bounded waits ran out.
int check_device_status(ddm_engine *e) {
    int st = 0;
    CUDA_TRY(cudaMemcpyAsync(&st, e->status_d, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    if (st != 0)
        return fail(DDM_ERR_CUDA, std::string(device_status_text(st)) + " (device status " + std::to_string(st) +
                                      "); results are incomplete");
    return DDM_OK;
}

inline int slot_of(const ddm_engine *e, long long label) {
    return label < 0 ? -1 : static_cast<int>(label % e->R);
}

// Unbiased: the new frames n0 .. n0+c-1 pair with the frames tau before each.
int lag_causal(ddm_engine *e, long long n0, int c) {
    Launch L;
    L.nreg = c;
    for (int j = 0; j < c; j++) L.reg[j] = slot_of(e, n0 + j);
    for (int i = e->T - 1; i >= 0; i--) {  // descending tau = ascending window start
        L.ent_acc.push_back(i);
        L.ent_w.push_back(e->tau_max - e->taus[i]);
        long long first = n0 - e->taus[i];  // partner of j = 0
        long long valid = std::max<long long>(0, std::min<long long>(c, first + c));
        e->pair_count[i] += static_cast<double>(valid);
    }
    L.pos.resize(c + e->tau_max);
    for (int p = 0; p < c + e->tau_max; p++) {
        long long f = n0 - e->tau_max + p;
        L.pos[p] = f >= 0 ? slot_of(e, f) : -1;
    }
    return launch_lag(e, L);
}

// Unbiased: pair every frame still waiting for a lag launch (compat runs the reference's
// iterations as their frames arrive and holds nothing back).
int flush_lag(ddm_engine *e) {
    if (e->estimator != DDM_EST_UNBIASED) return DDM_OK;
    while (e->lag_next < e->submitted) {
        const int c = static_cast<int>(std::min<long long>(e->lag_batch, e->submitted - e->lag_next));
        int st = lag_causal(e, e->lag_next, c);
        if (st) return st;
        e->lag_next += c;
    }
    return DDM_OK;
}

// Reference schedule: iteration `it` pairs A = start[fo] with position fo + tau of
// start|end (src/DDM.cu:250-255).
int lag_iteration(ddm_engine *e, const CompatIteration &it) {
    for (int f0 = 0; f0 < it.count; f0 += e->lag_batch) {
        Launch L;
        L.nreg = std::min(e->lag_batch, it.count - f0);
        for (int j = 0; j < L.nreg; j++) L.reg[j] = slot_of(e, it.start[f0 + j]);
        for (int i = 0; i < e->T; i++) {
            L.ent_acc.push_back(i);
            L.ent_w.push_back(e->taus[i]);
        }
        L.pos.resize(L.nreg + e->tau_max);
        for (int p = 0; p < L.nreg + e->tau_max; p++) {
            const int q = f0 + p;
            int lab = q < e->C ? it.start[q] : (q - e->C < e->C ? it.end[q - e->C] : kLabelUninit);
            L.pos[p] = slot_of(e, lab);
        }
        int st = launch_lag(e, L);
        if (st) return st;
    }
    return DDM_OK;
}

int run_azimuth(ddm_engine *e, const std::vector<double> &norm) {
    CUDA_TRY(cudaStreamWaitEvent(e->stream, e->ev_isf_read, 0));  // a result copy may still read isf_d
    // the upload reads its pinned half asynchronously: refill a half only once its previous
    // upload (two finalizes ago) has run; the upload into the device half waits for the
    // azimuthal average that last read it
    const int ns = e->norm_slot;
    e->norm_slot ^= 1;
    double *nh = e->norm_h + static_cast<size_t>(ns) * e->T;
    double *nd = e->norm_d + static_cast<size_t>(ns) * e->T;
    CUDA_TRY(cudaEventSynchronize(e->norm_ev[ns]));
    std::copy(norm.begin(), norm.end(), nh);
    CUDA_TRY(cudaStreamWaitEvent(e->upload_stream, e->norm_free[ns], 0));
    CUDA_TRY(cudaMemcpyAsync(nd, nh, sizeof(double) * e->T, cudaMemcpyHostToDevice, e->upload_stream));
    CUDA_TRY(cudaEventRecord(e->norm_ev[ns], e->upload_stream));
    CUDA_TRY(cudaStreamWaitEvent(e->stream, e->norm_ev[ns], 0));
    e->host_norm = norm;
    AzArgs a;
    std::memset(&a, 0, sizeof(a));
    a.S = e->S;
    a.T = e->T;
    a.Q = e->Q;
    for (int s = 0; s < e->S; s++) a.sc[s] = e->sd[s];
    a.acc = e->acc;
    a.E = e->E;
    a.idx = e->idx_d;
    a.chunk_beg = e->chunk_beg_d;
    a.chunk_end = e->chunk_end_d;
    a.chunk_first = e->chunk_first_d;
    a.chunk_count = e->chunk_count_d;
    a.counts = e->counts_d;
    a.norm = nd;
    a.partial = e->partial_d;
    a.isf = e->isf_d;
    a.items = e->az_items;
    a.bins = e->isf_size;
    TimedRange tr(e, 2);
    if (a.items > 0) {
        azimuth_partial_kernel<<<static_cast<unsigned>((a.items + kAzWarps - 1) / kAzWarps), kAzThreads, 0,
                                 e->stream>>>(a);
        CUDA_TRY(cudaGetLastError());
    }
    azimuth_final_kernel<<<static_cast<unsigned>((a.bins + kAzThreads - 1) / kAzThreads), kAzThreads, 0, e->stream>>>(a);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(e->norm_free[ns], e->stream));
    tr.end(a.items > 0 ? 2 : 1);
    e->tbytes[2] += e->az_bytes;
    e->launches += a.items > 0 ? 2 : 1;
    return DDM_OK;
}

int purge(ddm_engine *e) {
    CUDA_TRY(cudaMemsetAsync(e->acc, 0, sizeof(float2) * e->T * e->E, e->stream));
    std::fill(e->pair_count.begin(), e->pair_count.end(), 0.0);
    return DDM_OK;
}

int snapshot(ddm_engine *e, const std::vector<double> &norm) {
    int st = run_azimuth(e, norm);
    if (st) return st;
    std::vector<double> out(e->isf_size);
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    CUDA_TRY(cudaMemcpy(out.data(), e->isf_d, sizeof(double) * e->isf_size, cudaMemcpyDeviceToHost));
    e->dumps.push_back(std::move(out));
    return purge(e);
}

// Compat: run every pending iteration whose frames have all been submitted.
int run_ready_iterations(ddm_engine *e, bool final_pass) {
    while (e->next_it < e->its.size()) {
        const CompatIteration &it = e->its[e->next_it];
        if (it.max_label >= e->submitted) {
            if (!final_pass) break;
            return fail(DDM_ERR_NEED_FRAMES, "the reference schedule reads frame " +
                                                 std::to_string(it.max_label) + " but only " +
                                                 std::to_string(e->submitted) + " were submitted");
        }
        if (it.min_label < e->submitted - e->R)
            return fail(DDM_ERR_STATE, "internal: ring too small for the reference schedule");
        int st = lag_iteration(e, it);
        if (st) return st;
        e->next_it++;
        if (it.dump_after) {
            std::vector<double> norm(e->T, static_cast<double>(e->C) * e->G);  // src/DDM.cu:808
            st = snapshot(e, norm);
            if (st) return st;
        }
    }
    return DDM_OK;
}

}  // namespace

// =================================================================================
// C ABI
// =================================================================================

namespace {

// ddm_open; with plan_only it stops after the validation and sizing and reports the device
// bytes the engine's main buffers would take (the figure checked against the HBM budget).
int open_engine(const ddm_config *cfg, ddm_engine **out, size_t *need_out, bool plan_only) {
    if (!cfg || !out) return fail(DDM_ERR_INVALID_ARG, "ddm_open: null argument");
    *out = nullptr;
    if (!cfg->scales || !cfg->taus || !cfg->lambdas || cfg->scale_count <= 0 || cfg->tau_count <= 0 ||
        cfg->lambda_count <= 0)
        return fail(DDM_ERR_INVALID_ARG, "scale, tau and lambda lists must each hold at least one value");
    if (cfg->scale_count > kMaxScales)
        return fail(DDM_ERR_INVALID_ARG, "at most " + std::to_string(kMaxScales) + " scales");
    if (cfg->bytes_per_pixel != 1 && cfg->bytes_per_pixel != 2)
        return fail(DDM_ERR_INVALID_ARG, "bytes_per_pixel must be 1 or 2");
    if (cfg->pixel_mode == DDM_PIX_U16LE && cfg->bytes_per_pixel != 2)
        return fail(DDM_ERR_INVALID_ARG, "DDM_PIX_U16LE needs bytes_per_pixel = 2");
    if (cfg->pixel_mode != DDM_PIX_BYTE0 && cfg->pixel_mode != DDM_PIX_U16LE)
        return fail(DDM_ERR_INVALID_ARG, "unknown pixel_mode");
    if (cfg->estimator != DDM_EST_COMPAT && cfg->estimator != DDM_EST_UNBIASED)
        return fail(DDM_ERR_INVALID_ARG, "unknown estimator");

    ddm_engine *e = new ddm_engine;
    e->w = cfg->frame_width;
    e->h = cfg->frame_height;
    e->bpp = cfg->bytes_per_pixel;
    e->pixmode = cfg->pixel_mode;
    e->x_off = cfg->x_offset;
    e->y_off = cfg->y_offset;
    e->scales.assign(cfg->scales, cfg->scales + cfg->scale_count);
    e->taus.assign(cfg->taus, cfg->taus + cfg->tau_count);
    e->lambdas.assign(cfg->lambdas, cfg->lambdas + cfg->lambda_count);
    std::sort(e->taus.begin(), e->taus.end());  // src/DDM.cu:319-321
    std::sort(e->lambdas.begin(), e->lambdas.end());
    std::sort(e->scales.begin(), e->scales.end(), std::greater<int>());
    e->tol = cfg->tolerance;
    e->C = cfg->chunk_frames;
    e->estimator = cfg->estimator;
    e->multistream = cfg->multistream ? 1 : 0;
    e->N = cfg->total_frames;
    e->G = cfg->dump_every;
    e->lag_geom = cfg->lag_geometry ? 1 : 0;
    if (cfg->fft_group_frames < 0) {
        delete e;
        return fail(DDM_ERR_INVALID_ARG, "fft_group_frames must be >= 0");
    }
    e->fft_group = cfg->fft_group_frames;
    e->fft_per_tile = cfg->fft_per_tile ? 1 : 0;
    e->device = cfg->device;
    const bool compat = e->estimator == DDM_EST_COMPAT;

    auto bail = [&](int st) {
        free_all(e);
        delete e;
        return st;
    };
    std::string msg = validate_reference_params(e->scales, e->taus, e->lambdas, e->tol, e->C,
                                                /*enforce_tau_chunk=*/compat,
                                                /*enforce_lambda_scale=*/compat, nullptr);
    if (!msg.empty()) return bail(fail(DDM_ERR_INVALID_ARG, msg));
    e->M = e->scales[0];
    if (e->M > (1 << kFftMaxLog2))
        return bail(fail(DDM_ERR_INVALID_ARG, "the largest scale must be <= " + std::to_string(1 << kFftMaxLog2)));
    if (e->M + e->x_off > e->w || e->M + e->y_off > e->h || e->x_off < 0 || e->y_off < 0)
        return bail(fail(DDM_ERR_INVALID_ARG, "the specified out dimensions must be smaller than actual image size"));
    if (e->scales.back() < 2) return bail(fail(DDM_ERR_INVALID_ARG, "scales must be at least 2"));
    if (e->G < 0) return bail(fail(DDM_ERR_INVALID_ARG, "dump_every must be >= 0"));
    if (compat && e->N <= 0) return bail(fail(DDM_ERR_INVALID_ARG, "the reference schedule needs total_frames > 0"));
    e->S = static_cast<int>(e->scales.size());
    e->T = static_cast<int>(e->taus.size());
    e->Q = static_cast<int>(e->lambdas.size());
    e->tau_max = e->taus.back();
    if (lag_smem_bytes(kMaxJ, lag_table_capacity(e->T, kMaxJ + e->tau_max)) > static_cast<size_t>(kLagSmemMax))
        return bail(fail(DDM_ERR_INVALID_ARG, "tau list too long for the lag kernel's shared-memory table"));

    // Geometry
    long long off = 0, isf_off = 0;
    int q_base = 0;
    for (int s : e->scales) {
        ScaleDesc d;
        d.s = s;
        d.tiles = (e->M / s) * (e->M / s);
        d.n = static_cast<long long>(s) * (s / 2 + 1);
        d.off = off;
        d.isf_off = isf_off;
        d.q_base = q_base;
        d.inv_s4 = 1.0 / (static_cast<double>(s) * s * static_cast<double>(s) * s);
        off += d.tiles * d.n;
        isf_off += static_cast<long long>(d.tiles) * e->Q * e->T;
        q_base += e->Q;
        e->sd.push_back(d);
    }
    e->E = off;
    e->isf_size = isf_off;

    // Schedule and ring size
    e->jmax = std::min(kPieceFrames, e->C);
    if (cfg->lag_batch_frames < -1 || cfg->lag_batch_frames > kMaxJ)
        return bail(fail(DDM_ERR_INVALID_ARG, "lag_batch_frames must be -1.." + std::to_string(kMaxJ)));
    int lag_batch_cfg = cfg->lag_batch_frames;
    if (lag_batch_cfg == -1) {  // the tuned values for this shape, if a cache names them
        TunedValues tv;
        if (tune_lookup(std::getenv("DDM_TUNE_CACHE"), tune_key(cfg), &tv)) {
            lag_batch_cfg = tv.lag_batch;
            e->lag_geom = tv.lag_geometry;
            e->fft_group = tv.fft_group;
            e->fft_per_tile = tv.fft_per_tile;
        } else {
            lag_batch_cfg = 0;
        }
    }
    // default: unbiased launches of kPieceFrames (32) frames, the instantiated register-frame
    // count the kernel's cost per launch is set by (32 frames take about the time of 30);
    // compat iterations in blocks of one ingest piece
    e->lag_batch = lag_batch_cfg ? lag_batch_cfg : (compat ? e->jmax : kPieceFrames);
    if (compat) {
        e->its = compat_schedule(e->N, e->C, e->multistream, e->G, e->taus, &e->frames_read);
        // Frames arrive in pieces of jmax and iterations run in order, each once every
        // frame it reads is in: iteration j runs when at most run_j + jmax frames have
        // been submitted (run_j = the largest label read by iterations 0..j), so the ring
        // must still hold its oldest label then.
        int span = 1, run = -1;
        for (const CompatIteration &it : e->its) {
            run = std::max(run, it.max_label);
            if (it.max_label >= 0) span = std::max(span, run + e->jmax - it.min_label + 1);
        }
        e->R = span + e->jmax;  // + one piece: the next piece's FFT overlaps the running lag
    } else {
        // A lag launch reads its frames and tau_max frames further back while the next
        // piece's FFT (jmax frames) may already write; with lag_batch > jmax up to
        // lag_batch - 1 more frames wait in the ring for a fuller launch.
        e->R = e->tau_max + 2 * e->jmax + (e->lag_batch > e->jmax ? e->lag_batch - 1 : 0);
        e->pair_count.assign(e->T, 0.0);
    }

    // Budget check before any allocation
    const size_t ring_bytes = sizeof(float2) * static_cast<size_t>(e->R) * e->E;
    const size_t acc_bytes = sizeof(float2) * static_cast<size_t>(e->T) * e->E;
    const size_t stage_bytes = static_cast<size_t>(e->jmax) * e->M * e->M * e->bpp;
    e->tab_stride = lag_table_capacity(e->T, kMaxJ + e->tau_max);
    size_t need = ring_bytes + acc_bytes + stage_bytes + sizeof(double) * e->isf_size +
                  sizeof(int) * static_cast<size_t>(kTables) * e->tab_stride;
    if (need_out) *need_out = need;
    if (plan_only) return bail(DDM_OK);
    if (cfg->hbm_budget_bytes && need > cfg->hbm_budget_bytes)
        return bail(fail(DDM_ERR_OUT_OF_MEMORY, "engine needs " + std::to_string(need) +
                                                    " device bytes, over the budget of " +
                                                    std::to_string(cfg->hbm_budget_bytes)));

    // Device
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= e->device || e->device < 0)
        return bail(fail(DDM_ERR_NO_DEVICE, "no CUDA device " + std::to_string(e->device)));
    // two attribute queries, not cudaGetDeviceProperties: that one was measured to take up to
    // 0.3 s while the device is busy and to hold up other threads' launches meanwhile
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, e->device) != cudaSuccess || major != 10 ||
        cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, e->device) != cudaSuccess)
        return bail(fail(DDM_ERR_NO_DEVICE, "device " + std::to_string(e->device) + " is not an sm_100 GPU"));
    if (cudaSetDevice(e->device) != cudaSuccess) return bail(fail(DDM_ERR_CUDA, "cudaSetDevice failed"));
    if (cfg->stream) {
        e->stream = static_cast<cudaStream_t>(cfg->stream);
    } else {
        if (!(e->stream = stream_acquire(e->device))) return bail(fail(DDM_ERR_CUDA, "cudaStreamCreate failed"));
        e->own_stream = true;
    }
    // private streams from the process-wide pool (creating streams while the device is busy
    // is slow and holds up other threads' launches)
    if (!(e->fft_stream = stream_acquire(e->device)) || !(e->copy_stream = stream_acquire(e->device)) ||
        !(e->result_stream = stream_acquire(e->device)) || !(e->upload_stream = stream_acquire(e->device)) ||
        cudaEventCreateWithFlags(&e->ev_isf_ready, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->ev_isf_read, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->ev_copy, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->ev_stage, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->ev_fft, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->ev_guard[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->ev_guard[1], cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(DDM_ERR_CUDA, "stream/event creation failed"));
    int st;
    if ((st = dev_alloc(e, &e->ring, static_cast<size_t>(e->R) * e->E))) return bail(st);
    {
        std::string err = make_lag_maps(e->ring, e->E, e->R, &e->maps);
        if (!err.empty()) return bail(fail(DDM_ERR_CUDA, err));
    }
    if ((st = dev_alloc(e, &e->acc, static_cast<size_t>(e->T) * e->E))) return bail(st);
    if ((st = dev_alloc(e, &e->stage, stage_bytes))) return bail(st);
    if ((st = dev_alloc(e, &e->tables_d, static_cast<size_t>(kTables) * e->tab_stride))) return bail(st);
    if ((st = dev_alloc(e, &e->norm_d, 2 * e->T))) return bail(st);
    if ((st = dev_alloc(e, &e->isf_d, e->isf_size))) return bail(st);
    if ((st = dev_alloc(e, &e->status_d, 1))) return bail(st);
    if (cudaMemset(e->status_d, 0, sizeof(int)) != cudaSuccess) return bail(fail(DDM_ERR_CUDA, "status memset failed"));
    e->norm_h = static_cast<double *>(pinned_alloc(sizeof(double) * 2 * e->T));
    e->async_status_h = static_cast<int *>(pinned_alloc(sizeof(int) * kAsyncMax));
    if (!e->norm_h || !e->async_status_h) return bail(fail(DDM_ERR_OUT_OF_MEMORY, "pinned norm and status buffers"));
    for (int i = 0; i < 2; i++)
        if (cudaEventCreateWithFlags(&e->norm_ev[i], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&e->norm_free[i], cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(DDM_ERR_CUDA, "cudaEventCreate failed"));
    for (int i = 0; i < kAsyncMax; i++)
        if (cudaEventCreateWithFlags(&e->async_ev[i], cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(DDM_ERR_CUDA, "cudaEventCreate failed"));
    for (int i = 0; i < kSubmitEvents; i++)
        if (cudaEventCreateWithFlags(&e->submit_ev[i], cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(DDM_ERR_CUDA, "cudaEventCreate failed"));
    e->tables_h = static_cast<int *>(pinned_alloc(sizeof(int) * static_cast<size_t>(kTables) * e->tab_stride));
    if (!e->tables_h) return bail(fail(DDM_ERR_OUT_OF_MEMORY, "pinned table buffer"));
    for (int i = 0; i < kTables; i++)
        if (cudaEventCreateWithFlags(&e->tab_ev[i], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&e->tab_free[i], cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(DDM_ERR_CUDA, "cudaEventCreate failed"));

    // FFT twiddle tables (FP64 math rounded to FP32), one per transform length
    {
        e->small_dft = cfg->small_tile_dft != 0;
        if (e->small_dft)
            for (int s : e->scales) {
                const int l = log2i(s);
                if (l < kDftMinLog2 || l > kDftMaxLog2 || e->dft_tab[l - kDftMinLog2]) continue;
                const std::vector<uint16_t> t = dft_tables(s);
                uint4 **dst = &e->dft_tab[l - kDftMinLog2];
                if ((st = dev_alloc(e, dst, t.size() * 2 / sizeof(uint4)))) return bail(st);
                if (cudaMemcpy(*dst, t.data(), t.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess)
                    return bail(fail(DDM_ERR_CUDA, "DFT table upload failed"));
            }
        std::vector<float2> tw = fft_twiddle_tables(e->M);
        if ((st = dev_alloc(e, &e->tw, tw.size()))) return bail(st);
        if (cudaMemcpy(e->tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(fail(DDM_ERR_CUDA, "twiddle upload failed"));
    }

    // Masks (bit-exact host construction) as CSR per (scale, q), cut into chunks of at most
    // kAzChunk indices for the two-stage azimuthal reduction
    {
        std::vector<int> idx_all, cbeg, cend, cfirst, ccount;
        long long items = 0;
        for (int s = 0; s < e->S; s++) {
            std::vector<int> qp, idx, counts;
            build_masks(e->scales[s], e->lambdas, e->tol, &qp, &idx, &counts);
            const int base = static_cast<int>(idx_all.size());
            ScaleDesc &d = e->sd[s];
            d.chunk_off = static_cast<int>(cbeg.size());
            int nloc = 0;
            for (int q = 0; q < e->Q; q++) {
                cfirst.push_back(nloc);
                int n = 0;
                for (int b = qp[q]; b < qp[q + 1]; b += kAzChunk, n++) {
                    cbeg.push_back(base + b);
                    cend.push_back(base + std::min(b + kAzChunk, qp[q + 1]));
                }
                ccount.push_back(n);
                nloc += n;
            }
            d.nchunks = nloc;
            d.item_base = items;
            items += static_cast<long long>(d.tiles) * e->T * nloc;
            idx_all.insert(idx_all.end(), idx.begin(), idx.end());
            e->counts_h.insert(e->counts_h.end(), counts.begin(), counts.end());
            e->az_bytes += 8.0 * e->T * static_cast<double>(idx.size()) * d.tiles;
            e->q_ptr_s.push_back(qp);
            e->idx_s.push_back(std::move(idx));
        }
        e->az_items = items;
        auto up = [&](int **dst, const std::vector<int> &v) {
            int r = dev_alloc(e, dst, v.size());
            if (r) return r;
            if (!v.empty() && cudaMemcpy(*dst, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess)
                return fail(DDM_ERR_CUDA, "mask upload failed");
            return static_cast<int>(DDM_OK);
        };
        if ((st = up(&e->idx_d, idx_all)) || (st = up(&e->chunk_beg_d, cbeg)) || (st = up(&e->chunk_end_d, cend)) ||
            (st = up(&e->chunk_first_d, cfirst)) || (st = up(&e->chunk_count_d, ccount)) ||
            (st = up(&e->counts_d, e->counts_h)))
            return bail(st);
        if ((st = dev_alloc(e, &e->partial_d, static_cast<size_t>(std::max<long long>(items, 1))))) return bail(st);
    }

    // Kernel shared-memory limits (the FFT passes use up to 128 KB)
    if (cudaFuncSetAttribute(fft_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024) != cudaSuccess ||
        cudaFuncSetAttribute(fft_tile_kernel<5>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(fft_tile_smem_bytes(32))) != cudaSuccess ||
        cudaFuncSetAttribute(fft_tile_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(fft_tile_smem_bytes(64))) != cudaSuccess ||
        cudaFuncSetAttribute(fft_tile_kernel<7>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(fft_tile_smem_bytes(128))) != cudaSuccess ||
        cudaFuncSetAttribute(fft_cols_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<20>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<24>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<30>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<4, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<8, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<16, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<20, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<24, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<30, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(lag_pipe_kernel<32, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kLagSmemMax) != cudaSuccess ||
        cudaFuncSetAttribute(dft_bf16_kernel<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, dft_smem_bytes(32)) != cudaSuccess ||
        cudaFuncSetAttribute(dft_bf16_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, dft_smem_bytes(64)) != cudaSuccess ||
        cudaFuncSetAttribute(dft_bf16_kernel<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, dft_smem_bytes(128)) != cudaSuccess)
        return bail(fail(DDM_ERR_CUDA, "cudaFuncSetAttribute failed"));

    // Zero the accumulators on the engine's private FFT stream, ahead of its first FFT: every
    // lag launch waits for an FFT of that stream, so nothing else has to wait here (a
    // server's shared stream stays free while a new stream is set up). The unbiased
    // estimator never reads a ring slot before its frame is written, so only compat mode
    // (whose reference schedule can name frames it never wrote) clears the ring.
    if (cudaMemsetAsync(e->acc, 0, acc_bytes, e->fft_stream) != cudaSuccess ||
        (compat && cudaMemsetAsync(e->ring, 0, ring_bytes, e->fft_stream) != cudaSuccess) ||
        (e->own_stream && cudaStreamSynchronize(e->fft_stream) != cudaSuccess))
        return bail(fail(DDM_ERR_CUDA, "initial memset failed"));
    *out = e;
    return DDM_OK;
}

}  // namespace

extern "C" int ddm_open(const ddm_config *cfg, ddm_engine **out) {
    clear_error();
    return open_engine(cfg, out, nullptr, false);
}

namespace ddm {
int engine_plan_bytes(const ddm_config *cfg, size_t *need) {
    ddm_engine *unused = nullptr;
    return open_engine(cfg, &unused, need, true);
}
}  // namespace ddm

extern "C" int ddm_close(ddm_engine *e) {
    if (!e) return DDM_OK;
    if (e->result_stream) cudaStreamSynchronize(e->result_stream);
    if (e->fft_stream) cudaStreamSynchronize(e->fft_stream);
    if (e->stream) cudaStreamSynchronize(e->stream);
    free_all(e);
    delete e;
    return DDM_OK;
}

extern "C" int ddm_submit_frames(ddm_engine *e, const void *frames, int count, int on_device) {
    clear_error();
    if (!e || (!frames && count > 0) || count < 0) return fail(DDM_ERR_INVALID_ARG, "ddm_submit_frames: bad argument");
    const bool compat = e->estimator == DDM_EST_COMPAT;
    if (compat && e->finalized) return fail(DDM_ERR_STATE, "engine already finalized");
    if (compat && e->submitted + count > e->frames_read)
        return fail(DDM_ERR_STATE, "the reference schedule reads only " + std::to_string(e->frames_read) + " frames");
    const size_t frame_bytes = static_cast<size_t>(e->w) * e->h * e->bpp;
    const uint8_t *src = static_cast<const uint8_t *>(frames);
    int done = 0;
    while (done < count) {
        int piece = std::min(count - done, e->jmax);
        if (!compat && e->G > 0) {  // unbiased -G: cut pieces at snapshot boundaries
            const long long period = static_cast<long long>(e->G) * e->C;
            const long long to_edge = period - e->submitted % period;
            piece = static_cast<int>(std::min<long long>(piece, to_edge));
        }
        const uint8_t *p = src + frame_bytes * done;
        int st;
        // hold this piece's FFT until every lag issued before the previous piece's FFT is done
        if (e->pieces > 0) CUDA_TRY(cudaStreamWaitEvent(e->fft_stream, e->ev_guard[(e->pieces - 1) & 1], 0));
        CUDA_TRY(cudaEventRecord(e->ev_guard[e->pieces & 1], e->stream));
        e->pieces++;
        if (on_device) {
            st = launch_fft(e, p, static_cast<long long>(frame_bytes), static_cast<long long>(e->w) * e->bpp,
                            e->x_off, e->y_off, piece, e->submitted);
        } else {
            const size_t roi_row = static_cast<size_t>(e->M) * e->bpp;
            if (e->stage_busy) CUDA_TRY(cudaStreamWaitEvent(e->copy_stream, e->ev_stage, 0));
            auto copy_group = [&](int f0, int nf) -> int {
                if (e->M == e->h) {
                    // the ROI spans the frame's height: the rows of consecutive frames are
                    // evenly strided in the packed buffer, so the group is one 2-D copy
                    const uint8_t *fp = p + frame_bytes * f0 + static_cast<size_t>(e->x_off) * e->bpp;
                    CUDA_TRY(cudaMemcpy2DAsync(e->stage + static_cast<size_t>(f0) * e->M * roi_row, roi_row, fp,
                                               static_cast<size_t>(e->w) * e->bpp, roi_row,
                                               static_cast<size_t>(e->M) * nf, cudaMemcpyHostToDevice,
                                               e->copy_stream));
                    CUDA_TRY(cudaEventRecord(e->ev_copy, e->copy_stream));
                    CUDA_TRY(cudaStreamWaitEvent(e->fft_stream, e->ev_copy, 0));
                    return DDM_OK;
                }
                for (int f = f0; f < f0 + nf; f++) {
                    const uint8_t *fp = p + frame_bytes * f +
                                        (static_cast<size_t>(e->y_off) * e->w + e->x_off) * e->bpp;
                    CUDA_TRY(cudaMemcpy2DAsync(e->stage + static_cast<size_t>(f) * e->M * roi_row, roi_row, fp,
                                               static_cast<size_t>(e->w) * e->bpp, roi_row, e->M,
                                               cudaMemcpyHostToDevice, e->copy_stream));
                }
                CUDA_TRY(cudaEventRecord(e->ev_copy, e->copy_stream));
                CUDA_TRY(cudaStreamWaitEvent(e->fft_stream, e->ev_copy, 0));
                return DDM_OK;
            };
            st = launch_fft(e, e->stage, static_cast<long long>(e->M) * roi_row, static_cast<long long>(roi_row),
                            0, 0, piece, e->submitted, copy_group);
            if (!st) {
                CUDA_TRY(cudaEventRecord(e->ev_stage, e->fft_stream));
                e->stage_busy = true;
            }
        }
        if (st) return st;
        CUDA_TRY(cudaEventRecord(e->ev_fft, e->fft_stream));
        CUDA_TRY(cudaStreamWaitEvent(e->stream, e->ev_fft, 0));  // lags below read this piece
        e->submitted += piece;
        if (compat) {
            if ((st = run_ready_iterations(e, false))) return st;
        } else {
            while (e->submitted - e->lag_next >= e->lag_batch) {
                if ((st = lag_causal(e, e->lag_next, e->lag_batch))) return st;
                e->lag_next += e->lag_batch;
            }
            if (e->lag_batch <= e->jmax && (st = flush_lag(e))) return st;  // no batching
            if (e->G > 0 && e->submitted % (static_cast<long long>(e->G) * e->C) == 0) {
                if ((st = flush_lag(e))) return st;
                if ((st = snapshot(e, e->pair_count))) return st;
            }
        }
        done += piece;
    }
    // every copy of this call's host frames is queued on the copy stream by now
    CUDA_TRY(cudaEventRecord(e->submit_ev[e->submit_calls % kSubmitEvents], e->copy_stream));
    e->submit_calls++;
    return DDM_OK;
}

extern "C" int ddm_wait_frames_copied(ddm_engine *e, int back) {
    clear_error();
    if (!e || back < 0 || back >= kSubmitEvents)
        return fail(DDM_ERR_INVALID_ARG, "ddm_wait_frames_copied: back must be 0.." + std::to_string(kSubmitEvents - 1));
    if (back >= e->submit_calls) return DDM_OK;  // no such call
    CUDA_TRY(cudaEventSynchronize(e->submit_ev[(e->submit_calls - 1 - back) % kSubmitEvents]));
    return DDM_OK;
}

namespace ddm {

int engine_finalize_async(ddm_engine *e) {
    int st;
    std::vector<double> norm(e->T);
    if (e->estimator == DDM_EST_COMPAT) {
        if (e->finalized) return fail(DDM_ERR_STATE, "engine already finalized");
        if ((st = run_ready_iterations(e, true))) return st;
        std::fill(norm.begin(), norm.end(), static_cast<double>(e->N));  // src/DDM.cu:875
    } else {
        if ((st = flush_lag(e))) return st;
        norm = e->pair_count;
    }
    if ((st = run_azimuth(e, norm))) return st;
    e->finalized = true;
    return DDM_OK;
}

void engine_defer_lag(ddm_engine *e, bool on) { e->defer_lag = on; }

void engine_close_async(ddm_engine *e) {
    if (!e) return;
    free_all(e);
    delete e;
}

std::vector<DeferredLag> engine_take_deferred(ddm_engine *e) {
    std::vector<DeferredLag> out;
    out.swap(e->deferred);
    return out;
}

LagTarget engine_lag_target(const ddm_engine *e) { return LagTarget{e->ring, e->acc, e->E, e->status_d, &e->maps}; }

cudaStream_t engine_stream(const ddm_engine *e) { return e->stream; }
const double *engine_isf_device(const ddm_engine *e) { return e->isf_d; }
const int *engine_status_device(const ddm_engine *e) { return e->status_d; }

}  // namespace ddm

extern "C" int ddm_finalize(ddm_engine *e) {
    clear_error();
    if (!e) return fail(DDM_ERR_INVALID_ARG, "ddm_finalize: null engine");
    int st = engine_finalize_async(e);
    if (st) return st;
    return check_device_status(e);
}

extern "C" long ddm_isf_size(const ddm_engine *e) { return e ? static_cast<long>(e->isf_size) : 0; }

// Waits for the ddm_finalize_async result in `slot` and checks the device status word
// copied with it (the status of every kernel queued before that result).
static int wait_async_slot(ddm_engine *e, int slot) {
    if (!e->async_pending[slot]) return DDM_OK;
    e->async_pending[slot] = false;
    CUDA_TRY(cudaEventSynchronize(e->async_ev[slot]));
    if (e->async_status_h[slot] != 0)
        return fail(DDM_ERR_CUDA, std::string(device_status_text(e->async_status_h[slot])) + " (device status " +
                                      std::to_string(e->async_status_h[slot]) + "); results are incomplete");
    return DDM_OK;
}

extern "C" int ddm_finalize_async(ddm_engine *e, double *out, long capacity) {
    clear_error();
    if (!e || !out || capacity < e->isf_size) return fail(DDM_ERR_INVALID_ARG, "ddm_finalize_async: bad argument");
    const int slot = e->async_slot;
    int st = wait_async_slot(e, slot);  // async_depth results ago: already waited for by the call after it
    if (st) return st;
    // queue this result first, so the stream never idles while the host waits below
    if ((st = engine_finalize_async(e))) return st;
    CUDA_TRY(cudaEventRecord(e->ev_isf_ready, e->stream));
    CUDA_TRY(cudaStreamWaitEvent(e->result_stream, e->ev_isf_ready, 0));
    CUDA_TRY(cudaMemcpyAsync(out, e->isf_d, sizeof(double) * e->isf_size, cudaMemcpyDeviceToHost, e->result_stream));
    CUDA_TRY(cudaMemcpyAsync(e->async_status_h + slot, e->status_d, sizeof(int), cudaMemcpyDeviceToHost,
                             e->result_stream));
    CUDA_TRY(cudaEventRecord(e->async_ev[slot], e->result_stream));
    CUDA_TRY(cudaEventRecord(e->ev_isf_read, e->result_stream));
    e->async_pending[slot] = true;
    e->async_slot = (slot + 1) % e->async_depth;
    // the result of async_depth - 1 calls ago (the previous one at the default depth of 2):
    // its buffer is the caller's again
    return wait_async_slot(e, e->async_slot);
}

extern "C" int ddm_set_async_depth(ddm_engine *e, int depth) {
    clear_error();
    if (!e || depth < 2 || depth > kAsyncMax)
        return fail(DDM_ERR_INVALID_ARG, "ddm_set_async_depth: depth must be 2.." + std::to_string(kAsyncMax));
    for (int i = 0; i < kAsyncMax; i++)
        if (e->async_pending[i]) return fail(DDM_ERR_STATE, "ddm_set_async_depth: results still in flight (ddm_wait_isf)");
    e->async_depth = depth;
    e->async_slot = 0;
    return DDM_OK;
}

extern "C" int ddm_wait_isf(ddm_engine *e) {
    clear_error();
    if (!e) return fail(DDM_ERR_INVALID_ARG, "ddm_wait_isf: null engine");
    // oldest first: the slot of the next result holds the oldest one in flight, if any
    int st = DDM_OK;
    for (int i = 0; i < e->async_depth; i++) {
        const int s2 = wait_async_slot(e, (e->async_slot + i) % e->async_depth);
        if (!st) st = s2;
    }
    return st;
}

extern "C" int ddm_read_isf(ddm_engine *e, double *out, long capacity) {
    clear_error();
    if (!e || !out || capacity < e->isf_size) return fail(DDM_ERR_INVALID_ARG, "ddm_read_isf: bad argument");
    if (!e->finalized) return fail(DDM_ERR_STATE, "ddm_finalize has not run");
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    CUDA_TRY(cudaMemcpy(out, e->isf_d, sizeof(double) * e->isf_size, cudaMemcpyDeviceToHost));
    return DDM_OK;
}

extern "C" int ddm_dump_count(const ddm_engine *e) { return e ? static_cast<int>(e->dumps.size()) : 0; }

extern "C" int ddm_read_dump(ddm_engine *e, int index, double *out, long capacity) {
    clear_error();
    if (!e || !out || index < 0 || index >= static_cast<int>(e->dumps.size()) || capacity < e->isf_size)
        return fail(DDM_ERR_INVALID_ARG, "ddm_read_dump: bad argument");
    std::copy(e->dumps[index].begin(), e->dumps[index].end(), out);
    return DDM_OK;
}

extern "C" int ddm_reset_accumulators(ddm_engine *e) {
    clear_error();
    if (!e) return fail(DDM_ERR_INVALID_ARG, "null engine");
    int st = flush_lag(e);  // frames submitted before the reset belong to the discarded sums
    if (st) return st;
    return purge(e);
}

extern "C" int ddm_synchronize(ddm_engine *e) {
    clear_error();
    if (!e) return fail(DDM_ERR_INVALID_ARG, "null engine");
    int st = flush_lag(e);
    if (st) return st;
    CUDA_TRY(cudaStreamSynchronize(e->copy_stream));
    CUDA_TRY(cudaStreamSynchronize(e->fft_stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->result_stream));
    CUDA_TRY(cudaGetLastError());
    return check_device_status(e);
}

extern "C" int ddm_get_params(const ddm_engine *e, int *scales, int *taus, float *lambdas) {
    if (!e) return fail(DDM_ERR_INVALID_ARG, "null engine");
    if (scales) std::copy(e->scales.begin(), e->scales.end(), scales);
    if (taus) std::copy(e->taus.begin(), e->taus.end(), taus);
    if (lambdas) std::copy(e->lambdas.begin(), e->lambdas.end(), lambdas);
    return DDM_OK;
}

extern "C" int ddm_get_pixel_counts(const ddm_engine *e, int *counts) {
    if (!e || !counts) return fail(DDM_ERR_INVALID_ARG, "bad argument");
    std::copy(e->counts_h.begin(), e->counts_h.end(), counts);
    return DDM_OK;
}

extern "C" int ddm_get_mask(const ddm_engine *e, int si, unsigned char *mask, long capacity) {
    if (!e || !mask || si < 0 || si >= e->S) return fail(DDM_ERR_INVALID_ARG, "bad argument");
    const long long n = e->sd[si].n;
    if (capacity < n * e->Q) return fail(DDM_ERR_INVALID_ARG, "mask buffer too small");
    std::memset(mask, 0, static_cast<size_t>(n * e->Q));
    for (int q = 0; q < e->Q; q++)
        for (int i = e->q_ptr_s[si][q]; i < e->q_ptr_s[si][q + 1]; i++) mask[q * n + e->idx_s[si][i]] = 1;
    return DDM_OK;
}

extern "C" long ddm_frame_elements(const ddm_engine *e) { return e ? static_cast<long>(e->E) : 0; }

extern "C" int ddm_read_spectrum(ddm_engine *e, int frame, float *out, long capacity) {
    clear_error();
    if (!e || !out || capacity < 2 * e->E) return fail(DDM_ERR_INVALID_ARG, "bad argument");
    if (frame < 0 || frame >= e->submitted || frame < e->submitted - e->R)
        return fail(DDM_ERR_INVALID_ARG, "frame is not in the ring");
    CUDA_TRY(cudaStreamSynchronize(e->fft_stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    CUDA_TRY(cudaMemcpy(out, e->ring + static_cast<size_t>(frame % e->R) * e->E, sizeof(float2) * e->E,
                        cudaMemcpyDeviceToHost));
    return DDM_OK;
}

extern "C" int ddm_read_accumulators(ddm_engine *e, double *out, long capacity) {
    clear_error();
    if (!e || !out || capacity < static_cast<long>(e->T * e->E)) return fail(DDM_ERR_INVALID_ARG, "bad argument");
    int st = flush_lag(e);
    if (st) return st;
    std::vector<float2> tmp(static_cast<size_t>(e->T) * e->E);
    CUDA_TRY(cudaStreamSynchronize(e->fft_stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    CUDA_TRY(cudaMemcpy(tmp.data(), e->acc, sizeof(float2) * tmp.size(), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < tmp.size(); i++) out[i] = static_cast<double>(tmp[i].x) - static_cast<double>(tmp[i].y);
    return DDM_OK;
}

extern "C" int ddm_read_power_spectrum(ddm_engine *e, int frame, float *out, long capacity) {
    clear_error();
    if (!e || !out || capacity < e->E) return fail(DDM_ERR_INVALID_ARG, "ddm_read_power_spectrum: bad argument");
    std::vector<float> spec(2 * static_cast<size_t>(e->E));
    int st = ddm_read_spectrum(e, frame, spec.data(), static_cast<long>(spec.size()));
    if (st) return st;
    // src/DDM_kernel.cuh:107-121 (calculateAmplitude): v = F / s^2 in float, then |v|^2
    for (const ScaleDesc &d : e->sd) {
        const float fft_norm = 1.0f / static_cast<float>(d.s * d.s);
        const long long end = d.off + d.tiles * d.n;
        for (long long k = d.off; k < end; k++) {
            const float x = fft_norm * spec[2 * k], y = fft_norm * spec[2 * k + 1];
            out[k] = x * x + y * y;
        }
    }
    return DDM_OK;
}

extern "C" int ddm_read_unaveraged(ddm_engine *e, double *out, long capacity) {
    clear_error();
    if (!e || !out || capacity < static_cast<long>(e->T * e->E))
        return fail(DDM_ERR_INVALID_ARG, "ddm_read_unaveraged: bad argument");
    if (!e->finalized) return fail(DDM_ERR_STATE, "ddm_finalize has not run");
    std::vector<float2> tmp(static_cast<size_t>(e->T) * e->E);
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    CUDA_TRY(cudaMemcpy(tmp.data(), e->acc, sizeof(float2) * tmp.size(), cudaMemcpyDeviceToHost));
    for (int t = 0; t < e->T; t++) {
        const double nrm = e->host_norm[t];
        for (const ScaleDesc &d : e->sd) {
            const double f = nrm != 0.0 ? 2.0 * d.inv_s4 / nrm : 0.0;
            const size_t b = static_cast<size_t>(t) * e->E + d.off, n = static_cast<size_t>(d.tiles) * d.n;
            for (size_t k = b; k < b + n; k++)
                out[k] = (static_cast<double>(tmp[k].x) - static_cast<double>(tmp[k].y)) * f;
        }
    }
    return DDM_OK;
}

extern "C" long ddm_tile_count(const ddm_engine *e) {
    if (!e) return 0;
    long n = 0;
    for (const ScaleDesc &d : e->sd) n += d.tiles;
    return n;
}

extern "C" int ddm_fit_isf(ddm_engine *e, float fps, double um_per_px, int start, double *tile_fit,
                           double *scale_fit, double *tile_d, double *scale_d) {
    clear_error();
    if (!e) return fail(DDM_ERR_INVALID_ARG, "ddm_fit_isf: null engine");
    if (!e->finalized) return fail(DDM_ERR_STATE, "ddm_finalize has not run");
    if (!(um_per_px > 0.0) || !std::isfinite(um_per_px) || !std::isfinite(fps))
        return fail(DDM_ERR_INVALID_ARG, "ddm_fit_isf: um_per_px must be positive and fps finite");
    if (start != DDM_FIT_START_DATA && start != DDM_FIT_START_SCRIPT)
        return fail(DDM_ERR_INVALID_ARG, "ddm_fit_isf: unknown start");
    const int tiles_total = static_cast<int>(ddm_tile_count(e));
    const long tile_curves = static_cast<long>(tiles_total) * e->Q, scale_curves = static_cast<long>(e->S) * e->Q;
    // device layout: mean [S][Q][T], tau [T], q [Q], tile fits, scale fits, tile D, scale D
    const size_t n_mean = static_cast<size_t>(scale_curves) * e->T;
    const size_t n_all = n_mean + e->T + e->Q + (tile_curves + scale_curves) * kFitParams + 2 * (tiles_total + e->S);
    if (!e->fit_d) {
        int st = dev_alloc(e, &e->fit_d, n_all);
        if (st) return st;
    }
    FitArgs a;
    std::memset(&a, 0, sizeof(a));
    a.S = e->S, a.T = e->T, a.Q = e->Q;
    a.start = start == DDM_FIT_START_SCRIPT ? 1 : 0;
    int curve = 0;
    for (int si = 0; si < e->S; si++) {
        a.tiles[si] = e->sd[si].tiles;
        a.isf_off[si] = e->sd[si].isf_off;
        a.curve_off[si] = curve;
        curve += e->sd[si].tiles * e->Q;
    }
    a.tile_curves = static_cast<int>(tile_curves);
    a.isf = e->isf_d;
    a.mean = e->fit_d;
    double *tau_d = a.mean + n_mean, *q_d = tau_d + e->T;
    a.tau = tau_d, a.q = q_d;
    a.tile_fit = q_d + e->Q;
    a.scale_fit = a.tile_fit + tile_curves * kFitParams;
    a.tile_d = a.scale_fit + scale_curves * kFitParams;
    a.scale_d = a.tile_d + 2 * tiles_total;
    // lag times as the ISF files label them ((float)tau / fps, src/azimuthal_average.cu:131),
    // in frames when fps <= 0; q = 2 pi / (lambda * um_per_px) (plot_averaged.py:258-261)
    std::vector<double> host(static_cast<size_t>(e->T) + e->Q);
    for (int t = 0; t < e->T; t++)
        host[t] = fps > 0.0f ? static_cast<double>(static_cast<float>(e->taus[t]) / fps) : e->taus[t];
    const double two_pi = 6.283185307179586;
    for (int q = 0; q < e->Q; q++) host[e->T + q] = two_pi / (static_cast<double>(e->lambdas[q]) * um_per_px);
    CUDA_TRY(cudaMemcpyAsync(tau_d, host.data(), sizeof(double) * host.size(), cudaMemcpyHostToDevice, e->stream));
    fit_mean_kernel<<<static_cast<unsigned>((n_mean + kFitThreads - 1) / kFitThreads), kFitThreads, 0, e->stream>>>(a);
    CUDA_TRY(cudaGetLastError());
    fit_isf_kernel<<<static_cast<unsigned>((tile_curves + scale_curves + kFitThreads - 1) / kFitThreads), kFitThreads,
                     0, e->stream>>>(a);
    CUDA_TRY(cudaGetLastError());
    fit_diffusion_kernel<<<static_cast<unsigned>((tiles_total + e->S + kFitThreads - 1) / kFitThreads), kFitThreads, 0,
                           e->stream>>>(a, tiles_total);
    CUDA_TRY(cudaGetLastError());
    e->launches += 3;
    CUDA_TRY(cudaStreamSynchronize(e->stream));  // host is a local buffer the copy read from
    if (tile_fit)
        CUDA_TRY(cudaMemcpy(tile_fit, a.tile_fit, sizeof(double) * tile_curves * kFitParams, cudaMemcpyDeviceToHost));
    if (scale_fit)
        CUDA_TRY(cudaMemcpy(scale_fit, a.scale_fit, sizeof(double) * scale_curves * kFitParams, cudaMemcpyDeviceToHost));
    if (tile_d) CUDA_TRY(cudaMemcpy(tile_d, a.tile_d, sizeof(double) * 2 * tiles_total, cudaMemcpyDeviceToHost));
    if (scale_d) CUDA_TRY(cudaMemcpy(scale_d, a.scale_d, sizeof(double) * 2 * e->S, cudaMemcpyDeviceToHost));
    return DDM_OK;
}

extern "C" int ddm_get_info(const ddm_engine *e, ddm_info *info) {
    if (!e || !info) return fail(DDM_ERR_INVALID_ARG, "bad argument");
    info->frames_submitted = static_cast<long>(e->submitted);
    info->ring_slots = e->R;
    info->device_bytes = e->device_bytes;
    info->kernel_launches = static_cast<long>(e->launches);
    info->stream = e->stream;
    info->frames_needed = e->estimator == DDM_EST_COMPAT ? e->frames_read : 0;
    info->lag_batch_frames = e->lag_batch;
    info->lag_geometry = e->lag_geom;
    info->fft_group_frames = e->fft_group;
    info->fft_per_tile = e->fft_per_tile;
    return DDM_OK;
}

extern "C" const char *ddm_last_error(void) { return last_error(); }

extern "C" int ddm_set_wait_limit(ddm_engine *e, long long cycles) {
    clear_error();
    if (!e) return fail(DDM_ERR_INVALID_ARG, "null engine");
    if (cycles < 0) return fail(DDM_ERR_INVALID_ARG, "ddm_set_wait_limit: cycles must be >= 0");
    e->wait_cycles = cycles == 0 ? kWaitCycles : cycles;
    return DDM_OK;
}

extern "C" int ddm_inject_fault(ddm_engine *e, int fault) {
    clear_error();
    if (!e) return fail(DDM_ERR_INVALID_ARG, "null engine");
    if (fault != DDM_FAULT_NONE && fault != DDM_FAULT_LAG_WAIT)
        return fail(DDM_ERR_INVALID_ARG, "ddm_inject_fault: unknown fault");
    if (fault == DDM_FAULT_LAG_WAIT && e->defer_lag)
        return fail(DDM_ERR_STATE, "ddm_inject_fault: not for served streams");
    e->inject = fault;
    return DDM_OK;
}

extern "C" int ddm_set_timing(ddm_engine *e, int enabled) {
    if (!e) return fail(DDM_ERR_INVALID_ARG, "null engine");
    e->timing = enabled != 0;
    return DDM_OK;
}

extern "C" int ddm_kernel_times(ddm_engine *e, double *ms, long *launches) {
    return ddm_kernel_stats(e, ms, launches, nullptr);
}

extern "C" int ddm_kernel_stats(ddm_engine *e, double *ms, long *launches, double *bytes) {
    clear_error();
    if (!e || !ms || !launches) return fail(DDM_ERR_INVALID_ARG, "bad argument");
    for (int g = 0; g < 3; g++) {
        if (bytes) bytes[g] = e->tbytes[g];
        e->tbytes[g] = 0.0;
    }
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    for (int g = 0; g < 3; g++) {
        double total = 0.0;
        for (auto &pr : e->tev[g]) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, pr.first, pr.second) == cudaSuccess) total += t;
            e->tev_pool.push_back(pr.first);
            e->tev_pool.push_back(pr.second);
        }
        e->tev[g].clear();
        ms[g] = total;
        launches[g] = e->tlaunch[g];
        e->tlaunch[g] = 0;
    }
    return DDM_OK;
}

extern "C" int ddm_build_masks(int scale, const float *lambdas, int Q, float tol, unsigned char *mask,
                               int *counts) {
    clear_error();
    if (scale < 2 || (scale & (scale - 1)) || !lambdas || Q <= 0 || !counts)
        return fail(DDM_ERR_INVALID_ARG, "ddm_build_masks: bad argument");
    std::vector<int> qp, idx, cnt;
    build_masks(scale, std::vector<float>(lambdas, lambdas + Q), tol, &qp, &idx, &cnt);
    std::copy(cnt.begin(), cnt.end(), counts);
    if (mask) {
        const long long n = static_cast<long long>(scale) * (scale / 2 + 1);
        std::memset(mask, 0, static_cast<size_t>(n * Q));
        for (int q = 0; q < Q; q++)
            for (int i = qp[q]; i < qp[q + 1]; i++) mask[q * n + idx[i]] = 1;
    }
    return DDM_OK;
}

extern "C" int ddm_compat_schedule(int N, int C, int multistream, int G, const int *taus, int T, int max_calls,
                                   int *a_out, int *b_out, int *epoch_out, int *frames_read) {
    clear_error();
    if (N < 0 || C <= 0 || !taus || T <= 0 || !a_out || !b_out)
        return fail(DDM_ERR_INVALID_ARG, "ddm_compat_schedule: bad argument");
    std::vector<int> t(taus, taus + T);
    for (int v : t)
        if (v < 0 || v > C) return fail(DDM_ERR_INVALID_ARG, "taus must lie in [0, chunk]");
    int fr = 0;
    std::vector<CompatIteration> its = compat_schedule(N, C, multistream, G, t, &fr);
    long long calls = 0;
    for (const CompatIteration &it : its) calls += it.count;
    if (calls > max_calls) return -1;
    int c = 0, ep = 0;
    for (const CompatIteration &it : its) {
        for (int fo = 0; fo < it.count; fo++, c++) {
            a_out[c] = it.start[fo];
            for (int i = 0; i < T; i++) {
                const int p = fo + t[i];
                b_out[static_cast<long long>(c) * T + i] = p < C ? it.start[p] : it.end[p - C];
            }
            if (epoch_out) epoch_out[c] = ep;
        }
        if (it.dump_after) ep++;
    }
    if (frames_read) *frames_read = fr;
    return c;
}

extern "C" void *ddm_host_alloc(size_t bytes) {
    void *p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) {
        fail(DDM_ERR_OUT_OF_MEMORY, "cudaMallocHost of " + std::to_string(bytes) + " bytes failed");
        return nullptr;
    }
    return p;
}

extern "C" void ddm_host_free(void *p) {
    if (p) cudaFreeHost(p);
}

extern "C" const char *ddm_status_string(int status) {
    switch (status) {
        case DDM_OK: return "ok";
        case DDM_ERR_INVALID_ARG: return "invalid argument";
        case DDM_ERR_CUDA: return "CUDA error";
        case DDM_ERR_OUT_OF_MEMORY: return "out of device memory";
        case DDM_ERR_STATE: return "invalid state";
        case DDM_ERR_NEED_FRAMES: return "frames missing";
        case DDM_ERR_NO_DEVICE: return "no suitable CUDA device";
        case DDM_ERR_IO: return "I/O error";
        case DDM_ERR_BUSY: return "busy";
        default: return "unknown status";
    }
}

extern "C" int ddm_write_isf_file(const char *path, const double *isf_qt, const float *lambdas, int Q,
                                  const int *taus, int T, float fps) {
    clear_error();
    if (!path || !isf_qt || !lambdas || !taus || Q <= 0 || T <= 0)
        return fail(DDM_ERR_INVALID_ARG, "ddm_write_isf_file: bad argument");
    std::vector<float> l(lambdas, lambdas + Q);
    std::vector<int> t(taus, taus + T);
    if (!write_isf_file(path, isf_qt, l, t, fps))
        return fail(DDM_ERR_IO, std::string("[Out Error] Unable to open ") + path + ".");
    return DDM_OK;
}
