// Autotuner for the engine's blocking choices:
//   lag_batch_frames  the frames one lag launch pairs. A launch pairs its J register frames
//                     against the union of their partner frames, so larger J reads fewer
//                     partner bytes per frame, but J above the ingest piece holds frames back,
//                     and the kernel's per-element cost changes with J;
//   lag_geometry      one thread per element (4 consumer warps, 3 CTAs per SM) or two
//                     (8 consumer warps, 2 CTAs per SM): occupancy against per-entry overhead;
//   fft_group_frames  frames per FFT launch: fewer, larger launches against keeping the row
//                     pass's output in L2 and overlapping host copies with the FFT;
//   fft_per_tile      tiles of side 32..128 in the per-tile kernel or in the two passes.
// The best values depend on the frame size, scales, tau list and chunk. ddm_autotune times the
// (J, geometry) candidates, then the FFT groups with the fastest of those, on the caller's
// shape with synthetic frames resident on the device (the engine's steady state: every timed
// frame has all its lags), and keeps the winner in a JSON cache keyed by the shape, one key per
// line; engines opened with lag_batch_frames = -1 look their shape up in the cache named by the
// DDM_TUNE_CACHE environment variable.
#include "tune.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/ddm.h"
#include "errors.hpp"

namespace ddm {

namespace {

uint64_t fnv1a(const std::vector<int> &v) {
    uint64_t h = 1469598103934665603ull;
    for (int x : v)
        for (int b = 0; b < 4; b++) {
            h ^= static_cast<uint8_t>(static_cast<uint32_t>(x) >> (8 * b));
            h *= 1099511628211ull;
        }
    return h;
}

const int kCandidates[] = {16, 24, 30, 32, 64};
const int kFftGroups[] = {0, 4, 8, 16};

}  // namespace

std::string tune_key(const ddm_config *cfg) {
    std::vector<int> scales(cfg->scales, cfg->scales + cfg->scale_count);
    std::vector<int> taus(cfg->taus, cfg->taus + cfg->tau_count);
    std::sort(scales.rbegin(), scales.rend());
    std::sort(taus.begin(), taus.end());
    std::ostringstream k;
    k << "w" << cfg->frame_width << "h" << cfg->frame_height << "b" << cfg->bytes_per_pixel << "|s";
    for (size_t i = 0; i < scales.size(); i++) k << (i ? "," : "") << scales[i];
    char hash[20];
    std::snprintf(hash, sizeof(hash), "%016llx", static_cast<unsigned long long>(fnv1a(taus)));
    k << "|t" << taus.size() << ":" << (taus.empty() ? 0 : taus.back()) << ":" << hash << "|c" << cfg->chunk_frames
      << "|e" << cfg->estimator;
    if (cfg->small_tile_dft) k << "|dft";
    return k.str();
}

bool tune_lookup(const char *path, const std::string &key, TunedValues *out) {
    if (!path || !*path) return false;
    std::ifstream in(path);
    if (!in) return false;
    const std::string head = "\"" + key + "\": {";
    std::string line;
    // the value after "name": within this shape's line (-1 when absent)
    auto field = [&](size_t from, const char *name, double *v) {
        const std::string n = std::string("\"") + name + "\": ";
        const size_t a = line.find(n, from);
        if (a == std::string::npos) return false;
        *v = std::atof(line.c_str() + a + n.size());
        return true;
    };
    while (std::getline(in, line)) {
        const size_t p = line.find(head);
        if (p == std::string::npos) continue;
        double J = 0, G = 0, F = 0, V = 0, fps = 0;
        if (!field(p, "lag_batch_frames", &J) || J < 1 || J > 64) return false;
        field(p, "lag_geometry", &G);  // absent in caches written before these were tuned: 0
        field(p, "fft_group_frames", &F);
        field(p, "fft_per_tile", &V);
        field(p, "frames_per_s", &fps);
        out->lag_batch = static_cast<int>(J);
        out->lag_geometry = (G == 1 && J <= 32) ? 1 : 0;
        out->fft_group = F > 0 ? static_cast<int>(F) : 0;
        out->fft_per_tile = V == 1 ? 1 : 0;
        out->fps = fps;
        return true;
    }
    return false;
}

namespace {

// Rewrites the cache with `entry` for `key` (other keys kept, one per line); written to a
// temporary file first and renamed over the cache.
bool tune_store(const char *path, const std::string &key, const std::string &entry) {
    std::vector<std::string> keep;
    {
        std::ifstream in(path);
        std::string line;
        const std::string head = "\"" + key + "\": {";
        while (in && std::getline(in, line)) {
            if (line.size() < 2 || line[0] != '"' || line.find(head) == 0) continue;
            if (line.back() == ',') line.pop_back();
            keep.push_back(line);
        }
    }
    keep.push_back("\"" + key + "\": " + entry);
    const std::string tmp = std::string(path) + ".tmp";
    {
        std::ofstream out(tmp);
        if (!out) return false;
        out << "{\n";
        for (size_t i = 0; i < keep.size(); i++) out << keep[i] << (i + 1 < keep.size() ? ",\n" : "\n");
        out << "}\n";
        if (!out) return false;
    }
    return std::rename(tmp.c_str(), path) == 0;
}

// Frames/s of one engine with lag_batch_frames = J, lag_geometry = G, fft_group_frames = F and
// fft_per_tile = V on `frames` (device memory): pre-roll until
// every frame has all its lags, then `timed` chunks between two synchronisations.
int time_candidate(const ddm_config &base, int J, int G, int F, int V, const uint8_t *frames, int n_frames, int timed,
                   double *fps) {
    ddm_config c = base;
    c.lag_batch_frames = J;
    c.lag_geometry = G;
    c.fft_group_frames = F;
    c.fft_per_tile = V;
    c.dump_every = 0;
    ddm_engine *e = nullptr;
    int st = ddm_open(&c, &e);
    if (st) return st;
    const int C = c.chunk_frames;
    const int tau_max = *std::max_element(c.taus, c.taus + c.tau_count);
    const size_t frame_bytes = static_cast<size_t>(c.frame_width) * c.frame_height * c.bytes_per_pixel;
    int pos = 0;
    auto submit = [&]() {
        if (pos + C > n_frames) pos = 0;
        const int r = ddm_submit_frames(e, frames + frame_bytes * pos, C, 1);
        pos += C;
        return r;
    };
    const int preroll = (tau_max + C - 1) / C + 2;
    for (int i = 0; i < preroll && !st; i++) st = submit();
    if (!st) st = ddm_synchronize(e);
    ddm_info info;
    if (!st) st = ddm_get_info(e, &info);
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (!st && (cudaEventCreate(&t0) != cudaSuccess || cudaEventCreate(&t1) != cudaSuccess))
        st = fail(DDM_ERR_CUDA, "cudaEventCreate failed");
    if (!st) cudaEventRecord(t0, static_cast<cudaStream_t>(info.stream));
    for (int i = 0; i < timed && !st; i++) st = submit();
    if (!st) st = ddm_synchronize(e);  // pairs the frames a batch still holds back
    float ms = 0.f;
    if (!st) {
        cudaEventRecord(t1, static_cast<cudaStream_t>(info.stream));
        cudaEventSynchronize(t1);
        cudaEventElapsedTime(&ms, t0, t1);
        *fps = ms > 0.f ? 1000.0 * timed * C / ms : 0.0;
    }
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    ddm_close(e);
    return st;
}

}  // namespace

}  // namespace ddm

using namespace ddm;

extern "C" long ddm_tune_key(const ddm_config *cfg, char *out, long capacity) {
    if (!cfg || (cfg->scale_count > 0 && !cfg->scales) || (cfg->tau_count > 0 && !cfg->taus)) return -1;
    const std::string k = tune_key(cfg);
    if (out && capacity > 0) {
        const size_t n = std::min<size_t>(k.size(), static_cast<size_t>(capacity - 1));
        k.copy(out, n);
        out[n] = '\0';
    }
    return static_cast<long>(k.size());
}

extern "C" int ddm_autotune(const ddm_config *cfg, const char *cache_path, ddm_tuning *out) {
    clear_error();
    if (!cfg || !out || cfg->tau_count < 1 || !cfg->taus || cfg->chunk_frames < 1)
        return fail(DDM_ERR_INVALID_ARG, "ddm_autotune: bad argument");
    if (cfg->estimator != DDM_EST_UNBIASED)
        return fail(DDM_ERR_INVALID_ARG, "ddm_autotune: the lag blocking is tuned for the unbiased estimator");
    const std::string key = tune_key(cfg);
    *out = ddm_tuning{};
    TunedValues tv;
    if (tune_lookup(cache_path, key, &tv)) {
        out->lag_batch_frames = tv.lag_batch;
        out->lag_geometry = tv.lag_geometry;
        out->fft_group_frames = tv.fft_group;
        out->fft_per_tile = tv.fft_per_tile;
        out->frames_per_s = tv.fps;
        out->from_cache = 1;
        return DDM_OK;
    }
    // synthetic frames (a fixed LCG: the timing does not depend on their content) on the device
    const size_t frame_bytes = static_cast<size_t>(cfg->frame_width) * cfg->frame_height * cfg->bytes_per_pixel;
    const int n_frames = 4 * std::max(cfg->chunk_frames, 1);
    std::vector<uint8_t> host(frame_bytes * n_frames);
    uint32_t x = 12345u;
    for (auto &b : host) {
        x = x * 1664525u + 1013904223u;
        b = static_cast<uint8_t>(x >> 24);
    }
    if (cudaSetDevice(cfg->device) != cudaSuccess) return fail(DDM_ERR_NO_DEVICE, "cudaSetDevice failed");
    uint8_t *dev = nullptr;
    if (cudaMalloc(&dev, host.size()) != cudaSuccess) return fail(DDM_ERR_OUT_OF_MEMORY, "autotune frame buffer");
    if (cudaMemcpy(dev, host.data(), host.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(dev);
        return fail(DDM_ERR_CUDA, "autotune frame upload failed");
    }
    std::vector<int> cands(std::begin(kCandidates), std::end(kCandidates));
    if (cfg->chunk_frames <= 64) cands.push_back(cfg->chunk_frames);
    std::sort(cands.begin(), cands.end());
    cands.erase(std::unique(cands.begin(), cands.end()), cands.end());
    const int timed = std::max(4, (8 * 30 + cfg->chunk_frames - 1) / cfg->chunk_frames);
    std::ostringstream tried;
    int best = 0, best_g = 0, best_f = 0, best_v = 0, first_error = DDM_OK;
    std::string first_message;
    double best_fps = 0.0;
    // a candidate that cannot run here (e.g. its ring does not fit) is skipped
    auto run = [&](int J, int G, int F, int V) {
        double fps = 0.0;
        const int st = time_candidate(*cfg, J, G, F, V, dev, n_frames, timed, &fps);
        if (st) {
            if (!first_error) first_error = st, first_message = last_error();
            return;
        }
        char buf[64];
        std::snprintf(buf, sizeof(buf), "%s\"%d/%d/%d/%d\": %.1f", tried.tellp() > 0 ? ", " : "", J, G, F, V, fps);
        tried << buf;
        if (fps > best_fps) best_fps = fps, best = J, best_g = G, best_f = F, best_v = V;
    };
    for (int J : cands)
        for (int G = 0; G < (J <= 32 ? 2 : 1); G++) run(J, G, 0, 0);
    if (best > 0) {
        const int J = best, G = best_g;
        for (int F : kFftGroups)
            if (F > 0) run(J, G, F, 0);
        run(J, G, 0, 1);
    }
    cudaFree(dev);
    if (best == 0) return fail(first_error ? first_error : DDM_ERR_CUDA, "ddm_autotune: no candidate ran: " + first_message);
    out->lag_batch_frames = best;
    out->lag_geometry = best_g;
    out->fft_group_frames = best_f;
    out->fft_per_tile = best_v;
    out->frames_per_s = best_fps;
    out->from_cache = 0;
    if (cache_path && *cache_path) {
        char buf[192];
        std::snprintf(buf, sizeof(buf),
                      "{\"lag_batch_frames\": %d, \"lag_geometry\": %d, \"fft_group_frames\": %d, "
                      "\"fft_per_tile\": %d, \"frames_per_s\": %.1f, \"candidates\": {",
                      best, best_g, best_f, best_v, best_fps);
        if (!tune_store(cache_path, key, std::string(buf) + tried.str() + "}}"))
            return fail(DDM_ERR_INVALID_ARG, std::string("ddm_autotune: cannot write the cache ") + cache_path);
    }
    return DDM_OK;
}
