// Test-side harness around two of the reference's own host functions, linked from the
// reference sources by oracle/Makefile (target `ref`): buildAzimuthMask and
// analyseFFTDevice (src/azimuthal_average.cu:229-283, 292-346). It prints what they
// compute so the FP64 oracle can be pinned against them. TEST INFRASTRUCTURE ONLY.
//
//   ref_harness mask <scale> <tolerance> <lambda>...
//       -> "counts c0 c1 ...", then "fnv q <64-bit FNV-1a of mask bytes>" per lambda
//   ref_harness reduce <scale> <taus> <tolerance> <norm_frames> <seed> <lambda>...
//       fills a [taus][s*(s/2+1)] accumulator with the LCG values below, then prints
//       analyseFFTDevice's ISF as "isf q t value" lines (%.9g)
//
// Accumulator values: x_{i+1} = 6364136223846793005 x_i + 1442695040888963407 (mod 2^64),
// value_i = (x_i >> 40) / 2^24 * 1000, x_0 = seed.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

void buildAzimuthMask(bool *d_mask_out, int *h_pixel_counts, float *q_arr, int q_count,
                      float q_tolerance, int w, int h);
float *analyseFFTDevice(float *d_data_in, bool *d_mask, int *h_pixel_counts, float normalisation_factor,
                        int tau_count, int q_count, int tile_count, int w, int h);

static std::vector<float> q_of(int scale, int argc, char **argv, int first) {
    std::vector<float> q;
    for (int i = first; i < argc; i++) {
        float lambda = std::strtof(argv[i], nullptr);
        q.push_back(static_cast<float>(scale) / lambda);  // src/DDM.cu:102
    }
    return q;
}

int main(int argc, char **argv) {
    if (argc < 4) return 2;
    std::string mode = argv[1];
    const int s = std::atoi(argv[2]);
    const long n = static_cast<long>(s) * (s / 2 + 1);
    if (mode == "mask") {
        const float tol = std::strtof(argv[3], nullptr);
        std::vector<float> q = q_of(s, argc, argv, 4);
        const int Q = static_cast<int>(q.size());
        bool *d_mask = nullptr;
        if (cudaMalloc(&d_mask, sizeof(bool) * n * Q) != cudaSuccess) return 3;
        std::vector<int> counts(Q);
        buildAzimuthMask(d_mask, counts.data(), q.data(), Q, tol, s, s);
        std::vector<unsigned char> h(n * Q);
        if (cudaMemcpy(h.data(), d_mask, n * Q, cudaMemcpyDeviceToHost) != cudaSuccess) return 3;
        std::printf("counts");
        for (int c : counts) std::printf(" %d", c);
        std::printf("\n");
        for (int qi = 0; qi < Q; qi++) {
            uint64_t hsh = 1469598103934665603ULL;
            for (long k = 0; k < n; k++) {
                hsh ^= h[qi * n + k] ? 1u : 0u;
                hsh *= 1099511628211ULL;
            }
            std::printf("fnv %d %llu\n", qi, static_cast<unsigned long long>(hsh));
        }
        cudaFree(d_mask);
        return 0;
    }
    if (mode == "reduce" && argc >= 8) {
        const int T = std::atoi(argv[3]);
        const float tol = std::strtof(argv[4], nullptr);
        const int frames = std::atoi(argv[5]);
        uint64_t x = std::strtoull(argv[6], nullptr, 10);
        std::vector<float> q = q_of(s, argc, argv, 7);
        const int Q = static_cast<int>(q.size());
        std::vector<float> acc(n * T);
        for (auto &v : acc) {
            v = static_cast<float>(static_cast<double>(x >> 40) / 16777216.0 * 1000.0);
            x = x * 6364136223846793005ULL + 1442695040888963407ULL;
        }
        float *d_acc = nullptr;
        bool *d_mask = nullptr;
        if (cudaMalloc(&d_acc, sizeof(float) * n * T) != cudaSuccess) return 3;
        if (cudaMalloc(&d_mask, sizeof(bool) * n * Q) != cudaSuccess) return 3;
        cudaMemcpy(d_acc, acc.data(), sizeof(float) * n * T, cudaMemcpyHostToDevice);
        std::vector<int> counts(Q);
        buildAzimuthMask(d_mask, counts.data(), q.data(), Q, tol, s, s);
        const float norm = 1.0 / static_cast<float>(frames);  // src/DDM.cu:92
        float *isf = analyseFFTDevice(d_acc, d_mask, counts.data(), norm, T, Q, 1, s, s);
        for (int qi = 0; qi < Q; qi++)
            for (int t = 0; t < T; t++) std::printf("isf %d %d %.9g\n", qi, t, isf[qi * T + t]);
        cudaFree(d_acc);
        cudaFree(d_mask);
        return 0;
    }
    return 2;
}
