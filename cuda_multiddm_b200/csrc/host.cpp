// Host-side pieces of the DDM engine: masks, reference schedule, validation, ISF text.
#include "host.hpp"

#include <algorithm>
#include <cstdio>
#include <fstream>

namespace ddm {

float q_radius(int scale, float lambda) {
    volatile float s = static_cast<float>(scale);
    volatile float q = s / lambda;  // src/DDM.cu:102
    return q;
}

void build_masks(int scale, const std::vector<float> &lambdas, float tolerance,
                 std::vector<int> *q_ptr, std::vector<int> *idx, std::vector<int> *counts) {
    const int w = scale, h = scale, nx = w / 2 + 1;
    const int half_w = w / 2, half_h = h / 2;
    volatile float tol2 = tolerance * tolerance;  // src/azimuthal_average.cu:249
    q_ptr->assign(1, 0);
    idx->clear();
    counts->clear();
    // r2 depends only on (x', y'), so evaluate the float predicate per element in the
    // order the output wants (ky-major, kx fastest); the set of pixels is identical to
    // the reference's kx-major loop because each pixel's test is independent.
    for (float lambda : lambdas) {
        float q = q_radius(scale, lambda);
        volatile float q2 = q * q;  // src/azimuthal_average.cu:241-242
        int count = 0;
        for (int y = 0; y < h; y++) {
            const int ys = (y + half_h) % h - half_h;
            for (int x = 0; x < nx; x++) {
                const int xs = (x + half_w) % w - half_w;
                volatile float r2 = static_cast<float>(xs * xs + ys * ys);
                volatile float ratio = r2 / q2;
                if (1.0f <= ratio && ratio <= tol2) {
                    idx->push_back(y * nx + x);
                    count++;
                }
            }
        }
        counts->push_back(count);
        q_ptr->push_back(static_cast<int>(idx->size()));
    }
}

std::vector<CompatIteration> compat_schedule(int N, int C, int multistream, int G,
                                             const std::vector<int> &taus, int *frames_read) {
    // Buffers of C labels: two pinned host chunks (one when -Z), three FFT ring slots.
    std::vector<int> host_a(C, kLabelUninit), host_b(C, kLabelUninit);
    std::vector<int> slot0(C, kLabelUninit), slot1(C, kLabelUninit), slot2(C, kLabelUninit);
    std::vector<int> *h_cur = &host_a, *h_nxt = multistream ? &host_b : &host_a;
    std::vector<int> *start = &slot0, *end = &slot1, *junk = &slot2;
    int cursor = 0;
    auto load = [&](std::vector<int> *h, int n) {  // loadVideoToHost, src/video_reader.cpp:32
        for (int j = 0; j < n; j++) (*h)[j] = cursor++;
    };
    auto parse = [&](std::vector<int> *slot, const std::vector<int> *h, int n) {
        for (int j = 0; j < n; j++) (*slot)[j] = (*h)[j];  // H2D copy + parseChunk
    };
    const int K = N / C, L = N % C;
    const int tau_max = taus.empty() ? 0 : *std::max_element(taus.begin(), taus.end());
    std::vector<CompatIteration> its;
    auto record = [&](int count) {
        CompatIteration it;
        it.start = *start;
        it.end = *end;
        it.count = count;
        int lo = 1 << 30, hi = -1;
        for (int fo = 0; fo < count; fo++) {
            // the A frame and every partner position fo + tau in start|end
            auto see = [&](int lab) {
                if (lab >= 0) { lo = std::min(lo, lab); hi = std::max(hi, lab); }
            };
            see((*start)[fo]);
            for (int t : taus) {
                int p = fo + t;
                see(p < C ? (*start)[p] : (*end)[p - C]);
            }
        }
        (void)tau_max;
        it.min_label = hi < 0 ? 0 : lo;
        it.max_label = hi;
        its.push_back(std::move(it));
    };

    load(h_nxt, C);  // src/DDM.cu:752-753
    load(h_cur, C);
    parse(start, h_nxt, C);  // src/DDM.cu:755-760
    for (int i = 0; i < K; i++) {  // src/DDM.cu:765
        parse(end, h_cur, C);      // :767-771
        record(C);                 // :773-775
        if (K - i > 2)
            load(h_nxt, C);        // :780-781
        else if (L != 0 && K - i == 2)
            load(h_nxt, L);        // :782-783
        std::swap(h_cur, h_nxt);   // :788
        std::vector<int> *t = junk;  // :793 rotateThreePtr(junk, start, end)
        junk = start;
        start = end;
        end = t;
        if (G != 0 && i != 0 && i % G == 0) its.back().dump_after = true;  // :800
    }
    if (L != 0) {  // :830-843
        parse(end, h_cur, L);
        record(L);
    }
    if (frames_read) *frames_read = cursor;
    return its;
}

std::string validate_reference_params(const std::vector<int> &scales, const std::vector<int> &taus,
                                      const std::vector<float> &lambdas, float tolerance, int chunk,
                                      bool enforce_tau_chunk, bool enforce_lambda_scale,
                                      std::vector<std::string> *warnings) {
    if (scales.empty() || taus.empty() || lambdas.empty())
        return "scale, tau and lambda lists must each hold at least one value";
    for (size_t s = 0; s < scales.size(); s++) {  // src/DDM.cu:328-334
        unsigned int v = static_cast<unsigned int>(scales[s]);
        if (scales[s] <= 0 || (v & (v - 1))) return "scales must be powers of two (> 0)";
        if (s + 1 < scales.size() && !(scales[s] > scales[s + 1]))
            return "scales should be descending order";
    }
    for (size_t t = 0; t < taus.size(); t++) {  // src/DDM.cu:336-339 (all entries here)
        if (taus[t] < 0) return "Tau values should be positive";
        if (t + 1 < taus.size() && !(taus[t] < taus[t + 1]))
            return "Tau vector should be ascending order";
    }
    for (size_t q = 0; q < lambdas.size(); q++) {  // src/DDM.cu:341-344
        if (!(lambdas[q] >= 0)) return "q-vector values should be positive";
        if (q + 1 < lambdas.size() && !(lambdas[q] < lambdas[q + 1]))
            return "q-vector vector should be ascending order";
    }
    if (!(tolerance < 10 && tolerance > 1.0f) && warnings)  // src/DDM.cu:346-347
        warnings->push_back(
            "mask_tolerance is likely undesired value, refer to README for more information");
    if (enforce_lambda_scale && !(lambdas.back() <= scales.back()))  // src/DDM.cu:349-350
        return "The largest q-vector should be smaller than the smallest scale.";
    if (chunk <= 0) return "chunk frame count must be positive";
    if (enforce_tau_chunk && !(taus.back() <= chunk))  // src/DDM.cu:462-463
        return "the largest tau value must be smaller than number frames in a chunk";
    return std::string();
}

bool write_isf_file(const std::string &path, const double *isf, const std::vector<float> &lambdas,
                    const std::vector<int> &taus, float fps) {
    FILE *f = std::fopen(path.c_str(), "w");
    if (!f) return false;
    // std::ostream << float prints with "%g" (precision 6); the values are the reference's
    // floats, so round each to float first (src/azimuthal_average.cu:265,272,280).
    for (float l : lambdas) std::fprintf(f, "%g ", static_cast<double>(l));
    std::fputc('\n', f);
    for (int t : taus) std::fprintf(f, "%g ", static_cast<double>(static_cast<float>(t) / fps));
    std::fputc('\n', f);
    const size_t T = taus.size();
    for (size_t q = 0; q < lambdas.size(); q++) {
        for (size_t t = 0; t < T; t++)
            std::fprintf(f, "%g ", static_cast<double>(static_cast<float>(isf[q * T + t])));
        std::fputc('\n', f);
    }
    return std::fclose(f) == 0;
}

}  // namespace ddm
