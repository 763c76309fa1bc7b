// Seeded synthetic Brownian-particle video (ddm_synth_video in ddm.h).
//
// Random numbers: splitmix64 (Steele, Lea & Flood 2014) for uniforms, the Box-Muller
// transform for normals, and for Poisson shot noise Knuth's product method below mean
// 12 and Hoermann's PTRS transformed rejection (1993) above it. Particle paths come
// from one stream in a fixed order, so a (seed, sizes) pair always gives the same
// video; each frame's noise has its own stream, so frames render in parallel.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/ddm.h"
#include "errors.hpp"

namespace {

struct SplitMix64 {
    uint64_t state;
    explicit SplitMix64(uint64_t seed) : state(seed) {}
    uint64_t next() {
        uint64_t z = (state += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double uniform() { return static_cast<double>(next() >> 11) * 0x1.0p-53; }  // [0, 1)
    bool have_spare = false;
    double spare = 0.0;
    double normal() {  // Box-Muller, both outputs used
        if (have_spare) {
            have_spare = false;
            return spare;
        }
        const double two_pi = 6.283185307179586476925286766559;
        double u1 = 1.0 - uniform();  // (0, 1]
        double u2 = uniform();
        double r = std::sqrt(-2.0 * std::log(u1));
        spare = r * std::sin(two_pi * u2);
        have_spare = true;
        return r * std::cos(two_pi * u2);
    }
    long poisson(double lam) {
        if (lam <= 0) return 0;
        if (lam < 12.0) {  // Knuth: multiply uniforms until below e^-lam
            const double limit = std::exp(-lam);
            double prod = 1.0 - uniform();
            long k = 0;
            while (prod > limit) {
                prod *= 1.0 - uniform();
                k++;
            }
            return k;
        }
        // PTRS, W. Hoermann, "The transformed rejection method for generating Poisson
        // random variables", Insurance: Mathematics and Economics 12 (1993).
        const double slam = std::sqrt(lam), loglam = std::log(lam);
        const double b = 0.931 + 2.53 * slam;
        const double a = -0.059 + 0.02483 * b;
        const double inv_alpha = 1.1239 + 1.1328 / (b - 3.4);
        const double vr = 0.9277 - 3.6224 / (b - 2.0);
        for (;;) {
            double U = uniform() - 0.5;
            double V = uniform();
            double us = 0.5 - std::fabs(U);
            long k = static_cast<long>(std::floor((2.0 * a / us + b) * U + lam + 0.43));
            if (us >= 0.07 && V <= vr) return k;
            if (k < 0 || (us < 0.013 && V > us)) continue;
            if (std::log(V) + std::log(inv_alpha) - std::log(a / (us * us) + b) <=
                -lam + k * loglam - std::lgamma(static_cast<double>(k) + 1.0))
                return k;
        }
    }
};

}  // namespace

extern "C" int ddm_synth_video(uint64_t seed, int W, int H, int frames, int spots,
                               double spot_sigma, double amplitude, double background,
                               double step_var, double step_var_b, double noise_sd,
                               int max_value, void *out) {
    if (W <= 0 || H <= 0 || frames <= 0 || spots < 0 || spot_sigma <= 0 || max_value <= 0 ||
        max_value > 65535 || !out)
        return ddm::fail(DDM_ERR_INVALID_ARG, "ddm_synth_video: invalid argument");
    const int bpp = max_value <= 255 ? 1 : 2;
    // Particle paths, frame-major [frame][spot][x, y], generated serially.
    std::vector<double> pos(static_cast<size_t>(frames) * spots * 2);
    {
        SplitMix64 rng(seed);
        std::vector<double> x(spots), y(spots);
        for (int i = 0; i < spots; i++) {
            x[i] = rng.uniform() * W;
            y[i] = rng.uniform() * H;
        }
        const double sd_a = std::sqrt(step_var), sd_b = std::sqrt(step_var_b);
        for (int f = 0; f < frames; f++) {
            double *p = pos.data() + static_cast<size_t>(f) * spots * 2;
            for (int i = 0; i < spots; i++) {
                p[2 * i] = x[i];
                p[2 * i + 1] = y[i];
            }
            for (int i = 0; i < spots; i++) {
                const double sd = (i < spots - spots / 2) ? sd_a : sd_b;
                x[i] = std::fmod(x[i] + sd * rng.normal(), static_cast<double>(W));
                if (x[i] < 0) x[i] += W;
                y[i] = std::fmod(y[i] + sd * rng.normal(), static_cast<double>(H));
                if (y[i] < 0) y[i] += H;
            }
        }
    }
    const int reach = static_cast<int>(std::ceil(4.0 * spot_sigma));
    const double r2_max = 16.0 * spot_sigma * spot_sigma;
    const double inv_2s2 = 1.0 / (2.0 * spot_sigma * spot_sigma);
    unsigned char *dst = static_cast<unsigned char *>(out);
#pragma omp parallel
    {
        std::vector<double> img(static_cast<size_t>(W) * H);
#pragma omp for schedule(dynamic)
        for (int f = 0; f < frames; f++) {
            std::fill(img.begin(), img.end(), background);
            const double *p = pos.data() + static_cast<size_t>(f) * spots * 2;
            for (int i = 0; i < spots; i++) {
                const double cx = p[2 * i], cy = p[2 * i + 1];
                const int ix0 = static_cast<int>(std::floor(cx)), iy0 = static_cast<int>(std::floor(cy));
                for (int dy = -reach; dy <= reach; dy++) {
                    const int py = iy0 + dy;
                    const double ry = py - cy;
                    const int wy = ((py % H) + H) % H;
                    for (int dx = -reach; dx <= reach; dx++) {
                        const int px = ix0 + dx;
                        const double rx = px - cx;
                        const double r2 = rx * rx + ry * ry;
                        if (r2 > r2_max) continue;
                        const int wx = ((px % W) + W) % W;
                        img[static_cast<size_t>(wy) * W + wx] += amplitude * std::exp(-r2 * inv_2s2);
                    }
                }
            }
            SplitMix64 noise(seed ^ (0xD1B54A32D192ED03ULL * (static_cast<uint64_t>(f) + 1)));
            unsigned char *fr = dst + static_cast<size_t>(f) * W * H * bpp;
            for (size_t k = 0; k < static_cast<size_t>(W) * H; k++) {
                double v = img[k];
                if (noise_sd > 0)
                    v += noise_sd * noise.normal();
                else if (noise_sd < 0)
                    v = static_cast<double>(noise.poisson(v));
                v = std::nearbyint(v);  // round half to even (default rounding mode)
                if (v < 0) v = 0;
                if (v > max_value) v = max_value;
                const unsigned u = static_cast<unsigned>(v);
                if (bpp == 1) {
                    fr[k] = static_cast<unsigned char>(u);
                } else {
                    fr[2 * k] = static_cast<unsigned char>(u & 0xFF);
                    fr[2 * k + 1] = static_cast<unsigned char>(u >> 8);
                }
            }
        }
    }
    return DDM_OK;
}
