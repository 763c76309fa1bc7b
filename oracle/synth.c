/*
 * Seeded synthetic Brownian-particle video for the CPU side of the benchmark -- TEST
 * INFRASTRUCTURE ONLY (the reference arm and the CPU baseline generate their input here, so
 * that neither loads the product library).
 *
 * It restates the product's generator (ddm_synth_video) step for step, so that a (seed,
 * sizes) pair gives the same bytes from both; tests/test_host.py checks that they are
 * bit-identical. Random numbers: splitmix64 (Steele, Lea & Flood 2014) for uniforms,
 * Box-Muller for normals (both outputs used), Poisson by Knuth's product method below
 * mean 12 and Hoermann's PTRS transformed rejection (1993) above it. Particle paths come
 * from one stream in a fixed order; each frame's noise from its own stream.
 */
#include "ddm_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>

typedef struct {
    uint64_t state;
    int have_spare;
    double spare;
} orc_rng;

static uint64_t rng_next(orc_rng *r) {
    uint64_t z = (r->state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static double rng_uniform(orc_rng *r) { return (double)(rng_next(r) >> 11) * 0x1.0p-53; }

static double rng_normal(orc_rng *r) {
    if (r->have_spare) {
        r->have_spare = 0;
        return r->spare;
    }
    const double two_pi = 6.283185307179586476925286766559;
    double u1 = 1.0 - rng_uniform(r);
    double u2 = rng_uniform(r);
    double rad = sqrt(-2.0 * log(u1));
    r->spare = rad * sin(two_pi * u2);
    r->have_spare = 1;
    return rad * cos(two_pi * u2);
}

static long rng_poisson(orc_rng *r, double lam) {
    if (lam <= 0) return 0;
    if (lam < 12.0) {
        const double limit = exp(-lam);
        double prod = 1.0 - rng_uniform(r);
        long k = 0;
        while (prod > limit) {
            prod *= 1.0 - rng_uniform(r);
            k++;
        }
        return k;
    }
    const double slam = sqrt(lam), loglam = log(lam);
    const double b = 0.931 + 2.53 * slam;
    const double a = -0.059 + 0.02483 * b;
    const double inv_alpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    for (;;) {
        double U = rng_uniform(r) - 0.5;
        double V = rng_uniform(r);
        double us = 0.5 - fabs(U);
        long k = (long)floor((2.0 * a / us + b) * U + lam + 0.43);
        if (us >= 0.07 && V <= vr) return k;
        if (k < 0 || (us < 0.013 && V > us)) continue;
        if (log(V) + log(inv_alpha) - log(a / (us * us) + b) <= -lam + k * loglam - lgamma((double)k + 1.0))
            return k;
    }
}

int orc_synth_video(uint64_t seed, int W, int H, int frames, int spots, double spot_sigma, double amplitude,
                    double background, double step_var, double step_var_b, double noise_sd, int max_value,
                    unsigned char *out) {
    if (W <= 0 || H <= 0 || frames <= 0 || spots < 0 || spot_sigma <= 0 || max_value <= 0 || max_value > 65535 ||
        !out)
        return -1;
    const int bpp = max_value <= 255 ? 1 : 2;
    double *pos = (double *)malloc(sizeof(double) * (size_t)frames * (spots > 0 ? spots : 1) * 2);
    double *x = (double *)malloc(sizeof(double) * (spots > 0 ? spots : 1));
    double *y = (double *)malloc(sizeof(double) * (spots > 0 ? spots : 1));
    if (!pos || !x || !y) {
        free(pos);
        free(x);
        free(y);
        return -2;
    }
    orc_rng rng = {seed, 0, 0.0};
    for (int i = 0; i < spots; i++) {
        x[i] = rng_uniform(&rng) * W;
        y[i] = rng_uniform(&rng) * H;
    }
    const double sd_a = sqrt(step_var), sd_b = sqrt(step_var_b);
    for (int f = 0; f < frames; f++) {
        double *p = pos + (size_t)f * spots * 2;
        for (int i = 0; i < spots; i++) {
            p[2 * i] = x[i];
            p[2 * i + 1] = y[i];
        }
        for (int i = 0; i < spots; i++) {
            const double sd = (i < spots - spots / 2) ? sd_a : sd_b;
            x[i] = fmod(x[i] + sd * rng_normal(&rng), (double)W);
            if (x[i] < 0) x[i] += W;
            y[i] = fmod(y[i] + sd * rng_normal(&rng), (double)H);
            if (y[i] < 0) y[i] += H;
        }
    }
    free(x);
    free(y);
    const int reach = (int)ceil(4.0 * spot_sigma);
    const double r2_max = 16.0 * spot_sigma * spot_sigma;
    const double inv_2s2 = 1.0 / (2.0 * spot_sigma * spot_sigma);
    int bad = 0;
#pragma omp parallel
    {
        double *img = (double *)malloc(sizeof(double) * (size_t)W * H);
        if (!img) {
#pragma omp atomic write
            bad = 1;
        }
#pragma omp for schedule(dynamic)
        for (int f = 0; f < frames; f++) {
            if (!img) continue;
            for (size_t k = 0; k < (size_t)W * H; k++) img[k] = background;
            const double *p = pos + (size_t)f * spots * 2;
            for (int i = 0; i < spots; i++) {
                const double cx = p[2 * i], cy = p[2 * i + 1];
                const int ix0 = (int)floor(cx), iy0 = (int)floor(cy);
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
                        img[(size_t)wy * W + wx] += amplitude * exp(-r2 * inv_2s2);
                    }
                }
            }
            orc_rng noise = {seed ^ (0xD1B54A32D192ED03ULL * ((uint64_t)f + 1)), 0, 0.0};
            unsigned char *fr = out + (size_t)f * W * H * bpp;
            for (size_t k = 0; k < (size_t)W * H; k++) {
                double v = img[k];
                if (noise_sd > 0)
                    v += noise_sd * rng_normal(&noise);
                else if (noise_sd < 0)
                    v = (double)rng_poisson(&noise, v);
                v = nearbyint(v);
                if (v < 0) v = 0;
                if (v > max_value) v = max_value;
                const unsigned u = (unsigned)v;
                if (bpp == 1) {
                    fr[k] = (unsigned char)u;
                } else {
                    fr[2 * k] = (unsigned char)(u & 0xFF);
                    fr[2 * k + 1] = (unsigned char)(u >> 8);
                }
            }
        }
        free(img);
    }
    free(pos);
    return bad ? -2 : 0;
}
