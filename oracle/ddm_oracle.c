/*
 * FP64 CPU oracle for the multi-scale DDM path -- TEST INFRASTRUCTURE ONLY (the
 * checker for the CUDA engine; never linked into the product). See ddm_oracle.h for
 * what each function restates and where that code lives in the reference.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off, no fast-math, so that the
 * single-precision mask predicate rounds exactly as the reference's host code).
 */
#include "ddm_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
/* Masks: azimuthal_average.cu:229-283 and DDM.cu:101-105                     */
/* ------------------------------------------------------------------------- */

float orc_q_radius(int scale, float lambda) {
    /* DDM.cu:102: static_cast<float>(scale) / lambda, IEEE single division */
    volatile float s = (float)scale;
    volatile float q = s / lambda;
    return q;
}

int orc_mask_build(int scale, const float *lambda, int lambda_count, float tolerance,
                   unsigned char *mask, int *counts) {
    const int w = scale, h = scale;
    const int nx = w / 2 + 1;
    const long n = (long)nx * h;
    /* azimuthal_average.cu:249: tol2 = tol * tol (float) */
    volatile float tol2 = tolerance * tolerance;
    const int half_w = w / 2, half_h = h / 2;
    for (int qi = 0; qi < lambda_count; qi++) {
        float qr = orc_q_radius(scale, lambda[qi]);
        volatile float q2 = qr * qr; /* azimuthal_average.cu:241-242 */
        int count = 0;
        for (int x = 0; x < nx; x++) {
            for (int y = 0; y < h; y++) {
                /* azimuthal_average.cu:261-269: manual shift to signed frequency */
                int xs = (x + half_w) % w - half_w;
                int ys = (y + half_h) % h - half_h;
                volatile float r2 = (float)(xs * xs + ys * ys);
                volatile float ratio = r2 / q2;
                int px = (1.0f <= ratio) && (ratio <= tol2);
                count += px;
                if (mask) mask[qi * n + (long)y * nx + x] = (unsigned char)px;
            }
        }
        counts[qi] = count;
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Extraction: DDM_kernel.cuh:43-78                                           */
/* ------------------------------------------------------------------------- */

static inline double pixel_value(const unsigned char *p, int pixmode) {
    if (pixmode == ORC_PIX_U16LE) return (double)((unsigned)p[0] | ((unsigned)p[1] << 8));
    return (double)p[0];
}

void orc_extract(const unsigned char *frame, int w, int h, int bpp, int pixmode, int x_off,
                 int y_off, int main_scale, int scale, double *out) {
    (void)h;
    const int tiles_side = main_scale / scale;
    for (int y = 0; y < main_scale; y++) {
        for (int x = 0; x < main_scale; x++) {
            int tile = (y / scale) * tiles_side + (x / scale);
            int ly = y % scale, lx = x % scale;
            const unsigned char *p = frame + (size_t)bpp * ((size_t)(y + y_off) * w + (x + x_off));
            out[(size_t)tile * scale * scale + (size_t)ly * scale + lx] = pixel_value(p, pixmode);
        }
    }
}

/* ------------------------------------------------------------------------- */
/* FP64 FFT (stands in for cuFFT's R2C plan, DDM.cu:648-677)                   */
/* ------------------------------------------------------------------------- */

static void twiddles(int n, double *tw) {
    const double two_pi = 6.283185307179586476925286766559;
    for (int m = 0; m < n / 2; m++) {
        double a = two_pi * (double)m / (double)n;
        tw[2 * m] = cos(a);
        tw[2 * m + 1] = sin(a);
    }
}

/* In-place iterative radix-2 forward DFT, X[k] = sum x[j] e^{-2 pi i jk/n}. */
static void fft1d(double *z, int n, const double *tw) {
    for (int i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double tr = z[2 * i], ti = z[2 * i + 1];
            z[2 * i] = z[2 * j];
            z[2 * i + 1] = z[2 * j + 1];
            z[2 * j] = tr;
            z[2 * j + 1] = ti;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len / 2, step = n / len;
        for (int i = 0; i < n; i += len) {
            for (int k = 0; k < half; k++) {
                double wr = tw[2 * (k * step)], wi = -tw[2 * (k * step) + 1];
                double *u = z + 2 * (i + k), *v = z + 2 * (i + k + half);
                double vr = v[0] * wr - v[1] * wi, vi = v[0] * wi + v[1] * wr;
                v[0] = u[0] - vr;
                v[1] = u[1] - vi;
                u[0] += vr;
                u[1] += vi;
            }
        }
    }
}

void orc_fft2_r2c(const double *in, int s, double *out) {
    const int nx = s / 2 + 1;
    double *tw = (double *)malloc(sizeof(double) * s);
    double *row = (double *)malloc(sizeof(double) * 2 * s);
    double *half = (double *)malloc(sizeof(double) * 2 * (size_t)s * nx);
    twiddles(s, tw);
    for (int y = 0; y < s; y++) {
        for (int x = 0; x < s; x++) {
            row[2 * x] = in[(size_t)y * s + x];
            row[2 * x + 1] = 0.0;
        }
        fft1d(row, s, tw);
        memcpy(half + 2 * (size_t)y * nx, row, sizeof(double) * 2 * nx);
    }
    for (int kx = 0; kx < nx; kx++) {
        for (int y = 0; y < s; y++) {
            row[2 * y] = half[2 * ((size_t)y * nx + kx)];
            row[2 * y + 1] = half[2 * ((size_t)y * nx + kx) + 1];
        }
        fft1d(row, s, tw);
        for (int ky = 0; ky < s; ky++) {
            out[2 * ((size_t)ky * nx + kx)] = row[2 * ky];
            out[2 * ((size_t)ky * nx + kx) + 1] = row[2 * ky + 1];
        }
    }
    free(tw);
    free(row);
    free(half);
}

/* ------------------------------------------------------------------------- */
/* Schedule: DDM.cu:750-843, run on frame labels                              */
/* ------------------------------------------------------------------------- */

typedef struct {
    int cursor;
} reader_t;

static void load_labels(reader_t *r, int *h, int count) { /* loadVideoToHost, DDM.cu:752 */
    for (int j = 0; j < count; j++) h[j] = r->cursor++;
}

static void copy_labels(int *dst, const int *src, int count) { /* H2D copy + parseChunk */
    for (int j = 0; j < count; j++) dst[j] = src[j];
}

int orc_compat_schedule(int N, int C, int multistream, int G, const int *taus, int T,
                        int max_calls, int *A, int *B, int *epoch, int *frames_read) {
    if (C <= 0 || N < 0) return -1;
    const int K = N / C, L = N % C;
    if (K * C + L > max_calls) return -1;
    int *lab = (int *)malloc(sizeof(int) * 5 * C);
    for (int j = 0; j < 5 * C; j++) lab[j] = ORC_LABEL_UNINIT;
    int *h1 = lab, *h2 = multistream ? lab + C : lab;
    int *start = lab + 2 * C, *end = lab + 3 * C, *junk = lab + 4 * C;
    int *h_cur = h1, *h_nxt = h2;
    reader_t rd = {0};
    int ncalls = 0, ep = 0;

    load_labels(&rd, h_nxt, C); /* DDM.cu:752-753 */
    load_labels(&rd, h_cur, C);
    copy_labels(start, h_nxt, C); /* DDM.cu:755-760 */

#define EMIT(fo_)                                                                    \
    do {                                                                             \
        int fo__ = (fo_), left__ = C - fo__;                                         \
        A[ncalls] = start[fo__];                                                     \
        for (int t = 0; t < T; t++) /* DDM.cu:250-255 */                            \
            B[(long)ncalls * T + t] =                                                \
                taus[t] < left__ ? start[fo__ + taus[t]] : end[taus[t] - left__];    \
        if (epoch) epoch[ncalls] = ep;                                               \
        ncalls++;                                                                    \
    } while (0)

    for (int i = 0; i < K; i++) { /* DDM.cu:765-827 */
        copy_labels(end, h_cur, C);
        for (int fo = 0; fo < C; fo++) EMIT(fo);
        if (K - i > 2)
            load_labels(&rd, h_nxt, C);
        else if (L != 0 && K - i == 2)
            load_labels(&rd, h_nxt, L);
        {
            int *t = h_cur; /* DDM.cu:788 */
            h_cur = h_nxt;
            h_nxt = t;
        }
        {
            int *t = junk; /* DDM.cu:793 rotateThreePtr(junk, start, end) */
            junk = start;
            start = end;
            end = t;
        }
        if (G != 0 && i != 0 && i % G == 0) ep++; /* DDM.cu:800-826 */
    }
    if (L != 0) { /* DDM.cu:830-843 */
        copy_labels(end, h_cur, L);
        for (int fo = 0; fo < L; fo++) EMIT(fo);
    }
#undef EMIT
    if (frames_read) *frames_read = rd.cursor;
    free(lab);
    return ncalls;
}

/* ------------------------------------------------------------------------- */
/* Azimuthal average: azimuthal_average.cu:292-346 with DDM.cu:72-146          */
/* ------------------------------------------------------------------------- */

void orc_azimuthal(const double *acc, int scale, int tiles, int T, const float *lambdas, int Q,
                   float tolerance, const double *norm, double *out) {
    const long n = (long)scale * (scale / 2 + 1);
    unsigned char *mask = (unsigned char *)malloc((size_t)Q * n);
    int *counts = (int *)malloc(sizeof(int) * Q);
    orc_mask_build(scale, lambdas, Q, tolerance, mask, counts);
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int tile = 0; tile < tiles; tile++) {
        for (int q = 0; q < Q; q++) {
            for (int t = 0; t < T; t++) {
                double v = 0.0;
                if (counts[q] != 0 && norm[t] != 0.0) {
                    const double *a = acc + ((long)t * tiles + tile) * n;
                    const unsigned char *m = mask + (long)q * n;
                    double sum = 0.0;
                    for (long k = 0; k < n; k++)
                        if (m[k]) sum += a[k];
                    v = 2.0 * sum / (double)counts[q] / norm[t];
                }
                out[((long)tile * Q + q) * T + t] = v;
            }
        }
    }
    free(mask);
    free(counts);
}

long orc_isf_size(const int *scales, int S, int Q, int T) {
    long total = 0;
    for (int s = 0; s < S; s++) {
        long side = scales[0] / scales[s];
        total += side * side * Q * T;
    }
    return total;
}

/* ------------------------------------------------------------------------- */
/* Whole path                                                                 */
/* ------------------------------------------------------------------------- */

/* spectra[f][tile][k] (interleaved complex) of frames 0..nf-1 at one scale */
static double *transform_frames(const unsigned char *frames, int nf, int w, int h, int bpp,
                                int pixmode, int x_off, int y_off, int M, int s) {
    const int tiles = (M / s) * (M / s);
    const long n = (long)s * (s / 2 + 1);
    const size_t frame_bytes = (size_t)w * h * bpp;
    double *spec = (double *)malloc(sizeof(double) * 2 * (size_t)nf * tiles * n);
    if (!spec) return NULL;
#pragma omp parallel
    {
        double *px = (double *)malloc(sizeof(double) * (size_t)M * M);
#pragma omp for schedule(dynamic)
        for (int f = 0; f < nf; f++) {
            orc_extract(frames + frame_bytes * f, w, h, bpp, pixmode, x_off, y_off, M, s, px);
            for (int tile = 0; tile < tiles; tile++)
                orc_fft2_r2c(px + (size_t)tile * s * s, s,
                             spec + 2 * (((size_t)f * tiles + tile) * n));
        }
        free(px);
    }
    return spec;
}

static void accumulate_pair(double *acc_t, const double *fa, const double *fb, long count,
                            double inv_s4) {
#pragma omp parallel for schedule(static)
    for (long k = 0; k < count; k++) {
        double dr = fa[2 * k] - fb[2 * k], di = fa[2 * k + 1] - fb[2 * k + 1];
        acc_t[k] += (dr * dr + di * di) * inv_s4;
    }
}

static int ddm_run_impl(const unsigned char *frames, int nframes, int w, int h, int bpp, int pixmode,
                        int x_off, int y_off, const int *scales, int S, const int *taus, int T,
                        const float *lambdas, int Q, float tolerance, int N, int C, int multistream,
                        int estimator, int G, double *isf, double *dumps, int max_dumps, double *unav) {
    const int M = scales[0];
    long E_all = 0; /* complex elements per frame over all scales (unaveraged layout) */
    for (int si = 0; si < S; si++) E_all += (long)(M / scales[si]) * (M / scales[si]) * scales[si] * (scales[si] / 2 + 1);
    long e_off = 0;
    if (M + x_off > w || M + y_off > h) return -2;
    int ncalls_max = N + C;
    int *A = NULL, *B = NULL, *ep = NULL;
    int ncalls = 0, need = N, ndumps = 0;
    if (estimator == ORC_EST_COMPAT) {
        A = (int *)malloc(sizeof(int) * ncalls_max);
        B = (int *)malloc(sizeof(int) * (size_t)ncalls_max * T);
        ep = (int *)malloc(sizeof(int) * ncalls_max);
        ncalls = orc_compat_schedule(N, C, multistream, G, taus, T, ncalls_max, A, B, ep, &need);
        if (ncalls < 0) return -3;
        ndumps = ncalls > 0 ? ep[ncalls - 1] : 0;
    }
    if (need > nframes) {
        free(A);
        free(B);
        free(ep);
        return -4;
    }
    const long isf_block = orc_isf_size(scales, S, Q, T);
    long isf_off = 0;
    double *norm = (double *)malloc(sizeof(double) * T);
    for (int si = 0; si < S; si++) {
        const int s = scales[si];
        const int tiles = (M / s) * (M / s);
        const long n = (long)s * (s / 2 + 1);
        const long fsz = tiles * n; /* complex elements per frame at this scale */
        const double inv_s4 = 1.0 / ((double)s * s * (double)s * s);
        double *spec = transform_frames(frames, need, w, h, bpp, pixmode, x_off, y_off, M, s);
        double *acc = (double *)calloc((size_t)T * fsz, sizeof(double));
        if (!spec || !acc) return -5;
        if (estimator == ORC_EST_COMPAT) {
            int cur_ep = 0;
            for (int c = 0; c < ncalls; c++) {
                if (ep[c] != cur_ep) { /* a -G dump happened before this call */
                    if (dumps && cur_ep < max_dumps) {
                        for (int t = 0; t < T; t++) norm[t] = (double)C * G;
                        orc_azimuthal(acc, s, tiles, T, lambdas, Q, tolerance, norm,
                                      dumps + (long)cur_ep * isf_block + isf_off);
                    }
                    memset(acc, 0, sizeof(double) * T * fsz);
                    cur_ep = ep[c];
                }
                if (A[c] < 0) continue;
                for (int t = 0; t < T; t++) {
                    int b = B[(long)c * T + t];
                    if (b < 0) continue; /* reference reads never-written memory here */
                    accumulate_pair(acc + (long)t * fsz, spec + 2 * (size_t)A[c] * fsz,
                                    spec + 2 * (size_t)b * fsz, fsz, inv_s4);
                }
            }
            for (int t = 0; t < T; t++) norm[t] = (double)N; /* DDM.cu:875, :92 */
        } else {
            /* Every pair (a, a + tau) with a + tau < N. Blocked over elements so that a block's
             * frames stay in cache across all taus; each element still adds its pairs tau by tau,
             * a ascending, so the sums are those of the plain loop bit for bit. */
            const long KB = 256;
#pragma omp parallel for schedule(dynamic)
            for (long k0 = 0; k0 < fsz; k0 += KB) {
                const long k1 = k0 + KB < fsz ? k0 + KB : fsz;
                for (int t = 0; t < T; t++) {
                    double *at = acc + (long)t * fsz;
                    for (int a = 0; a + taus[t] < N; a++) {
                        const double *fa = spec + 2 * (size_t)a * fsz, *fb = spec + 2 * (size_t)(a + taus[t]) * fsz;
                        for (long k = k0; k < k1; k++) {
                            double dr = fa[2 * k] - fb[2 * k], di = fa[2 * k + 1] - fb[2 * k + 1];
                            at[k] += (dr * dr + di * di) * inv_s4;
                        }
                    }
                }
            }
            for (int t = 0; t < T; t++) norm[t] = N - taus[t] > 0 ? (double)(N - taus[t]) : 0.0;
        }
        orc_azimuthal(acc, s, tiles, T, lambdas, Q, tolerance, norm, isf + isf_off);
        isf_off += (long)tiles * Q * T;
        if (unav) { /* 2 * mean |dF|^2 / s^4 per element: its annulus means are the ISF */
            for (int t = 0; t < T; t++)
                for (long k = 0; k < fsz; k++)
                    unav[(long)t * E_all + e_off + k] = norm[t] > 0.0 ? 2.0 * acc[(long)t * fsz + k] / norm[t] : 0.0;
        }
        e_off += fsz;
        free(spec);
        free(acc);
    }
    free(norm);
    free(A);
    free(B);
    free(ep);
    return ndumps < max_dumps ? ndumps : max_dumps;
}

int orc_ddm_run(const unsigned char *frames, int nframes, int w, int h, int bpp, int pixmode,
                int x_off, int y_off, const int *scales, int S, const int *taus, int T,
                const float *lambdas, int Q, float tolerance, int N, int C, int multistream,
                int estimator, int G, double *isf, double *dumps, int max_dumps) {
    return ddm_run_impl(frames, nframes, w, h, bpp, pixmode, x_off, y_off, scales, S, taus, T, lambdas, Q,
                        tolerance, N, C, multistream, estimator, G, isf, dumps, max_dumps, NULL);
}

int orc_ddm_run_unaveraged(const unsigned char *frames, int nframes, int w, int h, int bpp, int pixmode,
                           int x_off, int y_off, const int *scales, int S, const int *taus, int T,
                           const float *lambdas, int Q, float tolerance, int N, int C, int multistream,
                           int estimator, double *isf, double *unav) {
    return ddm_run_impl(frames, nframes, w, h, bpp, pixmode, x_off, y_off, scales, S, taus, T, lambdas, Q,
                        tolerance, N, C, multistream, estimator, 0, isf, NULL, 0, unav);
}

/* ------------------------------------------------------------------------- */
/* CPU throughput sample (benchmark baseline)                                 */
/* ------------------------------------------------------------------------- */

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

double orc_bench_steady(const unsigned char *frames, int nframes, int w, int h, int bpp,
                        int pixmode, const int *scales, int S, const int *taus, int T,
                        int warm_frames, int timed_frames, int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    const int M = scales[0];
    const int tau_max = taus[T - 1];
    const int R = tau_max + 1;
    const size_t frame_bytes = (size_t)w * h * bpp;
    double total = 0.0;
    for (int si = 0; si < S; si++) {
        const int s = scales[si];
        const int tiles = (M / s) * (M / s);
        const long n = (long)s * (s / 2 + 1);
        const long fsz = tiles * n;
        const double inv_s4 = 1.0 / ((double)s * s * (double)s * s);
        double *ring = (double *)malloc(sizeof(double) * 2 * (size_t)R * fsz);
        double *acc = (double *)calloc((size_t)T * fsz, sizeof(double));
        double *px = (double *)malloc(sizeof(double) * (size_t)M * M);
        if (!ring || !acc || !px) {
            free(ring);
            free(acc);
            free(px);
            return -1.0;
        }
        /* untimed warm ring: a few transformed frames copied round the ring */
        int warm = nframes < 4 ? nframes : 4;
        for (int f = 0; f < warm; f++) {
            orc_extract(frames + frame_bytes * f, w, h, bpp, pixmode, 0, 0, M, s, px);
#pragma omp parallel for schedule(dynamic)
            for (int tile = 0; tile < tiles; tile++)
                orc_fft2_r2c(px + (size_t)tile * s * s, s, ring + 2 * ((size_t)f * fsz + tile * n));
        }
        for (int f = warm; f < R; f++)
            memcpy(ring + 2 * (size_t)f * fsz, ring + 2 * (size_t)(f % warm) * fsz,
                   sizeof(double) * 2 * fsz);
        double t0 = 0.0;
        for (int i = 0; i < warm_frames + timed_frames; i++) {
            if (i == warm_frames) t0 = now_s();
            const int b = R + i; /* frame number; ring slot b % R */
            double *fb = ring + 2 * (size_t)(b % R) * fsz;
            orc_extract(frames + frame_bytes * (i % nframes), w, h, bpp, pixmode, 0, 0, M, s, px);
#pragma omp parallel for schedule(dynamic)
            for (int tile = 0; tile < tiles; tile++)
                orc_fft2_r2c(px + (size_t)tile * s * s, s, fb + 2 * (size_t)tile * n);
            for (int t = 0; t < T; t++)
                accumulate_pair(acc + (long)t * fsz, fb,
                                ring + 2 * (size_t)((b - taus[t]) % R) * fsz, fsz, inv_s4);
        }
        total += now_s() - t0;
        free(ring);
        free(acc);
        free(px);
    }
    return total;
}

/* FNV-1a (64-bit) over n bytes: the hash the reference harness prints for each mask. */
uint64_t orc_fnv1a(const unsigned char *bytes, long n) {
    uint64_t h = 1469598103934665603ULL;
    for (long i = 0; i < n; i++) {
        h ^= bytes[i];
        h *= 1099511628211ULL;
    }
    return h;
}
