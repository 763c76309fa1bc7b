// On-device ISF fitting: the analysis the reference leaves to a Python script
// (resources/python_tools/plot_averaged.py:61-141), run on the GPU so that a stream's
// caller gets decay rates and diffusion coefficients without reading ISF files.
//
//   fit_mean_kernel   tile-averaged ISF per (scale, lambda, tau) (the script's ISF_scale,
//                     plot_averaged.py:246-252)
//   fit_isf_kernel    one thread per curve: I(tau) = A (1 - exp(-F tau)) + B (fit_func,
//                     :57-58) by Levenberg-Marquardt in FP64, from the script's fixed starting
//                     point p0 = (F, A, B) = (6, 0.03, 0.004) (:77) or from one read off the
//                     curve (fit_start_from_data), with the covariance scaling of
//                     scipy.optimize.curve_fit (absolute_sigma = False): cov = (J^T J)^-1 *
//                     RSS / (T - 3), errors = sqrt(diag(cov)) (:82)
//   fit_diffusion_kernel  ln F = ln D + 2 ln q over the lambdas with F > 0 (plot_diff_coeff,
//                     :93-136): with the slope fixed at 2 the least-squares intercept is the
//                     mean of ln F - 2 ln q, its variance the residual variance / n; q =
//                     2 pi / (lambda * um_per_px) (:261)
//
// The Levenberg-Marquardt iteration is the textbook one (Marquardt 1963): solve
// (J^T J + mu diag(J^T J)) d = -J^T r, accept the step if the cost falls (mu / 10), else
// retry with mu * 10; stop when a step changes the cost by less than 1e-15 of itself or the
// parameters by less than 1e-13 of themselves, or after kFitMaxIter iterations. The model's
// Jacobian is analytic. exp arguments are capped at 700, as the script's where= guard does.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ddm {

constexpr int kFitThreads = 128;
constexpr int kFitMaxIter = 400;
constexpr int kFitParams = 6;  // F, A, B, sigma_F, sigma_A, sigma_B per curve

struct FitArgs {
    int S, T, Q;
    int start;              // 0: from the curve (fit_start_from_data), 1: the script's p0
    int tiles[16];          // per scale
    long long isf_off[16];  // per scale, first bin of the scale in the ISF [scale][tile][q][tau]
    int curve_off[16];      // per scale, first tile curve of the scale
    int tile_curves;        // sum over scales of tiles * Q
    const double *isf;      // [bins]
    double *mean;           // [S][Q][T] tile-averaged ISF
    const double *tau;      // [T] lag times (seconds, or frames)
    const double *q;        // [Q] wave vectors 2 pi / (lambda um_per_px)
    double *tile_fit;       // [tile_curves][6]
    double *scale_fit;      // [S * Q][6]
    double *tile_d;         // [sum tiles][2]: D, sigma_D
    double *scale_d;        // [S][2]
};

__global__ void fit_mean_kernel(FitArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // (scale, q, tau)
    if (i >= a.S * a.Q * a.T) return;
    const int si = i / (a.Q * a.T), qt = i - si * a.Q * a.T;
    const double *p = a.isf + a.isf_off[si] + qt;  // tile 0; tiles are Q*T apart
    double s = 0.0;
    for (int t = 0; t < a.tiles[si]; t++) s += p[static_cast<long long>(t) * a.Q * a.T];
    a.mean[i] = s / a.tiles[si];
}

__device__ __forceinline__ double fit_exp(double x) { return exp(x < 700.0 ? x : 700.0); }

// Sum of squared residuals of (F, A, B) over the curve, and optionally J^T J and J^T r.
__device__ double fit_eval(const double *y, const double *tau, int T, const double p[3], double H[6],
                           double g[3], bool jac) {
    double cost = 0.0;
    if (jac) {
        for (int i = 0; i < 6; i++) H[i] = 0.0;
        for (int i = 0; i < 3; i++) g[i] = 0.0;
    }
    for (int i = 0; i < T; i++) {
        const double e = fit_exp(-p[0] * tau[i]);
        const double r = p[1] * (1.0 - e) + p[2] - y[i];
        cost += r * r;
        if (jac) {
            const double j0 = p[1] * tau[i] * e, j1 = 1.0 - e, j2 = 1.0;
            H[0] += j0 * j0, H[1] += j0 * j1, H[2] += j0 * j2;  // symmetric 3x3: 00 01 02 11 12 22
            H[3] += j1 * j1, H[4] += j1 * j2, H[5] += j2 * j2;
            g[0] += j0 * r, g[1] += j1 * r, g[2] += j2 * r;
        }
    }
    return cost;
}

// Solves the symmetric 3x3 system M x = b by Cramer's rule; false if singular.
__device__ bool fit_solve3(const double M[6], const double b[3], double x[3]) {
    const double a00 = M[0], a01 = M[1], a02 = M[2], a11 = M[3], a12 = M[4], a22 = M[5];
    const double c00 = a11 * a22 - a12 * a12, c01 = a02 * a12 - a01 * a22, c02 = a01 * a12 - a02 * a11;
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    if (!(fabs(det) > 0.0) || !isfinite(det)) return false;
    const double c11 = a00 * a22 - a02 * a02, c12 = a01 * a02 - a00 * a12, c22 = a00 * a11 - a01 * a01;
    x[0] = (c00 * b[0] + c01 * b[1] + c02 * b[2]) / det;
    x[1] = (c01 * b[0] + c11 * b[1] + c12 * b[2]) / det;
    x[2] = (c02 * b[0] + c12 * b[1] + c22 * b[2]) / det;
    return true;
}

// A start that works whatever the units of tau and I: the script's fixed p0 suits lag times
// in seconds and decay rates of a few per second only (from it, a curve whose F tau is large
// at the first lag has no F gradient and stalls). B from the first point, A from the largest
// rise above it, F = ln 2 over the first lag that reaches half the rise.
__device__ void fit_start_from_data(const double *y, const double *tau, int T, double p[3]) {
    const double b = y[0];
    double top = y[0];
    for (int i = 1; i < T; i++) top = fmax(top, y[i]);
    const double a = top - b > 0.0 ? top - b : fmax(fabs(b), 1e-300);
    double t_half = tau[T - 1];
    for (int i = 0; i < T; i++)
        if (y[i] >= b + 0.5 * a) {
            t_half = tau[i];
            break;
        }
    p[0] = 0.6931471805599453 / fmax(t_half, 1e-300);
    p[1] = a;
    p[2] = b;
}

__device__ void fit_curve(const double *y, const double *tau, int T, int start, double out[kFitParams]) {
    double p[3] = {6.0, 3e-2, 4e-3};  // plot_averaged.py:77
    if (start == 0) fit_start_from_data(y, tau, T, p);
    double H[6], g[3];
    double cost = fit_eval(y, tau, T, p, H, g, true);
    double mu = 1e-3;
    for (int it = 0; it < kFitMaxIter; it++) {
        bool accepted = false, done = false;
        while (mu < 1e20) {
            double M[6] = {H[0] * (1.0 + mu), H[1], H[2], H[3] * (1.0 + mu), H[4], H[5] * (1.0 + mu)};
            const double b[3] = {-g[0], -g[1], -g[2]};
            double d[3];
            if (!fit_solve3(M, b, d)) {
                mu *= 10.0;
                continue;
            }
            const double pn[3] = {p[0] + d[0], p[1] + d[1], p[2] + d[2]};
            double Hn[6], gn[3];
            const double cn = fit_eval(y, tau, T, pn, Hn, gn, true);
            if (isfinite(cn) && cn <= cost) {
                const bool small_step = fabs(d[0]) <= 1e-13 * fabs(p[0]) && fabs(d[1]) <= 1e-13 * fabs(p[1]) &&
                                        fabs(d[2]) <= 1e-13 * (fabs(p[2]) + 1e-300);
                done = (cost - cn) <= 1e-15 * cost || small_step;
                for (int i = 0; i < 3; i++) p[i] = pn[i], g[i] = gn[i];
                for (int i = 0; i < 6; i++) H[i] = Hn[i];
                cost = cn;
                mu = fmax(mu * 0.1, 1e-15);
                accepted = true;
                break;
            }
            mu *= 10.0;
        }
        if (!accepted || done) break;
    }
    out[0] = p[0], out[1] = p[1], out[2] = p[2];
    // covariance (J^T J)^-1 * RSS / (T - 3): the diagonal of the inverse from the cofactors
    const double a00 = H[0], a01 = H[1], a02 = H[2], a11 = H[3], a12 = H[4], a22 = H[5];
    const double c00 = a11 * a22 - a12 * a12, c11 = a00 * a22 - a02 * a02, c22 = a00 * a11 - a01 * a01;
    const double det = a00 * c00 + a01 * (a02 * a12 - a01 * a22) + a02 * (a01 * a12 - a02 * a11);
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    if (T > 3 && fabs(det) > 0.0 && isfinite(det)) {
        const double s2 = cost / (T - 3);
        out[3] = sqrt(fabs(c00 / det) * s2), out[4] = sqrt(fabs(c11 / det) * s2), out[5] = sqrt(fabs(c22 / det) * s2);
    } else {
        out[3] = out[4] = out[5] = inf;
    }
}

__global__ void fit_isf_kernel(FitArgs a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int total = a.tile_curves + a.S * a.Q;
    if (c >= total) return;
    const double *y;
    double *out;
    if (c < a.tile_curves) {
        int si = 0;
        while (si + 1 < a.S && c >= a.curve_off[si + 1]) si++;
        const int rel = c - a.curve_off[si];  // tile * Q + q
        y = a.isf + a.isf_off[si] + static_cast<long long>(rel) * a.T;
        out = a.tile_fit + static_cast<long long>(c) * kFitParams;
    } else {
        const int sc = c - a.tile_curves;  // scale * Q + q
        y = a.mean + static_cast<long long>(sc) * a.T;
        out = a.scale_fit + static_cast<long long>(sc) * kFitParams;
    }
    double r[kFitParams];
    fit_curve(y, a.tau, a.T, a.start, r);
    for (int i = 0; i < kFitParams; i++) out[i] = r[i];
}

// One thread per (scale, tile) and per scale: D from the Q decay rates of its curves.
__global__ void fit_diffusion_kernel(FitArgs a, int tiles_total) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= tiles_total + a.S) return;
    const double *fits;
    double *out;
    if (i < tiles_total) {
        fits = a.tile_fit + static_cast<long long>(i) * a.Q * kFitParams;  // tile curves are [tile][q]
        out = a.tile_d + 2 * i;
    } else {
        fits = a.scale_fit + static_cast<long long>(i - tiles_total) * a.Q * kFitParams;
        out = a.scale_d + 2 * (i - tiles_total);
    }
    double sum = 0.0;
    int n = 0;
    for (int q = 0; q < a.Q; q++) {
        const double F = fits[q * kFitParams];
        if (F > 0.0 && isfinite(F)) sum += log(F) - 2.0 * log(a.q[q]), n++;
    }
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    if (n == 0) {
        out[0] = nan, out[1] = nan;
        return;
    }
    const double c = sum / n;
    double rss = 0.0;
    for (int q = 0; q < a.Q; q++) {
        const double F = fits[q * kFitParams];
        if (F > 0.0 && isfinite(F)) {
            const double r = log(F) - 2.0 * log(a.q[q]) - c;
            rss += r * r;
        }
    }
    const double c_err = n > 1 ? sqrt(rss / (n - 1) / n) : inf;
    out[0] = exp(c);
    out[1] = c_err * out[0];
}

}  // namespace ddm
