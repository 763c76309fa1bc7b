/*
 * FP64 CPU oracle for the multi-scale DDM path. TEST INFRASTRUCTURE ONLY: tests,
 * the smoke check and the CPU-baseline leg of the benchmark may call it, as the
 * checker; the product (libddm_b200.so, the ddm CLI) never links or calls it.
 *
 * It restates, in plain C, what zhangyuyi99/cuda_multiDDM computes on the GPU:
 *   tile extraction           src/DDM_kernel.cuh:43-78  (parseBufferScalePow2)
 *   2-D R2C forward FFT       src/DDM.cu:648-677,189-192 (cuFFT plan/exec), here a
 *                             plain FP64 radix-2 DFT factorisation
 *   chunk/ring schedule       src/DDM.cu:750-843 (simulated symbolically, frame
 *                             labels instead of pixels, so every reference quirk
 *                             of which frame pairs with which is reproduced)
 *   lag accumulation          src/DDM_kernel.cuh:85-101 (processFFT), FP64 here
 *   annulus masks             src/azimuthal_average.cu:229-283 (buildAzimuthMask)
 *                             with q = s/lambda from src/DDM.cu:101-105, evaluated
 *                             in IEEE single precision exactly as the reference
 *   masked azimuthal average  src/azimuthal_average.cu:292-346 (analyseFFTDevice)
 *                             ISF = 2 * sum / pixel_count / frames, FP64 here
 *   -G rolling dumps          src/DDM.cu:800-826
 *
 * Parity pin: the reference has no tests or golden vectors of its own. The oracle
 * is pinned against outputs of the reference program itself, compiled from its
 * sources (oracle/Makefile target `ref`) and run on a GPU host by
 * tests/golden/make_golden.py; the fixtures live in tests/golden/.
 */
#ifndef DDM_ORACLE_H
#define DDM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Pixel decoding. */
#define ORC_PIX_BYTE0 0 /* first byte of each bpp-byte pixel (reference, DDM_kernel.cuh:74-75) */
#define ORC_PIX_U16LE 1 /* full little-endian 16-bit pixel (bpp must be 2) */

/* Estimators. */
#define ORC_EST_COMPAT 0   /* the reference's own pairing schedule, normalised by N */
#define ORC_EST_UNBIASED 1 /* every pair (t, t+tau) with t+tau < N, normalised by N - tau */

/* Frame labels produced by the schedule simulation. */
#define ORC_LABEL_UNINIT (-1) /* device memory the reference never wrote */

/* q radius in pixels of the spectrum for scale s and wavelength lambda (DDM.cu:102). */
float orc_q_radius(int scale, float lambda);

/* Boolean annulus masks [Q][s][s/2+1] and per-q pixel counts, bit-exact to
 * buildAzimuthMask. `mask` may be NULL (counts only). Returns 0. */
int orc_mask_build(int scale, const float *lambda, int lambda_count, float tolerance,
                   unsigned char *mask, int *counts);

/* Tile-major extraction of one frame for scale s: out[tile][ly][lx], tile id
 * (y/s)*(M/s) + x/s, ROI origin (x_off, y_off), ROI side M. */
void orc_extract(const unsigned char *frame, int w, int h, int bpp, int pixmode, int x_off,
                 int y_off, int main_scale, int scale, double *out);

/* Unnormalised forward 2-D R2C DFT of one s x s real tile (sign e^{-i}); output
 * interleaved complex [ky][kx], kx in [0, s/2]. */
void orc_fft2_r2c(const double *in, int scale, double *out);

/* Symbolic run of the reference's chunk loop (DDM.cu:750-843). For every
 * analyseChunk call, in order, writes the A-frame label to A[c] and the B-frame
 * label of each tau to B[c*T + t]. Labels are frame indices counted from the first
 * frame read, or ORC_LABEL_UNINIT. With dump_every = G > 0, epoch[c] counts the
 * accumulator purges that happened before call c, and dump_norm[e] receives the
 * frame count that dump e is normalised by (C*G). Returns the number of calls
 * (K*C + L), or -1 if the arrays are too small. *frames_read receives how many
 * frames the reference reads from its input. */
int orc_compat_schedule(int total_frames, int chunk, int multistream, int dump_every,
                        const int *taus, int tau_count, int max_calls, int *A, int *B,
                        int *epoch, int *frames_read);

/* Whole path on frames in host memory: frames[f] is w*h*bpp bytes, f < nframes.
 * scales sorted descending; taus ascending; lambdas ascending. Writes the final ISF
 * as isf[scale][tile][q][tau] (scales in the given order, tiles in tile order) and,
 * for compat runs with dump_every > 0, each dump into dumps (same layout, one block
 * per dump, up to max_dumps). Returns the number of dumps written, or a negative
 * error. */
int orc_ddm_run(const unsigned char *frames, int nframes, int w, int h, int bpp, int pixmode,
                int x_off, int y_off, const int *scales, int scale_count, const int *taus,
                int tau_count, const float *lambdas, int lambda_count, float tolerance,
                int total_frames, int chunk, int multistream, int estimator, int dump_every,
                double *isf, double *dumps, int max_dumps);

/* As orc_ddm_run without -G dumps, also writing the corrected -K output: for every tau and
 * spectrum element (layout [tau][scale][tile][ky][kx], all scales concatenated),
 * 2 * sum |dF|^2 / s^4 / norm[tau], the per-wave-vector values whose mean over each annulus
 * mask is the ISF (the reference writes raw accumulator rows, src/azimuthal_average.cu:62-106,
 * src/DDM.cu:120-134). */
int orc_ddm_run_unaveraged(const unsigned char *frames, int nframes, int w, int h, int bpp, int pixmode,
                           int x_off, int y_off, const int *scales, int scale_count, const int *taus,
                           int tau_count, const float *lambdas, int lambda_count, float tolerance,
                           int total_frames, int chunk, int multistream, int estimator, double *isf,
                           double *unaveraged);

/* Number of doubles in one ISF block: sum over scales of tiles*Q*T. */
long orc_isf_size(const int *scales, int scale_count, int lambda_count, int tau_count);

/* Masked azimuthal average of one accumulator block acc[tau][tile][k] (k over the
 * s*(s/2+1) half spectrum, values already scaled by 1/s^4), divided per tau by
 * norm[tau]; writes out[tile][q][tau]. */
void orc_azimuthal(const double *acc, int scale, int tiles, int tau_count, const float *lambdas,
                   int lambda_count, float tolerance, const double *norm, double *out);

/* Steady-state throughput sample of the causal (unbiased) path on the CPU: every
 * frame is extracted, transformed at every scale and paired with the frames at each tau
 * before it, FP64, OpenMP over tiles/elements with `threads` threads (0 = all). The ring
 * is first filled with copies of transformed frames, then `warm_frames` frames run
 * untimed, then `timed_frames` frames (frame i of the sample is frames[i % nframes]).
 * Returns the wall time in seconds of the timed frames (summed over the scales, which
 * run one after another). */
double orc_bench_steady(const unsigned char *frames, int nframes, int w, int h, int bpp,
                        int pixmode, const int *scales, int scale_count, const int *taus,
                        int tau_count, int warm_frames, int timed_frames, int threads);

/* 64-bit FNV-1a over n bytes (the hash the reference harness prints for each mask). */
uint64_t orc_fnv1a(const unsigned char *bytes, long n);

/* The synthetic particle video of the benchmark and the tests, restated from the product's
 * generator (ddm_synth_video, same arguments, bit-identical bytes) so that the CPU arms do
 * not load the product library. Returns 0, or a negative error. */
int orc_synth_video(uint64_t seed, int width, int height, int frames, int spots, double spot_sigma,
                    double amplitude, double background, double step_var, double step_var_b,
                    double noise_sd, int max_value, unsigned char *out);

#ifdef __cplusplus
}
#endif
#endif
