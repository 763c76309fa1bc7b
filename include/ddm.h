/*
 * ddm.h -- C ABI of the B200 multi-scale DDM engine (libddm_b200.so).
 *
 * The engine computes the image structure function D(q, tau) of a video at several
 * tile scales at once: every frame's square region of interest (side M = largest
 * scale) is cut into (M/s)^2 tiles per scale s, each tile gets a 2-D R2C FFT, the
 * spectra of the last frames stay in a device-resident ring, |F(t+tau) - F(t)|^2 is
 * accumulated per (tau, tile, k), and a masked azimuthal average over the annulus
 * |k| in [q, tol*q] (q = s/lambda) turns each (scale, tile) into ISF[lambda][tau].
 *
 * The reference program (zhangyuyi99/cuda_multiDDM) has no library API: everything
 * lives in one 24-argument function, runDDM (src/DDM.cu:268-292), driven by the ./ddm
 * command line (src/main.cpp). Each entry point below names the part of that program
 * it replaces. All calls return a ddm_status (0 = success) instead of exiting the
 * process (src/debug.cpp:10-15,33-45). The engine owns all device memory it
 * allocates; the caller owns every host buffer and every device buffer it passes in.
 * One engine is used from one host thread at a time.
 */
#ifndef DDM_B200_H
#define DDM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    DDM_OK = 0,
    DDM_ERR_INVALID_ARG = 1,   /* a parameter is out of range; see ddm_last_error() */
    DDM_ERR_CUDA = 2,          /* a CUDA runtime call failed */
    DDM_ERR_OUT_OF_MEMORY = 3, /* device allocation failed or the HBM budget is exceeded */
    DDM_ERR_STATE = 4,         /* call not valid in the engine's current state */
    DDM_ERR_NEED_FRAMES = 5,   /* finalize needs frames that were never submitted */
    DDM_ERR_NO_DEVICE = 6,     /* no CUDA device, or not an sm_100 device */
    DDM_ERR_IO = 7,            /* file could not be read or written */
    DDM_ERR_BUSY = 8           /* a server cannot admit the stream now; retry once streams leave */
} ddm_status;

/* How a source pixel becomes the FFT input value. */
typedef enum {
    DDM_PIX_BYTE0 = 0, /* first byte of each bytes_per_pixel-byte pixel: what the reference
                          does for every input, 16-bit included (src/DDM_kernel.cuh:74-75) */
    DDM_PIX_U16LE = 1  /* full little-endian 16-bit value (bytes_per_pixel must be 2) */
} ddm_pixel_mode;

/* Which frame pairs enter the accumulators and how each tau is normalised. */
typedef enum {
    DDM_EST_COMPAT = 0,  /* the reference's own schedule (src/DDM.cu:750-843), including which
                            frame each tail frame pairs with, normalised by N (src/DDM.cu:875);
                            needs total_frames and tau_max <= chunk_frames */
    DDM_EST_UNBIASED = 1 /* every pair (t, t+tau) with t + tau < frames seen, normalised by the
                            number of such pairs; no limit on tau_max */
} ddm_estimator;

typedef struct {
    int frame_width, frame_height; /* source frame size in pixels */
    int bytes_per_pixel;           /* 1 or 2 (also the channel stride for DDM_PIX_BYTE0) */
    int pixel_mode;                /* ddm_pixel_mode */
    int x_offset, y_offset;        /* ROI origin in the source frame (-x, -y) */
    const int *scales;             /* tile sides, powers of two (any order; sorted descending) */
    int scale_count;
    const int *taus;               /* lags in frames (any order; sorted ascending) */
    int tau_count;
    const float *lambdas;          /* wavelengths in pixels (any order; sorted ascending) */
    int lambda_count;
    float tolerance;               /* annulus outer radius / inner radius (reference default 1.2f) */
    int chunk_frames;              /* C: frames per ingest step (-C) */
    int estimator;                 /* ddm_estimator */
    int multistream;               /* compat only: 1 = reference default, 0 = its -Z schedule */
    int total_frames;              /* N (-N); required for DDM_EST_COMPAT, 0 = open-ended */
    int dump_every;                /* G (-G): ISF snapshot + accumulator purge every G chunks */
    size_t hbm_budget_bytes;       /* refuse to open if the engine would need more; 0 = no limit */
    int device;                    /* CUDA device ordinal */
    void *stream;                  /* cudaStream_t to run on; NULL = the engine creates one */
    int lag_batch_frames;          /* frames paired per lag launch, 1..64. Unbiased (0 = 32):
                                      up to lag_batch_frames - 1 frames may wait in the ring
                                      for a fuller launch (fuller launches read fewer partner
                                      bytes per frame); finalize/synchronize pair them. Compat
                                      (0 = min(C, 32)): A-frames per launch. -1: the value
                                      ddm_autotune cached for this shape in the file named by
                                      the DDM_TUNE_CACHE environment variable, else as 0. */
    int small_tile_dft;            /* 1: tiles of side 32, 64 and 128 are transformed by the
                                      split-BF16 tensor-core DFT (BF16 hi/lo operands, FP32
                                      accumulation; spectra within ~1e-5 of the tile maximum,
                                      ISF within 1e-3) instead of the FP32 FFT; 0: FP32 FFT for
                                      every scale (the reference uses cuFFT in FP32 for all,
                                      src/DDM.cu:648-677). Other scales always use the FP32 FFT. */
    int lag_geometry;              /* lag-kernel geometry for launches of up to 32 frames:
                                      0 = one thread per spectrum element, four consumer warps
                                      and three CTAs per SM; 1 = two threads per element (half
                                      the frames each), eight consumer warps and two CTAs per SM.
                                      The same pairs, their FP32 sums formed in another order
                                      (both within 1e-5 of the FP64 oracle). With
                                      lag_batch_frames = -1 the tuned geometry is used. */
    int fft_group_frames;          /* frames per FFT launch (both passes over every scale);
                                      0 = as many as 256 MB of spectra hold (at least 1). With
                                      lag_batch_frames = -1 the tuned value is used. */
    int fft_per_tile;              /* 1: tiles of side 32..128 are transformed by one kernel that
                                      keeps each tile in shared memory between its row and column
                                      passes (one HBM write per half spectrum); 0: every scale
                                      through the two-pass FFT (row pass to the ring, column pass
                                      in place), measured as fast or faster. Same arithmetic, the
                                      same spectra bit for bit. With lag_batch_frames = -1 the
                                      tuned value is used. */
} ddm_config;

typedef struct ddm_engine ddm_engine;

/* Validation, allocation, mask construction and ring set-up: replaces the first half of
 * runDDM (src/DDM.cu:301-744: sort + checks :319-355,459-463, buffers :493-641, cuFFT
 * plans :648-677, ring pointers :686-742) and buildAzimuthMask (src/azimuthal_average.cu:229).
 * Arrays in cfg are copied. */
int ddm_open(const ddm_config *cfg, ddm_engine **out);

/* Release every device and host resource of the engine. */
int ddm_close(ddm_engine *e);

/* Submit `count` consecutive source frames, each frame_height rows of
 * frame_width*bytes_per_pixel bytes, rows packed. `on_device` = 0: host memory (pinned
 * memory gives asynchronous copies); 1: device memory on the engine's device, read in
 * place. Frames are transformed into the ring and their lag pairs are accumulated; with
 * the unbiased estimator the lag work of up to lag_batch_frames - 1 frames may be held back
 * for a fuller launch, and ddm_finalize, ddm_synchronize, ddm_reset_accumulators and
 * ddm_read_accumulators queue it first. Replaces the chunk loop of runDDM
 * (src/DDM.cu:765-843: H2D copy :767, parseChunk :154 -> parseBufferScalePow2 +
 * cufftExecR2C, analyseChunk :222 -> processFFT). Returns once the work is queued on the
 * engine's stream. */
int ddm_submit_frames(ddm_engine *e, const void *frames, int count, int on_device);

/* Block until the host frames of the submit call `back` calls before the last (0 = the last
 * call, at most 7) have been copied to the device, so that buffer may be refilled while the
 * engine still transforms and pairs them: a reader that alternates two buffers calls it with
 * back = 1 before refilling the buffer of the call before last. Returns at once for calls
 * that read device memory or do not exist. */
int ddm_wait_frames_copied(ddm_engine *e, int back);

/* Queue the remaining pairs (compat tail, src/DDM.cu:830-843) and the masked azimuthal
 * average of every (scale, tile, lambda, tau) bin; the result is ready for
 * ddm_read_isf. Replaces combineAccumulators + analyse_accums + analyseFFTDevice
 * (src/DDM.cu:45-63,72-146,864-876; src/azimuthal_average.cu:292-346). */
int ddm_finalize(ddm_engine *e);

/* Number of doubles in one ISF result: sum over scales of tiles * lambda_count * tau_count. */
long ddm_isf_size(const ddm_engine *e);

/* Copy the finalized ISF, layout [scale (descending)][tile][lambda (ascending)][tau
 * (ascending)], into host memory (waits for the engine's stream). */
int ddm_read_isf(ddm_engine *e, double *isf_out, long capacity);

/* ddm_finalize + ddm_read_isf without stopping the stream: queues the finalize work and an
 * asynchronous copy of its result into `isf_out` (capacity >= ddm_isf_size; pinned host
 * memory for a copy that overlaps later work, pageable memory makes the call wait for it)
 * and returns. Frames submitted afterwards are paired after the copied result, so a caller
 * can submit chunk k+1 while the result of chunk k is on its way -- the rolling -G dump
 * (src/DDM.cu:800-826) without the pause of the chunk loop. The call queues its result and
 * then waits for the previous call's, so on return the previous buffer holds its result and
 * is the caller's again, and one result is in flight. Unbiased estimator: any number of
 * times; compat: once, as ddm_finalize. */
int ddm_finalize_async(ddm_engine *e, double *isf_out, long capacity);

/* Results ddm_finalize_async keeps in flight: with depth d (2..8, default 2) the call queues
 * its result and waits for the one of d - 1 calls before, so a caller cycles d buffers and d - 1
 * results are on their way at any time (for chunks whose GPU work is shorter than a result's
 * round trip). Only between results: DDM_ERR_STATE while any is in flight (ddm_wait_isf). */
int ddm_set_async_depth(ddm_engine *e, int depth);

/* Block until the last ddm_finalize_async result is in its buffer; returns DDM_ERR_CUDA if
 * a kernel queued before it reported a failure (the status ddm_finalize checks). */
int ddm_wait_isf(ddm_engine *e);

/* Autotuner (the reference has none: its block sizes are constants, src/constants.hpp:11-13,
 * and its lag work is one launch per (scale, tau, frame)). ddm_autotune times, on cfg's shape
 * (unbiased estimator only) with synthetic frames on the device in the engine's steady state,
 * first every lag blocking lag_batch_frames in {16, 24, 30, 32, 64, chunk} with each lag-kernel
 * geometry (lag_geometry 0 and 1; 64 frames run geometry 0 only), then, with the fastest of
 * those, the FFT launch group fft_group_frames in {0 (256 MB of spectra), 4, 8, 16} frames and
 * the per-tile FFT variant (fft_per_tile = 1, 256 MB groups), and returns the fastest
 * combination; with a cache path it first looks the shape up there and afterwards stores the
 * result (a JSON object, one shape key per line, with the frames/s of every candidate as
 * "J/G/F/V"). Engines opened with lag_batch_frames = -1 take all four tuned values. cfg's small_tile_dft is kept as given (it changes the precision, so it is never
 * chosen by timing). ddm_tune_key writes the shape key (frame size and depth, scales, tau
 * count / largest / hash, chunk, estimator, small_tile_dft) into out (capacity bytes, NUL
 * terminated) and returns its length, or -1. */
typedef struct {
    int lag_batch_frames;
    double frames_per_s;   /* of the winner, as timed (or as cached) */
    int from_cache;        /* 1: found in the cache, nothing timed */
    int lag_geometry;      /* the winner's lag-kernel geometry */
    int fft_group_frames;  /* the winner's FFT launch group (0 = the 256 MB rule) */
    int fft_per_tile;      /* the winner's FFT variant */
} ddm_tuning;
int ddm_autotune(const ddm_config *cfg, const char *cache_path, ddm_tuning *out);
long ddm_tune_key(const ddm_config *cfg, char *out, long capacity);

/* -G snapshots (src/DDM.cu:800-826): number of snapshots taken so far, and a copy of
 * snapshot `index` in the ddm_read_isf layout. */
int ddm_dump_count(const ddm_engine *e);
int ddm_read_dump(ddm_engine *e, int index, double *isf_out, long capacity);

/* Zero the accumulators and pair counts (the -G purge, src/DDM.cu:815-823). */
int ddm_reset_accumulators(ddm_engine *e);

/* Block until all queued work is done; returns the first asynchronous error. */
int ddm_synchronize(ddm_engine *e);

/* Sorted parameter arrays as the engine uses them (the reference sorts the caller's
 * arrays in place, src/DDM.cu:319-321; the engine leaves them alone and exposes the
 * sorted copies here). Any pointer may be NULL. */
int ddm_get_params(const ddm_engine *e, int *scales, int *taus, float *lambdas);

/* Annulus pixel counts per (scale, lambda) as [scale][lambda] (the h_pixel_counts of
 * buildAzimuthMask, src/azimuthal_average.cu:271), and the boolean mask of one scale as
 * [lambda][ky][kx] bytes, kx in [0, s/2]. */
int ddm_get_pixel_counts(const ddm_engine *e, int *counts_out);
int ddm_get_mask(const ddm_engine *e, int scale_index, unsigned char *mask_out, long capacity);

/* Spectrum of frame `frame` (0-based submission index, still in the ring) as interleaved
 * complex float [scale][tile][ky][kx]; and the raw accumulators as [tau][element]
 * (sum - compensation, unnormalised |dF|^2 sums), both for tests. */
long ddm_frame_elements(const ddm_engine *e);
int ddm_read_spectrum(ddm_engine *e, int frame, float *out, long capacity);
int ddm_read_accumulators(ddm_engine *e, double *out, long capacity);

/* The -A output (src/DDM.cu:196-211 with calculateAmplitude, src/DDM_kernel.cuh:107-121):
 * |F / s^2|^2 in float for every element of frame `frame` (still in the ring), layout
 * [scale][tile][ky][kx]. Unlike the reference, every element is written (its launch grid
 * covers only part of the array). */
int ddm_read_power_spectrum(ddm_engine *e, int frame, float *out, long capacity);

/* The -K output, corrected (the reference writes raw accumulator rows with a wrong row
 * stride, src/azimuthal_average.cu:62-106, from the tile offset of src/DDM.cu:122): after
 * ddm_finalize, for every tau and element [tau][scale][tile][ky][kx] the value
 * 2 * sum|dF|^2 / s^4 / norm[tau] with the norms that finalize used, i.e. the
 * per-wave-vector structure function whose mean over each annulus mask is the ISF bin. */
int ddm_read_unaveraged(ddm_engine *e, double *out, long capacity);

/* Tiles over all scales (sum of (M/s)^2): the row count of ddm_fit_isf's per-tile outputs. */
long ddm_tile_count(const ddm_engine *e);

/* Starting point of the ISF fits: read off each curve (B = first value, A = largest rise,
 * F = ln 2 / first lag reaching half of it), or the script's fixed (F, A, B) =
 * (6, 0.03, 0.004) (plot_averaged.py:77), which suits lags in seconds and F of a few per
 * second only. */
typedef enum { DDM_FIT_START_DATA = 0, DDM_FIT_START_SCRIPT = 1 } ddm_fit_start;

/* Fits the ISF of the last ddm_finalize on the GPU, the analysis of the reference's
 * resources/python_tools/plot_averaged.py:57-141 (run there with scipy on ISF files):
 * I(tau) = A (1 - exp(-F tau)) + B per (scale, tile, lambda) curve and per (scale, lambda)
 * curve of the tile-averaged ISF, by FP64 Levenberg-Marquardt from `start`
 * (ddm_fit_start), with 1-sigma errors as scipy's curve_fit reports them
 * (covariance (J^T J)^-1 * RSS / (T - 3)); then the diffusion coefficient from
 * ln F = ln D + 2 ln q (slope fixed at 2) over the lambdas with F > 0, q = 2 pi /
 * (lambda * um_per_px), per tile and per scale. Lag times are (float)tau / fps as the ISF
 * files label them, or frames when fps <= 0; D is then in um^2 per second (or per frame).
 * Outputs (each may be NULL): tile_fit [tiles][lambda][6] and scale_fit [scale][lambda][6]
 * hold F, A, B, sigma_F, sigma_A, sigma_B; tile_d [tiles][2] and scale_d [scale][2] hold D,
 * sigma_D (NaN where no lambda gave F > 0). Tiles run over scales (descending), then tile
 * index. The script itself fits the last tile's ISF where it means the average
 * (plot_averaged.py:280 passes the loop variable ISF, not ISF_scale); both are here. */
int ddm_fit_isf(ddm_engine *e, float fps, double um_per_px, int start, double *tile_fit, double *scale_fit,
                double *tile_d, double *scale_d);

/* Engine facts: frames submitted, ring slots, device bytes held, kernels launched so far,
 * the stream the engine runs on (a cudaStream_t), and for DDM_EST_COMPAT the number of
 * frames the reference schedule reads (max(N, 2C) when N < 2C, else N; 0 otherwise). */
typedef struct {
    long frames_submitted;
    int ring_slots;
    size_t device_bytes;
    long kernel_launches;
    void *stream;
    long frames_needed;
    int lag_batch_frames;          /* frames per lag launch in use (after defaults / tuning) */
    int lag_geometry;              /* lag-kernel geometry in use */
    int fft_group_frames;          /* frames per FFT launch in use */
    int fft_per_tile;              /* FFT variant in use */
} ddm_info;
int ddm_get_info(const ddm_engine *e, ddm_info *info);

/* Kernel timing: when enabled, the engine brackets every kernel it launches with CUDA
 * events on its stream. ddm_kernel_times waits for the stream, then returns for each
 * group -- 0 the FFT passes (parseChunk + cufftExecR2C in the reference), 1 the lag
 * kernel (processFFT), 2 the azimuthal reduction (analyseFFTDevice) -- the summed device
 * milliseconds and the number of launches since the last call, and clears them. */
int ddm_set_timing(ddm_engine *e, int enabled);
int ddm_kernel_times(ddm_engine *e, double *ms_out, long *launches_out);
/* As ddm_kernel_times, also returning per group the compulsory DRAM bytes of the kernels
 * launched since the last call (counted whether timing is on or not): FFT, the ROI's pixels
 * read once and every spectrum written once; lag, each register frame and each distinct
 * partner frame of a launch read once and each accumulator row read and written once;
 * azimuth, every masked accumulator element of every tau read once. bytes_out may be NULL. */
int ddm_kernel_stats(ddm_engine *e, double *ms_out, long *launches_out, double *bytes_out);

/* Host-only helpers (no GPU needed). ddm_build_masks: the annulus masks of one scale,
 * [lambda][ky][kx] bytes (kx in [0, s/2]; mask_out may be NULL) and per-lambda pixel
 * counts, bit-exact to buildAzimuthMask with q = s/lambda (src/azimuthal_average.cu:229-283,
 * src/DDM.cu:101-105). ddm_compat_schedule: the frame pairs of the reference's chunk loop
 * (src/DDM.cu:750-843) -- for each analysed frame c in order, the A-frame label a_out[c]
 * and the partner label of every tau b_out[c*tau_count + t] (labels count frames from the
 * first one read; -1 = device memory the reference never wrote), epoch_out[c] = -G purges
 * before c (may be NULL); returns the number of analysed frames, or -1 if max_calls is too
 * small; *frames_read = frames the reference reads from its source. */
int ddm_build_masks(int scale, const float *lambdas, int lambda_count, float tolerance,
                    unsigned char *mask_out, int *counts_out);
int ddm_compat_schedule(int total_frames, int chunk, int multistream, int dump_every, const int *taus,
                        int tau_count, int max_calls, int *a_out, int *b_out, int *epoch_out,
                        int *frames_read);

/* Lag accumulation on caller-owned device memory, with no device allocation at all. This
 * entry point has no counterpart in the reference. It exists for callers that cannot let a
 * library call cudaMalloc -- real-time acquisition loops that reserve all device memory at
 * start-up and must not stall mid-stream, and applications whose own pool allocator owns
 * every device buffer. For every element k < elements and tau row t < tau_count:
 *   acc[t][k] += sum over j < frame_count of |ring[a_slots[j]][k] - ring[b_slots[t*frame_count + j]][k]|^2
 * skipping pairs with a slot of -1; ring is float2[ring_slots][elements] (complex spectra,
 * elements even), acc is float2[tau_count][elements] holding {sum, Kahan compensation}
 * (value = sum - compensation), both device pointers on the current device; the engine's
 * lag kernel does the work, on `stream` (a cudaStream_t, NULL = default stream).
 * Limits: frame_count <= 32, tau_count <= 128, ring_slots <= 1048575; larger requests are
 * refused with DDM_ERR_INVALID_ARG. The kernel's pair table and status word live in one
 * static device array of about 37 KB that every GPU using the library keeps until exit and
 * that all calls share: calls are serialised in the process and each returns after its
 * kernel finished; kernels of calls made from other processes do not share it. The first
 * call on each device sets that device up (cudaGetSymbolAddress of the array and the
 * kernel's shared-memory limit), so make the first call before any stream capture. */
int ddm_lag_accumulate_static(const void *ring, int ring_slots, long long elements, void *acc,
                              const int *a_slots, int frame_count, const int *b_slots, int tau_count,
                              void *stream);

/* Page-locked host memory for frame buffers (asynchronous copies); NULL on failure. */
void *ddm_host_alloc(size_t bytes);
void ddm_host_free(void *ptr);

/* Bounded waits. Every wait in the lag kernel's copy pipeline gives up after `cycles` SM
 * clock cycles (0 = the default, 400,000,000: about 0.2 s at 1.965 GHz, orders of magnitude
 * above any legitimate copy latency). A wait that runs out makes the kernel finish its copies
 * in flight and return with a device status that the next ddm_finalize, ddm_synchronize or
 * ddm_wait_isf reports as DDM_ERR_CUDA ("... wait timed out ..."); the CUDA context stays
 * usable. The same report, worded "... shared memory was not 1 KB aligned", comes from a lag
 * kernel that found its dynamic shared memory off a 1 KB boundary: it returns before
 * issuing any copy. The reference has no such path: every error there ends the process
 * (src/debug.cpp:10-15). */
int ddm_set_wait_limit(ddm_engine *e, long long cycles);

/* Fault injection for tests of the error path (no counterpart in the reference).
 * DDM_FAULT_LAG_WAIT: the engine's next lag launch gets a pair table whose last tau window
 * reaches a group of partner frames that is never copied, so that launch's pipeline waits
 * run out and the error surfaces as above. Nothing faults on the GPU: every access of the
 * altered launch stays inside its buffers and every wait is bounded. One-shot; not for
 * streams of a server. */
typedef enum { DDM_FAULT_NONE = 0, DDM_FAULT_LAG_WAIT = 1 } ddm_fault;
int ddm_inject_fault(ddm_engine *e, int fault);

/* Text of the last error on this thread. */
const char *ddm_last_error(void);
const char *ddm_status_string(int status);

/* One (scale, tile) ISF text file, byte-compatible with writeIqtToFile
 * (src/azimuthal_average.cu:112-150): line 1 the lambdas, line 2 tau/fps with the frame
 * rate truncated to an integer as the reference does (src/DDM.cu:79,876), then one line
 * of tau values per lambda; every value %g with a trailing space. */
int ddm_write_isf_file(const char *path, const double *isf_qt, const float *lambdas,
                       int lambda_count, const int *taus, int tau_count, float fps);

/* Seeded synthetic Brownian-particle video (host memory, frame-major): background +
 * Gaussian spots of peak `amplitude` and width `spot_sigma`, positions uniform, each
 * frame every spot steps N(0, step_var) per axis (step_var_b for the second half of the
 * spots), periodic boundaries; then additive Gaussian noise of sd `noise_sd`
 * (noise_sd < 0: Poisson shot noise), rounded half-to-even and clipped to [0, max_value].
 * Pixels are 1 byte if max_value <= 255, else 2 bytes little-endian. */
int ddm_synth_video(uint64_t seed, int width, int height, int frames, int spots,
                    double spot_sigma, double amplitude, double background, double step_var,
                    double step_var_b, double noise_sd, int max_value, void *out);

/* ---------------------------------------------------------------------------------
 * Serving many streams on one GPU (no counterpart in the reference, which analyses one
 * video per process, src/DDM.cu:268-892). A server keeps every admitted stream's engine
 * (FFT ring, accumulators) resident and runs continuous batching: ddm_server_step takes the
 * next pending chunk of every stream (whose earlier results have been collected), runs each
 * stream's FFT on its own CUDA stream, then one lag-kernel launch over all of those streams'
 * lag work, then per stream the azimuthal average and the copy of its ISF to host memory.
 * A step returns once that work is queued; chunks submitted while it runs are taken by the
 * next step. Every chunk gets a result (the ISF of the stream so far, as ddm_finalize +
 * ddm_read_isf would give) with its submit and completion times on the server clock.
 * Streams use the unbiased estimator. Calls are thread-safe (one lock per server).
 * --------------------------------------------------------------------------------- */
typedef struct ddm_server ddm_server;

typedef struct {
    int device;                /* CUDA device ordinal */
    size_t hbm_budget_bytes;   /* device bytes the streams may hold; 0 = free memory - 2 GiB */
    int max_streams;           /* 0 = 64 */
    int results_per_stream;    /* chunks of a stream in flight or awaiting ddm_server_poll; 0 = 4 */
} ddm_server_config;

typedef struct {
    long chunk_index;  /* 0-based chunk of the stream */
    long frames;       /* frames of the stream analysed with this chunk */
    double submit_s;   /* server clock when the chunk was submitted */
    double done_s;     /* server clock when its ISF reached host memory */
} ddm_chunk_result;

typedef struct {
    int streams;            /* admitted */
    size_t device_bytes;    /* held by them */
    size_t budget_bytes;
    long batched_launches;  /* lag-kernel launches covering several streams' work */
    long chunks_pending;    /* submitted, not yet taken by a step */
    long steps;             /* ddm_server_step calls that took at least one chunk */
    double step_host_s;     /* host time spent inside those calls */
    double gpu_s;           /* GPU time of finished steps on the server's stream, from its first
                               operation to its last (queueing excluded) */
} ddm_server_stats;

/* Opens a server on cfg->device. At open it maps its HBM budget into the device's memory pool,
 * creates the private CUDA streams of every stream slot (4 each) and page-locks a 2 GiB host
 * arena for the streams' chunk and result buffers (once per process; skipped if refused), so
 * that admitting a stream later touches none of these slow driver paths. */
int ddm_server_open(const ddm_server_config *cfg, ddm_server **out);
int ddm_server_close(ddm_server *s);
/* Admit a stream (cfg as for ddm_open; its device, stream, lag_batch_frames and dump_every
 * are set by the server). DDM_ERR_BUSY: it does not fit the HBM budget or the stream
 * limit now; retry after streams leave. */
int ddm_server_add_stream(ddm_server *s, const ddm_config *cfg, int *stream_id);
/* Remove a stream: its device memory is released once the work queued for it has run
 * (without waiting here); its unpolled results are dropped. */
int ddm_server_remove_stream(ddm_server *s, int stream_id);
/* Queue one chunk of `count` frames from host memory (copied; the buffer is free on return). */
int ddm_server_submit(ddm_server *s, int stream_id, const void *frames, int count);
/* As ddm_server_submit without the copy: `frames` is page-locked host memory (cudaMallocHost,
 * cudaHostRegister) that the caller leaves unchanged until this chunk's result has been
 * returned by ddm_server_poll. */
int ddm_server_submit_pinned(ddm_server *s, int stream_id, const void *frames, int count);
/* One continuous-batching step; *chunks_issued = chunks taken. */
int ddm_server_step(ddm_server *s, int *chunks_issued);
/* The stream's oldest finished chunk: returns 1 and fills res / isf (ISF layout of
 * ddm_read_isf, capacity >= ddm_isf_size of the stream), or 0 if none is finished. */
int ddm_server_poll(ddm_server *s, int stream_id, ddm_chunk_result *res, double *isf, long capacity);
/* Block until all queued GPU work is done. */
int ddm_server_wait(ddm_server *s);
double ddm_server_clock(const ddm_server *s);  /* seconds since ddm_server_open */
int ddm_server_get_stats(const ddm_server *s, ddm_server_stats *stats);

/* Camera .movie files (src/video_reader.cpp:64-290): open, describe, read frames. */
typedef struct {
    int width, height, bytes_per_pixel;
    float fps;               /* 1e6 / (timestamp[1] - timestamp[0]), as the reference */
    int camera_type;         /* 1 IIDC, 2 Andor, 3 Ximea */
    int pixel_mode;          /* 1 mono8, 2 mono16 big-endian, 3 mono16 little-endian */
} ddm_movie_info;
typedef struct ddm_movie ddm_movie;
int ddm_movie_open(const char *path, int frame_offset, ddm_movie **out, ddm_movie_info *info);
int ddm_movie_read(ddm_movie *m, void *dst, int count); /* frames packed, w*h*bpp each */
int ddm_movie_close(ddm_movie *m);

#ifdef __cplusplus
}
#endif
#endif
