// ddm -- command-line front end of the B200 DDM engine, a drop-in for the reference's
// ./ddm (src/main.cpp + runDDM in src/DDM.cu). Same flags, parameter files, checks and
// messages, output file names and text layout, and the [Time elapsed] line; the
// computation runs through the C ABI in include/ddm.h.
//
// Flags kept from the reference (getopt string src/main.cpp:115):
//   -o PATH -N INT -Q PATH -T PATH -S PATH  outputs, frame count, lambda/tau/scale files
//   -f PATH -M                              .movie input (-f without -M needs OpenCV: unavailable)
//   -B ARG                                  benchmark mode on random frames (takes an argument,
//                                           as in the reference)
//   -s -x -y -I -v -Z -t -C -G -F -W        as in the reference; -F is accepted and, like the
//                                           reference, has no effect; -W is refused
//   -K ARG -A                               the reference's debug outputs, with corrected
//                                           contents (see write_unaveraged / write_power)
// Flags added here:
//   -D UM_PER_PX         fit the ISF on the GPU (ddm_fit_isf) and write <out>fit
//   -E compat|unbiased   estimator (default compat: the reference's own pairing)
//   -P byte0|u16         16-bit pixel decoding (default byte0: the reference's first byte)
//   -U CACHE             unbiased estimator: lag blocking, lag-kernel geometry and FFT launch
//                        shape from the autotuner (ddm_autotune; timed once per shape and kept
//                        in the JSON file CACHE)
//   -X                   split-BF16 tensor-core DFT for tiles of side 32..128 (ISF within 1e-3)
#include <getopt.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/ddm.h"

namespace {

bool g_verbose = false;

[[noreturn]] void die(const std::string &text) {  // conditionAssert(false, text, true)
    std::fprintf(stderr, "[Error] %s\n", text.c_str());
    std::exit(EXIT_FAILURE);
}

void warn(const std::string &text) { std::fprintf(stderr, "[Warning] %s\n", text.c_str()); }

void verbose(const char *fmt, const std::string &a = std::string()) {
    if (g_verbose) std::printf(fmt, a.c_str());
}

void print_help() {
    std::fprintf(stderr,
                 "\n multi-scale DDM (B200 engine)\n\n"
                 "  usage: ddm [OPTION]...\n"
                 "  -h           this help\n"
                 " required\n"
                 "  -o PATH      output path prefix; files are <PATH><scale>-<tile>\n"
                 "  -N INT       number of frames to analyse\n"
                 "  -Q PATH      lambda values (whitespace separated, pixels)\n"
                 "  -T PATH      tau values (whitespace separated, frames)\n"
                 "  -S PATH      scale values (whitespace separated, powers of two)\n"
                 " input (one of)\n"
                 "  -f PATH -M   camera .movie file\n"
                 "  -B ARG       benchmark mode on random frames\n"
                 " optional\n"
                 "  -s INT       skip this many frames at the start (default 0)\n"
                 "  -x INT -y INT  region-of-interest offset (default 0 0)\n"
                 "  -I           tau labels in frames instead of seconds\n"
                 "  -v           verbose\n"
                 "  -Z           single-stream schedule of the reference\n"
                 "  -t INT       annulus tolerance in percent (default 20: radii q .. 1.2 q)\n"
                 "  -C INT       frames per chunk (default 100)\n"
                 "  -G INT       write and reset the ISF every INT chunks\n"
                 "  -F FPS       accepted, no effect (as in the reference)\n"
                 "  -K ARG       also write <PATH><scale>-<tile>-nonAve: per tau, the structure\n"
                 "               function of every wave vector before the azimuthal average\n"
                 "  -A           also write <PATH>_fft_chunk_<k>-<scale>: |F/s^2|^2 of every\n"
                 "               frame and tile of chunk k\n"
                 "  -D UMPX      also fit A(1-exp(-F tau))+B to every ISF curve on the GPU and\n"
                 "               write <PATH>fit with F, A, B per curve and the diffusion\n"
                 "               coefficient per tile and scale (UMPX: micrometres per pixel)\n"
                 "  -E MODE      compat (default) or unbiased estimator\n"
                 "  -P MODE      byte0 (default) or u16 decoding of 16-bit pixels\n"
                 "  -U CACHE     with -E unbiased: lag blocking, lag-kernel geometry and FFT launch\n"
                 "               shape picked by the autotuner, timed once per shape and kept in\n"
                 "               the JSON file CACHE\n"
                 "  -X           tiles of side 32..128 through the split-BF16 tensor-core DFT\n"
                 "               (FP32 accumulation; ISF within 1e-3 instead of 1e-5)\n");
}

// Number text as std::ostream prints a float (6 significant digits), then one space, as
// the reference's writers do (src/azimuthal_average.cu:31-150).
inline void put_value(FILE *f, double v) { std::fprintf(f, "%g ", static_cast<double>(static_cast<float>(v))); }

FILE *open_out(const std::string &name) {
    FILE *f = std::fopen(name.c_str(), "w");
    if (!f) {
        std::fprintf(stderr, "[Out Error] Unable to open %s.\n", name.c_str());
        std::exit(EXIT_FAILURE);
    }
    return f;
}

// -K: <prefix><scale>-<tile>-nonAve (file name of src/DDM.cu:120). Header lines as the ISF
// file (lambdas, tau / fps); then one line per tau with the tile's s*(s/2+1) values of
// 2 * mean|dF|^2 / s^4 in [ky][kx] order, whose mean over an annulus mask is that ISF bin.
// (The reference's rows use a row stride of tau_count instead of the tile size and the
// accumulator tile offset of src/DDM.cu:122; this writes what those rows were meant to hold.)
void write_unaveraged(const std::string &prefix, const std::vector<double> &unav, long E,
                      const std::vector<int> &scales, const std::vector<float> &lambdas,
                      const std::vector<int> &taus, float fps) {
    long off = 0;
    for (int s : scales) {
        const int tiles = (scales[0] / s) * (scales[0] / s);
        const long n = static_cast<long>(s) * (s / 2 + 1);
        for (int tile = 0; tile < tiles; tile++, off += n) {
            FILE *f = open_out(prefix + std::to_string(s) + "-" + std::to_string(tile) + "-nonAve");
            for (float l : lambdas) put_value(f, l);
            std::fputc('\n', f);
            for (int t : taus) put_value(f, static_cast<float>(t) / fps);
            std::fputc('\n', f);
            for (size_t ti = 0; ti < taus.size(); ti++) {
                const double *row = unav.data() + static_cast<long>(ti) * E + off;
                for (long k = 0; k < n; k++) put_value(f, row[k]);
                std::fputc('\n', f);
            }
            std::fclose(f);
        }
    }
}

// -A: <prefix>_fft_chunk_<k>-<scale>, one line per (frame, tile) of chunk k with the
// tile's s*(s/2+1) values of |F/s^2|^2 (calculateAmplitude, src/DDM_kernel.cuh:107-121). The
// reference names every chunk's file _fft_chunk_<dumps so far> and so keeps only the last
// chunk's, and its launch grid leaves most of each line zero; here every chunk keeps its
// own file and every value is written.
struct PowerWriter {
    std::vector<FILE *> files;
    void open(const std::string &prefix, long chunk_index, const std::vector<int> &scales) {
        close();
        for (int s : scales)
            files.push_back(open_out(prefix + "_fft_chunk_" + std::to_string(chunk_index) + "-" + std::to_string(s)));
    }
    void frame(const std::vector<float> &pw, const std::vector<int> &scales) {
        long off = 0;
        for (size_t si = 0; si < scales.size(); si++) {
            const int s = scales[si];
            const int tiles = (scales[0] / s) * (scales[0] / s);
            const long n = static_cast<long>(s) * (s / 2 + 1);
            for (int tile = 0; tile < tiles; tile++, off += n) {
                for (long k = 0; k < n; k++) put_value(files[si], pw[off + k]);
                std::fputc('\n', files[si]);
            }
        }
    }
    void close() {
        for (FILE *f : files) std::fclose(f);
        files.clear();
    }
};

// -D: <prefix>fit. Per scale, a line "scale <s> D <D> sigma_D <err>" from the tile-averaged
// ISF, then per tile "tile <s> <index> D <D> sigma_D <err>", then per (tile, lambda)
// "curve <s> <index> <lambda> F A B sigma_F sigma_A sigma_B" (tile index -1: tile average).
void write_fits(const std::string &prefix, ddm_engine *eng, const std::vector<int> &scales,
                const std::vector<float> &lambdas, float fps, double um_per_px) {
    const long nt = ddm_tile_count(eng);
    const size_t S = scales.size(), Q = lambdas.size();
    std::vector<double> tile_fit(nt * Q * 6), scale_fit(S * Q * 6), tile_d(nt * 2), scale_d(S * 2);
    if (ddm_fit_isf(eng, fps, um_per_px, DDM_FIT_START_DATA, tile_fit.data(), scale_fit.data(), tile_d.data(),
                    scale_d.data()) != DDM_OK)
        die(ddm_last_error());
    FILE *f = open_out(prefix + "fit");
    std::fprintf(f, "# I(tau) = A (1 - exp(-F tau)) + B; tau in %s; D in um^2/%s (%g um per px)\n",
                 fps > 0 ? "s" : "frames", fps > 0 ? "s" : "frame", um_per_px);
    for (size_t si = 0; si < S; si++)
        std::fprintf(f, "scale %d D %.9g sigma_D %.9g\n", scales[si], scale_d[2 * si], scale_d[2 * si + 1]);
    long row = 0;
    for (size_t si = 0; si < S; si++) {
        const int tiles = (scales[0] / scales[si]) * (scales[0] / scales[si]);
        for (int t = 0; t < tiles; t++, row++)
            std::fprintf(f, "tile %d %d D %.9g sigma_D %.9g\n", scales[si], t, tile_d[2 * row], tile_d[2 * row + 1]);
    }
    auto curve = [&](int s, int t, float lam, const double *p) {
        std::fprintf(f, "curve %d %d %g %.9g %.9g %.9g %.9g %.9g %.9g\n", s, t, lam, p[0], p[1], p[2], p[3], p[4], p[5]);
    };
    row = 0;
    for (size_t si = 0; si < S; si++) {
        for (size_t q = 0; q < Q; q++) curve(scales[si], -1, lambdas[q], scale_fit.data() + (si * Q + q) * 6);
        const int tiles = (scales[0] / scales[si]) * (scales[0] / scales[si]);
        for (int t = 0; t < tiles; t++, row++)
            for (size_t q = 0; q < Q; q++) curve(scales[si], t, lambdas[q], tile_fit.data() + (row * Q + q) * 6);
    }
    std::fclose(f);
}

template <typename T>
std::vector<T> read_values(const std::string &path, const char *what) {
    std::ifstream in(path);
    if (!in.is_open()) die(what);
    std::vector<T> v;
    T x;
    while (in >> x) v.push_back(x);  // src/main.cpp:258-313: read until the first failure
    return v;
}

}  // namespace

int main(int argc, char **argv) {
    std::printf("DDM Start\n");
    std::fflush(stdout);

    std::string file_in, file_out, q_file, t_file, s_file;
    int frame_count = 0, frame_offset = 0, x_off = 0, y_off = 0, chunk = 100, rolling = 0;
    bool use_index_fps = false, multistream = true, bench = false, movie = false;
    bool input_specified = false, unaveraged_out = false, power_out = false;
    double fit_um_per_px = 0.0;  // -D
    float tolerance = 1.2f;
    int estimator = DDM_EST_COMPAT, pixel_mode = DDM_PIX_BYTE0;
    std::string tune_cache;  // -U
    bool small_tile_dft = false;  // -X

    for (;;) {
        int c = getopt(argc, argv, "ho:N:s:x:y:Q:T:S:If:W::vZt:C:MG:F:B:K:AE:P:D:U:X");
        if (c == -1) break;
        switch (c) {
            case '?':
            case 'h': print_help(); return -1;
            case 'o': file_out = optarg; break;
            case 'N': frame_count = std::atoi(optarg); break;
            case 'x': x_off = std::atoi(optarg); break;
            case 'y': y_off = std::atoi(optarg); break;
            case 'Q': q_file = optarg; break;
            case 'T': t_file = optarg; break;
            case 'S': s_file = optarg; break;
            case 'I': use_index_fps = true; break;
            case 's': frame_offset = std::atoi(optarg); break;
            case 'f':
                if (input_specified) die("Cannot use both in-filepath and web-cam option at same time.");
                file_in = optarg;
                input_specified = true;
                break;
            case 'W': die("web-camera input is unavailable in this build");
            case 'B': bench = true; input_specified = true; break;
            case 'v': g_verbose = true; break;
            case 'Z': multistream = false; break;
            case 't': tolerance = static_cast<float>(1.0 + std::atoi(optarg) / 100.0); break;  // src/main.cpp:195-200
            case 'C': chunk = std::atoi(optarg); break;
            case 'M': movie = true; break;
            case 'G': rolling = std::atoi(optarg); break;
            case 'F': break;  // the reference stores the value but never enables it (src/main.cpp:214-219)
            case 'K': unaveraged_out = true; break;  // takes an argument, as in the reference
            case 'A': power_out = true; break;
            case 'D':
                fit_um_per_px = std::atof(optarg);
                if (!(fit_um_per_px > 0.0)) die("-D takes the micrometres per pixel (> 0)");
                break;
            case 'E':
                if (!std::strcmp(optarg, "compat")) estimator = DDM_EST_COMPAT;
                else if (!std::strcmp(optarg, "unbiased")) estimator = DDM_EST_UNBIASED;
                else die("-E takes compat or unbiased");
                break;
            case 'U': tune_cache = optarg; break;
            case 'X': small_tile_dft = true; break;
            case 'P':
                if (!std::strcmp(optarg, "byte0")) pixel_mode = DDM_PIX_BYTE0;
                else if (!std::strcmp(optarg, "u16")) pixel_mode = DDM_PIX_U16LE;
                else die("-P takes byte0 or u16");
                break;
        }
    }
    if (optind != argc) {
        print_help();
        die("An unexpected option was found.");
    }
    if (!input_specified) die("Must specify input.");

    std::vector<float> lambdas = read_values<float>(q_file, "cannot open lambda-file.");
    std::vector<int> taus = read_values<int>(t_file, "cannot open tau-file");
    std::vector<int> scales = read_values<int>(s_file, "cannot open scales-file.");

    auto t_start = std::chrono::high_resolution_clock::now();
    if (scales.empty() || taus.empty() || lambdas.empty())
        die("scale, tau and lambda files must each hold at least one value");
    std::sort(taus.begin(), taus.end());  // src/DDM.cu:319-321
    std::sort(lambdas.begin(), lambdas.end());
    std::sort(scales.begin(), scales.end(), std::greater<int>());
    const bool compat = estimator == DDM_EST_COMPAT;

    // src/DDM.cu:327-350: the same checks in the same order, before any video set-up
    for (size_t s = 0; s < scales.size(); s++) {
        unsigned v = static_cast<unsigned>(scales[s]);
        if (scales[s] <= 0 || (v & (v - 1))) die("scales must be powers of two (> 0)");
        if (s + 1 < scales.size() && !(scales[s] > scales[s + 1])) die("scales should be descending order");
    }
    for (size_t t = 0; t + 1 < taus.size(); t++) {
        if (taus[t] < 0) die("Tau values should be positive");
        if (!(taus[t] < taus[t + 1])) die("Tau vector should be ascending order");
    }
    for (size_t q = 0; q + 1 < lambdas.size(); q++) {
        if (!(lambdas[q] >= 0)) die("q-vector values should be positive");
        if (!(lambdas[q] < lambdas[q + 1])) die("q-vector vector should be ascending order");
    }
    if (!(tolerance < 10 && tolerance > 1.0f))
        warn("mask_tolerance is likely undesired value, refer to README for more information");
    if (compat && !(lambdas.back() <= scales.back()))
        die("The largest q-vector should be smaller than the smallest scale.");

    // Video set-up (src/DDM.cu:390-452)
    int w = 0, h = 0, bpp = 1;
    float fps = 1.0f;
    ddm_movie *mv = nullptr;
    if (bench) {
        w = h = scales[0];
        bpp = 1;
        fps = 1.0f;
    } else if (movie) {
        ddm_movie_info info;
        if (ddm_movie_open(file_in.c_str(), frame_offset, &mv, &info) != DDM_OK) {
            std::fprintf(stderr, "%s\n", ddm_last_error());
            return EXIT_FAILURE;
        }
        w = info.width;
        h = info.height;
        bpp = info.bytes_per_pixel;
        fps = info.fps;
    } else {
        die("error opening video file with openCV");  // no OpenCV decoder in this build
    }
    if (use_index_fps) fps = 1.0f;
    if (!(scales[0] + x_off <= w && scales[0] + y_off <= h))  // src/DDM.cu:459-460
        die("the specified out dimensions must be smaller than actual image size");
    if (compat && !(taus.back() <= chunk))  // src/DDM.cu:462-463
        die("the largest tau value must be smaller than number frames in a chunk");

    ddm_config cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.frame_width = w;
    cfg.frame_height = h;
    cfg.bytes_per_pixel = bpp;
    cfg.pixel_mode = (bpp == 2) ? pixel_mode : DDM_PIX_BYTE0;
    cfg.x_offset = x_off;
    cfg.y_offset = y_off;
    cfg.scales = scales.data();
    cfg.scale_count = static_cast<int>(scales.size());
    cfg.taus = taus.data();
    cfg.tau_count = static_cast<int>(taus.size());
    cfg.lambdas = lambdas.data();
    cfg.lambda_count = static_cast<int>(lambdas.size());
    cfg.tolerance = tolerance;
    cfg.chunk_frames = chunk;
    cfg.estimator = estimator;
    cfg.multistream = multistream ? 1 : 0;
    cfg.total_frames = frame_count;
    cfg.dump_every = rolling;
    cfg.small_tile_dft = small_tile_dft ? 1 : 0;
    if (!tune_cache.empty()) {
        if (estimator != DDM_EST_UNBIASED) die("-U tunes the unbiased estimator (-E unbiased)");
        ddm_tuning tuned;
        if (ddm_autotune(&cfg, tune_cache.c_str(), &tuned) != DDM_OK) die(ddm_last_error());
        cfg.lag_batch_frames = tuned.lag_batch_frames;
        cfg.lag_geometry = tuned.lag_geometry;
        cfg.fft_group_frames = tuned.fft_group_frames;
        cfg.fft_per_tile = tuned.fft_per_tile;
        if (g_verbose)
            std::fprintf(stderr, "[Info] lag_batch_frames %d, lag_geometry %d, fft_group_frames %d (%s)\n",
                         tuned.lag_batch_frames, tuned.lag_geometry, tuned.fft_group_frames,
                         tuned.from_cache ? "cached" : "timed");
    }
    ddm_engine *eng = nullptr;
    if (ddm_open(&cfg, &eng) != DDM_OK) die(ddm_last_error());
    ddm_info info;
    ddm_get_info(eng, &info);
    const long frames_total = compat ? info.frames_needed : frame_count;
    const size_t frame_bytes = static_cast<size_t>(w) * h * bpp;

    // Two pinned chunk buffers: one is read from the file while the other is in flight.
    uint8_t *buf[2];
    for (int i = 0; i < 2; i++) {
        buf[i] = static_cast<uint8_t *>(ddm_host_alloc(frame_bytes * chunk));
        if (!buf[i]) die(ddm_last_error());
    }
    if (bench) {  // as src/DDM.cu:522-528: the first frame of each buffer gets rand() % 255
        for (int i = 0; i < 2; i++) {
            std::memset(buf[i], 0, frame_bytes * chunk);
            for (size_t k = 0; k < frame_bytes; k++) buf[i][k] = static_cast<uint8_t>(std::rand() % 255);
        }
    }
    const float int_fps = static_cast<float>(static_cast<int>(fps));  // analyse_accums takes int (src/DDM.cu:79)
    std::vector<double> isf(ddm_isf_size(eng));
    auto write_all = [&](const std::string &prefix) {  // analyse_accums file loop, src/DDM.cu:96-145
        const long block = static_cast<long>(lambdas.size() * taus.size());
        long off = 0;
        for (int s : scales) {
            const int tiles = (scales[0] / s) * (scales[0] / s);
            for (int tile = 0; tile < tiles; tile++) {
                std::string name = prefix + std::to_string(s) + "-" + std::to_string(tile);
                if (ddm_write_isf_file(name.c_str(), isf.data() + off, lambdas.data(),
                                       static_cast<int>(lambdas.size()), taus.data(),
                                       static_cast<int>(taus.size()), int_fps) != DDM_OK) {
                    std::fprintf(stderr, "%s\n", ddm_last_error());
                    std::exit(EXIT_FAILURE);
                }
                off += block;
            }
        }
    };

    int dumps_written = 0;
    long sent = 0;
    int which = 0;
    PowerWriter power;
    std::vector<float> pw(power_out ? ddm_frame_elements(eng) : 0);
    auto read_chunk = [&](int n) {
        if (!bench && ddm_movie_read(mv, buf[which], n) != DDM_OK) {
            std::fprintf(stderr, "%s\n", ddm_last_error());
            std::exit(EXIT_FAILURE);
        }
    };
    auto write_dumps = [&]() {
        while (dumps_written < ddm_dump_count(eng)) {  // -G snapshots, src/DDM.cu:800-826
            if (ddm_read_dump(eng, dumps_written, isf.data(), static_cast<long>(isf.size())) != DDM_OK)
                die(ddm_last_error());
            write_all(file_out + "_t" + std::to_string(dumps_written) + "_");
            dumps_written++;
        }
    };
    if (!power_out) {
        // Two buffers: chunk k+1 is read from the file while the engine transforms and pairs
        // chunk k; before a buffer is refilled, the copies of the submit call before last (its
        // frames) must have finished.
        int n = static_cast<int>(std::min<long>(chunk, frames_total));
        read_chunk(n);
        while (sent < frames_total) {
            if (ddm_submit_frames(eng, buf[which], n, 0) != DDM_OK) die(ddm_last_error());
            sent += n;
            which ^= 1;
            write_dumps();
            verbose("[Chunk complete]%s\n");
            if (sent < frames_total) {
                n = static_cast<int>(std::min<long>(chunk, frames_total - sent));
                if (!bench && ddm_wait_frames_copied(eng, 1) != DDM_OK) die(ddm_last_error());
                read_chunk(n);
            }
        }
    } else {
        while (sent < frames_total) {
            const int n = static_cast<int>(std::min<long>(chunk, frames_total - sent));
            read_chunk(n);
            // -A: submit in pieces no larger than the engine's ingest piece (min(C, 32) frames;
            // the ring holds at least that many latest frames), reading each piece's spectra
            power.open(file_out, sent / chunk, scales);
            const int step = std::max(1, std::min({chunk, 32, info.ring_slots}));
            for (int f0 = 0; f0 < n; f0 += step) {
                const int m = std::min(step, n - f0);
                if (ddm_submit_frames(eng, buf[which] + frame_bytes * f0, m, 0) != DDM_OK ||
                    ddm_synchronize(eng) != DDM_OK)
                    die(ddm_last_error());
                for (int f = 0; f < m; f++) {
                    if (ddm_read_power_spectrum(eng, static_cast<int>(sent + f0 + f), pw.data(),
                                                static_cast<long>(pw.size())) != DDM_OK)
                        die(ddm_last_error());
                    power.frame(pw, scales);
                }
            }
            power.close();
            sent += n;
            which ^= 1;
            write_dumps();
            verbose("[Chunk complete]%s\n");
        }
    }
    if (ddm_synchronize(eng) != DDM_OK) die(ddm_last_error());
    auto t_main = std::chrono::high_resolution_clock::now();

    if (ddm_finalize(eng) != DDM_OK) die(ddm_last_error());
    while (dumps_written < ddm_dump_count(eng)) {
        if (ddm_read_dump(eng, dumps_written, isf.data(), static_cast<long>(isf.size())) != DDM_OK)
            die(ddm_last_error());
        write_all(file_out + "_t" + std::to_string(dumps_written) + "_");
        dumps_written++;
    }
    if (ddm_read_isf(eng, isf.data(), static_cast<long>(isf.size())) != DDM_OK) die(ddm_last_error());
    write_all(file_out);
    if (unaveraged_out) {
        const long E = ddm_frame_elements(eng);
        std::vector<double> unav(static_cast<size_t>(E) * taus.size());
        if (ddm_read_unaveraged(eng, unav.data(), static_cast<long>(unav.size())) != DDM_OK) die(ddm_last_error());
        write_unaveraged(file_out, unav, E, scales, lambdas, taus, int_fps);
    }
    if (fit_um_per_px > 0.0) write_fits(file_out, eng, scales, lambdas, int_fps, fit_um_per_px);
    auto t_end = std::chrono::high_resolution_clock::now();

    ddm_close(eng);
    ddm_host_free(buf[0]);
    ddm_host_free(buf[1]);
    if (mv) ddm_movie_close(mv);

    const double d1 = std::chrono::duration_cast<std::chrono::microseconds>(t_main - t_start).count();
    const double d2 = std::chrono::duration_cast<std::chrono::microseconds>(t_end - t_main).count();
    std::printf("[Time elapsed] \n\tMain:\t\t%f s, \n\tRadial Average:\t%f s,\n\tTotal\t\t%f s,\t(%f frame / second)\n",
                d1 / 1e6, d2 / 1e6, (d1 + d2) / 1e6, frame_count * 1e6 / (d1 + d2));
    std::printf("DDM End\n");
    return 0;
}
