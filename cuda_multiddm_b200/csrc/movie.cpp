// Camera .movie reader (ddm_movie_* in ddm.h): the format read by initFile and
// loadMovieToHost (src/video_reader.cpp:64-290, structs src/video_reader.hpp:32-214).
//
// Layout: each frame is a camera header followed by length_data image bytes. Every
// header starts with the common 24-byte block {magic 'TemI' = 0x496d6554, version 1,
// camera type, pixel mode, header length, data length}; the full header is 172 bytes
// (IIDC), 128 (Andor) or 240 (Ximea). Frame size and the timestamp used for the frame
// rate sit at fixed offsets in those headers (read below as little-endian fields).
#include <unistd.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/ddm.h"
#include "errors.hpp"

namespace {

constexpr uint32_t kMagic = 0x496d6554;
constexpr int kIIDC = 1, kAndor = 2, kXimea = 3;
constexpr int kMono8 = 1;

uint32_t rd32(const unsigned char *p) {
    return uint32_t(p[0]) | uint32_t(p[1]) << 8 | uint32_t(p[2]) << 16 | uint32_t(p[3]) << 24;
}
uint64_t rd64(const unsigned char *p) { return uint64_t(rd32(p)) | uint64_t(rd32(p + 4)) << 32; }

int header_length(int type) {
    return type == kIIDC ? 172 : type == kAndor ? 128 : type == kXimea ? 240 : -1;
}

// Frame size and timestamp from one camera header (offsets per src/video_reader.hpp).
void decode(int type, const unsigned char *h, uint32_t *w, uint32_t *hh, uint64_t *ts) {
    if (type == kIIDC) {         // i_timestamp @48 (us), i_size_x @64, i_size_y @68
        *ts = rd64(h + 48);
        *w = rd32(h + 64);
        *hh = rd32(h + 68);
    } else if (type == kAndor) {  // a_timestamp_sec @24, x_start/end @48/52, y @56/60, bin @64/68
        *ts = rd64(h + 24);
        int32_t xs = int32_t(rd32(h + 48)), xe = int32_t(rd32(h + 52));
        int32_t ys = int32_t(rd32(h + 56)), ye = int32_t(rd32(h + 60));
        int32_t xb = int32_t(rd32(h + 64)), yb = int32_t(rd32(h + 68));
        *w = xb ? uint32_t((xe - xs + 1) / xb) : 0;
        *hh = yb ? uint32_t((ye - ys + 1) / yb) : 0;
    } else {                      // x_timestamp_sec @128, x_size_x @152, x_size_y @156
        *ts = rd64(h + 128);
        *w = rd32(h + 152);
        *hh = rd32(h + 156);
    }
}

}  // namespace

struct ddm_movie {
    FILE *f = nullptr;
    int type = 0;
    int header_len = 0;
    uint32_t length_data = 0;
    int w = 0, h = 0, bpp = 1;
    long long pos = 0;  // file offset of the next frame's header
};

extern "C" int ddm_movie_open(const char *path, int frame_offset, ddm_movie **out,
                              ddm_movie_info *info) {
    if (!path || !out || frame_offset < 0) return ddm::fail(DDM_ERR_INVALID_ARG, "ddm_movie_open: bad argument");
    FILE *f = std::fopen(path, "rb");
    if (!f) return ddm::fail(DDM_ERR_IO, "couldn't open .movie file");
    // Locate the first magic word, one byte at a time (src/video_reader.cpp:70-79).
    long magic_offset = 0;
    uint32_t word;
    unsigned char b4[4];
    while (std::fread(b4, 4, 1, f) == 1) {
        word = rd32(b4);
        if (word == kMagic) break;
        magic_offset++;
        std::fseek(f, magic_offset, SEEK_SET);
    }
    std::fseek(f, magic_offset, SEEK_SET);
    unsigned char common[24];
    auto bad = [&](const std::string &msg) {
        std::fclose(f);
        return ddm::fail(DDM_ERR_IO, msg);
    };
    if (std::fread(common, 24, 1, f) != 1)
        return bad("[.moviefile Initialise Error] Corrupted header at offset " + std::to_string(std::ftell(f)));
    if (rd32(common) != kMagic)
        return bad("[.moviefile Initialise Error] Wrong magic at offset " + std::to_string(std::ftell(f)));
    if (rd32(common + 4) != 1)
        return bad("[.moviefile Initialise Error] Unsupported movie version " + std::to_string(rd32(common + 4)));
    const int type = int(rd32(common + 8));
    const int hl = header_length(type);
    if (hl < 0) return bad("[Movie-file Init. Error] Unsupported camera type.");
    const uint32_t length_data = rd32(common + 20);
    std::fseek(f, -24, SEEK_CUR);
    unsigned char hdr[240];
    uint32_t w = 0, h = 0, w1, h1;
    uint64_t t0 = 0, t1 = 0;
    if (std::fread(hdr, hl, 1, f) != 1)
        return bad("[Movie-file Init Error] Corrupted header at offset " + std::to_string(std::ftell(f)));
    decode(type, hdr, &w, &h, &t0);
    std::fseek(f, length_data, SEEK_CUR);
    if (std::fread(hdr, hl, 1, f) != 1)  // second frame, for the frame rate
        return bad("[Movie-file Init. Error] Corrupted header at offset " + std::to_string(std::ftell(f)));
    decode(type, hdr, &w1, &h1, &t1);
    std::fseek(f, magic_offset + long(frame_offset) * (hl + long(length_data)), SEEK_SET);

    ddm_movie *m = new ddm_movie;
    m->f = f;
    m->pos = magic_offset + static_cast<long long>(frame_offset) * (hl + static_cast<long long>(length_data));
    m->type = type;
    m->header_len = hl;
    m->length_data = length_data;
    m->w = int(w);
    m->h = int(h);
    m->bpp = (rd32(common + 12) == kMono8) ? 1 : 2;  // src/video_reader.cpp:219
    if (uint64_t(m->w) * m->h * m->bpp != length_data) {
        std::fclose(f);
        delete m;
        return ddm::fail(DDM_ERR_IO, ".movie frame data length does not match width*height*bytes per pixel");
    }
    if (info) {
        info->width = m->w;
        info->height = m->h;
        info->bytes_per_pixel = m->bpp;
        // src/video_reader.cpp:221-222: 1.0e6 / static_cast<float>(frame_time)
        info->fps = static_cast<float>(1.0e6 / static_cast<float>(t1 - t0));
        info->camera_type = type;
        info->pixel_mode = int(rd32(common + 12));
    }
    *out = m;
    return DDM_OK;
}

namespace {
// All `n` bytes at file offset `at`, in as many positioned reads as the system returns.
bool read_at(int fd, void *dst, size_t n, long long at) {
    unsigned char *p = static_cast<unsigned char *>(dst);
    while (n > 0) {
        const ssize_t r = ::pread(fd, p, n, static_cast<off_t>(at));
        if (r <= 0) return false;
        p += r;
        at += r;
        n -= static_cast<size_t>(r);
    }
    return true;
}
constexpr int kReadThreads = 8;
}  // namespace

// Frames are fixed-size records (header + length_data bytes), so the frames of one call are
// read with positioned reads from up to kReadThreads threads at once: one reader of
// page-cached 1 MB frames moved about 4.6 GB/s, which was what bound the command line's
// file-to-ISF rate. The same checks as src/video_reader.cpp:240-284 (a header and a data
// block per frame); the file position advances by the frames read.
extern "C" int ddm_movie_read(ddm_movie *m, void *dst, int count) {
    if (!m || !dst || count < 0) return ddm::fail(DDM_ERR_INVALID_ARG, "ddm_movie_read: bad argument");
    unsigned char *out = static_cast<unsigned char *>(dst);
    const int fd = fileno(m->f);
    const long long rec = m->header_len + static_cast<long long>(m->length_data);
    long long bad_header = -1, bad_data = -1;  // offset of the first record that failed
    const int nt = std::max(1, std::min(count, kReadThreads));
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int i = 0; i < count; i++) {
        unsigned char hdr[240];
        const long long at = m->pos + i * rec;
        const bool hok = read_at(fd, hdr, static_cast<size_t>(m->header_len), at);
        const bool dok = hok && read_at(fd, out + size_t(i) * m->length_data, m->length_data, at + m->header_len);
        if (!hok || !dok) {
#pragma omp critical(ddm_movie_read_error)
            {
                long long &b = hok ? bad_data : bad_header;
                const long long off = hok ? at + m->header_len : at;
                if (b < 0 || off < b) b = off;
            }
        }
    }
    if (bad_header >= 0 && (bad_data < 0 || bad_header < bad_data))
        return ddm::fail(DDM_ERR_IO, "[.moviefile Read Error] Corrupted header at offset " + std::to_string(bad_header));
    if (bad_data >= 0)
        return ddm::fail(DDM_ERR_IO, "[.moviefile Read Error] Corrupted data at offset " + std::to_string(bad_data));
    m->pos += count * rec;
    return DDM_OK;
}

extern "C" int ddm_movie_close(ddm_movie *m) {
    if (!m) return DDM_OK;
    if (m->f) std::fclose(m->f);
    delete m;
    return DDM_OK;
}
