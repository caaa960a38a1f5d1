// Disparity, normal and plane images on disk, in the two formats cvt writes them in:
//   PFM     PFMSaver / PFMLoader (plugins/isaver/PFM/PFMSaver.cpp, plugins/iloader/PFM/PFMLoader.cpp):
//           text header "Pf" (grey) or "PF" (RGB), "<width> <height>", scale (negative: little
//           endian), then float rows from the bottom row up; an RGBA image is saved without its
//           alpha and loaded with alpha 1
//   CVTRaw  CVTRawSaver / CVTRawLoader (plugins/isaver/CVTRaw/CVTRawSaver.cpp,
//           plugins/iloader/CVTRaw/CVTRawLoader.cpp): four uint32 (width, height, stride in
//           bytes, IFormat id), then height rows of `stride` bytes
// Host code only; errors are status codes with a message (pm_io_last_error()).
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/cvtpm.h"

namespace {

thread_local std::string t_io_err;

int io_fail(int code, const std::string& msg)
{
    t_io_err = msg;
    return code;
}

bool little_endian()
{
    const uint32_t v = 1;
    uint8_t b;
    memcpy(&b, &v, 1);
    return b == 1;
}

uint32_t bswap32(uint32_t v) { return (v >> 24) | ((v >> 8) & 0xff00u) | ((v << 8) & 0xff0000u) | (v << 24); }

struct File {
    FILE* f = nullptr;
    explicit File(FILE* p) : f(p) {}
    ~File()
    {
        if (f) fclose(f);
    }
};

bool read_all(const char* path, std::vector<uint8_t>& data)
{
    File fh(fopen(path, "rb"));
    if (!fh.f) return false;
    uint8_t buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, fh.f)) > 0) data.insert(data.end(), buf, buf + n);
    return !ferror(fh.f);
}

// the next non-empty header line that does not start with '#', split at spaces and tabs
// (PFMLoader::nextDataLine); pos moves past its newline
bool next_tokens(const std::vector<uint8_t>& d, size_t& pos, std::vector<std::string>& tok)
{
    while (pos < d.size()) {
        size_t e = pos;
        while (e < d.size() && d[e] != '\n') e++;
        std::string line(reinterpret_cast<const char*>(d.data()) + pos, e - pos);
        pos = e < d.size() ? e + 1 : e;
        tok.clear();
        std::string cur;
        for (char c : line) {
            if (c == ' ' || c == '\t' || c == '\r') {
                if (!cur.empty()) tok.push_back(cur);
                cur.clear();
            } else {
                cur += c;
            }
        }
        if (!cur.empty()) tok.push_back(cur);
        if (!tok.empty() && tok[0][0] != '#') return true;
    }
    return false;
}

}  // namespace

extern "C" {

const char* pm_io_last_error(void) { return t_io_err.c_str(); }

int pm_pfm_save(const char* path, const float* data, int width, int height, int channels, size_t stride)
{
    if (!path || !data || width <= 0 || height <= 0 || (channels != 1 && channels != 4) ||
        stride < (size_t)width * channels * sizeof(float))
        return io_fail(PM_EINVAL_ARG, "pm_pfm_save: bad argument");
    File fh(fopen(path, "wb"));
    if (!fh.f) return io_fail(PM_EINVAL_ARG, std::string("Could not open file for output: ") + path);
    // PFMSaver::save: "PF" for a 4-channel float image (saved without alpha), "Pf" for grey
    fprintf(fh.f, "%s\n%d %d\n%s1.0\n", channels == 4 ? "PF" : "Pf", width, height, little_endian() ? "-" : "");
    std::vector<float> row((size_t)width * 3);
    for (int y = height - 1; y >= 0; y--) {   // bottom to top
        const float* src = reinterpret_cast<const float*>(reinterpret_cast<const uint8_t*>(data) + (size_t)y * stride);
        size_t n = (size_t)width;
        if (channels == 4) {
            for (int x = 0; x < width; x++) {
                row[3 * (size_t)x] = src[4 * (size_t)x];
                row[3 * (size_t)x + 1] = src[4 * (size_t)x + 1];
                row[3 * (size_t)x + 2] = src[4 * (size_t)x + 2];
            }
            src = row.data();
            n *= 3;
        }
        if (fwrite(src, sizeof(float), n, fh.f) != n) return io_fail(PM_EINVAL_ARG, "pm_pfm_save: write failed");
    }
    return PM_OK;
}

int pm_pfm_load(const char* path, float* out, size_t capacity, int* width, int* height, int* channels)
{
    if (!path || !width || !height || !channels) return io_fail(PM_EINVAL_ARG, "pm_pfm_load: bad argument");
    std::vector<uint8_t> d;
    if (!read_all(path, d)) return io_fail(PM_EINVAL_ARG, std::string("Could not open file: ") + path);
    size_t pos = 0;
    std::vector<std::string> tok;
    if (!next_tokens(d, pos, tok)) return io_fail(PM_EINVAL_ARG, "PFM header corrupt");
    int ch;
    if (tok[0] == "Pf") ch = 1;
    else if (tok[0] == "PF") ch = 4;
    else return io_fail(PM_EINVAL_ARG, "Unknown PFM type: " + tok[0]);
    if (!next_tokens(d, pos, tok) || tok.size() < 2) return io_fail(PM_EINVAL_ARG, "PFM header corrupt: expected <width> <height>");
    const long w = strtol(tok[0].c_str(), nullptr, 10), h = strtol(tok[1].c_str(), nullptr, 10);
    if (!next_tokens(d, pos, tok)) return io_fail(PM_EINVAL_ARG, "PFM header corrupt: expected <scale>");
    const float scale = strtof(tok[0].c_str(), nullptr);
    if (w <= 0 || h <= 0 || w > (1L << 20) || h > (1L << 20)) return io_fail(PM_EINVAL_SHAPE, "PFM size out of range");
    *width = (int)w;
    *height = (int)h;
    *channels = ch;
    const size_t n = (size_t)w * h;
    if (!out) return PM_OK;   // size query
    if (capacity < n * ch) return io_fail(PM_EINVAL_ARG, "pm_pfm_load: output buffer too small");
    const size_t per = ch == 4 ? 3 : 1;
    if (d.size() - pos < n * per * sizeof(float)) return io_fail(PM_EINVAL_ARG, "PFM: not enough data");
    // PFMLoader::load: the data is read as is when this host is little endian and the scale is
    // negative, byte-swapped otherwise
    const bool swap = !(little_endian() && scale < 0);
    const uint8_t* src = d.data() + pos;
    for (long y = h - 1; y >= 0; y--) {   // file rows run bottom to top
        float* dst = out + (size_t)y * w * ch;
        for (long x = 0; x < w; x++)
            for (size_t c = 0; c < per; c++) {
                uint32_t v;
                memcpy(&v, src, 4);
                src += 4;
                if (swap) v = bswap32(v);
                memcpy(&dst[(size_t)x * ch + c], &v, 4);
            }
        if (ch == 4)
            for (long x = 0; x < w; x++) dst[(size_t)x * 4 + 3] = 1.0f;
    }
    return PM_OK;
}

int pm_cvtraw_save(const char* path, const void* data, int width, int height, size_t stride, int format_id)
{
    if (!path || !data || width <= 0 || height <= 0 || stride == 0 || stride > 0xffffffffu)
        return io_fail(PM_EINVAL_ARG, "pm_cvtraw_save: bad argument");
    File fh(fopen(path, "wb"));
    if (!fh.f) return io_fail(PM_EINVAL_ARG, std::string("Could not open file for output: ") + path);
    const uint32_t hdr[4] = {(uint32_t)width, (uint32_t)height, (uint32_t)stride, (uint32_t)format_id};
    if (fwrite(hdr, 4, 4, fh.f) != 4 || fwrite(data, 1, (size_t)height * stride, fh.f) != (size_t)height * stride)
        return io_fail(PM_EINVAL_ARG, "pm_cvtraw_save: write failed");
    return PM_OK;
}

int pm_cvtraw_load(const char* path, void* out, size_t capacity, size_t out_stride, int* width, int* height,
                   size_t* stride, int* format_id)
{
    if (!path || !width || !height || !stride || !format_id) return io_fail(PM_EINVAL_ARG, "pm_cvtraw_load: bad argument");
    std::vector<uint8_t> d;
    if (!read_all(path, d)) return io_fail(PM_EINVAL_ARG, std::string("Could not open file: ") + path);
    if (d.size() < 16) return io_fail(PM_EINVAL_ARG, "CVTRaw: header truncated");
    uint32_t hdr[4];
    memcpy(hdr, d.data(), 16);
    *width = (int)hdr[0];
    *height = (int)hdr[1];
    *stride = hdr[2];
    *format_id = (int)hdr[3];
    if (!out) return PM_OK;   // size query
    const size_t row = out_stride ? out_stride : hdr[2];
    const size_t keep = hdr[2] < row ? hdr[2] : row;
    if (hdr[1] > 0 && capacity < (size_t)(hdr[1] - 1) * row + keep)
        return io_fail(PM_EINVAL_ARG, "pm_cvtraw_load: output buffer too small");
    if (d.size() - 16 < (size_t)hdr[1] * hdr[2]) return io_fail(PM_EINVAL_ARG, "CVTRaw: not enough data");
    // CVTRawLoader::load copies the rows; here each row's full saved stride is kept
    for (uint32_t y = 0; y < hdr[1]; y++)
        memcpy(static_cast<uint8_t*>(out) + (size_t)y * row, d.data() + 16 + (size_t)y * hdr[2], keep);
    return PM_OK;
}

}  // extern "C"
