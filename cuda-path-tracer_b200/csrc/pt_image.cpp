// pt_image.cpp — texture images for OBJ import: PNG (inflated with zlib), PPM (P3, P6) and
// baseline JPEG (pt_jpeg.cpp), turned
// into 8-bit RGB rows top first, the form the reference's image_texture holds
// (src/textures/texture.h:65-72 loads with 3 channels and indexes data[3*i + 3*nx*j]).
//
// PNG reduction to RGB follows what that loader (stb_image with 3 requested channels) does:
// grey g -> (g, g, g), alpha dropped, palette entries looked up, 16-bit samples keep their high
// byte, 1/2/4-bit grey scaled to 0..255 (x255, x85, x17).  Interlaced PNGs are de-interlaced
// (Adam7).  Baseline JPEG goes to pt_jpeg.cpp.
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>
#include <zlib.h>
#include "pt_image.h"

namespace ptb {
namespace {

uint32_t be32(const unsigned char *p) { return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | p[3]; }

int paeth(int a, int b, int c) {
    int p = a + b - c, pa = p > a ? p - a : a - p, pb = p > b ? p - b : b - p, pc = p > c ? p - c : c - p;
    if (pa <= pb && pa <= pc) return a;
    return pb <= pc ? b : c;
}

// Undoes the per-row filters of one (sub)image in place; `bpp` = bytes per complete pixel (>= 1).
bool unfilter(unsigned char *data, size_t rows, size_t stride, size_t bpp, std::string &err) {
    std::vector<unsigned char> prev(stride, 0);
    unsigned char *out = data;
    const unsigned char *in = data;
    for (size_t y = 0; y < rows; y++) {
        int type = in[0];
        const unsigned char *src = in + 1;
        std::vector<unsigned char> row(stride);
        for (size_t x = 0; x < stride; x++) {
            int a = x >= bpp ? row[x - bpp] : 0, b = prev[x], c = x >= bpp ? prev[x - bpp] : 0;
            int v = src[x];
            switch (type) {
                case 0: break;
                case 1: v += a; break;
                case 2: v += b; break;
                case 3: v += (a + b) >> 1; break;
                case 4: v += paeth(a, b, c); break;
                default: err = "PNG: invalid filter type"; return false;
            }
            row[x] = (unsigned char)v;
        }
        std::memcpy(out, row.data(), stride);
        prev = row;
        in += stride + 1;
        out += stride;
    }
    return true;
}

bool decode_png(const std::vector<unsigned char> &file, Image &img, std::string &err) {
    static const unsigned char sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (file.size() < 8 || std::memcmp(file.data(), sig, 8) != 0) { err = "not a PNG file"; return false; }
    size_t pos = 8;
    uint32_t w = 0, h = 0;
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<unsigned char> idat, palette;
    while (pos + 12 <= file.size()) {
        uint32_t len = be32(&file[pos]);
        const unsigned char *type = &file[pos + 4];
        if (pos + 12 + size_t(len) > file.size()) { err = "PNG: truncated chunk"; return false; }
        const unsigned char *data = &file[pos + 8];
        if (!std::memcmp(type, "IHDR", 4)) {
            if (len < 13) { err = "PNG: bad IHDR"; return false; }
            w = be32(data); h = be32(data + 4); depth = data[8]; ctype = data[9]; interlace = data[12];
            if (data[10] != 0 || data[11] != 0) { err = "PNG: unsupported compression or filter method"; return false; }
        } else if (!std::memcmp(type, "PLTE", 4)) {
            palette.assign(data, data + len);
        } else if (!std::memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), data, data + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            break;
        }
        pos += 12 + size_t(len);
    }
    if (!w || !h || w > (1u << 24) || h > (1u << 24) || uint64_t(w) * h > (uint64_t(1) << 30)) { err = "PNG: bad dimensions"; return false; }
    int channels;
    switch (ctype) {
        case 0: channels = 1; break;
        case 2: channels = 3; break;
        case 3: channels = 1; break;
        case 4: channels = 2; break;
        case 6: channels = 4; break;
        default: err = "PNG: unknown colour type"; return false;
    }
    bool ok_depth = ctype == 0 ? (depth == 1 || depth == 2 || depth == 4 || depth == 8 || depth == 16)
                  : ctype == 3 ? (depth == 1 || depth == 2 || depth == 4 || depth == 8) : (depth == 8 || depth == 16);
    if (!ok_depth) { err = "PNG: unsupported bit depth"; return false; }
    if (ctype == 3 && palette.size() < 3) { err = "PNG: palette missing"; return false; }
    const size_t bits = size_t(channels) * size_t(depth);
    const size_t bpp = bits >= 8 ? bits / 8 : 1;
    // Adam7 passes: (x0, y0, dx, dy); one pass covering everything when not interlaced
    static const int adam7[7][4] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4}, {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
    const int passes = interlace ? 7 : 1;
    size_t raw_size = 0;
    size_t pw[7], ph[7];
    for (int p = 0; p < passes; p++) {
        int x0 = interlace ? adam7[p][0] : 0, y0 = interlace ? adam7[p][1] : 0, dx = interlace ? adam7[p][2] : 1, dy = interlace ? adam7[p][3] : 1;
        pw[p] = w > uint32_t(x0) ? (w - x0 + dx - 1) / dx : 0;
        ph[p] = h > uint32_t(y0) ? (h - y0 + dy - 1) / dy : 0;
        if (pw[p] && ph[p]) raw_size += ph[p] * (1 + (pw[p] * bits + 7) / 8);
    }
    std::vector<unsigned char> raw(raw_size);
    uLongf out_len = uLongf(raw_size);
    int zr = uncompress(raw.data(), &out_len, idat.data(), uLong(idat.size()));
    if (zr != Z_OK || out_len != raw_size) { err = "PNG: corrupt image data"; return false; }
    img.width = int(w);
    img.height = int(h);
    img.rgb.assign(size_t(w) * h * 3, 0);
    size_t offset = 0;
    for (int p = 0; p < passes; p++) {
        if (!pw[p] || !ph[p]) continue;
        int x0 = interlace ? adam7[p][0] : 0, y0 = interlace ? adam7[p][1] : 0, dx = interlace ? adam7[p][2] : 1, dy = interlace ? adam7[p][3] : 1;
        const size_t stride = (pw[p] * bits + 7) / 8;
        if (!unfilter(raw.data() + offset, ph[p], stride, bpp, err)) return false;
        // after unfilter the rows are packed contiguously (stride bytes each) at `offset`
        const unsigned char *rows = raw.data() + offset;
        for (size_t y = 0; y < ph[p]; y++) {
            const unsigned char *row = rows + y * stride;
            for (size_t x = 0; x < pw[p]; x++) {
                unsigned char rgb[3];
                auto sample = [&](int c) -> int {   // channel c of pixel x as 8 bits (raw index for palettes)
                    if (depth == 16) return row[(x * channels + c) * 2];
                    if (depth == 8) return row[x * channels + c];
                    size_t bit = x * size_t(depth);
                    int v = (row[bit / 8] >> (8 - depth - int(bit % 8))) & ((1 << depth) - 1);
                    if (ctype == 3) return v;
                    return depth == 1 ? v * 255 : depth == 2 ? v * 85 : v * 17;
                };
                if (ctype == 3) {
                    size_t i = size_t(sample(0));
                    if (3 * i + 2 >= palette.size()) { err = "PNG: palette index out of range"; return false; }
                    rgb[0] = palette[3 * i]; rgb[1] = palette[3 * i + 1]; rgb[2] = palette[3 * i + 2];
                } else if (channels <= 2) {
                    rgb[0] = rgb[1] = rgb[2] = (unsigned char)sample(0);
                } else {
                    rgb[0] = (unsigned char)sample(0); rgb[1] = (unsigned char)sample(1); rgb[2] = (unsigned char)sample(2);
                }
                size_t X = size_t(x0) + x * size_t(dx), Y = size_t(y0) + y * size_t(dy);
                std::memcpy(&img.rgb[(Y * w + X) * 3], rgb, 3);
            }
        }
        offset += ph[p] * (1 + stride);
    }
    return true;
}

// PPM: P6 (binary) or P3 (ASCII), maxval <= 255 scaled to 0..255, > 255 (two bytes) high byte
bool decode_ppm(const std::vector<unsigned char> &file, Image &img, std::string &err) {
    size_t pos = 2;
    auto token = [&](long &value) {
        for (;;) {
            while (pos < file.size() && std::isspace(file[pos])) pos++;
            if (pos < file.size() && file[pos] == '#') { while (pos < file.size() && file[pos] != '\n') pos++; continue; }
            break;
        }
        if (pos >= file.size() || !std::isdigit(file[pos])) return false;
        value = 0;
        while (pos < file.size() && std::isdigit(file[pos])) { value = value * 10 + (file[pos] - '0'); pos++; if (value > (1 << 28)) return false; }
        return true;
    };
    bool binary = file[1] == '6';
    long w, h, maxval;
    if (!token(w) || !token(h) || !token(maxval) || w <= 0 || h <= 0 || maxval <= 0 || maxval > 65535 || w * h > (1l << 30)) {
        err = "PPM: bad header"; return false;
    }
    img.width = int(w); img.height = int(h);
    img.rgb.assign(size_t(w) * size_t(h) * 3, 0);
    const size_t n = img.rgb.size();
    if (binary) {
        pos++;   // one whitespace byte after maxval
        const size_t bytes = maxval > 255 ? 2 : 1;
        if (pos + n * bytes > file.size()) { err = "PPM: truncated"; return false; }
        for (size_t i = 0; i < n; i++) {
            long v = bytes == 2 ? (long(file[pos + 2 * i]) << 8) | file[pos + 2 * i + 1] : file[pos + i];
            img.rgb[i] = (unsigned char)(maxval == 255 ? v : bytes == 2 ? (v >> 8) : v * 255 / maxval);
        }
    } else {
        for (size_t i = 0; i < n; i++) {
            long v;
            if (!token(v)) { err = "PPM: truncated"; return false; }
            img.rgb[i] = (unsigned char)(maxval == 255 ? v : v * 255 / maxval);
        }
    }
    return true;
}

} // namespace

bool load_image(const std::string &path, Image &img, std::string &err) {
    std::ifstream in(path, std::ios::binary);
    if (!in) { err = "could not open image: " + path; return false; }
    std::vector<unsigned char> file((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    bool ok;
    if (file.size() >= 8 && file[0] == 137 && file[1] == 'P' && file[2] == 'N' && file[3] == 'G') ok = decode_png(file, img, err);
    else if (file.size() >= 3 && file[0] == 'P' && (file[1] == '6' || file[1] == '3')) ok = decode_ppm(file, img, err);
    else if (file.size() >= 3 && file[0] == 0xFF && file[1] == 0xD8) ok = decode_jpeg(file, img, err);
    else { err = "unknown image format"; ok = false; }
    if (!ok) err = path + ": " + err;
    return ok;
}

} // namespace ptb
