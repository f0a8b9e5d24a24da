// pt_jpeg.cpp — baseline (sequential, 8-bit, Huffman) JPEG decoding into 8-bit RGB for OBJ
// textures, with the sample arithmetic of the loader the reference's image_texture uses
// (third_party/stb_image.h of the reference, requested with 3 channels), so that decoded texels
// are the same bytes:
//   * coefficients dequantised while decoding and kept as int16;
//   * the integer inverse DCT of the IJG "islow" method (Loeffler–Ligtenberg–Moschytz, constants
//     in 12-bit fixed point), columns first with 2 extra bits kept (rounding 512 >> 10), rows
//     with rounding 2^16 and the +128 level shift before >> 17, clamped to 0..255; a column whose
//     AC terms are all zero takes 4 * DC;
//   * chroma upsampled to the full grid with the centred triangle filters (3:1 weights;
//     2x2: (3 * (3 n + f) + (3 n' + f') + 8) >> 4 inside a row, (3 n + f + 2) >> 2 at its ends;
//     2x1 and 1x2 likewise), other ratios by replication;
//   * YCbCr to RGB in fixed point: y << 20 plus 2^19, Cr * 1.402, Cr * -0.71414 plus the Cb term
//     * -0.34414 truncated to its upper 16 bits, Cb * 1.772, each constant rounded to 12 bits and
//     shifted by 8, result >> 20 clamped; three components stored as R, G, B directly when they
//     are labelled 'R' 'G' 'B' or an Adobe marker says so in a file without JFIF;
//   * one component: grey replicated.
// Progressive, lossless, arithmetic-coded, 12-bit and four-component files are rejected.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include "pt_image.h"

namespace ptb {
namespace {

const uint8_t kZigzag[64 + 15] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33,
                                  40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36,
                                  29, 22, 15, 23, 30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54,
                                  47, 55, 62, 63,
                                  // overrun guard: a run past 63 lands on 63
                                  63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63};

struct Huffman {
    // canonical code: for each length L, codes [mincode[L], maxcode[L]] map to values[valptr[L] + code - mincode[L]]
    int mincode[17], maxcode[18], valptr[17];
    uint8_t values[256];
    bool present = false;
};

struct Component {
    int id, h, v, tq, td, ta;
    int x, y, w2, h2;       // samples, padded plane width / height
    int dc;
    std::vector<uint8_t> plane;
};

struct Bits {
    const uint8_t *p, *end;
    uint32_t buffer = 0;
    int count = 0;
    int marker = -1;        // a marker met in the entropy-coded data (reading stops there)
    void fill() {
        while (count <= 24) {
            int byte = 0;
            if (marker < 0 && p < end) {
                byte = *p++;
                if (byte == 0xFF) {
                    int next = p < end ? *p : 0;
                    while (next == 0xFF && p + 1 < end) { p++; next = *p; }
                    if (next != 0) { marker = next; p++; byte = 0; }
                    else p++;
                }
            }
            buffer |= uint32_t(byte) << (24 - count);
            count += 8;
        }
    }
    int bits(int n) {
        if (n == 0) return 0;
        fill();
        int v = int(buffer >> (32 - n));
        buffer <<= n;
        count -= n;
        return v;
    }
    // EXTEND of the JPEG standard: an n-bit magnitude category to a signed value
    int receive_extend(int n) {
        if (n == 0) return 0;
        int v = bits(n);
        return v < (1 << (n - 1)) ? v - (1 << n) + 1 : v;
    }
    int decode(const Huffman &h) {
        fill();
        int code = 0;
        for (int len = 1; len <= 16; len++) {
            code = (code << 1) | int((buffer >> 31) & 1);
            buffer <<= 1;
            count--;
            if (count < 8) fill();
            if (h.maxcode[len] >= 0 && code <= h.maxcode[len] && code >= h.mincode[len]) return h.values[h.valptr[len] + code - h.mincode[len]];
        }
        return -1;
    }
    void restart() { buffer = 0; count = 0; marker = -1; }
};

inline uint8_t clamp8(int x) { return (unsigned)x > 255 ? (x < 0 ? 0 : 255) : uint8_t(x); }

// 12-bit fixed-point constants of the islow inverse DCT
constexpr int fix(float x) { return int(double(x * 4096) + 0.5); }

// one 8-point inverse DCT pass; s[] are the inputs at stride `stride`, results in out[8]
// before the caller's rounding/shift (even part x0..x3, odd part t0..t3 as in the islow method)
inline void idct_1d(const int *s, int stride, int &x0, int &x1, int &x2, int &x3, int &t0, int &t1, int &t2, int &t3) {
    int p2 = s[2 * stride], p3 = s[6 * stride];
    int p1 = (p2 + p3) * fix(0.5411961f);
    t2 = p1 + p3 * fix(-1.847759065f);
    t3 = p1 + p2 * fix(0.765366865f);
    p2 = s[0];
    p3 = s[4 * stride];
    t0 = (p2 + p3) * 4096;
    t1 = (p2 - p3) * 4096;
    x0 = t0 + t3; x3 = t0 - t3; x1 = t1 + t2; x2 = t1 - t2;
    t0 = s[7 * stride]; t1 = s[5 * stride]; t2 = s[3 * stride]; t3 = s[1 * stride];
    p3 = t0 + t2;
    int p4 = t1 + t3;
    p1 = t0 + t3;
    p2 = t1 + t2;
    int p5 = (p3 + p4) * fix(1.175875602f);
    t0 = t0 * fix(0.298631336f);
    t1 = t1 * fix(2.053119869f);
    t2 = t2 * fix(3.072711026f);
    t3 = t3 * fix(1.501321110f);
    p1 = p5 + p1 * fix(-0.899976223f);
    p2 = p5 + p2 * fix(-2.562915447f);
    p3 = p3 * fix(-1.961570560f);
    p4 = p4 * fix(-0.390180644f);
    t3 += p1 + p4;
    t2 += p2 + p3;
    t1 += p2 + p4;
    t0 += p1 + p3;
}

void idct_block(uint8_t *out, int stride, const int16_t coef[64]) {
    int tmp[64], in[64];
    for (int i = 0; i < 64; i++) in[i] = coef[i];
    for (int c = 0; c < 8; c++) {
        const int *d = in + c;
        if (!d[8] && !d[16] && !d[24] && !d[32] && !d[40] && !d[48] && !d[56]) {
            int dc = d[0] * 4;
            for (int r = 0; r < 8; r++) tmp[c + 8 * r] = dc;
            continue;
        }
        int x0, x1, x2, x3, t0, t1, t2, t3;
        idct_1d(d, 8, x0, x1, x2, x3, t0, t1, t2, t3);
        x0 += 512; x1 += 512; x2 += 512; x3 += 512;
        tmp[c + 0] = (x0 + t3) >> 10; tmp[c + 56] = (x0 - t3) >> 10;
        tmp[c + 8] = (x1 + t2) >> 10; tmp[c + 48] = (x1 - t2) >> 10;
        tmp[c + 16] = (x2 + t1) >> 10; tmp[c + 40] = (x2 - t1) >> 10;
        tmp[c + 24] = (x3 + t0) >> 10; tmp[c + 32] = (x3 - t0) >> 10;
    }
    for (int r = 0; r < 8; r++) {
        int x0, x1, x2, x3, t0, t1, t2, t3;
        idct_1d(tmp + 8 * r, 1, x0, x1, x2, x3, t0, t1, t2, t3);
        const int bias = 65536 + (128 << 17);
        x0 += bias; x1 += bias; x2 += bias; x3 += bias;
        uint8_t *o = out + r * stride;
        o[0] = clamp8((x0 + t3) >> 17); o[7] = clamp8((x0 - t3) >> 17);
        o[1] = clamp8((x1 + t2) >> 17); o[6] = clamp8((x1 - t2) >> 17);
        o[2] = clamp8((x2 + t1) >> 17); o[5] = clamp8((x2 - t1) >> 17);
        o[3] = clamp8((x3 + t0) >> 17); o[4] = clamp8((x3 - t0) >> 17);
    }
}

// One full-resolution row of a component from its stored rows `near` and `far` (w samples).
void upsample_row(uint8_t *out, const uint8_t *near, const uint8_t *far, int w, int hs, int vs) {
    if (hs == 1 && vs == 1) { std::memcpy(out, near, size_t(w)); return; }
    if (hs == 1 && vs == 2) { for (int i = 0; i < w; i++) out[i] = uint8_t((3 * near[i] + far[i] + 2) >> 2); return; }
    if (hs == 2 && vs == 1) {
        if (w == 1) { out[0] = out[1] = near[0]; return; }
        out[0] = near[0];
        out[1] = uint8_t((near[0] * 3 + near[1] + 2) >> 2);
        int i;
        for (i = 1; i < w - 1; i++) {
            int n = 3 * near[i] + 2;
            out[2 * i] = uint8_t((n + near[i - 1]) >> 2);
            out[2 * i + 1] = uint8_t((n + near[i + 1]) >> 2);
        }
        out[2 * i] = uint8_t((near[w - 2] * 3 + near[w - 1] + 2) >> 2);
        out[2 * i + 1] = near[w - 1];
        return;
    }
    if (hs == 2 && vs == 2) {
        if (w == 1) { out[0] = out[1] = uint8_t((3 * near[0] + far[0] + 2) >> 2); return; }
        int t1 = 3 * near[0] + far[0];
        out[0] = uint8_t((t1 + 2) >> 2);
        for (int i = 1; i < w; i++) {
            int t0 = t1;
            t1 = 3 * near[i] + far[i];
            out[2 * i - 1] = uint8_t((3 * t0 + t1 + 8) >> 4);
            out[2 * i] = uint8_t((3 * t1 + t0 + 8) >> 4);
        }
        out[2 * w - 1] = uint8_t((t1 + 2) >> 2);
        return;
    }
    for (int i = 0; i < w; i++)
        for (int j = 0; j < hs; j++) out[i * hs + j] = near[i];
}

constexpr int cfix(float x) { return int(x * 4096.0f + 0.5f) << 8; }

void ycbcr_row(uint8_t *out, const uint8_t *y, const uint8_t *cb, const uint8_t *cr, int count) {
    for (int i = 0; i < count; i++) {
        int yf = (y[i] << 20) + (1 << 19);
        int r_ = cr[i] - 128, b_ = cb[i] - 128;
        int r = yf + r_ * cfix(1.40200f);
        int g = yf + (r_ * -cfix(0.71414f)) + int(unsigned(b_ * -cfix(0.34414f)) & 0xffff0000u);
        int b = yf + b_ * cfix(1.77200f);
        out[3 * i] = clamp8(r >> 20);
        out[3 * i + 1] = clamp8(g >> 20);
        out[3 * i + 2] = clamp8(b >> 20);
    }
}

bool build_huffman(Huffman &h, const uint8_t counts[16], const uint8_t *symbols, int total) {
    int code = 0, k = 0;
    for (int len = 1; len <= 16; len++) {
        h.valptr[len] = k;
        h.mincode[len] = code;
        code += counts[len - 1];
        k += counts[len - 1];
        h.maxcode[len] = counts[len - 1] ? code - 1 : -1;
        if (code > (1 << len)) return false;
        code <<= 1;
    }
    if (total > 256) return false;
    std::memcpy(h.values, symbols, size_t(total));
    h.present = true;
    return true;
}

} // namespace

bool decode_jpeg(const std::vector<unsigned char> &file, Image &img, std::string &err) {
    const uint8_t *p = file.data(), *end = file.data() + file.size();
    if (file.size() < 4 || p[0] != 0xFF || p[1] != 0xD8) { err = "not a JPEG file"; return false; }
    p += 2;
    uint16_t quant[4][64] = {};
    Huffman dc[4], ac[4];
    std::vector<Component> comps;
    int width = 0, height = 0, restart_interval = 0, hmax = 1, vmax = 1, app14 = -1;
    bool jfif = false, frame = false;
    auto be16 = [&](const uint8_t *q) { return (q[0] << 8) | q[1]; };
    for (;;) {
        while (p < end && *p != 0xFF) p++;        // skip to a marker
        while (p < end && *p == 0xFF) p++;
        if (p >= end) break;
        int m = *p++;
        if (m == 0xD9) break;                    // EOI
        if (m == 0x00 || m == 0x01 || (m >= 0xD0 && m <= 0xD7)) continue;   // stuffed byte, TEM, stray RSTn
        if (p + 2 > end) { err = "JPEG: truncated marker"; return false; }
        int len = be16(p);
        if (len < 2 || p + len > end) { err = "JPEG: bad marker length"; return false; }
        const uint8_t *seg = p + 2, *seg_end = p + len;
        p += len;
        if (m == 0xDB) {                                      // DQT
            while (seg < seg_end) {
                int pq = *seg >> 4, tq = *seg & 15;
                seg++;
                if (tq > 3 || pq > 1) { err = "JPEG: bad quantisation table"; return false; }
                for (int i = 0; i < 64; i++) {
                    quant[tq][kZigzag[i]] = uint16_t(pq ? be16(seg) : *seg);
                    seg += pq ? 2 : 1;
                }
            }
        } else if (m == 0xC4) {                               // DHT
            while (seg + 17 <= seg_end) {
                int tc = *seg >> 4, th = *seg & 15;
                uint8_t counts[16];
                std::memcpy(counts, seg + 1, 16);
                int total = 0;
                for (int i = 0; i < 16; i++) total += counts[i];
                if (tc > 1 || th > 3 || seg + 17 + total > seg_end) { err = "JPEG: bad Huffman table"; return false; }
                if (!build_huffman(tc ? ac[th] : dc[th], counts, seg + 17, total)) { err = "JPEG: bad Huffman table"; return false; }
                seg += 17 + total;
            }
        } else if (m == 0xDD) {                               // DRI
            restart_interval = be16(seg);
        } else if (m == 0xE0) {                               // APP0
            if (seg_end - seg >= 5 && std::memcmp(seg, "JFIF\0", 5) == 0) jfif = true;
        } else if (m == 0xEE) {                               // APP14 (Adobe)
            if (seg_end - seg >= 12 && std::memcmp(seg, "Adobe", 5) == 0) app14 = seg[11];
        } else if (m == 0xC0 || m == 0xC1) {                  // SOF0 / SOF1 (Huffman, sequential)
            if (seg[0] != 8) { err = "JPEG: only 8-bit samples are supported"; return false; }
            height = be16(seg + 1);
            width = be16(seg + 3);
            int n = seg[5];
            if (width <= 0 || height <= 0 || (n != 1 && n != 3) || 6 + 3 * n > seg_end - seg) {
                err = n == 4 ? "JPEG: four-component (CMYK) files are not supported" : "JPEG: bad frame header";
                return false;
            }
            if (uint64_t(width) * uint64_t(height) > (uint64_t(1) << 30)) { err = "JPEG: image too large"; return false; }
            comps.resize(size_t(n));
            for (int i = 0; i < n; i++) {
                Component &c = comps[size_t(i)];
                c.id = seg[6 + 3 * i]; c.h = seg[7 + 3 * i] >> 4; c.v = seg[7 + 3 * i] & 15; c.tq = seg[8 + 3 * i];
                if (c.h < 1 || c.h > 4 || c.v < 1 || c.v > 4 || c.tq > 3) { err = "JPEG: bad component"; return false; }
                hmax = std::max(hmax, c.h); vmax = std::max(vmax, c.v);
            }
            const int mcu_x = (width + hmax * 8 - 1) / (hmax * 8), mcu_y = (height + vmax * 8 - 1) / (vmax * 8);
            for (Component &c : comps) {
                c.x = (width * c.h + hmax - 1) / hmax;
                c.y = (height * c.v + vmax - 1) / vmax;
                c.w2 = mcu_x * c.h * 8;
                c.h2 = mcu_y * c.v * 8;
                c.plane.assign(size_t(c.w2) * size_t(c.h2), 0);
            }
            frame = true;
        } else if ((m >= 0xC2 && m <= 0xCF) && m != 0xC4 && m != 0xC8 && m != 0xCC) {
            err = m == 0xC2 ? "JPEG: progressive files are not supported" : "JPEG: unsupported coding process";
            return false;
        } else if (m == 0xDA) {                               // SOS: decode the scan
            if (!frame) { err = "JPEG: scan before frame"; return false; }
            int ns = seg[0];
            if (ns < 1 || ns > int(comps.size()) || 1 + 2 * ns + 3 > seg_end - seg) { err = "JPEG: bad scan header"; return false; }
            std::vector<Component *> sc;
            for (int i = 0; i < ns; i++) {
                int id = seg[1 + 2 * i];
                Component *c = nullptr;
                for (Component &k : comps) if (k.id == id) c = &k;
                if (!c) { err = "JPEG: scan names an unknown component"; return false; }
                c->td = seg[2 + 2 * i] >> 4; c->ta = seg[2 + 2 * i] & 15;
                if (c->td > 3 || c->ta > 3 || !dc[c->td].present || !ac[c->ta].present) { err = "JPEG: missing Huffman table"; return false; }
                c->dc = 0;
                sc.push_back(c);
            }
            Bits bits{p, end};
            int16_t coef[64];
            auto block = [&](Component &c, int bx, int by) -> bool {
                std::memset(coef, 0, sizeof coef);
                int t = bits.decode(dc[c.td]);
                if (t < 0 || t > 15) return false;
                c.dc += bits.receive_extend(t);
                coef[0] = int16_t(c.dc * quant[c.tq][0]);
                for (int k = 1; k < 64;) {
                    int rs = bits.decode(ac[c.ta]);
                    if (rs < 0) return false;
                    int r = rs >> 4, s = rs & 15;
                    if (s == 0) {
                        if (rs != 0xF0) break;
                        k += 16;
                        continue;
                    }
                    k += r;
                    int zig = kZigzag[k > 63 ? 63 : k];
                    k++;
                    coef[zig] = int16_t(bits.receive_extend(s) * quant[c.tq][zig]);
                }
                idct_block(&c.plane[size_t(by) * 8 * size_t(c.w2) + size_t(bx) * 8], c.w2, coef);
                return true;
            };
            int todo = restart_interval ? restart_interval : 0x7fffffff;
            // after each restart interval but the scan's last: an RSTn, then fresh predictions
            auto after_unit = [&](bool last) {
                if (--todo > 0 || last) return;
                // expect RSTn: drop buffered bits, reset predictions
                if (bits.marker < 0) {
                    bits.count = 0;
                    while (bits.p + 1 < end && !(bits.p[0] == 0xFF && bits.p[1] >= 0xD0 && bits.p[1] <= 0xD7)) bits.p++;
                    if (bits.p + 1 < end) bits.p += 2;
                }
                bits.restart();
                for (Component &c : comps) c.dc = 0;
                todo = restart_interval;
            };
            if (ns == 1) {
                Component &c = *sc[0];
                const int bw = (c.x + 7) >> 3, bh = (c.y + 7) >> 3;
                for (int by = 0; by < bh; by++)
                    for (int bx = 0; bx < bw; bx++) {
                        if (!block(c, bx, by)) { err = "JPEG: corrupt entropy-coded data"; return false; }
                        after_unit(by == bh - 1 && bx == bw - 1);
                    }
            } else {
                const int mcu_x = (width + hmax * 8 - 1) / (hmax * 8), mcu_y = (height + vmax * 8 - 1) / (vmax * 8);
                for (int my = 0; my < mcu_y; my++)
                    for (int mx = 0; mx < mcu_x; mx++) {
                        for (Component *c : sc)
                            for (int v = 0; v < c->v; v++)
                                for (int u = 0; u < c->h; u++)
                                    if (!block(*c, mx * c->h + u, my * c->v + v)) { err = "JPEG: corrupt entropy-coded data"; return false; }
                        after_unit(my == mcu_y - 1 && mx == mcu_x - 1);
                    }
            }
            // continue after the scan's data: the next marker
            p = bits.p;
            if (bits.marker >= 0) p -= 2;
            if (p < file.data() + 2) p = file.data() + 2;
        }
    }
    if (!frame || comps.empty()) { err = "JPEG: no image"; return false; }
    img.width = width;
    img.height = height;
    img.rgb.assign(size_t(width) * size_t(height) * 3, 0);
    const size_t n = comps.size();
    std::vector<std::vector<uint8_t>> line(n, std::vector<uint8_t>(size_t(width) + 3 * 4 + 8));
    struct Cursor { int hs, vs, ystep, ypos, w_lores; const uint8_t *line0, *line1; };
    std::vector<Cursor> cur(n);
    for (size_t k = 0; k < n; k++) {
        Component &c = comps[k];
        cur[k].hs = hmax / c.h; cur[k].vs = vmax / c.v;
        cur[k].ystep = cur[k].vs >> 1; cur[k].ypos = 0;
        cur[k].w_lores = (width + cur[k].hs - 1) / cur[k].hs;
        cur[k].line0 = cur[k].line1 = c.plane.data();
        if (size_t(cur[k].w_lores) * size_t(cur[k].hs) + 8 > line[k].size()) line[k].resize(size_t(cur[k].w_lores) * size_t(cur[k].hs) + 8);
    }
    const bool is_rgb = n == 3 && ((comps[0].id == 'R' && comps[1].id == 'G' && comps[2].id == 'B') || (app14 == 0 && !jfif));
    std::vector<const uint8_t *> row(n);
    for (int y = 0; y < height; y++) {
        for (size_t k = 0; k < n; k++) {
            Cursor &r = cur[k];
            const bool bottom = r.ystep >= (r.vs >> 1);
            const uint8_t *near = bottom ? r.line1 : r.line0, *far = bottom ? r.line0 : r.line1;
            if (r.hs == 1 && r.vs == 1) row[k] = near;
            else { upsample_row(line[k].data(), near, far, r.w_lores, r.hs, r.vs); row[k] = line[k].data(); }
            if (++r.ystep >= r.vs) {
                r.ystep = 0;
                r.line0 = r.line1;
                if (++r.ypos < comps[k].y) r.line1 += comps[k].w2;
            }
        }
        uint8_t *out = &img.rgb[size_t(y) * size_t(width) * 3];
        if (n == 3) {
            if (is_rgb) for (int i = 0; i < width; i++) { out[3 * i] = row[0][i]; out[3 * i + 1] = row[1][i]; out[3 * i + 2] = row[2][i]; }
            else ycbcr_row(out, row[0], row[1], row[2], width);
        } else {
            for (int i = 0; i < width; i++) out[3 * i] = out[3 * i + 1] = out[3 * i + 2] = row[0][i];
        }
    }
    return true;
}

} // namespace ptb
