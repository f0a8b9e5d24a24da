// pt_jpeg.cpp — baseline (sequential, 8-bit, Huffman) JPEG decoding into 8-bit RGB for OBJ
// textures (ITU-T T.81), with the sample arithmetic of the loader the reference's image_texture
// uses (its third_party image loader, requested with 3 channels), so that decoded texels are the
// same bytes.  The arithmetic is fixed by that bar; the code is this library's own:
//   * coefficients dequantised while decoding and kept as int16;
//   * the inverse DCT is the islow integer method (Loeffler-Ligtenberg-Moschytz constants in
//     12-bit fixed point), evaluated as two passes of an integer basis-matrix product (columns
//     kept with 2 extra bits, rounding 2^9 >> 10; rows with rounding 2^16 and the +128 level
//     shift before >> 17; clamped to 0..255) — the same integers the factorised flow produces;
//   * chroma upsampled to the full grid with centred triangle filters (3:1 weights; 2x2:
//     (3 v + v' + 8) >> 4 over the vertical blend v = 3 near + far, clamped at the row ends;
//     2x1 and 1x2 likewise), other ratios by replication;
//   * YCbCr to RGB in 20-bit fixed point from per-chroma lookup tables (1.402, -0.71414 and
//     -0.34414 with its product truncated to the upper 16 bits, 1.772), result >> 20 clamped;
//     three components stored as R, G, B directly when they are labelled 'R' 'G' 'B' or an
//     Adobe marker says so in a file without JFIF;
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

// 12-bit fixed point, rounded as (int)(x * 4096 + 0.5) of the signed value (so a negative
// constant rounds toward zero after the + 0.5).
constexpr int q12(float x) { return int(double(x * 4096) + 0.5); }

// Inverse-DCT basis: kBasis.m[n][k] multiplies frequency k in sample n.  The islow method
// evaluates the Loeffler-Ligtenberg-Moschytz factorisation: shared butterflies with 12 rounded
// rotation constants.  Every step of it is an exact integer addition or multiplication, so each
// sample of a 1-D pass equals the dot product of the frequencies with one row of an integer
// matrix, whose entry is the sum of the rounded constants on the flow graph's paths from that
// frequency to that sample; this table holds those sums.
struct IdctBasis { int m[8][8]; };
constexpr IdctBasis make_idct_basis() {
    IdctBasis b{};
    const int r0541 = q12(0.5411961f), r0765 = q12(0.765366865f), n1847 = q12(-1.847759065f);
    const int r1175 = q12(1.175875602f), r0298 = q12(0.298631336f), r2053 = q12(2.053119869f);
    const int r3072 = q12(3.072711026f), r1501 = q12(1.501321110f), n0899 = q12(-0.899976223f);
    const int n2562 = q12(-2.562915447f), n1961 = q12(-1.961570560f), n0390 = q12(-0.390180644f);
    // even frequencies 0, 2, 4, 6: four sums, sample m and sample 7 - m both add sum m
    const int even[4][4] = {{4096, r0541 + r0765, 4096, r0541},
                            {4096, r0541, -4096, r0541 + n1847},
                            {4096, -r0541, -4096, -(r0541 + n1847)},
                            {4096, -(r0541 + r0765), 4096, -r0541}};
    // odd frequencies 1, 3, 5, 7: four sums, sample m adds sum m and sample 7 - m subtracts it;
    // each carries r1175 (f1 + f3 + f5 + f7) and the rotations of its own paths
    const int odd[4][4] = {{r1175 + r1501 + n0899 + n0390, r1175, r1175 + n0390, r1175 + n0899},
                           {r1175, r1175 + r3072 + n2562 + n1961, r1175 + n2562, r1175 + n1961},
                           {r1175 + n0390, r1175 + n2562, r1175 + r2053 + n2562 + n0390, r1175},
                           {r1175 + n0899, r1175 + n1961, r1175, r1175 + r0298 + n0899 + n1961}};
    for (int m = 0; m < 4; m++) {
        for (int j = 0; j < 4; j++) {
            b.m[m][2 * j] = even[m][j];
            b.m[7 - m][2 * j] = even[m][j];
            b.m[m][2 * j + 1] = odd[m][j];
            b.m[7 - m][2 * j + 1] = -odd[m][j];
        }
    }
    return b;
}
constexpr IdctBasis kIdct = make_idct_basis();

// 8x8 inverse DCT of dequantised coefficients (natural order) into 8-bit samples: a pass over the
// columns kept with 2 extra bits (x 2^-10, rounded), a pass over the rows (x 2^-17, rounded, with
// the +128 level shift), clamped to 0..255.  Sums wrap modulo 2^32 as 32-bit integer code does.
void idct8x8(uint8_t *out, int stride, const int16_t coef[64]) {
    int mid[64];
    for (int c = 0; c < 8; c++) {
        for (int n = 0; n < 8; n++) {
            int64_t acc = 512;
            for (int k = 0; k < 8; k++) acc += int64_t(kIdct.m[n][k]) * coef[8 * k + c];
            mid[8 * n + c] = int32_t(uint32_t(acc)) >> 10;
        }
    }
    const int64_t bias = 65536 + (int64_t(128) << 17);
    for (int r = 0; r < 8; r++) {
        for (int n = 0; n < 8; n++) {
            int64_t acc = bias;
            for (int k = 0; k < 8; k++) acc += int64_t(kIdct.m[n][k]) * mid[8 * r + k];
            out[r * stride + n] = clamp8(int32_t(uint32_t(acc)) >> 17);
        }
    }
}

// One full-resolution row of a component from its stored rows `near` (nearest to the output
// row) and `far` (the one beyond it), w stored samples, hs x vs subsampling.  Triangle filters:
// vertically 3 near + far; horizontally every output sample weighs its own stored sample 3:1
// against the neighbour on its side, the neighbour clamped to the row.  For 2x1 the loader the
// reference uses computes the second-to-last sample of a row (w >= 2) from the last two stored
// samples weighted 3:1 toward the earlier one; that is kept.
void upsample_row(uint8_t *out, const uint8_t *near, const uint8_t *far, int w, int hs, int vs) {
    if (hs == 1 && vs == 1) { std::memcpy(out, near, size_t(w)); return; }
    if (hs == 1 && vs == 2) { for (int i = 0; i < w; i++) out[i] = uint8_t((3 * near[i] + far[i] + 2) >> 2); return; }
    if (hs == 2 && (vs == 1 || vs == 2)) {
        // v[i]: the vertical blend in quarter units (vs == 2) or the stored sample (vs == 1)
        auto v = [&](int i) { return vs == 2 ? 3 * near[i] + far[i] : int(near[i]); };
        const int shift = vs == 2 ? 4 : 2, round = 1 << (shift - 1);
        int prev = v(0), cur = prev;
        for (int i = 0; i < w; i++) {
            int next = i + 1 < w ? v(i + 1) : cur;
            out[2 * i] = uint8_t((3 * cur + prev + round) >> shift);
            out[2 * i + 1] = uint8_t((3 * cur + next + round) >> shift);
            prev = cur;
            cur = next;
        }
        if (vs == 1 && w >= 2) out[2 * w - 2] = uint8_t((3 * near[w - 2] + near[w - 1] + 2) >> 2);
        return;
    }
    for (int i = 0; i < w; i++)
        for (int j = 0; j < hs; j++) out[i * hs + j] = near[i];
}

// YCbCr to RGB in 20-bit fixed point with the JFIF matrix (1.402, -0.71414, -0.34414, 1.772,
// each rounded to 12 bits then scaled by 2^8), the products looked up per chroma value; the Cb
// term of green keeps only its upper 16 bits, as the reference's loader computes it.
struct ChromaTables { int cr_r[256], cr_g[256], cb_g[256], cb_b[256]; };
constexpr int q20(float x) { return int(x * 4096.0f + 0.5f) << 8; }
constexpr ChromaTables make_chroma_tables() {
    ChromaTables t{};
    for (int value = 0; value < 256; value++) {
        const int c = value - 128;
        t.cr_r[value] = c * q20(1.40200f);
        t.cr_g[value] = c * -q20(0.71414f);
        t.cb_g[value] = int(unsigned(c * -q20(0.34414f)) & 0xffff0000u);
        t.cb_b[value] = c * q20(1.77200f);
    }
    return t;
}
constexpr ChromaTables kChroma = make_chroma_tables();

void ycbcr_to_rgb(uint8_t *rgb, const uint8_t *y, const uint8_t *cb, const uint8_t *cr, int count) {
    for (int i = 0; i < count; i++) {
        const int base = (int(y[i]) << 20) | (1 << 19);
        rgb[3 * i + 0] = clamp8((base + kChroma.cr_r[cr[i]]) >> 20);
        rgb[3 * i + 1] = clamp8((base + kChroma.cr_g[cr[i]] + kChroma.cb_g[cb[i]]) >> 20);
        rgb[3 * i + 2] = clamp8((base + kChroma.cb_b[cb[i]]) >> 20);
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
                idct8x8(&c.plane[size_t(by) * 8 * size_t(c.w2) + size_t(bx) * 8], c.w2, coef);
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
            else ycbcr_to_rgb(out, row[0], row[1], row[2], width);
        } else {
            for (int i = 0; i < width; i++) out[3 * i] = out[3 * i + 1] = out[3 * i + 2] = row[0][i];
        }
    }
    return true;
}

} // namespace ptb
