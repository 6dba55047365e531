// riv_oracle.cpp -- CPU oracle (test infrastructure only) for the riv2 P-frame encoder.
//
// A plain, single-threaded restatement of the reference's encoder path, residual codec,
// DCT, rANS coders and decoder.  Every function cites the reference file:line it
// restates; paths are relative to the reference project root:
//   enc/  = reitero_video/reitero_encode/src/
//   com/  = reitero_video/reitero_video_common/src/
//   res/  = reitero_video/reitero_residual/src/
//   dct/  = reitero_video/reitero_dct/src/
//   dec/  = reitero_video/reitero_decode/src/
// Build flags: -O2 -fwrapv -ffp-contract=off (no FMA contraction the reference lacks;
// wrapping i32 where the reference uses Wrapping / i32x8 arithmetic).  glibc logf /
// exp2f / log2 / pow are called exactly where the reference calls f32::ln / exp2 /
// f64::log2 / powf.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this.
#include "riv_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

namespace {

typedef std::vector<uint8_t> Bytes;

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int64_t clampl(int64_t v, int64_t lo, int64_t hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int8_t sat_i8(int v) { return (int8_t)clampi(v, -128, 127); }

// Rust `f32 as i16`: saturating, NaN -> 0.
static inline int16_t f32_as_i16(float f) {
    if (std::isnan(f)) return 0;
    if (f <= -32768.0f) return -32768;
    if (f >= 32767.0f) return 32767;
    return (int16_t)f;
}
static inline int32_t f32_as_i32(float f) {
    if (std::isnan(f)) return 0;
    if (f <= -2147483648.0f) return INT32_MIN;
    if (f >= 2147483647.0f) return INT32_MAX;
    return (int32_t)f;
}
static inline int64_t f64_as_i64(double d) {
    if (std::isnan(d)) return 0;
    if (d <= -9223372036854775808.0) return INT64_MIN;
    if (d >= 9223372036854775807.0) return INT64_MAX;
    return (int64_t)d;
}

// ----------------------------------------------------------------------------------
// MotionVector  (com/motion_vector.rs:3-117)
// ----------------------------------------------------------------------------------
struct MV {
    int8_t dx = 0, dy = 0, sx = 0, sy = 0;
    bool skip = false;
};
static inline int8_t clamp_sub(int8_t v) { return v < -1 ? -1 : (v > 1 ? 1 : v); }
static inline MV mv_new(int8_t dx, int8_t dy, int8_t sx, int8_t sy, bool skip) {  // :15-30
    MV m;
    m.dx = dx; m.dy = dy; m.sx = clamp_sub(sx); m.sy = clamp_sub(sy); m.skip = skip;
    return m;
}
static inline int dx_hp(const MV& m) { return (int)m.dx * 2 + m.sx; }  // :68
static inline int dy_hp(const MV& m) { return (int)m.dy * 2 + m.sy; }  // :70
static inline uint8_t mv_flags(const MV& m) {                          // :81-95
    uint8_t f = 0;
    if (m.sx == 1) f |= 0x01; else if (m.sx == -1) f |= 0x02;
    if (m.sy == 1) f |= 0x04; else if (m.sy == -1) f |= 0x08;
    if (m.skip) f |= 0x40;
    return f;
}
static inline MV mv_canon(MV m) {  // :103-117
    if (m.dx == -128 && m.sx == -1) m.sx = 0;
    if (m.dy == -128 && m.sy == -1) m.sy = 0;
    if (m.sx == -1) { m.sx = 1; m.dx = (int8_t)std::max(-128, (int)m.dx - 1); }
    if (m.sy == -1) { m.sy = 1; m.dy = (int8_t)std::max(-128, (int)m.dy - 1); }
    return m;
}
struct Tup { int8_t dx, dy, sx, sy; };
static inline bool operator==(const Tup& a, const Tup& b) {
    return a.dx == b.dx && a.dy == b.dy && a.sx == b.sx && a.sy == b.sy;
}
static inline Tup tup(const MV& m) { return Tup{m.dx, m.dy, m.sx, m.sy}; }

// ----------------------------------------------------------------------------------
// Planar YUV 4:2:0 frame (com/yuv.rs:187-322)
// ----------------------------------------------------------------------------------
struct Yuv {
    int w = 0, h = 0;
    Bytes y, u, v;
    void alloc(int W, int H) {
        w = W; h = H;
        y.assign((size_t)W * H, 0);
        u.assign((size_t)(W / 2) * (H / 2), 0);
        v.assign((size_t)(W / 2) * (H / 2), 0);
    }
};

// pad_rgb24 (enc/encoder.rs:1049-1096): right pad repeats the last pixel of each
// row, bottom pad repeats the last (padded) display row.
static Bytes pad_rgb24(const uint8_t* d, int dw, int dh, int sw, int sh) {
    Bytes out((size_t)sw * sh * 3, 0);
    for (int y = 0; y < dh; y++) {
        const uint8_t* src = d + (size_t)y * dw * 3;
        uint8_t* dst = out.data() + (size_t)y * sw * 3;
        memcpy(dst, src, (size_t)dw * 3);
        for (int x = dw; x < sw; x++) memcpy(dst + x * 3, src + (dw - 1) * 3, 3);
    }
    for (int y = dh; y < sh; y++)
        memcpy(out.data() + (size_t)y * sw * 3, out.data() + (size_t)(dh - 1) * sw * 3, (size_t)sw * 3);
    return out;
}

// RGB24 -> YUV 4:2:0, BT.709 limited range.  The reference calls the un-vendored
// `yuv` 0.8.9 crate (com/yuv.rs:56-65, Limited / Bt709 / Balanced); its exact integer
// arithmetic is not available here, so this is the project's own definition (13-bit
// fixed point, chroma from the rounded 2x2 RGB mean).  The CUDA path uses the same
// constants, so GPU == oracle holds bit-exactly; parity with the crate is unpinned.
static const int YR = 1496, YG = 5032, YB = 508;      // round(8192*K*219/255)
static const int UR = -824, UG = -2774, UB = 3598;     // Cb row, 224/255 scale
static const int VR = 3598, VG = -3268, VB = -330;     // Cr row
static void rgb_to_yuv420(const uint8_t* rgb, int w, int h, Yuv& out) {
    out.alloc(w, h);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            const uint8_t* p = rgb + ((size_t)y * w + x) * 3;
            int v = (YR * p[0] + YG * p[1] + YB * p[2] + (16 << 13) + (1 << 12)) >> 13;
            out.y[(size_t)y * w + x] = (uint8_t)clampi(v, 16, 235);
        }
    int cw = w / 2;
    for (int cy = 0; cy < h / 2; cy++)
        for (int cx = 0; cx < cw; cx++) {
            int s[3] = {0, 0, 0};
            for (int k = 0; k < 4; k++) {
                const uint8_t* p = rgb + ((size_t)(2 * cy + (k >> 1)) * w + 2 * cx + (k & 1)) * 3;
                s[0] += p[0]; s[1] += p[1]; s[2] += p[2];
            }
            int r = (s[0] + 2) >> 2, g = (s[1] + 2) >> 2, b = (s[2] + 2) >> 2;
            int cb = (UR * r + UG * g + UB * b + (128 << 13) + (1 << 12)) >> 13;
            int cr = (VR * r + VG * g + VB * b + (128 << 13) + (1 << 12)) >> 13;
            out.u[(size_t)cy * cw + cx] = (uint8_t)clampi(cb, 16, 240);
            out.v[(size_t)cy * cw + cx] = (uint8_t)clampi(cr, 16, 240);
        }
}

// YUV 4:2:0 -> RGB24 for the decoder's output (dec/decoder.rs:445-456: `to_rgb24`, then
// `crop_rgb24` to the display size; com/yuv.rs:94-110 calls the `yuv` crate's
// `yuv420_to_rgb`, limited range, BT.709, absent here).  The project's own definition, the
// inverse of rgb_to_yuv420: BT.709 (Kr 0.2126, Kb 0.0722) limited range in 13-bit fixed point,
// each chroma sample covering its 2x2 luma quad.  Parity with the crate is unpinned.
static const int IY = 9539;                   // round(8192*255/219)
static const int IRV = 14686, IBU = 17305;    // round(8192*255/224*1.5748), *1.8556
static const int IGU = 1747, IGV = 4366;      // round(8192*255/224*2Kb(1-Kb)/Kg), *2Kr(1-Kr)/Kg
static void yuv420_to_rgb24_crop(const Yuv& f, int dw, int dh, uint8_t* rgb) {
    const int cw = f.w / 2;
    for (int y = 0; y < dh; y++)
        for (int x = 0; x < dw; x++) {
            const int yv = IY * ((int)f.y[(size_t)y * f.w + x] - 16);
            const int u = (int)f.u[(size_t)(y / 2) * cw + x / 2] - 128, v = (int)f.v[(size_t)(y / 2) * cw + x / 2] - 128;
            uint8_t* p = rgb + ((size_t)y * dw + x) * 3;
            p[0] = (uint8_t)clampi((yv + IRV * v + (1 << 12)) >> 13, 0, 255);
            p[1] = (uint8_t)clampi((yv - IGU * u - IGV * v + (1 << 12)) >> 13, 0, 255);
            p[2] = (uint8_t)clampi((yv + IBU * u + (1 << 12)) >> 13, 0, 255);
        }
}

// ----------------------------------------------------------------------------------
// Deblocking filter (com/deblock.rs)
// ----------------------------------------------------------------------------------
static int deblock_level_from_quant_step(float qs) {  // :34-36
    float v = roundf(qs * 0.6f);
    if (v < 0.0f) v = 0.0f;
    if (v > 63.0f) v = 63.0f;
    return (int)v;
}
static void thresholds(int level, bool intra, int& e, int& i_lim, int& hev) {  // :40-58
    i_lim = std::max(level, 1);
    e = (level + 2) * 2 + i_lim;
    if (intra) hev = level >= 40 ? 2 : (level >= 15 ? 1 : 0);
    else hev = level >= 40 ? 3 : (level >= 20 ? 2 : (level >= 15 ? 1 : 0));
}
static inline int c128(int x) { return clampi(x, -128, 127); }
static void mb_filter_line(int* px, int E, int I, int H) {  // :68-115
    int p3 = px[0], p2 = px[1], p1 = px[2], p0 = px[3], q0 = px[4], q1 = px[5], q2 = px[6], q3 = px[7];
    bool mask = 2 * abs(p0 - q0) + abs(q1 - p1) / 2 <= E && abs(p3 - p2) <= I && abs(p2 - p1) <= I &&
                abs(p1 - p0) <= I && abs(q1 - q0) <= I && abs(q2 - q1) <= I && abs(q3 - q2) <= I;
    if (!mask) return;
    int ps2 = p2 - 128, ps1 = p1 - 128, ps0 = p0 - 128, qs0 = q0 - 128, qs1 = q1 - 128, qs2 = q2 - 128;
    bool hev = abs(p1 - p0) > H || abs(q1 - q0) > H;
    int w = c128(c128(ps1 - qs1) + 3 * (qs0 - ps0));
    if (hev) {
        int f1 = c128(w + 4) >> 3;
        int f2 = c128(w + 3) >> 3;
        px[4] = clampi(c128(qs0 - f1) + 128, 0, 255);
        px[3] = clampi(c128(ps0 + f2) + 128, 0, 255);
    } else {
        int a = c128((27 * w + 63) >> 7);
        int nq0 = c128(qs0 - a), np0 = c128(ps0 + a);
        a = c128((18 * w + 63) >> 7);
        int nq1 = c128(qs1 - a), np1 = c128(ps1 + a);
        a = c128((9 * w + 63) >> 7);
        int nq2 = c128(qs2 - a), np2 = c128(ps2 + a);
        px[1] = clampi(np2 + 128, 0, 255);
        px[2] = clampi(np1 + 128, 0, 255);
        px[3] = clampi(np0 + 128, 0, 255);
        px[4] = clampi(nq0 + 128, 0, 255);
        px[5] = clampi(nq1 + 128, 0, 255);
        px[6] = clampi(nq2 + 128, 0, 255);
    }
}
static void deblock_plane(uint8_t* plane, int w, int h, int grid, int E, int I, int H,
                          const uint8_t* mask) {  // :129-177
    int bw = w / grid;
    int px[8];
    for (int x = grid; x < w; x += grid) {
        int bx = x / grid;
        for (int y = 0; y < h; y++) {
            if (mask && !(mask[(y / grid) * bw + bx - 1] || mask[(y / grid) * bw + bx])) continue;
            size_t i = (size_t)y * w + x;
            for (int k = 0; k < 8; k++) px[k] = plane[i - 4 + k];
            mb_filter_line(px, E, I, H);
            for (int k = 0; k < 8; k++) plane[i - 4 + k] = (uint8_t)px[k];
        }
    }
    for (int y = grid; y < h; y += grid) {
        int by = y / grid;
        for (int x = 0; x < w; x++) {
            if (mask && !(mask[(by - 1) * bw + x / grid] || mask[by * bw + x / grid])) continue;
            for (int k = 0; k < 8; k++) px[k] = plane[(size_t)(y - 4 + k) * w + x];
            mb_filter_line(px, E, I, H);
            for (int k = 0; k < 8; k++) plane[(size_t)(y - 4 + k) * w + x] = (uint8_t)px[k];
        }
    }
}
static void deblock_yuv420(Yuv& f, int level, bool intra, const uint8_t* mask) {  // :189-202
    if (level <= 0) return;
    int E, I, H;
    thresholds(level, intra, E, I, H);
    deblock_plane(f.y.data(), f.w, f.h, 16, E, I, H, mask);
    deblock_plane(f.u.data(), f.w / 2, f.h / 2, 8, E, I, H, mask);
    deblock_plane(f.v.data(), f.w / 2, f.h / 2, 8, E, I, H, mask);
}

// ----------------------------------------------------------------------------------
// Motion search (enc/motion/scalar.rs, satd_scalar.rs, satd_simd.rs; non-`threads` build)
// Luma samples are u8; the reference's i32<<8 `MotionLuma` representation only adds a
// scale that `to_satd_sample` removes again (enc/motion/luma.rs:19-21,31-38).
// ----------------------------------------------------------------------------------
static const int HEX[6][2] = {{2, 0}, {1, 2}, {-1, 2}, {-2, 0}, {-1, -2}, {1, -2}};  // scalar.rs:8
static const int CARD[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};                    // scalar.rs:7

// satd_scalar.rs:4-100 -- per-4x4 sub-block clamped reference origin, early exit.
static int64_t sad_int_scalar(const uint8_t* prev, const uint8_t* curr, int w, int h, int x0, int y0, int dx,
                              int dy, int64_t limit) {
    int64_t sad = 0;
    for (int by = 0; by < 4; by++)
        for (int bx = 0; bx < 4; bx++) {
            int sx0 = x0 + bx * 4, sy0 = y0 + by * 4;
            if (sx0 < 0 || sy0 < 0 || sx0 >= w || sy0 >= h) continue;
            int rx0 = sx0 + dx, ry0 = sy0 + dy;
            if (rx0 < 0) rx0 = 0;
            if (ry0 < 0) ry0 = 0;
            if (rx0 + 4 > w) rx0 = std::max(w - 4, 0);
            if (ry0 + 4 > h) ry0 = std::max(h - 4, 0);
            bool in_c = sy0 + 4 <= h && sx0 + 4 <= w;
            bool in_p = ry0 + 4 <= h && rx0 + 4 <= w;
            if (in_c && in_p) {
                for (int sy = 0; sy < 4; sy++)
                    for (int sx = 0; sx < 4; sx++)
                        sad += abs((int)curr[(size_t)(sy0 + sy) * w + sx0 + sx] -
                                   (int)prev[(size_t)(ry0 + sy) * w + rx0 + sx]);
            } else {
                for (int sy = 0; sy < 4; sy++)
                    for (int sx = 0; sx < 4; sx++) {
                        int cy = sy0 + sy, cx = sx0 + sx, ry = ry0 + sy, rx = rx0 + sx;
                        if (cy >= 0 && cy < h && cx >= 0 && cx < w && ry >= 0 && ry < h && rx >= 0 && rx < w)
                            sad += abs((int)curr[(size_t)cy * w + cx] - (int)prev[(size_t)ry * w + rx]);
                    }
            }
            if (sad > limit) return sad;
        }
    return sad;
}
// satd_simd.rs:15-53 -- full-block in-bounds fast path (no early exit), else scalar.
static int64_t sad_int(const uint8_t* prev, const uint8_t* curr, int w, int h, int x0, int y0, int dx, int dy,
                       int64_t limit) {
    int rx = x0 + dx, ry = y0 + dy;
    bool in_c = x0 >= 0 && y0 >= 0 && x0 + 16 <= w && y0 + 16 <= h;
    bool in_p = rx >= 0 && ry >= 0 && rx + 16 <= w && ry + 16 <= h;
    if (in_c && in_p) {
        int64_t s = 0;
        for (int r = 0; r < 16; r++)
            for (int c = 0; c < 16; c++)
                s += abs((int)curr[(size_t)(y0 + r) * w + x0 + c] - (int)prev[(size_t)(ry + r) * w + rx + c]);
        return s;
    }
    return sad_int_scalar(prev, curr, w, h, x0, y0, dx, dy, limit);
}
// Floor-averaged half-pel luma sample (satd_scalar.rs:107-168): the reference averages
// values pre-scaled by 256, so the +1 / +2 rounding terms vanish after `>> 8`.
static inline int sample_hp_floor(const uint8_t* p, int w, int h, int xh, int yh) {
    xh = clampi(xh, 0, (w - 1) * 2);
    yh = clampi(yh, 0, (h - 1) * 2);
    int x0 = xh / 2, y0 = yh / 2;
    bool xo = xh & 1, yo = yh & 1;
    int x1 = x0 + 1 < w ? x0 + 1 : x0, y1 = y0 + 1 < h ? y0 + 1 : y0;
    int a = p[(size_t)y0 * w + x0];
    if (!xo && !yo) return a;
    int b = p[(size_t)y0 * w + x1], d = p[(size_t)y1 * w + x0], e = p[(size_t)y1 * w + x1];
    int A = a << 8, B = b << 8, D = d << 8, E = e << 8;
    int f;
    if (xo && !yo) f = (A + B + 1) / 2;
    else if (!xo && yo) f = (A + D + 1) / 2;
    else f = (A + B + D + E + 2) / 4;
    return f >> 8;
}
// satd_scalar.rs:171-222 (per-pixel early exit)
static int64_t sad_hp_scalar(const uint8_t* prev, const uint8_t* curr, int w, int h, int x0, int y0, int dxh,
                             int dyh, int64_t limit) {
    int64_t sad = 0;
    for (int yy = 0; yy < 16; yy++)
        for (int xx = 0; xx < 16; xx++) {
            int cx = x0 + xx, cy = y0 + yy;
            int r = sample_hp_floor(prev, w, h, cx * 2 + dxh, cy * 2 + dyh);
            sad += abs((int)curr[(size_t)cy * w + cx] - r);
            if (sad > limit) return sad;
        }
    return sad;
}
// satd_simd.rs:386-469 -- interior fast path (full SAD), else the scalar path.
static int64_t sad_hp(const uint8_t* prev, const uint8_t* curr, int w, int h, int x0, int y0, int dxh, int dyh,
                      int64_t limit) {
    int max_x = (w - 1) * 2, max_y = (h - 1) * 2;
    bool x_in = x0 * 2 + dxh >= 0 && (x0 + 15) * 2 + dxh <= max_x;
    bool y_in = y0 * 2 + dyh >= 0 && (y0 + 15) * 2 + dyh <= max_y;
    int xe = (dxh & 1) ? 1 : 0, ye = (dyh & 1) ? 1 : 0;
    bool inb = x0 >= 0 && y0 >= 0 && x0 + 16 + xe <= w && y0 + 16 + ye <= h;
    if (inb && x_in && y_in) {
        int64_t s = 0;
        for (int yy = 0; yy < 16; yy++)
            for (int xx = 0; xx < 16; xx++)
                s += abs((int)curr[(size_t)(y0 + yy) * w + x0 + xx] -
                         sample_hp_floor(prev, w, h, (x0 + xx) * 2 + dxh, (y0 + yy) * 2 + dyh));
        return s;
    }
    return sad_hp_scalar(prev, curr, w, h, x0, y0, dxh, dyh, limit);
}

static inline int median3(int a, int b, int c) {  // scalar.rs:24-43
    if (a > b) {
        if (b > c) return b;
        else if (a > c) return c;
        else return a;
    } else {
        if (a > c) return a;
        else if (b > c) return c;
        else return b;
    }
}
struct MvCostCtx {
    int nx, ny, rx, ry, mx, my;  // nearest, near, median
    double lambda;
};
static inline double mv_bits(int d) { return d == 0 ? 1.0 : 2.0 * log2((double)d) + 2.0; }
static int64_t estimate_mv_cost(int dx, int dy, const MvCostCtx& c) {  // scalar.rs:453-544
    if (c.lambda == 0.0) return 0;
    const double scale = 2.0;
    int64_t best = INT64_MAX;
    if (dx == c.nx && dy == c.ny) best = std::min(best, f64_as_i64(c.lambda * scale * 1.5));
    if (dx == c.rx && dy == c.ry) best = std::min(best, f64_as_i64(c.lambda * scale * 1.5));
    if (dx == c.mx && dy == c.my) best = std::min(best, f64_as_i64(c.lambda * scale * 1.5));
    if (dx == 0 && dy == 0) best = std::min(best, f64_as_i64(c.lambda * scale * 0.5));
    {
        double bx = mv_bits(abs(dx - c.nx)), by = mv_bits(abs(dy - c.ny));
        best = std::min(best, f64_as_i64(c.lambda * scale * (6.0 + bx + by)));
    }
    {
        double bx = mv_bits(abs(dx - c.rx)), by = mv_bits(abs(dy - c.ry));
        best = std::min(best, f64_as_i64(c.lambda * scale * (6.0 + bx + by)));
    }
    return best;
}
static inline int64_t sat_sub(int64_t a, int64_t b) {
    if (b > 0 && a < INT64_MIN + b) return INT64_MIN;
    if (b < 0 && a > INT64_MAX + b) return INT64_MAX;
    return a - b;
}
struct St { int dx, dy; int64_t cost; };

static void process_block_hex(int bx, int by, int w, int h, int sr, const std::vector<std::pair<int, int>>& cands,
                              const uint8_t* prev, const uint8_t* curr, int64_t zthr, int64_t pthr,
                              const MvCostCtx& mc, MV& out_mv, int64_t& out_sad) {  // scalar.rs:546-636
    // block_origin (scalar.rs:159-167): storage dims are multiples of 16, so no clamp occurs.
    int x0 = (bx * 16 + 16 <= w) ? bx * 16 : std::max(w - 16, 0);
    int y0 = (by * 16 + 16 <= h) ? by * 16 : std::max(h - 16, 0);
    // block_is_identical (scalar.rs:169-203) short-circuits to 0, which is the SAD anyway.
    int64_t zero_sad = sad_int(prev, curr, w, h, x0, y0, 0, 0, INT64_MAX);
    St st{0, 0, zero_sad + estimate_mv_cost(0, 0, mc)};
    bool skip_int = zthr > 0 && zero_sad <= zthr;
    if (!skip_int) {
        for (auto& c : cands) {  // evaluate_seed_candidates scalar.rs:638-678
            int dx = c.first, dy = c.second;
            if ((dx == 0 && dy == 0) || abs(dx) > sr || abs(dy) > sr) continue;
            int64_t mvc = estimate_mv_cost(dx, dy, mc);
            int64_t limit = sat_sub(st.cost, mvc);
            if (limit < 0) continue;
            int64_t sad = sad_int(prev, curr, w, h, x0, y0, dx, dy, limit);
            if (sad + mvc < st.cost) st = {dx, dy, sad + mvc};
        }
        int64_t cur_sad = st.cost - estimate_mv_cost(st.dx, st.dy, mc);
        if (pthr > 0 && cur_sad <= pthr) skip_int = true;
    }
    if (!skip_int) {  // refine_integer_motion scalar.rs:680-757
        for (;;) {
            bool improved = false;
            int cx = st.dx, cy = st.dy;
            for (int k = 0; k < 6; k++) {
                int dx = cx + HEX[k][0], dy = cy + HEX[k][1];
                if (abs(dx) > sr || abs(dy) > sr) continue;
                int64_t mvc = estimate_mv_cost(dx, dy, mc);
                int64_t limit = sat_sub(st.cost, mvc);
                if (limit < 0) continue;
                int64_t sad = sad_int(prev, curr, w, h, x0, y0, dx, dy, limit);
                if (sad + mvc < st.cost) { st = {dx, dy, sad + mvc}; improved = true; }
            }
            if (!improved) break;
        }
        int cx = st.dx, cy = st.dy;
        for (int k = 0; k < 4; k++) {
            int dx = cx + CARD[k][0], dy = cy + CARD[k][1];
            if (abs(dx) > sr || abs(dy) > sr) continue;
            int64_t mvc = estimate_mv_cost(dx, dy, mc);
            int64_t limit = sat_sub(st.cost, mvc);
            if (limit < 0) continue;
            int64_t sad = sad_int(prev, curr, w, h, x0, y0, dx, dy, limit);
            if (sad + mvc < st.cost) st = {dx, dy, sad + mvc};
        }
    }
    // refine_halfpel scalar.rs:759-839
    int bdx = st.dx * 2, bdy = st.dy * 2, best_dx = bdx, best_dy = bdy;
    int64_t best_total = sad_hp(prev, curr, w, h, x0, y0, bdx, bdy, INT64_MAX);
    int64_t best_sad = best_total;
    for (int sy = -1; sy <= 1; sy++)
        for (int sx = -1; sx <= 1; sx++) {
            if (sx == 0 && sy == 0) continue;
            int dxh = bdx + sx, dyh = bdy + sy;
            if ((st.dx == -128 && sx == -1) || (st.dy == -128 && sy == -1)) continue;
            bool frac = (dxh % 2 != 0) || (dyh % 2 != 0);
            int64_t pen = frac ? f64_as_i64(mc.lambda * 2.0 * 1.5) : 0;
            int64_t limit = sat_sub(best_total, pen);
            if (limit < 0) continue;
            int64_t sad = sad_hp(prev, curr, w, h, x0, y0, dxh, dyh, limit);
            if (sad + pen < best_total) { best_total = sad + pen; best_sad = sad; best_dx = dxh; best_dy = dyh; }
        }
    int dxh = clampi(best_dx, -255, 255), dyh = clampi(best_dy, -255, 255);
    // Rust `/` and `%` truncate toward zero, like C.
    out_mv = mv_canon(mv_new(sat_i8(dxh / 2), sat_i8(dyh / 2), (int8_t)(dxh % 2), (int8_t)(dyh % 2), false));
    out_sad = best_sad;
}

static void push_candidate(std::vector<std::pair<int, int>>& v, int dx, int dy, int sr) {  // scalar.rs:46-53
    if (abs(dx) > sr || abs(dy) > sr) return;
    for (auto& c : v)
        if (c.first == dx && c.second == dy) return;
    v.push_back({dx, dy});
}

// hex_search_impl, non-`threads` loop (scalar.rs:233-449) with
// gather_local_motion_candidates (scalar.rs:56-156).
static void hex_search(const uint8_t* prev, const uint8_t* curr, int w, int h, int sr_u8, const MV* prev_mvs,
                       int64_t zthr, int64_t pthr, double lambda, std::vector<MV>& mvs,
                       std::vector<int64_t>& sads) {
    int bw = (w + 15) / 16, bh = (h + 15) / 16;
    int sr = sr_u8;
    mvs.assign((size_t)bw * bh, mv_new(0, 0, 0, 0, false));
    sads.assign((size_t)bw * bh, 0);
    std::vector<std::pair<int, int>> cands;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            int idx = by * bw + bx;
            std::vector<std::pair<int, int>> preds;
            if (bx > 0) preds.push_back({mvs[idx - 1].dx, mvs[idx - 1].dy});
            if (by > 0) {
                const MV& t = mvs[(by - 1) * bw + bx];
                preds.push_back({t.dx, t.dy});
                if (bx + 1 < bw) preds.push_back({mvs[(by - 1) * bw + bx + 1].dx, mvs[(by - 1) * bw + bx + 1].dy});
                if (bx > 0) preds.push_back({mvs[(by - 1) * bw + bx - 1].dx, mvs[(by - 1) * bw + bx - 1].dy});
            }
            if (prev_mvs) preds.push_back({prev_mvs[idx].dx, prev_mvs[idx].dy});
            std::vector<std::pair<int, int>> uniq;
            for (auto& p : preds)
                if (std::find(uniq.begin(), uniq.end(), p) == uniq.end()) uniq.push_back(p);
            if (uniq.empty()) uniq.push_back({0, 0});
            if (uniq.size() == 1) uniq.push_back({0, 0});
            MvCostCtx mc;
            mc.nx = uniq[0].first; mc.ny = uniq[0].second;
            mc.rx = uniq[1].first; mc.ry = uniq[1].second;
            int lx = 0, ly = 0, tx = 0, ty = 0, trx = 0, try_ = 0;
            if (bx > 0) { lx = mvs[idx - 1].dx; ly = mvs[idx - 1].dy; }
            if (by > 0) { tx = mvs[(by - 1) * bw + bx].dx; ty = mvs[(by - 1) * bw + bx].dy; }
            if (by > 0 && bx + 1 < bw) { trx = mvs[(by - 1) * bw + bx + 1].dx; try_ = mvs[(by - 1) * bw + bx + 1].dy; }
            else if (by > 0 && bx > 0) { trx = mvs[(by - 1) * bw + bx - 1].dx; try_ = mvs[(by - 1) * bw + bx - 1].dy; }
            mc.mx = median3(lx, tx, trx);
            mc.my = median3(ly, ty, try_);
            mc.lambda = lambda;
            cands.clear();
            push_candidate(cands, 0, 0, sr);
            for (auto& p : preds) push_candidate(cands, p.first, p.second, sr);
            process_block_hex(bx, by, w, h, sr, cands, prev, curr, zthr, pthr, mc, mvs[idx], sads[idx]);
        }
}

// ----------------------------------------------------------------------------------
// Motion-compensated prediction
// ----------------------------------------------------------------------------------
static inline uint8_t sample_round(const uint8_t* p, int w, int h, int xh, int yh) {  // com/motion.rs:28-59
    xh = clampi(xh, 0, (w - 1) * 2);
    yh = clampi(yh, 0, (h - 1) * 2);
    int x0 = xh / 2, y0 = yh / 2;
    bool xo = xh & 1, yo = yh & 1;
    int x1 = x0 + 1 < w ? x0 + 1 : x0, y1 = y0 + 1 < h ? y0 + 1 : y0;
    int a = p[(size_t)y0 * w + x0];
    if (!xo && !yo) return (uint8_t)a;
    int b = p[(size_t)y0 * w + x1], d = p[(size_t)y1 * w + x0], e = p[(size_t)y1 * w + x1];
    if (xo && !yo) return (uint8_t)((a + b + 1) / 2);
    if (!xo && yo) return (uint8_t)((a + d + 1) / 2);
    return (uint8_t)((a + b + d + e + 2) / 4);
}

// build_predicted (com/fast_motion.rs:103-352).  The normative predictor: its row-wise
// fast paths reduce to per-sample clamped rounded bilinear sampling, except the integer
// MV copy path, whose chroma copies from the truncated (x0+dx)/2 origin.
static void build_predicted(const Yuv& prev, const std::vector<MV>& mvs, Yuv& out) {
    int w = prev.w, h = prev.h, cw = w / 2, ch = h / 2;
    out.alloc(w, h);
    int bw = (w + 15) / 16, bh = (h + 15) / 16;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            const MV& mv = mvs[(size_t)by * bw + bx];
            int mdx = dx_hp(mv), mdy = dy_hp(mv);
            int x0 = bx * 16, y0 = by * 16;
            if ((mdx & 1) == 0 && (mdy & 1) == 0) {  // :135-199
                int dx = mdx / 2, dy = mdy / 2;
                int sx0 = x0 + dx, sy0 = y0 + dy;
                if (sx0 >= 0 && sy0 >= 0 && sx0 + 15 < w && sy0 + 15 < h) {
                    for (int r = 0; r < 16; r++)
                        memcpy(&out.y[(size_t)(y0 + r) * w + x0], &prev.y[(size_t)(sy0 + r) * w + sx0], 16);
                    int csx = sx0 / 2, csy = sy0 / 2;
                    if (csx + 8 <= cw && csy + 8 <= ch) {
                        for (int r = 0; r < 8; r++) {
                            memcpy(&out.u[(size_t)(y0 / 2 + r) * cw + x0 / 2], &prev.u[(size_t)(csy + r) * cw + csx], 8);
                            memcpy(&out.v[(size_t)(y0 / 2 + r) * cw + x0 / 2], &prev.v[(size_t)(csy + r) * cw + csx], 8);
                        }
                    } else {  // :171-196 (unreachable for in-bounds luma; kept as restated)
                        for (int yy = 0; yy < 16; yy++) {
                            int y = clampi(y0 + yy, 0, h - 1);
                            if (y & 1) continue;
                            int ryh = y * 2 + mdy;
                            int rxh = x0 * 2 + mdx;
                            for (int xx = 0; xx < 16; xx += 2) {
                                int x = x0 + xx;
                                size_t ci = (size_t)(y / 2) * cw + x / 2;
                                out.u[ci] = sample_round(prev.u.data(), cw, ch, rxh >> 1, ryh >> 1);
                                out.v[ci] = sample_round(prev.v.data(), cw, ch, rxh >> 1, ryh >> 1);
                                rxh += 2;
                            }
                        }
                    }
                    continue;
                }
            }
            for (int yy = 0; yy < 16; yy++) {  // :201-346
                int y = clampi(y0 + yy, 0, h - 1);
                int ryh = clampi(y * 2 + mdy, 0, (h - 1) * 2);
                for (int xx = 0; xx < 16; xx++) {
                    int x = clampi(x0 + xx, 0, w - 1);
                    out.y[(size_t)y * w + x] = sample_round(prev.y.data(), w, h, x0 * 2 + mdx + 2 * xx, ryh);
                }
                if ((y & 1) == 0) {
                    int rxh0 = x0 * 2 + mdx, ryh_raw = y * 2 + mdy;
                    for (int xx = 0; xx < 16; xx += 2) {
                        size_t ci = (size_t)(y / 2) * cw + (x0 + xx) / 2;
                        out.u[ci] = sample_round(prev.u.data(), cw, ch, (rxh0 + xx * 2) >> 1, ryh_raw >> 1);
                        out.v[ci] = sample_round(prev.v.data(), cw, ch, (rxh0 + xx * 2) >> 1, ryh_raw >> 1);
                    }
                }
            }
        }
}
// reference_build_predicted (com/motion.rs:152-283): the scalar predictor used by the
// reference's own equivalence test (tests/fast_pred.rs).
static void reference_build_predicted(const Yuv& prev, const std::vector<MV>& mvs, Yuv& out) {
    int w = prev.w, h = prev.h, cw = w / 2, ch = h / 2;
    out.alloc(w, h);
    int bw = (w + 15) / 16, bh = (h + 15) / 16;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            const MV& mv = mvs[(size_t)by * bw + bx];
            int mdx = dx_hp(mv), mdy = dy_hp(mv);
            int x0 = bx * 16, y0 = by * 16;
            if ((mdx & 1) == 0 && (mdy & 1) == 0) {
                int sx0 = x0 + mdx / 2, sy0 = y0 + mdy / 2;
                if (sx0 >= 0 && sy0 >= 0 && sx0 + 15 < w && sy0 + 15 < h) {
                    for (int r = 0; r < 16; r++)
                        memcpy(&out.y[(size_t)(y0 + r) * w + x0], &prev.y[(size_t)(sy0 + r) * w + sx0], 16);
                    int csx = sx0 / 2, csy = sy0 / 2;
                    if (csx + 8 <= cw && csy + 8 <= ch)
                        for (int r = 0; r < 8; r++) {
                            memcpy(&out.u[(size_t)(y0 / 2 + r) * cw + x0 / 2], &prev.u[(size_t)(csy + r) * cw + csx], 8);
                            memcpy(&out.v[(size_t)(y0 / 2 + r) * cw + x0 / 2], &prev.v[(size_t)(csy + r) * cw + csx], 8);
                        }
                    continue;
                }
            }
            for (int yy = 0; yy < 16; yy++) {
                int y = clampi(y0 + yy, 0, h - 1);
                int ryh = y * 2 + mdy;
                int rxh = x0 * 2 + mdx;
                for (int xx = 0; xx < 16; xx++) {
                    int x = clampi(x0 + xx, 0, w - 1);
                    out.y[(size_t)y * w + x] = sample_round(prev.y.data(), w, h, rxh, ryh);
                    if ((y & 1) == 0 && (x & 1) == 0) {
                        size_t ci = (size_t)(y / 2) * cw + x / 2;
                        out.u[ci] = sample_round(prev.u.data(), cw, ch, rxh >> 1, ryh >> 1);
                        out.v[ci] = sample_round(prev.v.data(), cw, ch, rxh >> 1, ryh >> 1);
                    }
                    rxh += 2;
                }
            }
        }
}

// ----------------------------------------------------------------------------------
// RDO skip decision (enc/rdo.rs)
// ----------------------------------------------------------------------------------
static float quant_step_from_quality(uint8_t q) {  // res/residual.rs:13-23
    if (q == 100) return 1.0f;
    if (q == 1) return 112.0f;
    float qf = (float)q;
    float range = 112.0f - 1.0f;
    return 1.0f + (100.0f - qf) / 99.0f * range;
}
struct Lambda {
    double lambda, retention, slope, icpt, skip_bits, keep_bits;
};
static Lambda lambda_for_quality(uint8_t quality, double mult) {  // rdo.rs:23-48,75-86
    quality = (uint8_t)clampi(quality, 1, 100);
    uint32_t inv = 100u - quality;
    int qp = (int)round((double)inv * 0.6);
    qp = clampi(qp, 0, 60);
    Lambda L;
    L.lambda = mult * pow(2.0, ((double)qp - 12.0) / 3.0);
    double nq = (double)quality / 100.0;
    double q = (double)quant_step_from_quality(quality);
    L.slope = 0.5 / q;
    L.icpt = 5.0 + 0.56 * q;
    L.retention = 0.15 + ((q - 1.0) / 111.0) * 0.55;
    L.skip_bits = 0.55 - nq * 0.15;
    L.keep_bits = 1.20 + nq * 0.35;
    return L;
}
static bool rdo_decide(const Lambda& L, bool allow, double guard, int64_t satd_i, bool int_aligned) {  // :140-178
    double satd = (double)std::max<int64_t>(satd_i, 0);
    double skip_cost = satd + L.lambda * L.skip_bits;
    double est = L.icpt + L.slope * satd;
    if (est < 0.0) est = 0.0;
    double coded_cost = satd * L.retention + L.lambda * (L.keep_bits + est);
    if (!allow) return false;
    if (!int_aligned) return false;
    if (satd > guard) return false;
    return skip_cost <= coded_cost;
}

// ----------------------------------------------------------------------------------
// DCT (dct/)
// ----------------------------------------------------------------------------------
static int32_t T16[16][16], T8[8][8];  // T[i][j]: sample i, frequency j (dct16.rs:7-145, dct8.rs:6-25)
static bool g_tables = false;
static int32_t round_half_away(double v) { return (int32_t)(v >= 0 ? floor(v + 0.5) : -floor(-v + 0.5)); }
static void init_tables() {
    if (g_tables) return;
    const double PI = 3.14159265358979323846;
    for (int i = 0; i < 16; i++)
        for (int j = 0; j < 16; j++) {
            double c = j == 0 ? sqrt(1.0 / 16) : sqrt(2.0 / 16);
            T16[i][j] = round_half_away(262144.0 * c * cos((2 * i + 1) * j * PI / 32));
        }
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) {
            double c = j == 0 ? sqrt(1.0 / 8) : 0.5;
            T8[i][j] = round_half_away(262144.0 * c * cos((2 * i + 1) * j * PI / 16));
        }
    g_tables = true;
}
// fdct_1d_16 / fdct_1d_8 (dct16.rs:151-194, dct8.rs:32-52): i64 accumulate, +2^17 >> 18.
template <int N>
static void fdct_1d(const int32_t* in, int32_t* out, const int32_t (*T)[N]) {
    int64_t acc[N] = {0};
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) acc[j] += (int64_t)in[i] * (int64_t)T[i][j];
    for (int j = 0; j < N; j++) out[j] = (int32_t)clampl((acc[j] + (1LL << 17)) >> 18, INT32_MIN, INT32_MAX);
}
template <int N>
static void fdct_2d(const int32_t* blk, int32_t* out, const int32_t (*T)[N]) {  // rows, then columns
    int32_t rows[N * N], col[N], res[N];
    for (int r = 0; r < N; r++) fdct_1d<N>(blk + r * N, rows + r * N, T);
    for (int c = 0; c < N; c++) {
        for (int r = 0; r < N; r++) col[r] = rows[r * N + c];
        fdct_1d<N>(col, res, T);
        for (int r = 0; r < N; r++) out[r * N + c] = res[r];
    }
}
static inline int16_t quant_aq(int32_t c, float qs, float dz) {  // dct16.rs:325-331
    float r = (float)c / qs;
    if (fabsf(r) < dz) return 0;
    return f32_as_i16(roundf(r));
}
// idct_1d_16 (dct16.rs:201-233): wrapping i32 multiply-accumulate, +2^17 >> 18.
static void idct_1d_16(const int32_t* in, int32_t* out) {
    for (int x = 0; x < 16; x++) {
        uint32_t acc = 0;
        for (int i = 0; i < 16; i++) acc += (uint32_t)in[i] * (uint32_t)T16[x][i];
        out[x] = (int32_t)(acc + (1u << 17)) >> 18;
    }
}
static void idct16_2d(const int32_t* deq, int16_t* out) {  // dct16.rs:387-407
    int32_t rows[256], col[16], res[16];
    for (int v = 0; v < 16; v++) idct_1d_16(deq + v * 16, rows + v * 16);
    for (int x = 0; x < 16; x++) {
        for (int v = 0; v < 16; v++) col[v] = rows[v * 16 + x];
        idct_1d_16(col, res);
        for (int y = 0; y < 16; y++) out[y * 16 + x] = (int16_t)clampi(res[y], -32768, 32767);
    }
}
// 8x8 AAN-style IDCT (dct/fast_dct8.rs:123-174,273-330): the reference's own integer
// constants, wrapping i32 arithmetic, first pass over horizontal frequency (>>10,
// +512 bias), second over vertical frequency (>>17, +65536 bias).
static const int32_t K0541 = 2218, K1848 = -7572, K0765 = 3136, K1176 = 4817, K0299 = 1223, K2053 = 8411,
                     K3073 = 12595, K1501 = 6150, K0900 = -3685, K2563 = -10496, K1962 = -8035, K0390 = -1598;
static inline int32_t wmul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }
static inline int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
static inline int32_t wsub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
static void aan_1d(const int32_t s[8], int32_t xs[4], int32_t ts[4], int32_t bias) {
    int32_t p1 = wmul(wadd(s[2], s[6]), K0541);
    int32_t t2 = wadd(p1, wmul(s[6], K1848));
    int32_t t3 = wadd(p1, wmul(s[2], K0765));
    int32_t t0 = (int32_t)((uint32_t)wadd(s[0], s[4]) << 12);
    int32_t t1 = (int32_t)((uint32_t)wsub(s[0], s[4]) << 12);
    xs[0] = wadd(wadd(t0, t3), bias);
    xs[3] = wadd(wsub(t0, t3), bias);
    xs[1] = wadd(wadd(t1, t2), bias);
    xs[2] = wadd(wsub(t1, t2), bias);
    int32_t a0 = s[7], a1 = s[5], a2 = s[3], a3 = s[1];
    int32_t q3 = wadd(a0, a2), q4 = wadd(a1, a3), q1 = wadd(a0, a3), q2 = wadd(a1, a2);
    int32_t q5 = wmul(wadd(q3, q4), K1176);
    a0 = wmul(a0, K0299); a1 = wmul(a1, K2053); a2 = wmul(a2, K3073); a3 = wmul(a3, K1501);
    q1 = wadd(q5, wmul(q1, K0900));
    q2 = wadd(q5, wmul(q2, K2563));
    q3 = wmul(q3, K1962);
    q4 = wmul(q4, K0390);
    ts[3] = wadd(a3, wadd(q1, q4));
    ts[2] = wadd(a2, wadd(q2, q3));
    ts[1] = wadd(a1, wadd(q2, q4));
    ts[0] = wadd(a0, wadd(q1, q3));
}
static void idct8_aan(const int16_t* coef, const uint16_t* qt, int16_t* out) {
    int32_t tmp[8][8];  // tmp[x][v]
    for (int v = 0; v < 8; v++) {
        int32_t s[8], xs[4], ts[4];
        for (int u = 0; u < 8; u++) s[u] = (int32_t)coef[v * 8 + u] * (int32_t)qt[v * 8 + u];
        aan_1d(s, xs, ts, 512);
        tmp[0][v] = wadd(xs[0], ts[3]) >> 10; tmp[7][v] = wsub(xs[0], ts[3]) >> 10;
        tmp[1][v] = wadd(xs[1], ts[2]) >> 10; tmp[6][v] = wsub(xs[1], ts[2]) >> 10;
        tmp[2][v] = wadd(xs[2], ts[1]) >> 10; tmp[5][v] = wsub(xs[2], ts[1]) >> 10;
        tmp[3][v] = wadd(xs[3], ts[0]) >> 10; tmp[4][v] = wsub(xs[3], ts[0]) >> 10;
    }
    for (int x = 0; x < 8; x++) {
        int32_t xs[4], ts[4];
        aan_1d(tmp[x], xs, ts, 65536);
        int32_t r[8] = {wadd(xs[0], ts[3]) >> 17, wadd(xs[1], ts[2]) >> 17, wadd(xs[2], ts[1]) >> 17,
                        wadd(xs[3], ts[0]) >> 17, wsub(xs[3], ts[0]) >> 17, wsub(xs[2], ts[1]) >> 17,
                        wsub(xs[1], ts[2]) >> 17, wsub(xs[0], ts[3]) >> 17};
        for (int y = 0; y < 8; y++) out[y * 8 + x] = (int16_t)clampi(r[y], -32768, 32767);
    }
}

// ----------------------------------------------------------------------------------
// Residual codec (res/residual.rs)
// ----------------------------------------------------------------------------------
static const float JPEG_LUMA[64] = {16, 11, 10, 16, 24,  40,  51,  61,  12, 12, 14, 19, 26,  58,  60,  55,
                                    14, 13, 16, 24, 40,  57,  69,  56,  14, 17, 22, 29, 51,  87,  80,  62,
                                    18, 22, 37, 56, 68,  109, 103, 77,  24, 35, 55, 64, 81,  104, 113, 92,
                                    49, 64, 78, 87, 103, 121, 120, 101, 72, 92, 95, 98, 112, 100, 103, 99};
static const float JPEG_CHROMA[64] = {17, 18, 24, 47, 99, 99, 99, 99, 18, 21, 26, 66, 99, 99, 99, 99,
                                      24, 26, 56, 99, 99, 99, 99, 99, 47, 66, 99, 99, 99, 99, 99, 99,
                                      99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99,
                                      99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99};
static uint16_t f32_round_max1_u16(float s) {
    float r = roundf(s);
    if (r < 1.0f) r = 1.0f;
    if (r >= 65535.0f) return 65535;
    return (uint16_t)r;
}
static void build_intra_y_table(float qs, uint16_t* t) {  // residual.rs:58-85
    for (int v = 0; v < 16; v++)
        for (int u = 0; u < 16; u++) {
            float fx = (float)u * 7.0f / 15.0f, fy = (float)v * 7.0f / 15.0f;
            int x0 = (int)fx, y0 = (int)fy;
            int x1 = std::min(x0 + 1, 7), y1 = std::min(y0 + 1, 7);
            float dx = fx - (float)x0, dy = fy - (float)y0;
            float val = JPEG_LUMA[y0 * 8 + x0] * (1.0f - dx) * (1.0f - dy) + JPEG_LUMA[y0 * 8 + x1] * dx * (1.0f - dy) +
                        JPEG_LUMA[y1 * 8 + x0] * (1.0f - dx) * dy + JPEG_LUMA[y1 * 8 + x1] * dx * dy;
            float scaled = (val / JPEG_LUMA[0]) * qs;
            t[v * 16 + u] = f32_round_max1_u16(scaled);
        }
}
static void build_intra_uv_table(float qs, uint16_t* t) {  // residual.rs:89-96
    for (int i = 0; i < 64; i++) t[i] = f32_round_max1_u16((JPEG_CHROMA[i] / JPEG_CHROMA[0]) * qs);
}
// compute_aq_quant_steps (residual.rs:116-167): f32 arithmetic, glibc logf/exp2f,
// sequential f32 sum.
static void aq_steps(const uint8_t* py, int stride, int w, int h, float base, std::vector<float>& out) {
    int bw = w / 16, bh = h / 16, n = bw * bh;
    std::vector<float> var(n);
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            uint64_t s = 0, s2 = 0;
            for (int y = 0; y < 16; y++)
                for (int x = 0; x < 16; x++) {
                    uint64_t v = py[(size_t)(by * 16 + y) * stride + bx * 16 + x];
                    s += v; s2 += v * v;
                }
            float vv = (float)(s2 * 256 - s * s) / (float)(256 * 256);
            var[by * bw + bx] = std::max(vv, 4.0f);
        }
    float sum = 0.0f;
    for (int i = 0; i < n; i++) sum += logf(var[i]);
    float avg = sum / (float)n;
    out.resize(n);
    for (int i = 0; i < n; i++) {
        float off = 0.8f * (logf(var[i]) - avg);
        out[i] = base * exp2f(off / 6.0f);
    }
}

// ----------------------------------------------------------------------------------
// rANS core (com/rans.rs)
// ----------------------------------------------------------------------------------
static uint8_t ZERO_PROB[65536];
static bool g_zp = false;
static void init_zero_prob() {  // :30-42
    if (g_zp) return;
    ZERO_PROB[0] = 1;
    for (int i = 1; i < 65536; i++) {
        int zeros = i >> 8, ones = i & 0xff;
        uint8_t p = (uint8_t)((zeros << 8) / (zeros + ones));
        ZERO_PROB[i] = p ? p : 1;
    }
    g_zp = true;
}
struct BinProb {
    uint16_t packed = 0x0101;
    uint8_t p0() const { return ZERO_PROB[packed]; }
    void observe(bool bit) {  // :73-84
        uint16_t rot = bit ? (uint16_t)((packed << 8) | (packed >> 8)) : packed;
        uint32_t sum = (uint32_t)rot + 0x100u;
        uint16_t upd = (uint16_t)sum;
        if (sum > 0xFFFFu) {
            uint16_t mask = rot == 0xff01 ? 0xff00 : 0x8100;
            upd = (uint16_t)(((uint16_t)(rot + 0x101)) >> 1) | mask;
        }
        packed = bit ? (uint16_t)((upd << 8) | (upd >> 8)) : upd;
    }
};
static const int BATCH = 16386;  // :201
struct RansEnc {  // :215-292
    Bytes* sink;
    std::vector<std::pair<bool, uint8_t>> stack;  // stack[BATCH-1] is the oldest entry
    int sp = BATCH;
    explicit RansEnc(Bytes* s) : sink(s), stack(BATCH) {}
    static void put_sym(uint32_t& r, std::vector<uint16_t>& pushes, bool bit, uint8_t p) {
        uint32_t start = bit ? p : 0, freq = bit ? 256u - p : p;
        uint32_t xmax = ((65536u >> 8) << 16) * freq;
        if (r >= xmax) { pushes.push_back((uint16_t)r); r >>= 16; }
        r = ((r / freq) << 8) | ((r % freq) + start);
    }
    void drain() {  // :231-269
        uint32_t r0 = 65536, r1 = 65536;
        std::vector<uint16_t> pushes;  // push_front order
        int i = sp;
        if (i & 1) {
            uint8_t p = stack[i].second ? stack[i].second : 1;
            put_sym(r0, pushes, stack[i].first, p);
            i++;
            std::swap(r0, r1);
        }
        while (i < BATCH) {
            uint8_t pa = stack[i].second ? stack[i].second : 1, pb = stack[i + 1].second ? stack[i + 1].second : 1;
            put_sym(r0, pushes, stack[i].first, pa);
            put_sym(r1, pushes, stack[i + 1].first, pb);
            i += 2;
        }
        pushes.push_back((uint16_t)(r0 >> 16)); pushes.push_back((uint16_t)(r0 & 0xffff));
        pushes.push_back((uint16_t)(r1 >> 16)); pushes.push_back((uint16_t)(r1 & 0xffff));
        for (size_t k = pushes.size(); k-- > 0;) {
            sink->push_back((uint8_t)(pushes[k] & 0xff));
            sink->push_back((uint8_t)(pushes[k] >> 8));
        }
        sp = BATCH;
    }
    void put(bool bit, BinProb& ctx) {  // :271-279
        uint8_t p = ctx.p0();
        ctx.observe(bit);
        if (sp == 0) drain();
        sp--;
        stack[sp] = {bit, p};
    }
    void put_bypass(bool bit) {
        if (sp == 0) drain();
        sp--;
        stack[sp] = {bit, 128};
    }
    void finish() { drain(); }
};
struct RansDec {  // :299-354
    const uint8_t* src; size_t len, pos = 0;
    uint32_t r0 = 0, r1 = 0;
    int count = 0;
    bool err = false;
    uint16_t rd16() {
        if (pos + 2 > len) { err = true; pos = len; return 0; }
        uint16_t v = (uint16_t)(src[pos] | (src[pos + 1] << 8));
        pos += 2;
        return v;
    }
    uint32_t rd32() { uint32_t lo = rd16(); uint32_t hi = rd16(); return lo | (hi << 16); }
    RansDec(const uint8_t* s, size_t n) : src(s), len(n) { r0 = rd32(); r1 = rd32(); }
    void reload() {
        if (count == BATCH) { count = 0; r0 = rd32(); r1 = rd32(); }
        count++;
    }
    void adv(uint32_t& r, uint32_t start, uint32_t freq) {
        r = freq * (r >> 8) + (r & 255) - start;
        if (r < 65536) r = (r << 16) | rd16();
    }
    bool get(BinProb& ctx) {
        reload();
        uint32_t r = r0;
        r0 = r1;
        uint8_t p = ctx.p0();
        bool bit = (r & 255) >= p;
        ctx.observe(bit);
        adv(r, bit ? p : 0, bit ? 256u - p : p);
        r1 = r;
        return bit;
    }
    bool get_bypass() {
        reload();
        uint32_t r = r0;
        r0 = r1;
        uint32_t start = r & 0x80;
        adv(r, start, 128);
        r1 = r;
        return start != 0;
    }
};

// ----------------------------------------------------------------------------------
// DCT coefficient coder (res/rans.rs)
// ----------------------------------------------------------------------------------
static inline int eob_class(unsigned v) { return v <= 1 ? (int)v : 32 - __builtin_clz(v); }  // :46-53
static inline int luma_band(int p) { return p == 0 ? 0 : (p < 16 ? 1 : (p < 64 ? 2 : 3)); }
static inline int chroma_band(int p) { return p == 0 ? 0 : (p < 8 ? 1 : 2); }
static bool g_overflow = false;  // set where the reference would panic (index out of bounds)
// Class nctx is still coded (nctx continue bits, no stop bit), as the reference does,
// although its decoder stops at class nctx - 1; from class nctx + 1 the reference indexes
// contexts[nctx] and panics (reitero_residual/src/rans.rs:81-83).
static void enc_class_value(RansEnc& w, unsigned value, BinProb* ctx, int nctx) {  // :72-98,133-159
    int maxc = nctx - 1, cls = eob_class(value);
    if (cls > nctx) { g_overflow = true; return; }  // the reference panics here
    for (int c = 0; c < cls; c++) w.put(true, ctx[c]);
    if (cls < maxc) w.put(false, ctx[cls]);
    if (cls >= 2) {
        unsigned off = value - (1u << (cls - 1));
        for (int b = cls - 2; b >= 0; b--) w.put_bypass((off >> b) & 1);
    }
}
static unsigned dec_class_value(RansDec& r, BinProb* ctx, int nctx) {
    int maxc = nctx - 1, cls = 0;
    while (cls < maxc) {
        if (!r.get(ctx[cls])) break;
        cls++;
    }
    if (cls <= 1) return (unsigned)cls;
    unsigned off = 0;
    for (int k = 0; k < cls - 1; k++) off = (off << 1) | (unsigned)r.get_bypass();
    return (1u << (cls - 1)) + off;
}
struct DctCtx {
    BinProb sig_y[256], sig_c[64], mag_y[4][13], mag_c[3][13], eob_y[9], eob_c[7];
    int16_t prev_dc[3] = {0, 0, 0};
    bool dcp = false;
};
static void dct_encode_plane(RansEnc& w, DctCtx& c, const int16_t* plane, int n, bool luma, int pi) {  // :248-321
    int16_t dcv;
    int last;
    if (c.dcp) {
        int16_t d0 = plane[0], pred = c.prev_dc[pi];
        int16_t delta = (int16_t)(d0 - pred);
        c.prev_dc[pi] = d0;
        last = 0;
        for (int i = n - 1; i >= 1; i--)
            if (plane[i] != 0) { last = i; break; }
        dcv = delta;
    } else {
        last = 0;
        for (int i = n - 1; i >= 0; i--)
            if (plane[i] != 0) { last = i; break; }
        dcv = plane[0];
    }
    if (luma) enc_class_value(w, (unsigned)last, c.eob_y, 9);
    else enc_class_value(w, (unsigned)last, c.eob_c, 7);
    BinProb* sig = luma ? c.sig_y : c.sig_c;
    for (int i = 0; i <= last; i++) {
        int16_t v = i == 0 ? dcv : plane[i];
        w.put(v != 0, sig[i]);
        if (v != 0) {
            w.put_bypass(v < 0);
            unsigned a = (unsigned)abs((int)v) - 1;
            BinProb* mc = luma ? c.mag_y[luma_band(i)] : c.mag_c[chroma_band(i)];
            enc_class_value(w, a, mc, 13);
        }
    }
}
static void dct_decode_plane(RansDec& r, DctCtx& c, int16_t* blk, int n, bool luma, int pi) {  // :392-459
    int16_t dcpred = c.dcp ? c.prev_dc[pi] : 0;
    unsigned end = luma ? dec_class_value(r, c.eob_y, 9) : dec_class_value(r, c.eob_c, 7);
    if ((int)end >= n) { r.err = true; return; }
    BinProb* sig = luma ? c.sig_y : c.sig_c;
    for (unsigned i = 0; i <= end; i++) {
        if (r.get(sig[i])) {
            bool neg = r.get_bypass();
            BinProb* mc = luma ? c.mag_y[luma_band(i)] : c.mag_c[chroma_band(i)];
            int16_t a = (int16_t)(dec_class_value(r, mc, 13) + 1);
            blk[i] = neg ? (int16_t)-a : a;
        }
    }
    if (c.dcp) {
        blk[0] = (int16_t)(blk[0] + dcpred);
        c.prev_dc[pi] = blk[0];
    }
}

// ----------------------------------------------------------------------------------
// MV predictors (res/mv_predictor.rs) and MV entropy coder (res/mv_rans*)
// ----------------------------------------------------------------------------------
enum Mode { Z = 0, NEAREST = 1, NEAR = 2, TR = 3, TL = 4, NEW = 5, TEMPORAL = 6 };
struct Neigh {
    bool has_l = false, has_t = false, has_tr = false, has_tl = false, has_tm = false;
    Tup l{}, t{}, tr{}, tl{}, tm{};
};
static Neigh gather_neighbors(const std::vector<MV>& cur, const MV* prev, int bw, int bx, int by) {  // :59-118
    Neigh n;
    size_t idx = (size_t)by * bw + bx;
    if (bx > 0) { n.has_l = true; n.l = tup(cur[idx - 1]); }
    if (by > 0) {
        n.has_t = true; n.t = tup(cur[idx - bw]);
        if (bx + 1 < bw) { n.has_tr = true; n.tr = tup(cur[idx - bw + 1]); }
        if (bx > 0) { n.has_tl = true; n.tl = tup(cur[idx - bw - 1]); }
    }
    if (prev) { n.has_tm = true; n.tm = tup(prev[idx]); }
    return n;
}
struct Preds { Tup nearest, near, temporal; };
static Preds derive_predictors(const Neigh& n) {  // :135-163, :181-272
    std::vector<Tup> c;
    auto add = [&](const Tup& t) {
        for (auto& e : c)
            if (e == t) return;
        c.push_back(t);
    };
    if (n.has_l) add(n.l);
    if (n.has_t) add(n.t);
    if (n.has_tr) add(n.tr);
    if (n.has_tl) add(n.tl);
    if (n.has_tm) add(n.tm);
    Tup zero{0, 0, 0, 0};
    if (c.empty()) c.push_back(zero);
    if (c.size() == 1) c.push_back(zero);
    Preds p;
    p.nearest = c[0]; p.near = c[1];
    p.temporal = n.has_tm ? n.tm : zero;
    return p;
}
static int mode_context(const std::vector<int>& modes, int bw, int bx, int by) {  // :275-308
    int idx = by * bw + bx, score = 0;
    auto sc = [](int m) { return m == Z ? 2 : (m == NEW ? 0 : 1); };
    if (bx > 0 && idx - 1 < (int)modes.size()) score += sc(modes[idx - 1]);
    if (by > 0 && idx >= bw && idx - bw < (int)modes.size()) score += sc(modes[idx - bw]);
    return std::min(score, 3);
}
static int mv_class(unsigned mag) {  // res/mv_rans.rs:80-86
    if (mag == 0) return 0;
    int msb = 31 - __builtin_clz(mag);
    return std::min(msb + 1, 10);
}
enum Sub { SZ = 0, SP = 1, SM = 2 };  // Subpel, declaration order = Ord (mv_rans.rs:17-22)
struct Coded { int mode, base; int8_t dx, dy; int spx, spy; bool skip; };
typedef std::tuple<int8_t, int8_t, int, int> CandKey;
struct MvCoder {  // res/mv_rans/encoder.rs:60-412, decoder.rs:57-330
    BinProb skip, m_new[4], m_nz[4], m_near[4], m_tmp[4], m_tr[4], m_tl[4], b_nearest[4], b_near[4], b_tr[4],
        b_tl[4], cls_x[4], cls_y[4], sign_x, sign_y, mag_x[10], mag_y[10], sub_x, sub_y, hit[3], cidx[4];
    std::vector<CandKey> cands;
    std::map<CandKey, uint32_t> counts;
    uint32_t total = 0;
    void reset() { *this = MvCoder(); }
    static void enc_class(RansEnc& w, BinProb* ctx, int cls) {
        int lo = 0, hi = 10, d = 0;
        while (lo < hi) {
            int mid = (lo + hi) / 2;
            bool hiside = cls > mid;
            w.put(hiside, ctx[d]);
            if (hiside) lo = mid + 1; else hi = mid;
            d++;
        }
    }
    static int dec_class(RansDec& r, BinProb* ctx) {
        int lo = 0, hi = 10, d = 0;
        while (lo < hi) {
            int mid = (lo + hi) / 2;
            if (r.get(ctx[d])) lo = mid + 1; else hi = mid;
            d++;
        }
        return lo;
    }
    static void enc_comp(RansEnc& w, int8_t delta, BinProb* cls, BinProb& sign, BinProb* mag) {
        unsigned m = (unsigned)abs((int)delta);
        int c = mv_class(m);
        enc_class(w, cls, c);
        if (c == 0) return;
        w.put(delta < 0, sign);
        unsigned base = 1u << (c - 1), bits = c <= 1 ? 0 : c - 1, off = m - base;
        for (unsigned b = 0; b < bits; b++) w.put((off >> b) & 1, mag[b]);
    }
    static int8_t dec_comp(RansDec& r, BinProb* cls, BinProb& sign, BinProb* mag) {
        int c = dec_class(r, cls);
        if (c == 0) return 0;
        bool s = r.get(sign);
        unsigned base = 1u << (c - 1), bits = c <= 1 ? 0 : c - 1, off = 0;
        for (unsigned b = 0; b < bits; b++)
            if (r.get(mag[b])) off |= 1u << b;
        int v = (int)(base + off);
        return sat_i8(s ? -v : v);
    }
    void update(const std::vector<Coded>& blocks) {  // encoder.rs:370-412
        for (auto& kv : counts) kv.second = (kv.second * 7) / 8;
        total = (total * 7) / 8;
        for (auto& b : blocks)
            if (b.mode == NEW) {
                if (b.spx == SM || b.spy == SM) continue;  // (encoder panics; never reached)
                counts[CandKey(b.dx, b.dy, b.spx, b.spy)] += 1;
                total++;
            }
        for (auto it = counts.begin(); it != counts.end();)
            if (it->second == 0) it = counts.erase(it); else ++it;
        cands.clear();
        if (total < 100) return;
        std::vector<std::pair<CandKey, uint32_t>> s(counts.begin(), counts.end());
        std::stable_sort(s.begin(), s.end(), [](const std::pair<CandKey, uint32_t>& a, const std::pair<CandKey, uint32_t>& b) {
            if (a.second != b.second) return a.second > b.second;
            return a.first < b.first;
        });
        uint32_t thr = total / 100;
        for (auto& e : s) {
            if (cands.size() >= 16) break;
            if (e.second > thr) cands.push_back(e.first);
        }
    }
    Bytes encode_frame(const std::vector<Coded>& blocks, int bw) {  // encoder.rs:145-255,351-368
        Bytes out;
        RansEnc w(&out);
        std::vector<int> modes;
        std::vector<bool> hits;
        for (size_t i = 0; i < blocks.size(); i++) {
            const Coded& b = blocks[i];
            int bx = (int)(i % bw), by = (int)(i / bw);
            w.put(b.skip, skip);
            int ctx = mode_context(modes, bw, bx, by);
            bool is_new = b.mode == NEW;
            w.put(is_new, m_new[ctx]);
            if (!is_new) {
                bool nz = b.mode != Z;
                w.put(nz, m_nz[ctx]);
                if (nz) {
                    bool nr = b.mode == NEAR;
                    w.put(nr, m_near[ctx]);
                    if (!nr) {
                        bool tm = b.mode == TEMPORAL;
                        w.put(tm, m_tmp[ctx]);
                        if (!tm) {
                            bool tr = b.mode == TR;
                            w.put(tr, m_tr[ctx]);
                            if (!tr) w.put(b.mode == TL, m_tl[ctx]);
                        }
                    }
                }
            }
            if (is_new) {
                bool e0 = b.base == 0;
                w.put(e0, b_nearest[ctx]);
                if (!e0) {
                    bool e1 = b.base == 1;
                    w.put(e1, b_near[ctx]);
                    if (!e1) {
                        bool e2 = b.base == 2;
                        w.put(e2, b_tr[ctx]);
                        if (!e2) w.put(b.base == 3, b_tl[ctx]);
                    }
                }
                bool via_cand = false;
                if (!cands.empty()) {
                    int ci = -1;
                    for (size_t k = 0; k < cands.size(); k++)
                        if (cands[k] == CandKey(b.dx, b.dy, b.spx, b.spy)) { ci = (int)k; break; }
                    bool hit_ = ci >= 0;
                    bool lh = bx > 0 ? hits[i - 1] : false, th = by > 0 ? hits[i - bw] : false;
                    w.put(hit_, hit[(int)lh + (int)th]);
                    if (hit_) {
                        int lo = 0, hi = 16, d = 0;
                        while (hi - lo > 1) {
                            int mid = (lo + hi) / 2;
                            bool g = ci >= mid;
                            w.put(g, cidx[d]);
                            if (g) lo = mid; else hi = mid;
                            d++;
                        }
                        via_cand = true;
                    } else {
                        enc_comp(w, b.dx, cls_x, sign_x, mag_x);
                        enc_comp(w, b.dy, cls_y, sign_y, mag_y);
                    }
                    hits.push_back(hit_);
                } else {
                    enc_comp(w, b.dx, cls_x, sign_x, mag_x);
                    enc_comp(w, b.dy, cls_y, sign_y, mag_y);
                    hits.push_back(false);
                }
                if (!via_cand) {
                    w.put(b.spx != SZ, sub_x);
                    w.put(b.spy != SZ, sub_y);
                }
            } else {
                hits.push_back(false);
            }
            modes.push_back(b.mode);
        }
        w.finish();
        update(blocks);
        return out;
    }
    bool decode_frame(const uint8_t* data, size_t len, int bw, int bh, std::vector<Coded>& out) {  // decoder.rs:149-283
        RansDec r(data, len);
        int n = bw * bh;
        out.clear();
        std::vector<int> modes;
        std::vector<bool> hits;
        for (int i = 0; i < n; i++) {
            int bx = i % bw, by = i / bw;
            Coded b{};
            b.skip = r.get(skip);
            int ctx = mode_context(modes, bw, bx, by);
            int mode;
            if (r.get(m_new[ctx])) mode = NEW;
            else if (!r.get(m_nz[ctx])) mode = Z;
            else if (r.get(m_near[ctx])) mode = NEAR;
            else if (r.get(m_tmp[ctx])) mode = TEMPORAL;
            else if (r.get(m_tr[ctx])) mode = TR;
            else if (r.get(m_tl[ctx])) mode = TL;
            else mode = NEAREST;
            b.mode = mode;
            b.spx = SZ; b.spy = SZ; b.dx = 0; b.dy = 0; b.base = 0;
            if (mode == NEW) {
                if (r.get(b_nearest[ctx])) b.base = 0;
                else if (r.get(b_near[ctx])) b.base = 1;
                else if (r.get(b_tr[ctx])) b.base = 2;
                else b.base = r.get(b_tl[ctx]) ? 3 : 4;
                bool via = false;
                if (!cands.empty()) {
                    bool lh = bx > 0 ? hits[i - 1] : false, th = by > 0 ? hits[i - bw] : false;
                    bool h = r.get(hit[(int)lh + (int)th]);
                    if (h) {
                        int lo = 0, hi = 16, d = 0;
                        while (hi - lo > 1) {
                            int mid = (lo + hi) / 2;
                            if (r.get(cidx[d])) lo = mid; else hi = mid;
                            d++;
                        }
                        if (lo < (int)cands.size()) {
                            b.dx = std::get<0>(cands[lo]); b.dy = std::get<1>(cands[lo]);
                            b.spx = std::get<2>(cands[lo]); b.spy = std::get<3>(cands[lo]);
                            via = true;
                        }
                    } else {
                        b.dx = dec_comp(r, cls_x, sign_x, mag_x);
                        b.dy = dec_comp(r, cls_y, sign_y, mag_y);
                    }
                    hits.push_back(h);
                } else {
                    b.dx = dec_comp(r, cls_x, sign_x, mag_x);
                    b.dy = dec_comp(r, cls_y, sign_y, mag_y);
                    hits.push_back(false);
                }
                if (!via) {
                    b.spx = r.get(sub_x) ? SP : SZ;
                    b.spy = r.get(sub_y) ? SP : SZ;
                }
            } else {
                hits.push_back(false);
            }
            out.push_back(b);
            modes.push_back(mode);
        }
        update(out);
        return !r.err;
    }
};

// ----------------------------------------------------------------------------------
// Packed frame records (com/format.rs)
// ----------------------------------------------------------------------------------
static void put_le(Bytes& b, uint64_t v, int n) {
    for (int i = 0; i < n; i++) b.push_back((uint8_t)(v >> (8 * i)));
}
static uint64_t get_le(const uint8_t* p, int n) {
    uint64_t v = 0;
    for (int i = 0; i < n; i++) v |= (uint64_t)p[i] << (8 * i);
    return v;
}
static Bytes header_bytes(const oracle_config& c, uint64_t frame_count) {  // :64-88
    Bytes b = {'R', 'I', 'V', 0};
    put_le(b, 5, 4);
    put_le(b, c.display_width, 4); put_le(b, c.display_height, 4);
    put_le(b, c.storage_width, 4); put_le(b, c.storage_height, 4);
    put_le(b, c.fps, 4);
    put_le(b, frame_count, 8);
    return b;
}

// ----------------------------------------------------------------------------------
// Encoder (enc/encoder.rs)
// ----------------------------------------------------------------------------------
// EncodeFrameStats of a P-frame (enc/encoder.rs:436-733 mode loop telemetry, :768-800 delta
// statistics after the bias, :822 mv_raw_bytes, :873-884 zero deltas, :886-941 the rest), in
// the order of oracle_enc_last_stats.  mvs: raw search MVs, coded: coded_prefix, prev: the
// previous P-frame's coded MVs or nullptr, modes / bases / deltas: the mode decision's
// outputs, opt: the optimized skip mask.
static std::vector<double> inter_stats(int bw, int bh, const std::vector<MV>& mvs, const std::vector<MV>& coded,
                                       const MV* prev, const std::vector<int64_t>& sads, const Lambda& L, bool allow,
                                       double guard, const std::vector<uint8_t>& modes, const std::vector<uint8_t>& bases,
                                       const std::vector<std::pair<int8_t, int8_t>>& raw_delta, int8_t biasx, int8_t biasy,
                                       const std::vector<bool>& opt, size_t mv_bytes, size_t res_bytes, size_t total) {
    const int n = bw * bh;
    double mode_counts[7] = {0}, base_counts[5] = {0}, best_ref[5] = {0}, cls[11] = {0}, match[6] = {0};
    double saved = 0, new_blocks = 0, zero_pre = 0, zero_post = 0, axes_x = 0, axes_y = 0, mag_sum = 0, mag_sq = 0;
    double uniq_total = 0, uniq_samples = 0, uniq_min = 1e30, uniq_max = 0, nonzero = 0, any_sp = 0, any_tm = 0;
    double evaluated = 0, chosen = 0, f_frac = 0, f_thr = 0, f_dis = 0, tot_skip = 0.0, tot_coded = 0.0;
    double zero_delta = 0, skipped = 0;
    for (int i = 0; i < n; i++) {
        const MV& mv = mvs[i];
        const int bx = i % bw, by = i / bw;
        // RdoContext::decide + RdoTelemetry::record (enc/rdo.rs:140-178, :220-234)
        double satd = (double)std::max<int64_t>(sads[i], 0);
        double skip_cost = satd + L.lambda * L.skip_bits;
        double est = L.icpt + L.slope * satd;
        if (est < 0.0) est = 0.0;
        double coded_cost = satd * L.retention + L.lambda * (L.keep_bits + est);
        evaluated += 1;
        if (!allow) f_dis += 1;
        else if (mv.sx != 0 || mv.sy != 0) f_frac += 1;
        else if (satd > guard) f_thr += 1;
        else if (skip_cost <= coded_cost) chosen += 1;
        tot_skip += skip_cost;
        tot_coded += coded_cost;
        // derive_mv_predictors_with_stats (res/mv_predictor.rs:135-163) on coded_prefix
        std::vector<MV> before(coded.begin(), coded.begin() + i);
        Neigh ng = gather_neighbors(before, prev, bw, bx, by);
        std::vector<Tup> c;
        auto add = [&](bool has, const Tup& t) {
            if (!has) return;
            for (auto& e : c)
                if (e == t) return;
            c.push_back(t);
        };
        add(ng.has_l, ng.l); add(ng.has_t, ng.t); add(ng.has_tr, ng.tr); add(ng.has_tl, ng.tl); add(ng.has_tm, ng.tm);
        double u = c.empty() ? 1 : (double)c.size();
        uniq_total += u; uniq_samples += 1;
        uniq_min = std::min(uniq_min, u); uniq_max = std::max(uniq_max, u);
        Preds P = derive_predictors(ng);
        Tup act = tup(mv);
        bool zero_el = mv.dx == 0 && mv.dy == 0 && mv.sx == 0 && mv.sy == 0;
        if (!zero_el) {  // :483-515
            nonzero += 1;
            bool ml = ng.has_l && ng.l == act, mt = ng.has_t && ng.t == act, mtr = ng.has_tr && ng.tr == act,
                 mtl = ng.has_tl && ng.tl == act, mtm = ng.has_tm && ng.tm == act;
            if (ml || mt || mtr || mtl) any_sp += 1;
            if (mtm) any_tm += 1;
            match[ml ? 0 : mt ? 1 : mtr ? 2 : mtl ? 3 : mtm ? 4 : 5] += 1;
        }
        int mode = modes[i];
        mode_counts[mode] += 1;
        if (mode == NEW) {  // :567-660
            int ax = mv.dx, ay = mv.dy;
            auto l1 = [&](const Tup& b) { return (uint32_t)(std::abs(ax - b.dx) + std::abs(ay - b.dy)); };
            uint32_t cn = l1(P.nearest), cr = l1(P.near);
            bool has[5] = {true, true, ng.has_tr, ng.has_tl, true};
            uint32_t cost[5] = {cn, cr, ng.has_tr ? l1(ng.tr) : 0u, ng.has_tl ? l1(ng.tl) : 0u, l1(P.temporal)};
            int best = 0;
            uint32_t bc = cn;
            for (int k = 0; k < 5; k++)
                if (has[k] && cost[k] < bc) { bc = cost[k]; best = k; }
            best_ref[best] += 1;
            uint32_t cur = std::min(cn, cr);
            if (bc < cur) saved += (double)(cur - bc);
            base_counts[bases[i]] += 1;
            new_blocks += 1;
            if (raw_delta[i].first == 0 && raw_delta[i].second == 0) zero_pre += 1;
            // after the bias (:776-798)
            int8_t dx = sat_i8(raw_delta[i].first - biasx), dy = sat_i8(raw_delta[i].second - biasy);
            double fx = (double)dx, fy = (double)dy, mag = sqrt(fx * fx + fy * fy);
            mag_sum += mag;
            mag_sq += mag * mag;
            cls[mv_class((unsigned)std::abs((int)dx))] += 1;
            cls[mv_class((unsigned)std::abs((int)dy))] += 1;
            if (dx == 0) axes_x += 1;
            if (dy == 0) axes_y += 1;
            if (dx == 0 && dy == 0) zero_post += 1;
            if (raw_delta[i].first == 0 && raw_delta[i].second == 0) zero_delta += 1;  // :873-884
        } else {
            zero_delta += 1;
        }
        if (opt[i]) skipped += 1;
    }
    std::vector<double> o;
    auto put = [&](double v) { o.push_back(v); };
    put(2); put((double)total); put((double)mv_bytes); put((double)(n * 2 + new_blocks * 2)); put((double)res_bytes);
    put(n); put(skipped); put(zero_delta);
    for (double v : mode_counts) put(v);
    put(zero_pre); put(zero_post); put(axes_x); put(axes_y);
    for (double v : base_counts) put(v);
    for (double v : best_ref) put(v);
    put(saved); put(new_blocks); put(new_blocks); put(mag_sum); put(mag_sq);
    for (double v : cls) put(v);
    put(biasx); put(biasy);
    put(uniq_total); put(uniq_samples); put(uniq_samples ? uniq_min : 0); put(uniq_max);
    for (double v : match) put(v);
    put(nonzero); put(any_sp); put(any_tm);
    put((double)((n - skipped) * 384 * 2)); put((double)res_bytes);
    put(L.lambda); put(evaluated); put(chosen); put(f_frac); put(f_thr); put(f_dis);
    put(evaluated ? tot_skip / evaluated : 0.0); put(evaluated ? tot_coded / evaluated : 0.0);
    return o;
}

struct Encoder {
    oracle_config cfg;
    Bytes out;
    uint64_t pos = 0, header_pos = 0, frame_count = 0;
    bool has_prev = false;
    Yuv prev_recon;
    bool has_prev_mvs = false;
    std::vector<MV> prev_mvs;
    MvCoder mvc;
    // intermediates of the last frame
    int last_type = 0;
    Yuv curr, pred, recon_pre, recon;
    std::vector<MV> raw, coded;
    std::vector<int64_t> sads;
    std::vector<uint8_t> side;  // 8 per MB
    std::vector<float> qs;
    std::vector<int16_t> coeffs;
    int8_t bias[2] = {0, 0};
    Bytes record;
    std::vector<double> stats;  // EncodeFrameStats of the last frame, ORACLE_STATS_* order

    void write(const Bytes& b) {  // VecWriter semantics (enc/writer.rs:49-69)
        if (pos + b.size() > out.size()) out.resize(pos + b.size(), 0);
        memcpy(out.data() + pos, b.data(), b.size());
        pos += b.size();
    }
};

static int est_selector_bits(int base) { return base == 0 ? 1 : base == 1 ? 2 : base == 2 ? 3 : 4; }  // encoder.rs:128-139
static int est_comp_bits(int8_t d) {  // encoder.rs:142-154
    int c = mv_class((unsigned)abs((int)d));
    return c == 0 ? 4 : 4 + c;
}
static void compute_bias(const std::vector<std::pair<int8_t, int8_t>>& d, int8_t& bx, int8_t& by) {  // :1002-1048
    bx = 0; by = 0;
    if (d.empty()) return;
    int64_t bzx = -1, bzy = -1, bcx = INT64_MAX, bcy = INT64_MAX;
    for (int bias = -24; bias <= 24; bias++) {
        int64_t zx = 0, cx = 0, zy = 0, cy = 0;
        for (auto& p : d) {
            // `adj.abs() as i32` on an i8: i8::abs wraps at -128 in the release build.
            int ax = clampi(p.first - bias, -128, 127);
            if (ax == 0) zx++;
            cx += ax == -128 ? -128 : abs(ax);
            int ay = clampi(p.second - bias, -128, 127);
            if (ay == 0) zy++;
            cy += ay == -128 ? -128 : abs(ay);
        }
        if (zx > bzx || (zx == bzx && cx < bcx)) { bzx = zx; bcx = cx; bx = (int8_t)bias; }
        if (zy > bzy || (zy == bzy && cy < bcy)) { bzy = zy; bcy = cy; by = (int8_t)bias; }
    }
}

// ResidualEncoder::encode_intra (res/residual.rs:267-388)
static Bytes encode_intra(const Yuv& cur, uint8_t quality, Yuv& recon, std::vector<int16_t>& all) {
    init_tables();
    int w = cur.w, h = cur.h, cw = w / 2, bw = w / 16, bh = h / 16, n = bw * bh;
    float qs = quant_step_from_quality(quality);
    uint16_t yt[256], ct[64];
    build_intra_y_table(qs, yt);
    build_intra_uv_table(qs, ct);
    all.assign((size_t)n * 384, 0);
    for (int b = 0; b < n; b++) {
        int bx = b % bw, by = b / bw;
        int32_t blk[256], c[256];
        for (int y = 0; y < 16; y++)
            for (int x = 0; x < 16; x++) blk[y * 16 + x] = (int)cur.y[(size_t)(by * 16 + y) * w + bx * 16 + x] - 128;
        fdct_2d<16>(blk, c, T16);
        for (int i = 0; i < 256; i++) all[(size_t)b * 384 + i] = f32_as_i16(roundf((float)c[i] / (float)std::max<uint16_t>(yt[i], 1)));
        for (int pl = 0; pl < 2; pl++) {
            const Bytes& P = pl == 0 ? cur.u : cur.v;
            int32_t b8[64], c8[64];
            for (int y = 0; y < 8; y++)
                for (int x = 0; x < 8; x++) b8[y * 8 + x] = (int)P[(size_t)(by * 8 + y) * cw + bx * 8 + x] - 128;
            fdct_2d<8>(b8, c8, T8);
            for (int i = 0; i < 64; i++)
                all[(size_t)b * 384 + 256 + pl * 64 + i] = f32_as_i16(roundf((float)c8[i] / (float)std::max<uint16_t>(ct[i], 1)));
        }
    }
    Bytes data;
    RansEnc w_(&data);
    DctCtx ctx;
    ctx.dcp = true;
    for (int b = 0; b < n; b++) {
        const int16_t* p = &all[(size_t)b * 384];
        dct_encode_plane(w_, ctx, p, 256, true, 0);
        dct_encode_plane(w_, ctx, p + 256, 64, false, 1);
        dct_encode_plane(w_, ctx, p + 320, 64, false, 2);
    }
    if (n > 0) w_.finish();
    recon.alloc(w, h);
    for (int b = 0; b < n; b++) {
        int bx = b % bw, by = b / bw;
        const int16_t* p = &all[(size_t)b * 384];
        int32_t deq[256];
        int16_t r[256];
        for (int i = 0; i < 256; i++) deq[i] = (int32_t)p[i] * (int32_t)std::max<uint16_t>(yt[i], 1);
        idct16_2d(deq, r);
        for (int y = 0; y < 16; y++)
            for (int x = 0; x < 16; x++)
                recon.y[(size_t)(by * 16 + y) * w + bx * 16 + x] = (uint8_t)clampi(r[y * 16 + x] + 128, 0, 255);
        for (int pl = 0; pl < 2; pl++) {
            int16_t r8[64];
            uint16_t ct1[64];
            for (int i = 0; i < 64; i++) ct1[i] = std::max<uint16_t>(ct[i], 1);
            idct8_aan(p + 256 + pl * 64, ct1, r8);
            Bytes& P = pl == 0 ? recon.u : recon.v;
            for (int y = 0; y < 8; y++)
                for (int x = 0; x < 8; x++) P[(size_t)(by * 8 + y) * cw + bx * 8 + x] = (uint8_t)clampi(r8[y * 8 + x] + 128, 0, 255);
        }
    }
    return data;
}

// ResidualEncoder::encode_inter (res/residual.rs:396-809)
// Residual, transforms, quantisation and reconstruction of encode_inter (residual.rs:520-752)
// for given AQ steps; the coefficient coding of the coded MBs follows separately, in MB order.
static void residual_inter(const Yuv& cur, const Yuv& pred, const std::vector<bool>& skip_mask,
                           const std::vector<float>& qsv, float dz, Yuv& recon, std::vector<bool>& opt_skip,
                           std::vector<int16_t>& all) {
    init_tables();
    int w = cur.w, h = cur.h, cw = w / 2, bw = w / 16, bh = h / 16, n = bw * bh;
    all.assign((size_t)n * 384, 0);
    opt_skip.assign(n, true);
    for (int b = 0; b < n; b++) {
        if (skip_mask[b]) continue;
        int bx = b % bw, by = b / bw;
        float q = qsv[b];
        int16_t tmp[384];
        int32_t blk[256], c[256];
        for (int y = 0; y < 16; y++)
            for (int x = 0; x < 16; x++) {
                size_t i = (size_t)(by * 16 + y) * w + bx * 16 + x;
                blk[y * 16 + x] = (int16_t)((int)cur.y[i] - (int)pred.y[i]);
            }
        fdct_2d<16>(blk, c, T16);
        for (int i = 0; i < 256; i++) tmp[i] = quant_aq(c[i], q, dz);
        for (int pl = 0; pl < 2; pl++) {
            const Bytes& C = pl == 0 ? cur.u : cur.v;
            const Bytes& P = pl == 0 ? pred.u : pred.v;
            int32_t b8[64], c8[64];
            for (int y = 0; y < 8; y++)
                for (int x = 0; x < 8; x++) {
                    size_t i = (size_t)(by * 8 + y) * cw + bx * 8 + x;
                    b8[y * 8 + x] = (int16_t)((int)C[i] - (int)P[i]);
                }
            fdct_2d<8>(b8, c8, T8);
            for (int i = 0; i < 64; i++) tmp[256 + pl * 64 + i] = quant_aq(c8[i], q, dz);
        }
        bool zero = true;
        for (int i = 0; i < 384; i++)
            if (tmp[i]) { zero = false; break; }
        if (zero) continue;
        opt_skip[b] = false;
        memcpy(&all[(size_t)b * 384], tmp, sizeof(tmp));
    }
    recon = pred;
    for (int b = 0; b < n; b++) {
        if (opt_skip[b]) continue;
        int bx = b % bw, by = b / bw;
        const int16_t* p = &all[(size_t)b * 384];
        float q = qsv[b];
        int32_t qfp = f32_as_i32(roundf(q * 16384.0f));
        int32_t deq[256];
        int16_t r[256];
        for (int i = 0; i < 256; i++) deq[i] = wadd(wmul((int32_t)p[i], qfp), 8192) >> 14;
        idct16_2d(deq, r);
        for (int y = 0; y < 16; y++)
            for (int x = 0; x < 16; x++) {
                size_t i = (size_t)(by * 16 + y) * w + bx * 16 + x;
                recon.y[i] = (uint8_t)clampi((int)recon.y[i] + r[y * 16 + x], 0, 255);
            }
        float qr = roundf(q);
        if (qr < 1.0f) qr = 1.0f;
        uint16_t q8 = qr >= 65535.0f ? 65535 : (uint16_t)qr;
        uint16_t qt[64];
        for (int i = 0; i < 64; i++) qt[i] = q8;
        for (int pl = 0; pl < 2; pl++) {
            int16_t r8[64];
            idct8_aan(p + 256 + pl * 64, qt, r8);
            Bytes& P = pl == 0 ? recon.u : recon.v;
            for (int y = 0; y < 8; y++)
                for (int x = 0; x < 8; x++) {
                    size_t i = (size_t)(by * 8 + y) * cw + bx * 8 + x;
                    P[i] = (uint8_t)clampi((int)P[i] + r8[y * 8 + x], 0, 255);
                }
        }
    }
}

static Bytes encode_inter(const Yuv& cur, const Yuv& pred, const std::vector<bool>& skip_mask, uint8_t quality,
                          float dz, Yuv& recon, std::vector<bool>& opt_skip, std::vector<float>& qsv,
                          std::vector<int16_t>& all) {  // residual.rs:396-809
    const int n = (cur.w / 16) * (cur.h / 16);
    aq_steps(pred.y.data(), cur.w, cur.w, cur.h, quant_step_from_quality(quality), qsv);
    residual_inter(cur, pred, skip_mask, qsv, dz, recon, opt_skip, all);
    // the inline DCT-rANS coder (residual.rs:618-674) sees the coded MBs in raster order
    Bytes data;
    RansEnc* w_ = nullptr;
    DctCtx ctx;
    for (int b = 0; b < n; b++) {
        if (opt_skip[b]) continue;
        const int16_t* tmp = &all[(size_t)b * 384];
        if (!w_) w_ = new RansEnc(&data);
        dct_encode_plane(*w_, ctx, tmp, 256, true, 0);
        dct_encode_plane(*w_, ctx, tmp + 256, 64, false, 1);
        dct_encode_plane(*w_, ctx, tmp + 320, 64, false, 2);
    }
    if (w_) {
        w_->finish();
        delete w_;
    }
    return data;
}

static int encode_frame_yuv(Encoder& E, Yuv& cur, uint64_t ts) {  // encoder.rs:258-947
    const oracle_config& c = E.cfg;
    g_overflow = false;
    int w = (int)c.storage_width, h = (int)c.storage_height, bw = w / 16, bh = h / 16, n = bw * bh;
    bool intra;
    if (c.keyframe_mode == 0) intra = true;
    else if (c.keyframe_mode == 1) intra = E.frame_count % 30 == 0;
    else intra = E.frame_count % c.keyframe_interval == 0;
    if (!E.has_prev) intra = true;
    E.curr = cur;
    Bytes rec;
    if (intra) {
        Yuv recon;
        Bytes data = encode_intra(cur, c.intra_quality, recon, E.coeffs);
        E.recon_pre = recon;
        deblock_yuv420(recon, deblock_level_from_quant_step(quant_step_from_quality(c.intra_quality)), true, nullptr);
        E.prev_recon = recon;
        E.recon = recon;
        E.has_prev = true;
        put_le(rec, ts, 8);
        rec.push_back(1);
        rec.push_back(c.intra_quality);
        put_le(rec, data.size(), 4);
        rec.insert(rec.end(), data.begin(), data.end());
        E.has_prev_mvs = false;
        E.prev_mvs.clear();
        E.mvc.reset();
        E.last_type = 1;
        {  // EncodeFrameStats of a key frame (enc/encoder.rs:338-385): sizes only, Options None
            const int n = (w / 16) * (h / 16);
            const size_t total = data.size() + 14;
            E.stats.assign(ORACLE_STATS_N, 0.0);
            E.stats[0] = 1; E.stats[1] = (double)total; E.stats[4] = (double)data.size(); E.stats[5] = n;
            E.stats[ORACLE_STATS_RESI_RAW] = -1; E.stats[ORACLE_STATS_RESI_RAW + 1] = -1;
        }
        E.raw.assign(n, MV()); E.coded.assign(n, MV()); E.sads.assign(n, 0);
        E.side.assign((size_t)n * 8, 0);
        E.qs.assign(n, 0.0f);
        E.bias[0] = E.bias[1] = 0;
        E.pred.alloc(w, h);
    } else {
        const Yuv& prev = E.prev_recon;
        Lambda L = lambda_for_quality(c.inter_quality, c.rdo_lambda_mult);
        bool allow = c.skip_threshold > 0;
        double guard = (double)768 * (double)c.skip_threshold;
        const MV* pm = E.has_prev_mvs ? E.prev_mvs.data() : nullptr;
        std::vector<MV> mvs;
        std::vector<int64_t> sads;
        hex_search(prev.y.data(), cur.y.data(), w, h, c.search_range, pm, c.me_zero_mv_threshold,
                   c.me_predictor_threshold, L.lambda, mvs, sads);
        Yuv pred;
        build_predicted(prev, mvs, pred);
        std::vector<bool> skip_mask(n);
        std::vector<std::pair<int8_t, int8_t>> raw_delta(n, {0, 0});
        std::vector<uint8_t> flags(n), modes(n), bases(n);
        std::vector<MV> coded;
        coded.reserve(n);
        for (int i = 0; i < n; i++) {  // :447-733
            const MV& mv = mvs[i];
            int bx = i % bw, by = i / bw;
            bool int_al = mv.sx == 0 && mv.sy == 0;
            skip_mask[i] = rdo_decide(L, allow, guard, sads[i], int_al);
            Neigh ng = gather_neighbors(coded, pm, bw, bx, by);
            Preds P = derive_predictors(ng);
            bool zero_el = mv.dx == 0 && mv.dy == 0 && mv.sx == 0 && mv.sy == 0;
            int mode;
            auto hpx = [](const Tup& t) { return (int)t.dx * 2 + t.sx; };
            auto hpy = [](const Tup& t) { return (int)t.dy * 2 + t.sy; };
            int mx = dx_hp(mv), my = dy_hp(mv);
            if (zero_el) mode = Z;
            else if (mx == hpx(P.nearest) && my == hpy(P.nearest)) mode = NEAREST;
            else if (mx == hpx(P.near) && my == hpy(P.near)) mode = NEAR;
            else if (ng.has_tr && mx == hpx(ng.tr) && my == hpy(ng.tr)) mode = TR;
            else if (ng.has_tl && mx == hpx(ng.tl) && my == hpy(ng.tl)) mode = TL;
            else if (mx == hpx(P.temporal) && my == hpy(P.temporal)) mode = TEMPORAL;
            else mode = NEW;
            int chosen = 0;
            int8_t rdx = 0, rdy = 0;
            if (mode == NEW) {
                int ax = mv.dx, ay = mv.dy;
                bool has[5] = {true, true, ng.has_tr, ng.has_tl, true};
                Tup bases5[5] = {P.nearest, P.near, ng.tr, ng.tl, P.temporal};
                uint32_t best = UINT32_MAX;
                int bbx = P.nearest.dx, bby = P.nearest.dy;
                for (int k = 0; k < 5; k++) {
                    if (!has[k]) continue;
                    int8_t ddx = sat_i8(ax - bases5[k].dx), ddy = sat_i8(ay - bases5[k].dy);
                    uint32_t cost = (uint32_t)(est_selector_bits(k) + est_comp_bits(ddx) + est_comp_bits(ddy));
                    if (cost < best) { best = cost; chosen = k; bbx = bases5[k].dx; bby = bases5[k].dy; }
                }
                rdx = sat_i8(ax - bbx);
                rdy = sat_i8(ay - bby);
            }
            raw_delta[i] = {rdx, rdy};
            modes[i] = (uint8_t)mode;
            bases[i] = (uint8_t)chosen;
            MV rmv = mv;
            if (mode == NEAREST) rmv = mv_new(P.nearest.dx, P.nearest.dy, P.nearest.sx, P.nearest.sy, mv.skip);
            else if (mode == NEAR) rmv = mv_new(P.near.dx, P.near.dy, P.near.sx, P.near.sy, mv.skip);
            else if (mode == TR) rmv = mv_new(ng.tr.dx, ng.tr.dy, ng.tr.sx, ng.tr.sy, mv.skip);
            else if (mode == TL) rmv = mv_new(ng.tl.dx, ng.tl.dy, ng.tl.sx, ng.tl.sy, mv.skip);
            else if (mode == TEMPORAL) rmv = mv_new(P.temporal.dx, P.temporal.dy, P.temporal.sx, P.temporal.sy, mv.skip);
            else if (mode == NEW) {
                Tup b = chosen == 0 ? P.nearest : chosen == 1 ? P.near : chosen == 2 ? (ng.has_tr ? ng.tr : P.nearest)
                        : chosen == 3 ? (ng.has_tl ? ng.tl : P.nearest) : P.temporal;
                rmv.dx = sat_i8(b.dx + rdx);
                rmv.dy = sat_i8(b.dy + rdy);
            }
            coded.push_back(rmv);
            uint8_t f = mode == NEW ? (uint8_t)(mv_flags(mv) & 0x0F) : 0;
            if (skip_mask[i]) f |= 0x40;
            flags[i] = f;
        }
        Yuv recon;
        std::vector<bool> opt;
        std::vector<float> qsv;
        Bytes data = encode_inter(cur, pred, skip_mask, c.inter_quality, c.inter_dead_zone, recon, opt, qsv, E.coeffs);
        std::vector<std::pair<int8_t, int8_t>> nd;
        for (int i = 0; i < n; i++)
            if (modes[i] == NEW) nd.push_back(raw_delta[i]);
        int8_t bx_, by_;
        compute_bias(nd, bx_, by_);
        std::vector<Coded> blocks(n);
        for (int i = 0; i < n; i++) {
            Coded& b = blocks[i];
            b.mode = modes[i];
            b.base = bases[i];
            b.dx = 0; b.dy = 0;
            if (modes[i] == NEW) {
                b.dx = sat_i8(raw_delta[i].first - bx_);
                b.dy = sat_i8(raw_delta[i].second - by_);
                b.spx = mvs[i].sx == 1 ? SP : (mvs[i].sx == -1 ? SM : SZ);
                b.spy = mvs[i].sy == 1 ? SP : (mvs[i].sy == -1 ? SM : SZ);
            } else {
                b.spx = SZ; b.spy = SZ;
            }
            b.skip = opt[i];
        }
        Bytes mvdata = E.mvc.encode_frame(blocks, bw);
        E.stats = inter_stats(bw, h / 16, mvs, coded, pm, sads, L, allow, guard, modes, bases, raw_delta, bx_, by_, opt,
                              mvdata.size(), data.size(), 8 + 1 + 1 + 2 + 1 + 4 + mvdata.size() + 4 + data.size());
        std::vector<uint8_t> fmask(n);
        for (int i = 0; i < n; i++)
            fmask[i] = (!opt[i] || coded[i].dx != 0 || coded[i].dy != 0 || coded[i].sx != 0 || coded[i].sy != 0) ? 1 : 0;
        E.recon_pre = recon;
        deblock_yuv420(recon, deblock_level_from_quant_step(quant_step_from_quality(c.inter_quality)), false, fmask.data());
        E.prev_recon = recon;
        E.recon = recon;
        E.prev_mvs = coded;
        E.has_prev_mvs = true;
        put_le(rec, ts, 8);
        rec.push_back(2);
        rec.push_back(c.inter_quality);
        rec.push_back((uint8_t)bx_);
        rec.push_back((uint8_t)by_);
        rec.push_back(0);  // global_mv flags: no subpel, no skip
        put_le(rec, mvdata.size(), 4);
        rec.insert(rec.end(), mvdata.begin(), mvdata.end());
        put_le(rec, data.size(), 4);
        rec.insert(rec.end(), data.begin(), data.end());
        E.last_type = 2;
        E.raw = mvs; E.coded = coded; E.sads = sads; E.pred = pred; E.qs = qsv;
        E.bias[0] = bx_; E.bias[1] = by_;
        E.side.assign((size_t)n * 8, 0);
        for (int i = 0; i < n; i++) {
            uint8_t* s = &E.side[(size_t)i * 8];
            s[0] = modes[i]; s[1] = bases[i]; s[2] = (uint8_t)raw_delta[i].first; s[3] = (uint8_t)raw_delta[i].second;
            s[4] = flags[i]; s[5] = skip_mask[i]; s[6] = opt[i]; s[7] = fmask[i];
        }
    }
    if (g_overflow) return 3;  // EncodeError::EncodingFailed (the reference panics)
    E.write(rec);
    E.record = rec;
    E.frame_count++;
    return 0;
}

// ----------------------------------------------------------------------------------
// Decoder (dec/decoder.rs:195-460)
// ----------------------------------------------------------------------------------
struct Decoder {
    Bytes data;
    size_t pos = 0;
    uint32_t dw = 0, dh = 0, sw = 0, sh = 0, fps = 0;
    uint64_t frame_count = 0, current = 0;
    bool has_prev = false;
    Yuv prev;
    bool has_prev_mvs = false;
    std::vector<MV> prev_mvs;
    MvCoder mvc;
};

static void decode_intra(const uint8_t* d, size_t len, int w, int h, uint8_t quality, Yuv& out) {  // residual.rs:815-887
    init_tables();
    int cw = w / 2, bw = w / 16, bh = h / 16, n = bw * bh;
    float qs = quant_step_from_quality(quality);
    uint16_t yt[256], ct[64];
    build_intra_y_table(qs, yt);
    build_intra_uv_table(qs, ct);
    for (int i = 0; i < 64; i++) ct[i] = std::max<uint16_t>(ct[i], 1);
    std::vector<int16_t> all((size_t)n * 384, 0);
    if (len) {
        RansDec r(d, len);
        DctCtx ctx;
        ctx.dcp = true;
        for (int b = 0; b < n; b++) {
            int16_t* p = &all[(size_t)b * 384];
            dct_decode_plane(r, ctx, p, 256, true, 0);
            dct_decode_plane(r, ctx, p + 256, 64, false, 1);
            dct_decode_plane(r, ctx, p + 320, 64, false, 2);
        }
    }
    out.alloc(w, h);
    for (int b = 0; b < n; b++) {
        int bx = b % bw, by = b / bw;
        const int16_t* p = &all[(size_t)b * 384];
        int32_t deq[256];
        int16_t r[256];
        for (int i = 0; i < 256; i++) deq[i] = (int32_t)p[i] * (int32_t)std::max<uint16_t>(yt[i], 1);
        idct16_2d(deq, r);
        for (int y = 0; y < 16; y++)
            for (int x = 0; x < 16; x++)
                out.y[(size_t)(by * 16 + y) * w + bx * 16 + x] = (uint8_t)clampi(r[y * 16 + x] + 128, 0, 255);
        for (int pl = 0; pl < 2; pl++) {
            int16_t r8[64];
            idct8_aan(p + 256 + pl * 64, ct, r8);
            Bytes& P = pl == 0 ? out.u : out.v;
            for (int y = 0; y < 8; y++)
                for (int x = 0; x < 8; x++) P[(size_t)(by * 8 + y) * cw + bx * 8 + x] = (uint8_t)clampi(r8[y * 8 + x] + 128, 0, 255);
        }
    }
}

static void decode_inter(const uint8_t* d, size_t len, const Yuv& pred, const std::vector<bool>& skip,
                         uint8_t quality, Yuv& out) {  // residual.rs:889-1079
    init_tables();
    int w = pred.w, h = pred.h, cw = w / 2, bw = w / 16, bh = h / 16, n = bw * bh;
    std::vector<int16_t> all((size_t)n * 384, 0);
    if (len) {
        RansDec r(d, len);
        DctCtx ctx;
        for (int b = 0; b < n; b++) {
            if (skip[b]) continue;
            int16_t* p = &all[(size_t)b * 384];
            dct_decode_plane(r, ctx, p, 256, true, 0);
            dct_decode_plane(r, ctx, p + 256, 64, false, 1);
            dct_decode_plane(r, ctx, p + 320, 64, false, 2);
        }
    }
    std::vector<float> qsv;
    aq_steps(pred.y.data(), w, w, h, quant_step_from_quality(quality), qsv);
    out = pred;
    for (int b = 0; b < n; b++) {
        if (skip[b]) continue;
        int bx = b % bw, by = b / bw;
        const int16_t* p = &all[(size_t)b * 384];
        float q = qsv[b];
        int32_t qfp = f32_as_i32(roundf(q * 16384.0f));
        int32_t deq[256];
        int16_t r[256];
        for (int i = 0; i < 256; i++) deq[i] = wadd(wmul((int32_t)p[i], qfp), 8192) >> 14;
        idct16_2d(deq, r);
        for (int y = 0; y < 16; y++)
            for (int x = 0; x < 16; x++) {
                size_t i = (size_t)(by * 16 + y) * w + bx * 16 + x;
                out.y[i] = (uint8_t)clampi((int)out.y[i] + r[y * 16 + x], 0, 255);
            }
        float qr = roundf(q);
        if (qr < 1.0f) qr = 1.0f;
        uint16_t q8 = qr >= 65535.0f ? 65535 : (uint16_t)qr, qt[64];
        for (int i = 0; i < 64; i++) qt[i] = q8;
        for (int pl = 0; pl < 2; pl++) {
            int16_t r8[64];
            idct8_aan(p + 256 + pl * 64, qt, r8);
            Bytes& P = pl == 0 ? out.u : out.v;
            for (int y = 0; y < 8; y++)
                for (int x = 0; x < 8; x++) {
                    size_t i = (size_t)(by * 8 + y) * cw + bx * 8 + x;
                    P[i] = (uint8_t)clampi((int)P[i] + r8[y * 8 + x], 0, 255);
                }
        }
    }
}

static int decode_next(Decoder& D, Yuv& out) {
    if (D.current >= D.frame_count) return -1;
    const uint8_t* b = D.data.data() + D.pos;
    size_t left = D.data.size() - D.pos;
    if (left < 9) return -2;
    uint64_t ts = get_le(b, 8);
    (void)ts;
    int type = b[8];
    int w = (int)D.sw, h = (int)D.sh, bw = w / 16, bh = h / 16, n = bw * bh;
    if (type == 1) {
        if (left < 14) return -2;
        uint8_t q = b[9];
        size_t sz = get_le(b + 10, 4);
        if (left < 14 + sz) return -2;
        decode_intra(b + 14, sz, w, h, q, out);
        deblock_yuv420(out, deblock_level_from_quant_step(quant_step_from_quality(q)), true, nullptr);
        D.pos += 14 + sz;
        D.prev = out;
        D.has_prev = true;
        D.has_prev_mvs = false;
        D.prev_mvs.clear();
        D.mvc.reset();
    } else if (type == 2) {
        if (left < 17 || !D.has_prev) return -2;
        uint8_t q = b[9];
        int16_t biasx = (int8_t)b[10], biasy = (int8_t)b[11];
        size_t mvs = get_le(b + 13, 4);
        if (left < 17 + mvs + 4) return -2;
        const uint8_t* mvd = b + 17;
        size_t rs = get_le(b + 17 + mvs, 4);
        if (left < 21 + mvs + rs) return -2;
        const uint8_t* rd = b + 21 + mvs;
        std::vector<Coded> blocks;
        if (!D.mvc.decode_frame(mvd, mvs, bw, bh, blocks)) return -3;
        std::vector<MV> mv;
        mv.reserve(n);
        std::vector<bool> skip(n);
        const MV* pm = D.has_prev_mvs ? D.prev_mvs.data() : nullptr;
        for (int i = 0; i < n; i++) {
            const Coded& cb = blocks[i];
            int bx = i % bw, by = i / bw;
            int8_t ddx = cb.mode == NEW ? sat_i8(cb.dx + biasx) : 0;
            int8_t ddy = cb.mode == NEW ? sat_i8(cb.dy + biasy) : 0;
            Neigh ng = gather_neighbors(mv, pm, bw, bx, by);
            Preds P = derive_predictors(ng);
            Tup base{0, 0, 0, 0};
            switch (cb.mode) {
                case Z: break;
                case NEAREST: base = P.nearest; break;
                case NEAR: base = P.near; break;
                case TR: base = ng.has_tr ? ng.tr : P.nearest; break;
                case TL: base = ng.has_tl ? ng.tl : P.nearest; break;
                case TEMPORAL: base = P.temporal; break;
                default:
                    base = cb.base == 0 ? P.nearest : cb.base == 1 ? P.near
                           : cb.base == 2 ? (ng.has_tr ? ng.tr : P.nearest)
                           : cb.base == 3 ? (ng.has_tl ? ng.tl : P.nearest) : cb.base == 4 ? P.temporal : P.nearest;
            }
            int8_t dx = sat_i8(base.dx + ddx), dy = sat_i8(base.dy + ddy);
            MV m;
            if (cb.mode == NEW) m = mv_new(dx, dy, cb.spx == SP ? 1 : (cb.spx == SM ? -1 : 0), cb.spy == SP ? 1 : (cb.spy == SM ? -1 : 0), cb.skip);
            else m = mv_new(dx, dy, base.sx, base.sy, cb.skip);
            mv.push_back(m);
            skip[i] = cb.skip;
        }
        Yuv pred;
        build_predicted(D.prev, mv, pred);
        decode_inter(rd, rs, pred, skip, q, out);
        std::vector<uint8_t> fm(n);
        for (int i = 0; i < n; i++) fm[i] = (!mv[i].skip || mv[i].dx || mv[i].dy || mv[i].sx || mv[i].sy) ? 1 : 0;
        deblock_yuv420(out, deblock_level_from_quant_step(quant_step_from_quality(q)), false, fm.data());
        D.pos += 21 + mvs + rs;
        D.prev = out;
        D.prev_mvs = mv;
        D.has_prev_mvs = true;
    } else {
        return -2;
    }
    D.current++;
    return type;
}

static Yuv yuv_from(const uint8_t* y, const uint8_t* u, const uint8_t* v, int w, int h) {
    Yuv f;
    f.alloc(w, h);
    memcpy(f.y.data(), y, f.y.size());
    memcpy(f.u.data(), u, f.u.size());
    memcpy(f.v.data(), v, f.v.size());
    return f;
}
static void yuv_to(const Yuv& f, uint8_t* y, uint8_t* u, uint8_t* v) {
    if (y) memcpy(y, f.y.data(), f.y.size());
    if (u) memcpy(u, f.u.data(), f.u.size());
    if (v) memcpy(v, f.v.data(), f.v.size());
}
static std::vector<MV> mvs_from(const int8_t* m4, int n) {
    std::vector<MV> v(n);
    for (int i = 0; i < n; i++) v[i] = mv_new(m4[4 * i], m4[4 * i + 1], m4[4 * i + 2], m4[4 * i + 3], false);
    return v;
}

}  // namespace

// ==================================================================================
// C interface
// ==================================================================================
extern "C" {

void oracle_config_default(oracle_config* c, uint32_t w, uint32_t h, uint32_t fps) {  // enc/config.rs:56-77
    memset(c, 0, sizeof(*c));
    c->display_width = w; c->display_height = h;
    c->storage_width = (w + 15) / 16 * 16; c->storage_height = (h + 15) / 16 * 16;
    c->fps = fps;
    c->keyframe_mode = 2; c->keyframe_interval = 30;
    c->intra_quality = 90; c->inter_quality = 35; c->search_range = 12; c->mv_deflate_level = 6;
    c->skip_threshold = 3;
    c->rdo_lambda_mult = 0.49;
    c->inter_dead_zone = 0.75f;
}

void* oracle_enc_new(const oracle_config* c, int* status) {  // enc/encoder.rs:162-188, config.rs:129-164
    init_zero_prob();
    init_tables();
    int st = 0;
    if (c->display_width == 0 || c->display_height == 0) st = 2;
    else if (c->storage_width < c->display_width || c->storage_height < c->display_height) st = 2;
    else if (c->fps == 0) st = 2;
    else if (c->search_range > 127) st = 2;
    else if (c->mv_deflate_level > 10) st = 2;
    else if (c->keyframe_mode == 2 && c->keyframe_interval == 0) st = 2;
    else if (c->storage_width % 16 || c->storage_height % 16) st = 2;
    if (status) *status = st;
    if (st) return nullptr;
    Encoder* E = new Encoder();
    E->cfg = *c;
    E->write(header_bytes(*c, 0));
    return E;
}
int oracle_enc_frame_yuv(void* h, const uint8_t* y, const uint8_t* u, const uint8_t* v, uint64_t ts) {
    Encoder& E = *(Encoder*)h;
    Yuv f = yuv_from(y, u, v, (int)E.cfg.storage_width, (int)E.cfg.storage_height);
    return encode_frame_yuv(E, f, ts);
}
int oracle_enc_frame_rgb(void* h, const uint8_t* rgb, uint32_t w, uint32_t hgt, uint64_t ts) {
    Encoder& E = *(Encoder*)h;
    if (w != E.cfg.display_width || hgt != E.cfg.display_height) return 5;
    Bytes pad = pad_rgb24(rgb, (int)w, (int)hgt, (int)E.cfg.storage_width, (int)E.cfg.storage_height);
    Yuv f;
    rgb_to_yuv420(pad.data(), (int)E.cfg.storage_width, (int)E.cfg.storage_height, f);
    return encode_frame_yuv(E, f, ts);
}
int oracle_enc_finish(void* h) {  // enc/encoder.rs:950-961
    Encoder& E = *(Encoder*)h;
    uint64_t end = E.pos;
    E.pos = E.header_pos;
    E.write(header_bytes(E.cfg, E.frame_count));
    E.pos = end;
    return 0;
}
size_t oracle_enc_bytes(void* h, const uint8_t** d) {
    Encoder& E = *(Encoder*)h;
    *d = E.out.data();
    return E.out.size();
}
void oracle_enc_free(void* h) { delete (Encoder*)h; }
int oracle_enc_last_type(void* h) { return ((Encoder*)h)->last_type; }
void oracle_enc_last_recon(void* h, uint8_t* y, uint8_t* u, uint8_t* v) { yuv_to(((Encoder*)h)->recon, y, u, v); }
void oracle_enc_last_recon_pre(void* h, uint8_t* y, uint8_t* u, uint8_t* v) { yuv_to(((Encoder*)h)->recon_pre, y, u, v); }
void oracle_enc_last_curr(void* h, uint8_t* y, uint8_t* u, uint8_t* v) { yuv_to(((Encoder*)h)->curr, y, u, v); }
void oracle_enc_last_pred(void* h, uint8_t* y, uint8_t* u, uint8_t* v) { yuv_to(((Encoder*)h)->pred, y, u, v); }
void oracle_enc_last_mvs(void* h, int8_t* raw, int8_t* coded, int64_t* best_sad) {
    Encoder& E = *(Encoder*)h;
    for (size_t i = 0; i < E.raw.size(); i++) {
        if (raw) { raw[4 * i] = E.raw[i].dx; raw[4 * i + 1] = E.raw[i].dy; raw[4 * i + 2] = E.raw[i].sx; raw[4 * i + 3] = E.raw[i].sy; }
        if (coded) { coded[4 * i] = E.coded[i].dx; coded[4 * i + 1] = E.coded[i].dy; coded[4 * i + 2] = E.coded[i].sx; coded[4 * i + 3] = E.coded[i].sy; }
        if (best_sad) best_sad[i] = E.sads[i];
    }
}
void oracle_enc_last_side(void* h, uint8_t* side) {
    Encoder& E = *(Encoder*)h;
    memcpy(side, E.side.data(), E.side.size());
}
void oracle_enc_last_qsteps(void* h, float* qs) {
    Encoder& E = *(Encoder*)h;
    memcpy(qs, E.qs.data(), E.qs.size() * sizeof(float));
}
void oracle_enc_last_coeffs(void* h, int16_t* c) {
    Encoder& E = *(Encoder*)h;
    memcpy(c, E.coeffs.data(), E.coeffs.size() * sizeof(int16_t));
}
size_t oracle_enc_last_stats(void* h, double* out, size_t n) {
    Encoder& E = *(Encoder*)h;
    for (size_t i = 0; i < n && i < E.stats.size(); i++) out[i] = E.stats[i];
    return E.stats.size();
}
void oracle_enc_last_bias(void* h, int8_t* b) {
    Encoder& E = *(Encoder*)h;
    b[0] = E.bias[0]; b[1] = E.bias[1];
}
size_t oracle_enc_last_record(void* h, const uint8_t** d) {
    Encoder& E = *(Encoder*)h;
    *d = E.record.data();
    return E.record.size();
}

void* oracle_dec_new(const uint8_t* s, size_t len, int* status) {  // dec/decoder.rs:112-171
    init_zero_prob();
    init_tables();
    if (len < 36 || memcmp(s, "RIV\0", 4) != 0 || get_le(s + 4, 4) != 5) {
        if (status) *status = 1;
        return nullptr;
    }
    Decoder* D = new Decoder();
    D->data.assign(s, s + len);
    D->dw = (uint32_t)get_le(s + 8, 4); D->dh = (uint32_t)get_le(s + 12, 4);
    D->sw = (uint32_t)get_le(s + 16, 4); D->sh = (uint32_t)get_le(s + 20, 4);
    D->fps = (uint32_t)get_le(s + 24, 4);
    D->frame_count = get_le(s + 28, 8);
    D->pos = 36;
    if (status) *status = 0;
    return D;
}
int oracle_dec_next(void* h, uint8_t* y, uint8_t* u, uint8_t* v) {
    Decoder& D = *(Decoder*)h;
    Yuv out;
    int t = decode_next(D, out);
    if (t > 0) yuv_to(out, y, u, v);
    return t;
}
void oracle_dec_dims(void* h, uint32_t* d) {
    Decoder& D = *(Decoder*)h;
    d[0] = D.dw; d[1] = D.dh; d[2] = D.sw; d[3] = D.sh; d[4] = D.fps; d[5] = (uint32_t)D.frame_count;
}
void oracle_dec_free(void* h) { delete (Decoder*)h; }

void oracle_rgb_to_yuv420(const uint8_t* rgb, uint32_t dw, uint32_t dh, uint32_t sw, uint32_t sh, uint8_t* y,
                          uint8_t* u, uint8_t* v) {
    Bytes pad = pad_rgb24(rgb, (int)dw, (int)dh, (int)sw, (int)sh);
    Yuv f;
    rgb_to_yuv420(pad.data(), (int)sw, (int)sh, f);
    yuv_to(f, y, u, v);
}
void oracle_yuv_to_rgb(const uint8_t* y, const uint8_t* u, const uint8_t* v, uint32_t sw, uint32_t sh, uint32_t dw,
                       uint32_t dh, uint8_t* rgb) {
    Yuv f = yuv_from(y, u, v, (int)sw, (int)sh);
    yuv420_to_rgb24_crop(f, (int)dw, (int)dh, rgb);
}
void oracle_deblock(uint8_t* y, uint8_t* u, uint8_t* v, uint32_t w, uint32_t h, int level, int intra,
                    const uint8_t* mask) {
    Yuv f = yuv_from(y, u, v, (int)w, (int)h);
    deblock_yuv420(f, level, intra != 0, mask);
    yuv_to(f, y, u, v);
}
int oracle_deblock_level(uint8_t q) { return deblock_level_from_quant_step(quant_step_from_quality(q)); }
float oracle_quant_step(uint8_t q) { return quant_step_from_quality(q); }
void oracle_build_predicted(const uint8_t* py, const uint8_t* pu, const uint8_t* pv, uint32_t w, uint32_t h,
                            const int8_t* mvs4, uint8_t* oy, uint8_t* ou, uint8_t* ov) {
    Yuv p = yuv_from(py, pu, pv, (int)w, (int)h), o;
    build_predicted(p, mvs_from(mvs4, (int)(((w + 15) / 16) * ((h + 15) / 16))), o);
    yuv_to(o, oy, ou, ov);
}
void oracle_reference_build_predicted(const uint8_t* py, const uint8_t* pu, const uint8_t* pv, uint32_t w,
                                      uint32_t h, const int8_t* mvs4, uint8_t* oy, uint8_t* ou, uint8_t* ov) {
    Yuv p = yuv_from(py, pu, pv, (int)w, (int)h), o;
    reference_build_predicted(p, mvs_from(mvs4, (int)(((w + 15) / 16) * ((h + 15) / 16))), o);
    yuv_to(o, oy, ou, ov);
}
void oracle_motion_search(const uint8_t* prev_y, const uint8_t* curr_y, uint32_t w, uint32_t h, uint8_t sr,
                          const int8_t* prev_mvs4, int64_t zthr, int64_t pthr, double lambda, int8_t* out4,
                          int64_t* sads_out) {
    int n = (int)(((w + 15) / 16) * ((h + 15) / 16));
    std::vector<MV> pm;
    if (prev_mvs4) pm = mvs_from(prev_mvs4, n);
    std::vector<MV> mvs;
    std::vector<int64_t> sads;
    hex_search(prev_y, curr_y, (int)w, (int)h, sr, prev_mvs4 ? pm.data() : nullptr, zthr, pthr, lambda, mvs, sads);
    for (int i = 0; i < n; i++) {
        out4[4 * i] = mvs[i].dx; out4[4 * i + 1] = mvs[i].dy; out4[4 * i + 2] = mvs[i].sx; out4[4 * i + 3] = mvs[i].sy;
        sads_out[i] = sads[i];
    }
}
int64_t oracle_sad_int(const uint8_t* prev, const uint8_t* curr, uint32_t w, uint32_t h, int x0, int y0, int dx,
                       int dy, int64_t limit, int force_scalar) {
    if (force_scalar) return sad_int_scalar(prev, curr, (int)w, (int)h, x0, y0, dx, dy, limit);
    return sad_int(prev, curr, (int)w, (int)h, x0, y0, dx, dy, limit);
}
int64_t oracle_sad_halfpel(const uint8_t* prev, const uint8_t* curr, uint32_t w, uint32_t h, int x0, int y0,
                           int dxh, int dyh, int64_t limit, int force_scalar) {
    if (force_scalar) return sad_hp_scalar(prev, curr, (int)w, (int)h, x0, y0, dxh, dyh, limit);
    return sad_hp(prev, curr, (int)w, (int)h, x0, y0, dxh, dyh, limit);
}
void oracle_aq_steps(const uint8_t* py, uint32_t w, uint32_t h, float base, float* out) {
    std::vector<float> v;
    aq_steps(py, (int)w, (int)w, (int)h, base, v);
    memcpy(out, v.data(), v.size() * sizeof(float));
}
double oracle_rdo_lambda(uint8_t q, double mult) { return lambda_for_quality(q, mult).lambda; }
void oracle_residual_inter(const uint8_t* cur_yuv, const uint8_t* pred_yuv, uint32_t w, uint32_t h, const uint8_t* skip,
                           const float* qs, float dz, int16_t* coeffs, uint8_t* opt_skip, uint8_t* recon_yuv) {
    const size_t ys = (size_t)w * h, cs = ys / 4;
    const int n = (int)((w / 16) * (h / 16));
    Yuv c = yuv_from(cur_yuv, cur_yuv + ys, cur_yuv + ys + cs, (int)w, (int)h);
    Yuv p = yuv_from(pred_yuv, pred_yuv + ys, pred_yuv + ys + cs, (int)w, (int)h), r;
    std::vector<bool> sk(n), os;
    for (int b = 0; b < n; b++) sk[b] = skip[b] != 0;
    std::vector<float> q(qs, qs + n);
    std::vector<int16_t> all;
    residual_inter(c, p, sk, q, dz, r, os, all);
    memcpy(coeffs, all.data(), all.size() * 2);
    for (int b = 0; b < n; b++) opt_skip[b] = os[b] ? 1 : 0;
    yuv_to(r, recon_yuv, recon_yuv + ys, recon_yuv + ys + cs);
}
void oracle_fdct16_quant(const int16_t* blk, float qs, float dz, int16_t* out) {
    init_tables();
    int32_t b[256], c[256];
    for (int i = 0; i < 256; i++) b[i] = blk[i];
    fdct_2d<16>(b, c, T16);
    for (int i = 0; i < 256; i++) out[i] = quant_aq(c[i], qs, dz);
}
void oracle_fdct8_quant(const int16_t* blk, float qs, float dz, int16_t* out) {
    init_tables();
    int32_t b[64], c[64];
    for (int i = 0; i < 64; i++) b[i] = blk[i];
    fdct_2d<8>(b, c, T8);
    for (int i = 0; i < 64; i++) out[i] = quant_aq(c[i], qs, dz);
}
void oracle_idct16_aq(const int16_t* coeffs, float qs, int16_t* out) {
    init_tables();
    int32_t qfp = f32_as_i32(roundf(qs * 16384.0f)), deq[256];
    for (int i = 0; i < 256; i++) deq[i] = wadd(wmul((int32_t)coeffs[i], qfp), 8192) >> 14;
    idct16_2d(deq, out);
}
void oracle_idct8_aq(const int16_t* coeffs, float qs, int16_t* out) {
    float qr = roundf(qs);
    if (qr < 1.0f) qr = 1.0f;
    uint16_t q = qr >= 65535.0f ? 65535 : (uint16_t)qr, qt[64];
    for (int i = 0; i < 64; i++) qt[i] = q;
    idct8_aan(coeffs, qt, out);
}
size_t oracle_rans_roundtrip(const uint8_t* bits, const uint8_t* bypass, size_t n, uint8_t* out_bits,
                             uint8_t* stream, size_t cap) {
    init_zero_prob();
    Bytes s;
    {
        RansEnc w(&s);
        BinProb ctx[4];
        for (size_t i = 0; i < n; i++) {
            if (bypass[i]) w.put_bypass(bits[i] != 0);
            else w.put(bits[i] != 0, ctx[i & 3]);
        }
        w.finish();
    }
    RansDec r(s.data(), s.size());
    BinProb ctx[4];
    for (size_t i = 0; i < n; i++) out_bits[i] = bypass[i] ? r.get_bypass() : r.get(ctx[i & 3]);
    if (stream && cap) memcpy(stream, s.data(), std::min(cap, s.size()));
    return s.size();
}
double oracle_glibc_logf_check(void) { return (double)logf(10.0f); }

// The coefficient decoder of one frame (res/rans.rs:340-459): blocks with coded[b] == 0 are
// not in the stream and stay zero.  Returns 1 where the stream is malformed (read past its
// end, an EOB beyond the plane), where the reference decoder panics; the blocks then hold
// what was decoded.
int oracle_dct_decode(const uint8_t* d, size_t len, const uint8_t* coded, int n, int intra, int16_t* out) {
    init_zero_prob();
    std::fill(out, out + (size_t)n * 384, (int16_t)0);
    if (len == 0) return 0;
    RansDec r(d, len);
    DctCtx ctx;
    ctx.dcp = intra != 0;
    for (int b = 0; b < n && !r.err; b++) {
        if (!coded[b]) continue;
        int16_t* p = out + (size_t)b * 384;
        dct_decode_plane(r, ctx, p, 256, true, 0);
        if (!r.err) dct_decode_plane(r, ctx, p + 256, 64, false, 1);
        if (!r.err) dct_decode_plane(r, ctx, p + 320, 64, false, 2);
    }
    return r.err ? 1 : 0;
}

// The MV coder over nframes frames with one coder (res/mv_rans/encoder.rs:60-412): frame f
// has dims[2f] x dims[2f+1] blocks of 7 bytes (mode, NEW base, dx, dy, subpel x, subpel y,
// skip).  Returns the total size (frame_len[f] per frame, up to cap bytes copied), SIZE_MAX
// where the reference encoder panics: a NEW block with a raw -1/2 subpel reaches
// encode_fractional (:335-336), no candidate ever holding one (:379-381).
static Coded oracle_coded(const uint8_t* r) {
    Coded b;
    b.mode = r[0];
    b.base = r[1];
    b.dx = (int8_t)r[2];
    b.dy = (int8_t)r[3];
    b.spx = r[4];
    b.spy = r[5];
    b.skip = r[6] != 0;
    return b;
}
size_t oracle_mv_encode(const uint8_t* blk, const uint32_t* dims, int nframes, uint8_t* out, size_t cap,
                        uint32_t* frame_len) {
    init_zero_prob();
    MvCoder c;
    Bytes all;
    size_t k = 0;
    for (int f = 0; f < nframes; f++) {
        const size_t n = (size_t)dims[2 * f] * dims[2 * f + 1];
        std::vector<Coded> v(n);
        for (size_t i = 0; i < n; i++, k++) {
            v[i] = oracle_coded(blk + 7 * k);
            if (v[i].mode == NEW && (v[i].spx == SM || v[i].spy == SM)) return SIZE_MAX;
        }
        Bytes fb = c.encode_frame(v, (int)dims[2 * f]);
        frame_len[f] = (uint32_t)fb.size();
        all.insert(all.end(), fb.begin(), fb.end());
    }
    if (out && cap) memcpy(out, all.data(), std::min(cap, all.size()));
    return all.size();
}
// Inverse of oracle_mv_encode with a fresh coder (res/mv_rans/decoder.rs:149-283); 1 where
// the data is malformed.
int oracle_mv_decode(const uint8_t* data, const uint32_t* frame_len, const uint32_t* dims, int nframes,
                     uint8_t* blk) {
    init_zero_prob();
    MvCoder c;
    std::vector<Coded> v;
    size_t pos = 0, k = 0;
    for (int f = 0; f < nframes; f++) {
        if (!c.decode_frame(data + pos, frame_len[f], (int)dims[2 * f], (int)dims[2 * f + 1], v)) return 1;
        pos += frame_len[f];
        for (const Coded& b : v) {
            uint8_t* r = blk + 7 * k++;
            r[0] = (uint8_t)b.mode;
            r[1] = (uint8_t)b.base;
            r[2] = (uint8_t)b.dx;
            r[3] = (uint8_t)b.dy;
            r[4] = (uint8_t)b.spx;
            r[5] = (uint8_t)b.spy;
            r[6] = b.skip ? 1 : 0;
        }
    }
    return 0;
}

// compute_delta_bias_for_new (enc/encoder.rs:984-1048) over n NEW-block raw deltas.
void oracle_delta_bias(const int8_t* dx, const int8_t* dy, uint32_t n, int8_t* bx, int8_t* by) {
    std::vector<std::pair<int8_t, int8_t>> d(n);
    for (uint32_t i = 0; i < n; i++) d[i] = {dx[i], dy[i]};
    compute_bias(d, *bx, *by);
}

// Returns SIZE_MAX where the reference encoder panics (a magnitude class above 13).
size_t oracle_dct_encode(const int16_t* blocks, int n, int intra, uint8_t* stream, size_t cap) {  // res/rans.rs:195-330
    init_zero_prob();
    g_overflow = false;
    Bytes s;
    if (n > 0) {
        RansEnc w(&s);
        DctCtx ctx;
        ctx.dcp = intra != 0;
        for (int b = 0; b < n; b++) {
            const int16_t* p = blocks + (size_t)b * 384;
            dct_encode_plane(w, ctx, p, 256, true, 0);
            dct_encode_plane(w, ctx, p + 256, 64, false, 1);
            dct_encode_plane(w, ctx, p + 320, 64, false, 2);
        }
        w.finish();
    }
    if (g_overflow) return SIZE_MAX;
    if (stream && cap) memcpy(stream, s.data(), std::min(cap, s.size()));
    return s.size();
}

}  // extern "C"
