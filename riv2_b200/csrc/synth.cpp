// synth.cpp -- seeded synthetic RGB24 clip generator (host, C ABI).
//
// Stands in for the public test sequences the reference benchmarks on (foreman CIF,
// park_joy 1080p), which are not available here.  Scene model:
//   * background: 128 + sum of 3 sinusoidal gratings (frequency U[0.01,0.1] cycles/px,
//     orientation U[0,pi), phase U[0,2pi), per-channel amplitude U[20,60]), panned by a
//     constant global velocity U[-pan,pan] px/frame;
//   * N opaque rectangles (sides U[side_min,side_max]) filled with bilinear value noise
//     (lattice L px, lattice values U[0,255] per channel), constant velocity
//     U[-vmax,vmax] quantised to 0.5 px/frame, wrapping around the frame;
//   * i.i.d. Gaussian noise (sigma) per sample, then rounding and clamping to 0..255.
// Randomness: SplitMix64.  Scene parameters come from a sequential stream seeded by
// (seed, clip); per-sample noise is counter-based on (clip seed, frame, sample index),
// so any frame can be generated independently and in parallel.  Gaussian samples use
// Box-Muller in f64.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "riv_synth.h"

namespace {
static inline uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline uint64_t mix(uint64_t a) {
    uint64_t s = a;
    return splitmix(s);
}
static inline double u01(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }
struct Rng {
    uint64_t s;
    double uni(double lo, double hi) { return lo + (hi - lo) * u01(splitmix(s)); }
    int uint_range(int lo, int hi) { return lo + (int)(u01(splitmix(s)) * (double)(hi - lo + 1)); }
};
struct Grating { double f, c, s, phase, amp[3]; };
struct Rect {
    int w, h;
    double x0, y0, vx, vy;
    int lw, lh;  // lattice size
    std::vector<uint8_t> lat;  // lh*lw*3
};
struct Synth {
    riv_synth_params p;
    uint64_t clip_seed;
    Grating g[3];
    double pan_x, pan_y;
    std::vector<Rect> rects;
};
static const double TWO_PI = 6.283185307179586476925286766559;
}  // namespace

extern "C" {

void riv_synth_preset(riv_synth_params* p, const char* name, uint32_t seed, uint32_t clip) {
    memset(p, 0, sizeof(*p));
    p->seed = seed;
    p->clip = clip;
    p->sigma = 2.0;
    if (!strcmp(name, "1080p")) {
        p->width = 1920; p->height = 1080; p->n_rects = 16; p->side_min = 64; p->side_max = 384;
        p->vmax = 16.0; p->lattice = 16; p->pan_max = 4.0;
    } else if (!strcmp(name, "720p")) {
        p->width = 1280; p->height = 720; p->n_rects = 12; p->side_min = 48; p->side_max = 256;
        p->vmax = 24.0; p->lattice = 12; p->pan_max = 3.0;
    } else if (!strcmp(name, "4k")) {
        p->width = 3840; p->height = 2160; p->n_rects = 24; p->side_min = 128; p->side_max = 768;
        p->vmax = 48.0; p->lattice = 32; p->pan_max = 8.0; p->sigma = 4.0;
    } else {  // "cif"
        p->width = 352; p->height = 288; p->n_rects = 8; p->side_min = 16; p->side_max = 96;
        p->vmax = 6.0; p->lattice = 8; p->pan_max = 2.0;
    }
}

void* riv_synth_new(const riv_synth_params* params) {
    if (!params || params->width == 0 || params->height == 0 || params->lattice == 0) return nullptr;
    Synth* S = new Synth();
    S->p = *params;
    S->clip_seed = mix(((uint64_t)params->seed << 32) ^ (uint64_t)params->clip ^ 0x5249563242323030ull);
    Rng r{S->clip_seed};
    for (int k = 0; k < 3; k++) {
        double f = r.uni(0.01, 0.1), th = r.uni(0.0, TWO_PI / 2);
        S->g[k].f = f;
        S->g[k].c = cos(th);
        S->g[k].s = sin(th);
        S->g[k].phase = r.uni(0.0, TWO_PI);
        for (int c = 0; c < 3; c++) S->g[k].amp[c] = r.uni(20.0, 60.0);
    }
    S->pan_x = r.uni(-params->pan_max, params->pan_max);
    S->pan_y = r.uni(-params->pan_max, params->pan_max);
    for (uint32_t i = 0; i < params->n_rects; i++) {
        Rect R;
        R.w = r.uint_range((int)params->side_min, (int)params->side_max);
        R.h = r.uint_range((int)params->side_min, (int)params->side_max);
        R.x0 = floor(r.uni(0.0, (double)params->width));
        R.y0 = floor(r.uni(0.0, (double)params->height));
        R.vx = round(r.uni(-params->vmax, params->vmax) * 2.0) / 2.0;
        R.vy = round(r.uni(-params->vmax, params->vmax) * 2.0) / 2.0;
        int L = (int)params->lattice;
        R.lw = R.w / L + 3;
        R.lh = R.h / L + 3;
        R.lat.resize((size_t)R.lw * R.lh * 3);
        for (auto& v : R.lat) v = (uint8_t)(splitmix(r.s) >> 56);
        S->rects.push_back(std::move(R));
    }
    return S;
}

void riv_synth_free(void* h) { delete (Synth*)h; }

// Generates frame t (RGB24, width*height*3 bytes, row-major).
void riv_synth_frame(void* h, uint32_t t, uint8_t* out) {
    const Synth& S = *(const Synth*)h;
    const int W = (int)S.p.width, H = (int)S.p.height;
    const double L = (double)S.p.lattice;
    const double ox = S.pan_x * t, oy = S.pan_y * t;
    // Per-rectangle position at frame t, wrapped so objects re-enter from the other side.
    std::vector<double> rx(S.rects.size()), ry(S.rects.size());
    for (size_t i = 0; i < S.rects.size(); i++) {
        const Rect& R = S.rects[i];
        double spanx = (double)(W + R.w), spany = (double)(H + R.h);
        double px = fmod(R.x0 + R.vx * t + R.w, spanx);
        if (px < 0) px += spanx;
        double py = fmod(R.y0 + R.vy * t + R.h, spany);
        if (py < 0) py += spany;
        rx[i] = px - R.w;
        ry[i] = py - R.h;
    }
    const uint64_t fseed = mix(S.clip_seed ^ ((uint64_t)t * 0xD1B54A32D192ED03ull));
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; y++) {
        for (int x = 0; x < W; x++) {
            double v[3];
            int top = -1;
            for (int i = (int)S.rects.size() - 1; i >= 0; i--) {
                const Rect& R = S.rects[i];
                if ((double)x >= rx[i] && (double)x < rx[i] + R.w && (double)y >= ry[i] && (double)y < ry[i] + R.h) {
                    top = i;
                    break;
                }
            }
            if (top >= 0) {
                const Rect& R = S.rects[top];
                double u = ((double)x - rx[top]) / L, w = ((double)y - ry[top]) / L;
                int iu = (int)floor(u), iw = (int)floor(w);
                double fu = u - iu, fw = w - iw;
                if (iu < 0) { iu = 0; fu = 0; }
                if (iw < 0) { iw = 0; fw = 0; }
                if (iu > R.lw - 2) { iu = R.lw - 2; fu = 1; }
                if (iw > R.lh - 2) { iw = R.lh - 2; fw = 1; }
                for (int c = 0; c < 3; c++) {
                    double a = R.lat[((size_t)iw * R.lw + iu) * 3 + c], b = R.lat[((size_t)iw * R.lw + iu + 1) * 3 + c];
                    double d = R.lat[((size_t)(iw + 1) * R.lw + iu) * 3 + c],
                           e = R.lat[((size_t)(iw + 1) * R.lw + iu + 1) * 3 + c];
                    v[c] = (a * (1 - fu) + b * fu) * (1 - fw) + (d * (1 - fu) + e * fu) * fw;
                }
            } else {
                double X = x + ox, Y = y + oy;
                v[0] = v[1] = v[2] = 128.0;
                for (int k = 0; k < 3; k++) {
                    double sv = sin(TWO_PI * S.g[k].f * (X * S.g[k].c + Y * S.g[k].s) + S.g[k].phase);
                    for (int c = 0; c < 3; c++) v[c] += S.g[k].amp[c] * sv;
                }
            }
            uint64_t ctr = fseed ^ ((uint64_t)y * (uint64_t)W + (uint64_t)x) * 0x9E3779B97F4A7C15ull;
            uint64_t r0 = mix(ctr), r1 = mix(ctr ^ 0xA5A5A5A5A5A5A5A5ull);
            double u1 = (double)((r0 >> 11) + 1) * (1.0 / 9007199254740993.0);
            double u2 = u01(r1);
            double rad = sqrt(-2.0 * log(u1));
            double n0 = rad * cos(TWO_PI * u2), n1 = rad * sin(TWO_PI * u2);
            uint64_t r2 = mix(ctr ^ 0x3C3C3C3C3C3C3C3Cull), r3 = mix(ctr ^ 0x7E7E7E7E7E7E7E7Eull);
            double u3 = (double)((r2 >> 11) + 1) * (1.0 / 9007199254740993.0);
            double n2 = sqrt(-2.0 * log(u3)) * cos(TWO_PI * u01(r3));
            double nz[3] = {n0, n1, n2};
            uint8_t* o = out + ((size_t)y * W + x) * 3;
            for (int c = 0; c < 3; c++) {
                double s = floor(v[c] + S.p.sigma * nz[c] + 0.5);
                o[c] = (uint8_t)(s < 0 ? 0 : (s > 255 ? 255 : s));
            }
        }
    }
}

}  // extern "C"
