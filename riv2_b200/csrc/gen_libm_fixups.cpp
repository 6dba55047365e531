// gen_libm_fixups.cpp -- build-time generator of the glibc logf / exp2f fix-up tables.
//
// The reference's adaptive quantiser uses f32::ln and f32::exp2, which on linux-gnu are
// glibc logf / exp2f -- accurate but not correctly rounded.  The device evaluates the
// correctly rounded value (double function rounded to float) and patches the inputs
// where glibc returns the other neighbour.  This program runs glibc over the whole
// input domain the quantiser can reach and records those inputs:
//   logf : every float in [4, 16384]   (variance floor 4, 8-bit luma variance <= 16256.25)
//   exp2f: every float with |x| <= 2   (x = 0.8*(ln v - mean)/6, |x| < 1.11)
// Output: "RIVLIBM1", u32 nlog, u32 nexp, then nlog and nexp (input bits, output bits)
// pairs sorted by input bits.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

static inline float f_of(uint32_t b) { float f; memcpy(&f, &b, 4); return f; }
static inline uint32_t b_of(float f) { uint32_t b; memcpy(&b, &f, 4); return b; }

template <class F>
static void scan(uint32_t lo, uint32_t hi, F fn, std::vector<uint32_t>& out) {
    const int NT = 64;
    std::vector<std::vector<uint32_t>> part(NT);
    uint64_t span = (uint64_t)hi - lo + 1;
#pragma omp parallel for schedule(static)
    for (int t = 0; t < NT; t++) {
        uint64_t a = lo + span * t / NT, b = lo + span * (t + 1) / NT;
        for (uint64_t k = a; k < b; k++) {
            uint32_t bits = (uint32_t)k;
            float x = f_of(bits);
            float g, c;
            fn(x, g, c);
            if (b_of(g) != b_of(c)) {
                part[t].push_back(bits);
                part[t].push_back(b_of(g));
            }
        }
    }
    for (auto& p : part) out.insert(out.end(), p.begin(), p.end());
}

int main(int argc, char** argv) {
    if (argc < 2) {
        fprintf(stderr, "usage: %s out.bin\n", argv[0]);
        return 2;
    }
    std::vector<uint32_t> lg, ex;
    auto flog = [](float x, float& g, float& c) {
        g = logf(x);
        c = (float)log((double)x);
    };
    auto fexp = [](float x, float& g, float& c) {
        g = exp2f(x);
        c = (float)exp2((double)x);
    };
    scan(b_of(4.0f), b_of(16384.0f), flog, lg);
    // positive floats 0..2 then negative floats -0..-2 (bit order: pairs stay sorted by
    // key because the two ranges are disjoint and appended in increasing key order)
    scan(0u, b_of(2.0f), fexp, ex);
    scan(0x80000000u, b_of(-2.0f), fexp, ex);
    FILE* f = fopen(argv[1], "wb");
    if (!f) return 1;
    uint32_t n[2] = {(uint32_t)(lg.size() / 2), (uint32_t)(ex.size() / 2)};
    fwrite("RIVLIBM1", 1, 8, f);
    fwrite(n, 4, 2, f);
    fwrite(lg.data(), 4, lg.size(), f);
    fwrite(ex.data(), 4, ex.size(), f);
    fclose(f);
    printf("libm fixups: logf %u, exp2f %u\n", n[0], n[1]);
    return 0;
}
