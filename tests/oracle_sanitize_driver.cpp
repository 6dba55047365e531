// The oracle (oracle/riv_oracle.cpp, test infrastructure) under AddressSanitizer and
// UndefinedBehaviorSanitizer: small moving clips through the oracle encoder and decoder at a
// few sizes and settings, with every decoded frame equal to the encoder's reconstruction.
// Built and run by tests/test_host_sanitizers.py.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "riv_oracle.h"

namespace {

// A textured background panning by (t, t/2) with a bright square moving the other way.
std::vector<uint8_t> frame_rgb(uint32_t w, uint32_t h, int t) {
    std::vector<uint8_t> rgb((size_t)w * h * 3);
    for (uint32_t y = 0; y < h; y++)
        for (uint32_t x = 0; x < w; x++) {
            const int sx = (int)x + t, sy = (int)y + t / 2;
            uint32_t v = (uint32_t)(sx * 7 + sy * 13) ^ (uint32_t)(sx * sy);
            uint8_t* p = &rgb[((size_t)y * w + x) * 3];
            p[0] = (uint8_t)(v & 0xff);
            p[1] = (uint8_t)((v >> 3) & 0xff);
            p[2] = (uint8_t)((sx * 5 + sy * 3) & 0xff);
            const int qx = (int)w / 2 - 2 * t, qy = (int)h / 3 + t;
            if ((int)x >= qx && (int)x < qx + 12 && (int)y >= qy && (int)y < qy + 12) p[0] = p[1] = p[2] = 235;
        }
    return rgb;
}

int run(uint32_t w, uint32_t h, uint8_t sr, uint8_t iq, uint8_t pq, int frames) {
    oracle_config c;
    oracle_config_default(&c, w, h, 30);
    c.search_range = sr;
    c.intra_quality = iq;
    c.inter_quality = pq;
    c.keyframe_mode = 2;
    c.keyframe_interval = 1000;
    int st = 0;
    void* e = oracle_enc_new(&c, &st);
    if (!e || st) return 10;
    const uint32_t sw = c.storage_width, sh = c.storage_height;
    std::vector<std::vector<uint8_t>> recon;
    for (int t = 0; t < frames; t++) {
        std::vector<uint8_t> rgb = frame_rgb(w, h, t);
        if (oracle_enc_frame_rgb(e, rgb.data(), w, h, (uint64_t)t * 33)) return 11;
        std::vector<uint8_t> r((size_t)sw * sh * 3 / 2);
        oracle_enc_last_recon(e, r.data(), r.data() + (size_t)sw * sh, r.data() + (size_t)sw * sh * 5 / 4);
        recon.push_back(r);
    }
    if (oracle_enc_finish(e)) return 12;
    const uint8_t* data = nullptr;
    const size_t len = oracle_enc_bytes(e, &data);
    std::vector<uint8_t> stream(data, data + len);
    oracle_enc_free(e);
    void* d = oracle_dec_new(stream.data(), stream.size(), &st);
    if (!d || st) return 13;
    for (int t = 0; t < frames; t++) {
        std::vector<uint8_t> r((size_t)sw * sh * 3 / 2);
        if (oracle_dec_next(d, r.data(), r.data() + (size_t)sw * sh, r.data() + (size_t)sw * sh * 5 / 4) < 0) return 14;
        if (r != recon[t]) return 15;
    }
    oracle_dec_free(d);
    return 0;
}

}  // namespace

int main() {
    struct Case { uint32_t w, h; uint8_t sr, iq, pq; int frames; } cases[] = {
        {64, 48, 12, 85, 80, 5}, {100, 70, 31, 95, 90, 4}, {16, 16, 12, 85, 80, 3}, {96, 64, 15, 60, 40, 4}};
    for (const Case& k : cases) {
        const int rc = run(k.w, k.h, k.sr, k.iq, k.pq, k.frames);
        if (rc) {
            std::fprintf(stderr, "FAIL case %ux%u sr %u: code %d\n", k.w, k.h, k.sr, rc);
            return 1;
        }
    }
    std::printf("oracle sanitizer driver: ok\n");
    return 0;
}
