/* riv_synth.h -- seeded synthetic RGB24 clip generator (host C ABI); see synth.cpp. */
#ifndef RIV_SYNTH_H
#define RIV_SYNTH_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct {
    uint32_t width, height;
    uint32_t n_rects, side_min, side_max, lattice;
    double vmax, pan_max, sigma;
    uint32_t seed, clip;
} riv_synth_params;

/* name: "cif" (352x288), "720p", "1080p", "4k" */
void riv_synth_preset(riv_synth_params* p, const char* name, uint32_t seed, uint32_t clip);
void* riv_synth_new(const riv_synth_params* p);
void riv_synth_frame(void* h, uint32_t t, uint8_t* rgb_out);
void riv_synth_free(void* h);
#ifdef __cplusplus
}
#endif
#endif
