/*
 * riv_oracle.h -- C interface of the CPU oracle for the riv2 P-frame encoder path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain, single-threaded C++
 * restatement of the reference encoder (reitero_encode), its residual/DCT/rANS
 * crates and its decoder (reitero_decode), written to be read side by side with
 * the reference sources cited in riv_oracle.cpp.  It is the checker for the CUDA
 * path: only the test suite, the smoke check and the CPU-baseline leg of the
 * benchmark load it.  Nothing in the product links or calls it.
 *
 * Parity status: pinned by the reference's own deblock known-answer tests and by
 * its DCT / IDCT constant tables (tests/golden); everything else is a faithful
 * restatement checked for encoder/decoder self-consistency.  RGB->YUV lives in
 * the un-vendored `yuv` 0.8.9 crate and is parity-unpinned (own BT.709 limited
 * range fixed-point definition, shared with the CUDA path).
 */
#ifndef RIV_ORACLE_H
#define RIV_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors reitero_encode::EncoderConfig (enc/config.rs:24-53). */
typedef struct {
    uint32_t display_width, display_height;
    uint32_t storage_width, storage_height;
    uint32_t fps;
    uint32_t keyframe_mode;      /* 0 = AllIntra, 1 = Automatic, 2 = Fixed */
    uint64_t keyframe_interval;  /* used when keyframe_mode == 2 */
    uint8_t intra_quality, inter_quality, search_range, mv_deflate_level, skip_threshold;
    uint8_t _pad[3];
    int64_t me_zero_mv_threshold, me_predictor_threshold;
    double rdo_lambda_mult;
    float inter_dead_zone;
    uint32_t _pad2;
} oracle_config;

void oracle_config_default(oracle_config* c, uint32_t w, uint32_t h, uint32_t fps);

/* ---- whole-encoder / decoder ---- */
void* oracle_enc_new(const oracle_config* c, int* status);
int oracle_enc_frame_rgb(void* h, const uint8_t* rgb, uint32_t w, uint32_t hgt, uint64_t ts);
int oracle_enc_frame_yuv(void* h, const uint8_t* y, const uint8_t* u, const uint8_t* v, uint64_t ts);
int oracle_enc_finish(void* h);
size_t oracle_enc_bytes(void* h, const uint8_t** data);
void oracle_enc_free(void* h);
/* Per-frame intermediates of the last encoded frame (sizes: mbs = (w/16)*(h/16)). */
int oracle_enc_last_type(void* h);
void oracle_enc_last_recon(void* h, uint8_t* y, uint8_t* u, uint8_t* v);          /* after deblock */
void oracle_enc_last_recon_pre(void* h, uint8_t* y, uint8_t* u, uint8_t* v);      /* before deblock */
void oracle_enc_last_curr(void* h, uint8_t* y, uint8_t* u, uint8_t* v);           /* converted input */
void oracle_enc_last_pred(void* h, uint8_t* y, uint8_t* u, uint8_t* v);
/* raw: 4 bytes/MB (dx,dy,sx,sy) canonical search MV; coded: same for the coded_prefix MV */
void oracle_enc_last_mvs(void* h, int8_t* raw, int8_t* coded, int64_t* best_sad);
/* side: 8 bytes/MB = mode, new_base, raw_dx, raw_dy, flags(pre-residual), rdo_skip, opt_skip, filter */
void oracle_enc_last_side(void* h, uint8_t* side);
void oracle_enc_last_qsteps(void* h, float* qs);
void oracle_enc_last_coeffs(void* h, int16_t* coeffs); /* 384 per MB: Y256,U64,V64 */
void oracle_enc_last_bias(void* h, int8_t* bias2);
/* EncodeFrameStats of the last frame as ORACLE_STATS_N doubles: frame_type, total_bytes,
 * mv_bytes, mv_raw_bytes, residual_bytes, blocks_total, blocks_skipped, mv_zero_delta_blocks,
 * mv_mode_counts[7], mv_new_zero_pre_bias, _post_bias, _axes_x, _axes_y, mv_new_base_counts[5],
 * mv_new_best_ref_counts[5], mv_new_best_ref_l1_saved_sum, mv_new_blocks, mv_new_delta_count,
 * mv_new_delta_mag_sum, _sq_sum, mv_class_histogram[11], mv_bias_dx, _dy,
 * mv_candidate_unique_total, _samples, _min, _max, mv_match_source_counts[6],
 * mv_match_nonzero_blocks, _any_spatial, _any_temporal, resi_raw, resi_rans (-1 = None),
 * rdo_lambda, rdo_blocks_evaluated, rdo_blocks_selected_skip, rdo_forced_fractional,
 * _threshold, _disabled, rdo_avg_skip_cost, rdo_avg_coded_cost.  Returns the count written. */
#define ORACLE_STATS_N 70
#define ORACLE_STATS_RESI_RAW 60
size_t oracle_enc_last_stats(void* h, double* out, size_t n);
size_t oracle_enc_last_record(void* h, const uint8_t** data);

void* oracle_dec_new(const uint8_t* stream, size_t len, int* status);
/* returns frame type (1/2) or negative on error / end of stream */
int oracle_dec_next(void* h, uint8_t* y, uint8_t* u, uint8_t* v);
void oracle_dec_dims(void* h, uint32_t* dims6); /* dw, dh, sw, sh, fps, frame_count(lo) */
void oracle_dec_free(void* h);

/* ---- stage functions ---- */
void oracle_rgb_to_yuv420(const uint8_t* rgb, uint32_t dw, uint32_t dh, uint32_t sw, uint32_t sh,
                          uint8_t* y, uint8_t* u, uint8_t* v);
void oracle_deblock(uint8_t* y, uint8_t* u, uint8_t* v, uint32_t w, uint32_t h, int level, int intra,
                    const uint8_t* mask /* nullable, one byte per MB */);
int oracle_deblock_level(uint8_t quality);
float oracle_quant_step(uint8_t quality);
void oracle_build_predicted(const uint8_t* py, const uint8_t* pu, const uint8_t* pv, uint32_t w, uint32_t h,
                            const int8_t* mvs4, uint8_t* oy, uint8_t* ou, uint8_t* ov);
void oracle_reference_build_predicted(const uint8_t* py, const uint8_t* pu, const uint8_t* pv, uint32_t w,
                                      uint32_t h, const int8_t* mvs4, uint8_t* oy, uint8_t* ou, uint8_t* ov);
/* hex search over luma planes; prev_mvs4 nullable; out: raw mvs (4 B/MB) + best sads */
void oracle_motion_search(const uint8_t* prev_y, const uint8_t* curr_y, uint32_t w, uint32_t h,
                          uint8_t search_range, const int8_t* prev_mvs4, int64_t zthr, int64_t pthr,
                          double lambda, int8_t* out_mvs4, int64_t* out_sads);
int64_t oracle_sad_int(const uint8_t* prev_y, const uint8_t* curr_y, uint32_t w, uint32_t h, int x0, int y0,
                       int dx, int dy, int64_t limit, int force_scalar);
int64_t oracle_sad_halfpel(const uint8_t* prev_y, const uint8_t* curr_y, uint32_t w, uint32_t h, int x0,
                           int y0, int dx_hp, int dy_hp, int64_t limit, int force_scalar);
void oracle_aq_steps(const uint8_t* pred_y, uint32_t w, uint32_t h, float base, float* out);
/* Residual, 16x16/8x8 FDCT, dead-zone quantisation, optimized skip and reconstruction of
 * encode_inter (res/residual.rs:520-752) for given per-MB AQ steps; skip = RDO-skipped MBs;
 * coeffs: 384 per MB; planes contiguous Y, U, V. */
void oracle_residual_inter(const uint8_t* cur_yuv, const uint8_t* pred_yuv, uint32_t w, uint32_t h, const uint8_t* skip,
                           const float* qs, float dz, int16_t* coeffs, uint8_t* opt_skip, uint8_t* recon_yuv);
double oracle_rdo_lambda(uint8_t inter_quality, double mult);
/* forward transforms + quant of one block; inverse of one block */
void oracle_fdct16_quant(const int16_t* blk256, float qs, float dead_zone, int16_t* out256);
void oracle_fdct8_quant(const int16_t* blk64, float qs, float dead_zone, int16_t* out64);
void oracle_idct16_aq(const int16_t* coeffs256, float qs, int16_t* out256);
void oracle_idct8_aq(const int16_t* coeffs64, float qs, int16_t* out64);
/* rANS helpers for round-trip tests */
size_t oracle_rans_roundtrip(const uint8_t* bits, const uint8_t* bypass, size_t n, uint8_t* out_bits,
                             uint8_t* stream, size_t stream_cap);
double oracle_glibc_logf_check(void);
/* DCT-coefficient coder of one frame (res/rans.rs:195-330) on n dense blocks of 384 i16
 * (Y 256, U 64, V 64), DC prediction when intra; returns the stream size, copies up to cap
 * bytes. */
size_t oracle_dct_encode(const int16_t* blocks, int n, int intra, uint8_t* stream, size_t cap);
/* Decoder output: storage-size YUV 4:2:0 to display-size RGB24 (BT.709 limited range, the
 * project's definition; dec/decoder.rs:445-456). */
void oracle_yuv_to_rgb(const uint8_t* y, const uint8_t* u, const uint8_t* v, uint32_t sw, uint32_t sh, uint32_t dw,
                       uint32_t dh, uint8_t* rgb);

#ifdef __cplusplus
}
#endif
#endif
