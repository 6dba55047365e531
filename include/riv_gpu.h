/*
 * riv_gpu.h -- C ABI of the B200 riv2 P-frame encoder (drop-in for reitero_encode).
 *
 * Each declaration names the reference interface it replaces (paths relative to the
 * reference project root; enc/ = reitero_video/reitero_encode/src/).  A Rust caller
 * binds these through an `extern "C"` block; Python binds them with ctypes
 * (riv2_b200/encoder.py).  No CUDA or torch types appear here: buffers
 * are plain pointers and sizes.
 *
 * Threading: one encoder per host thread.  riv_encode_frame may keep up to
 * `pipeline_depth` frames in flight (GPU work and host entropy coding overlap across
 * frames); records still reach the writer strictly in frame order, and riv_finish
 * flushes everything.  With pipeline_depth == 0 every call returns only after its own
 * record has been handed to the writer, exactly like Encoder::encode_frame.
 */
#ifndef RIV_GPU_H
#define RIV_GPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* EncodeError variants (enc/error.rs:4-20) plus device-side failures. */
typedef enum {
    RIV_OK = 0,
    RIV_ERR_IO = 1,               /* EncodeError::Io -- a writer callback failed */
    RIV_ERR_INVALID_CONFIG = 2,   /* EncodeError::InvalidConfig */
    RIV_ERR_ENCODING_FAILED = 3,  /* EncodeError::EncodingFailed */
    RIV_ERR_UNSUPPORTED_CODEC = 4,/* EncodeError::UnsupportedCodec (never produced) */
    RIV_ERR_FRAME = 5,            /* EncodeError::FrameError -- bad dimensions / sizes */
    RIV_ERR_CUDA = 6,             /* a CUDA runtime call failed */
    RIV_ERR_DEVICE_TIMEOUT = 7    /* a bounded device-side wait expired */
} riv_status;

/* KeyframeInterval (enc/config.rs:5-19): AllIntra, Automatic (= fixed 30), Fixed(n). */
typedef enum { RIV_KEYFRAME_ALL_INTRA = 0, RIV_KEYFRAME_AUTOMATIC = 1, RIV_KEYFRAME_FIXED = 2 } riv_keyframe_mode;

/* EncoderConfig (enc/config.rs:24-53).  The trailing device fields never change bits. */
typedef struct {
    uint32_t display_width, display_height;
    uint32_t storage_width, storage_height;
    uint32_t fps;
    uint32_t keyframe_mode;     /* riv_keyframe_mode */
    uint64_t keyframe_interval; /* for RIV_KEYFRAME_FIXED */
    uint8_t intra_quality, inter_quality, search_range, mv_deflate_level, skip_threshold;
    uint8_t _pad[3];
    int64_t me_zero_mv_threshold, me_predictor_threshold;
    double rdo_lambda_mult;
    float inter_dead_zone;
    /* device / host-runtime tuning */
    int32_t device;          /* CUDA device ordinal */
    uint32_t pipeline_depth; /* frames in flight (0 = synchronous, like the reference) */
    uint32_t entropy_threads;/* host threads for the DCT-coefficient rANS coder (0 = auto) */
    /* Encode form (riv_encode_form; no counterpart in the reference, which has only the plain
     * search).  The plain form reproduces the reference encoder byte for byte; the learned
     * form seeds a parallel search with the proposal network (riv_encoder_set_proposal) and
     * writes a different, equally valid stream.  proposal_margin: SAD margin above which a
     * macroblock's proposals count as failed and it falls back to the hexagon search. */
    uint32_t encode_form;
    uint32_t proposal_margin;
} riv_config;

/* RIV_FORM_PLAIN: the reference's raster-order search (byte-identical streams).
 * RIV_FORM_LEARNED: every MB searched at once from the proposal network's four candidates and
 * the previous P-frame's MV predictors (short diamond + half-pel; hexagon search as fallback);
 * mode decisions for all MBs at once.  Needs search_range <= 63 and riv_encoder_set_proposal.
 * RIV_FORM_PARALLEL: the same parallel search without the network: every MB runs the hexagon
 * search from its best predictor (the learned form's method without its network). */
typedef enum { RIV_FORM_PLAIN = 0, RIV_FORM_LEARNED = 1, RIV_FORM_PARALLEL = 2 } riv_encode_form;

/* EncoderConfig::new (enc/config.rs:56-77): defaults, storage rounded up to 16. */
void riv_config_default(riv_config* cfg, uint32_t width, uint32_t height, uint32_t fps);

/* VideoWriter (enc/writer.rs:5-18).  Callbacks return 0 on success. */
typedef struct {
    int (*write)(void* user, const uint8_t* data, size_t len);
    uint64_t (*position)(void* user);
    int (*seek)(void* user, uint64_t pos);
    int (*flush)(void* user);
    void* user;
} riv_writer_vtable;

/* EncodeFrameStats (enc/encoder.rs:58-124), field for field except `rle_stats` (its sizes are
 * resi_raw / resi_rans).  Option fields: -1 = None.  The fields marked (*) need the frame's
 * per-MB search results and are filled only for the frame whose riv_encode_frame call passed
 * a stats pointer (the others leave them 0); the rest are filled for every frame. */
typedef struct {
    uint64_t frame_index, timestamp_ms;
    uint32_t frame_type; /* 1 = intra, 2 = inter (FrameType, com/format.rs:12-20) */
    uint32_t total_bytes, mv_bytes, mv_raw_bytes, residual_bytes;
    uint32_t storage_width, storage_height;
    uint32_t blocks_total, blocks_skipped;
    uint32_t mv_zero_delta_blocks;
    uint32_t mv_mode_counts[7];
    uint32_t mv_new_zero_pre_bias, mv_new_zero_post_bias, mv_new_zero_axes_x, mv_new_zero_axes_y;
    uint32_t mv_new_base_counts[5];
    uint32_t mv_new_best_ref_counts[5];      /* (*) */
    uint64_t mv_new_best_ref_l1_saved_sum;   /* (*) */
    uint32_t mv_new_blocks, mv_new_delta_count;
    double mv_new_delta_mag_sum, mv_new_delta_mag_sq_sum;
    uint64_t mv_class_histogram[11];
    int32_t mv_bias_dx, mv_bias_dy;
    uint32_t mv_candidate_unique_total, mv_candidate_unique_samples; /* (*) */
    uint32_t mv_candidate_unique_min, mv_candidate_unique_max;       /* (*) */
    uint32_t mv_match_source_counts[6];                              /* (*) */
    uint32_t mv_match_nonzero_blocks, mv_match_any_spatial, mv_match_any_temporal; /* (*) */
    int64_t resi_raw, resi_rans;
    double rdo_lambda;
    uint32_t rdo_blocks_evaluated, rdo_blocks_selected_skip;                    /* (*) */
    uint32_t rdo_forced_fractional, rdo_forced_threshold, rdo_forced_disabled; /* (*) */
    double rdo_avg_skip_cost, rdo_avg_coded_cost;                               /* (*) */
} riv_frame_stats;

typedef struct riv_encoder riv_encoder;

/* Encoder::new (enc/encoder.rs:162-188): validates, writes the 36-byte header now. */
riv_status riv_encoder_new(const riv_config* cfg, const riv_writer_vtable* writer, riv_encoder** out);
/* Encoder::encode_frame / encode_frame_with_stats (enc/encoder.rs:229-256): RGB24,
 * display size, row-major, no padding; `rgb` is only read during the call.
 * `stats` (nullable) forces this frame to complete before returning. */
riv_status riv_encode_frame(riv_encoder* enc, const uint8_t* rgb, uint32_t width, uint32_t height,
                            uint64_t timestamp_ms, riv_frame_stats* stats);
/* Same input already resident in device memory (display-size RGB24). */
riv_status riv_encode_frame_device(riv_encoder* enc, const void* d_rgb, uint64_t timestamp_ms, riv_frame_stats* stats);
/* Test hook: storage-size YUV 4:2:0 planes (the input of the path after RGB->YUV). */
riv_status riv_encode_frame_yuv(riv_encoder* enc, const uint8_t* y, const uint8_t* u, const uint8_t* v,
                                uint64_t timestamp_ms, riv_frame_stats* stats);
/* Encoder::finish (enc/encoder.rs:950-961): drains, rewrites frame_count, flushes. */
riv_status riv_finish(riv_encoder* enc);
void riv_encoder_free(riv_encoder* enc);
/* No counterpart in the reference.  Loads the proposal network's parameters for
 * RIV_FORM_LEARNED: n = 91,536 f32 values (bf16-rounded weights of conv1..4, fc1..3, then
 * their biases; the layout of riv_nn.h), as written by this library's trainer.  Call before
 * the first P-frame; RIV_ERR_INVALID_CONFIG when n does not match. */
riv_status riv_encoder_set_proposal(riv_encoder* enc, const float* params, size_t n);
/* No counterpart in the reference.  Learned and parallel forms: P-frame MBs searched so far,
 * MBs that fell back to the hexagon search, MBs that kept an unrefined whole-pixel candidate
 * (the network's skip shortcut).  Synchronises the device. */
riv_status riv_learned_counters(riv_encoder* enc, uint64_t* mbs, uint64_t* fallbacks, uint64_t* shortcuts);
/* Message of the last failure ("" if none). */
const char* riv_last_error(const riv_encoder* enc);
uint64_t riv_frame_count(const riv_encoder* enc);

/* Reconstruction (deblocked reference) of the last frame whose GPU work finished;
 * storage-size planes.  Synchronises the device. */
riv_status riv_last_recon(riv_encoder* enc, uint8_t* y, uint8_t* u, uint8_t* v);
/* Per-frame GPU timing of the last completed frame that carried stage timing events (every
 * frame at pipeline_depth 0 or with per-frame stats, else one in 8), microseconds: [0] rgb->yuv
 * [1] integer-SAD table (plain form) or proposal network (learned form) [2] search/mode
 * (the wavefront, or the learned forms' parallel search + mode decision) [3] predict [4] aq
 * [5] residual [6] deblock [7] compact [8] total */
riv_status riv_last_kernel_times(riv_encoder* enc, float* us9);

/* Cumulative counters since riv_encoder_new: us9 = per-stage GPU time summed over all
 * P-frames (same stage order as riv_last_kernel_times), io2 = {host->device bytes,
 * device->host bytes}, n4 = {P-frames, kernel launches, P-frames whose residual and deblock
 * ran inside the next P-frame's search launch, P-frames with stage timings}.  With
 * pipeline_depth > 0 only one frame in 8 carries stage timing events (timing-enabled
 * events between back-to-back search launches idle the GPU for microseconds each), so us9
 * sums over the timed P-frames: divide by n4[3]. */
riv_status riv_counters(riv_encoder* enc, double* us9, uint64_t* io2, uint64_t* n4);
/* Cumulative host-side milliseconds: [0] GPU submission, [1] retiring finished frames,
 * [2] motion-vector coding, [3] DCT-coefficient coding (summed over worker threads),
 * [4] record writes, [5] waiting for a frame's entropy coding to finish. */
riv_status riv_host_times(riv_encoder* enc, double* ms6);

/* ---- Multi-clip encoding.  No counterpart in the reference (one stream per Encoder). ----
 * A batch holds n independent clips -- each with its own config (any mix of sizes, qualities
 * and keyframe settings; plain form; one device) and its own writer -- whose frames are
 * encoded together one step at a time.  A step takes at most one frame per clip; its GPU work
 * is one launch per stage over every clip of the step (conversion, SAD tables, the search --
 * one cooperative launch in which each clip's CTAs run its MB rows as a wavefront --,
 * prediction, AQ mean, residual, deblock, compaction), so the clips fill the SMs that one
 * clip's wavefront leaves idle; each clip's entropy coding and records then run as in
 * riv_encode_frame, on thread pools the clips share.  Every clip's stream is byte-identical
 * to what riv_encoder_new + riv_encode_frame + riv_finish write for that clip alone.
 * Tile shapes (search CTAs, SAD table or not, MBs per residual CTA, deblock tile width) are
 * chosen by an autotuner during the first all-P-frame steps (they do not change the output),
 * or fixed by riv_batch_set_tune. */
#define RIV_BATCH_MAX_CLIPS 256
typedef struct riv_batch riv_batch;
typedef struct {
    int32_t search_rows_pct; /* search CTAs per step, percent of what fits on the device (1..100) */
    int32_t res_mbs;         /* MBs per residual CTA: 2, 4 or 8 */
    int32_t db_tw;           /* deblock tile width, luma columns: 64, 128 or 256 */
    int32_t sad_table;       /* 1: search from an exhaustive SAD table (search ranges <= 15), 0: SADs on the way */
} riv_batch_tune;
/* cfgs[i] / writers[i]: clip i (n <= RIV_BATCH_MAX_CLIPS).  Headers are written now. */
riv_status riv_batch_new(const riv_config* cfgs, const riv_writer_vtable* writers, uint32_t n, riv_batch** out);
/* One step: frames[i] = clip i's next RGB24 frame (display size, host memory, read during
 * the call) or NULL when clip i has none in this step; ts[i] its timestamp. */
riv_status riv_batch_encode(riv_batch* b, const uint8_t* const* frames, const uint64_t* ts);
/* The same with the frames already in device memory. */
riv_status riv_batch_encode_device(riv_batch* b, const void* const* d_frames, const uint64_t* ts);
/* Encoder::finish of every clip (drains, rewrites each header's frame count, flushes). */
riv_status riv_batch_finish(riv_batch* b);
void riv_batch_free(riv_batch* b);
const char* riv_batch_last_error(const riv_batch* b);
/* Fixes the tile shapes (the autotuner stops); RIV_ERR_INVALID_CONFIG for values not listed. */
riv_status riv_batch_set_tune(riv_batch* b, const riv_batch_tune* t);
/* The shapes in use; *tuned = 0 still tuning, 1 chosen by the autotuner, 2 fixed. */
riv_status riv_batch_get_tune(const riv_batch* b, riv_batch_tune* t, int* tuned);
/* c7 = {steps, frames, MBs, kernel launches, timed steps, host->device bytes, device->host
 * bytes}; stage_us10 = mean GPU microseconds per timed step: conversion, SAD tables, search,
 * prediction, AQ mean, residual, deblock, scan, pack, whole step.  Either may be NULL. */
riv_status riv_batch_counters(const riv_batch* b, uint64_t* c7, double* stage_us10);
/* Cumulative host milliseconds: [0] waiting for a clip's earlier records before its next
 * frame (pipeline full), [1] descriptors and launches, [2] copies back and bookkeeping,
 * [3] advancing the clips' pipelines after each step, [4] riv_batch_finish. */
riv_status riv_batch_host_times(const riv_batch* b, double* ms5);
/* Reconstruction (storage-size planes) of clip `clip`'s last submitted frame.  Synchronises. */
riv_status riv_batch_last_recon(riv_batch* b, uint32_t clip, uint8_t* y, uint8_t* u, uint8_t* v);
/* Records written so far for clip `clip`, and its host milliseconds (as riv_host_times). */
riv_status riv_batch_clip_counters(const riv_batch* b, uint32_t clip, uint64_t* frames_written, double* host_ms6);

/* In-memory writer (VecWriter, enc/writer.rs:20-69). */
typedef struct riv_memwriter riv_memwriter;
riv_memwriter* riv_memwriter_new(void);
void riv_memwriter_vtable(riv_memwriter* w, riv_writer_vtable* out);
size_t riv_memwriter_size(const riv_memwriter* w);
const uint8_t* riv_memwriter_data(const riv_memwriter* w);
void riv_memwriter_free(riv_memwriter* w);

/* ---- Stage entry points (one kernel each, host buffers in/out) for parity tests ---- */
/* Yuv420Frame::from_rgb after pad_rgb24 (com/yuv.rs:41-74, enc/encoder.rs:1049-1096). */
riv_status riv_stage_rgb_to_yuv(const uint8_t* rgb, uint32_t dw, uint32_t dh, uint32_t sw, uint32_t sh,
                                uint8_t* yuv_out);
/* deblock_yuv420 (com/deblock.rs:189-202); mask: one byte per MB or NULL. */
riv_status riv_stage_deblock(uint8_t* yuv, uint32_t w, uint32_t h, int level, int intra, const uint8_t* mask);
/* No reference counterpart.  riv_stage_deblock without any device allocation, for callers
 * that cannot call cudaMalloc/cudaFree around each stage: applications whose device
 * memory is handed in full to their own pool allocator (a framework's caching allocator),
 * where a raw cudaMalloc fails or fragments the pool, and latency-critical threads, where
 * cudaFree would synchronise the whole device and stall the work already in flight.  The
 * planes and the optional mask are staged in one fixed device scratch area (a file-scope
 * __device__ array of RIV_DEBLOCK_NOALLOC_MAX_BYTES bytes, 256-byte aligned, held by every
 * GPU that loads the library until the process exits) instead of memory allocated and
 * freed on every call.  Same arguments and result as riv_stage_deblock, on the current
 * CUDA device.
 * Limit: w*h*3/2 bytes, plus (w/16)*(h/16) when mask != NULL, at most
 * RIV_DEBLOCK_NOALLOC_MAX_BYTES (4 MiB: storage sizes up to 1920x1088); larger requests
 * return RIV_ERR_FRAME and write the reason to errbuf (nullable, errbuf_len bytes).
 * Set-up: the first call on a device looks up the scratch address
 * (cudaGetSymbolAddress, device current) and keeps it for the life of the process; make
 * that first call before any stream capture on that device.  The kept address belongs to
 * the device's primary context: after cudaDeviceReset, or with another context current,
 * it is stale, so do not call this entry point after either.
 * Zero state: nothing in the scratch has to start at zero; each call writes every byte
 * it reads.
 * Calls that overlap on one device (from several host threads) share the scratch and
 * race: serialise them. */
#define RIV_DEBLOCK_NOALLOC_MAX_BYTES (4u << 20)
riv_status riv_stage_deblock_noalloc(uint8_t* yuv, uint32_t w, uint32_t h, int level, int intra,
                                     const uint8_t* mask, char* errbuf, size_t errbuf_len);
/* build_predicted (com/fast_motion.rs:103-352) and compute_aq_quant_steps
 * (res/residual.rs:116-167): the motion-compensated prediction of storage-size planes
 * ref_yuv (Y, U, V contiguous) for one MV per MB (mv4: dx, dy, sx, sy as i8, raster order),
 * then the per-MB AQ steps (qs, nullable) from the prediction's luma with the base step of
 * `quality` (quant_step_from_quality, res/residual.rs:13-23). */
riv_status riv_stage_predict(const uint8_t* ref_yuv, const int8_t* mv4, uint32_t w, uint32_t h, uint8_t quality,
                             uint8_t* pred_yuv, float* qs);
/* The residual part of ResidualEncoder::encode_inter (res/residual.rs:520-752): current minus
 * prediction, 16x16 / 8x8 FDCT, dead-zone quantisation with the per-MB steps qs, optimized
 * skip of all-zero MBs, dequantisation, inverse transforms and the pre-deblock
 * reconstruction.  rdo_skip: one byte per MB (RDO-skipped MBs keep the prediction);
 * coded4 (nullable): coded MVs, for the deblock mask (fmask, nullable: 1 where the MB is
 * coded or its MV is not zero).  coeffs: 384 i16 per MB (Y 16x16, U 8x8, V 8x8, row-major). */
riv_status riv_stage_residual(const uint8_t* cur_yuv, const uint8_t* pred_yuv, const float* qs, const uint8_t* rdo_skip,
                              const int8_t* coded4, float dead_zone, uint32_t w, uint32_t h, int16_t* coeffs,
                              uint8_t* opt_skip, uint8_t* recon_yuv, uint8_t* fmask);
/* glibc-exact logf (which=0) / exp2f (which=1) on the device over n inputs. */
riv_status riv_stage_libm(int which, const float* in, float* out, size_t n);
/* Test hook: device state left by the most recent frame (synchronises the device; meant
 * for pipeline_depth == 0).  what: 0 per-MB search/mode output (20 B/MB), 1 AQ steps
 * (f32/MB), 2 prediction (YUV), 3 converted input (YUV), 4 quantised coefficients
 * (384 x i16 per MB), 5 optimized skip (u8/MB), 6 search-kernel phase stamps (32 x i64 per
 * MB: words 0-15 SM clock cycles, 16-27 global-timer nanoseconds of the search start, the
 * deferred residual / deblock / SAD-table tasks and the loaders' reference waits; only when
 * the encoder was created with RIV_PROFILE_SEARCH set in the environment).
 * Returns RIV_ERR_FRAME if `size` is short. */
riv_status riv_debug_frame_state(riv_encoder* enc, int what, void* out, size_t size);
/* Test hook (no reference counterpart): the device logf (which=0), exp2f (which=1) and the
 * four-wide batched logf of the AQ warps (which=2) on every f32 whose bit pattern lies in
 * [lo_bits, hi_bits], compared bit for bit with the host's glibc logf / exp2f (the functions
 * f32::ln / f32::exp2 call on linux-gnu, res/residual.rs:116-167).  *mismatches = number of
 * inputs that differ, *first_bad_bits = the smallest such bit pattern (0 if none). */
riv_status riv_test_libm_range(int which, uint32_t lo_bits, uint32_t hi_bits, uint64_t* mismatches,
                               uint32_t* first_bad_bits);
/* Test hook (no reference counterpart): runs the bounded device waits of the search launch
 * on flags nothing sets (which: 0 wavefront record, 1 worker-queue counter, 2 search -> mode
 * hand-off slot, 3 mbarrier phase) with a spin limit of spin_limit polls (1 .. 2^20).  The
 * waits give up, the kernel returns, and the status word (*status_word) carries the same
 * timeout bit the encoder maps to RIV_ERR_DEVICE_TIMEOUT, which this call returns. */
riv_status riv_test_wait_expiry(int which, int64_t spin_limit, uint32_t* status_word);
/* Number of glibc fix-up entries loaded for logf / exp2f. */
riv_status riv_libm_fixup_counts(uint32_t* nlog, uint32_t* nexp);
/* The DCT bases the device uses (T16[i][j], T8[i][j]: sample i, frequency j). */
void riv_dct_tables(int32_t* t16, int32_t* t8);
/* Test hook (host only, no reference counterpart): the encoder's DCT-coefficient coder on n
 * dense blocks of 384 i16 (Y 256, U 64, V 64), laid out as the GPU compaction does, with DC
 * prediction when intra; threads > 0 codes it in parallel on this thread and a pool of that
 * many threads, as the encoder does for the newest frame of a drain (frames of 16K to 2M
 * coded coefficients; smaller ones model here and hand the full rANS batches to the pool).
 * *len = stream size; up to cap bytes copied.  RIV_ERR_ENCODING_FAILED where the reference
 * encoder panics (a magnitude class above 13). */
riv_status riv_test_dct_encode(const int16_t* blocks, uint32_t n, int intra, uint32_t threads, uint8_t* out, size_t cap,
                               size_t* len);
/* Test hook (host only, no reference counterpart): the decoder's DCT-coefficient decoder on one
 * frame's coefficient stream; n blocks of 384 i16 out, blocks with coded[b] == 0 are not in the
 * stream and stay zero; DC prediction when intra.  RIV_OK, or RIV_ERR_FRAME where the stream is
 * malformed (read past its end, an EOB beyond the plane: the reference decoder panics). */
riv_status riv_test_dct_decode(const uint8_t* data, size_t len, const uint8_t* coded, uint32_t n, int intra,
                               int16_t* out);
/* Test hook (host only, no reference counterpart): the NEW-delta bias the encoder writes in
 * each P-frame record (compute_delta_bias_for_new, enc/encoder.rs:984-1048) over n raw deltas. */
riv_status riv_test_delta_bias(const int8_t* dx, const int8_t* dy, uint32_t n, int8_t* bx, int8_t* by);
/* Test hooks (host only, no reference counterpart): the MV coder over nframes frames with one
 * coder (contexts and candidate history carry across frames, res/mv_rans/encoder.rs:60-412).
 * Frame f has dims[2f] x dims[2f+1] blocks; a block is 7 bytes: mode (MvMode order: Zero,
 * Nearest, Near, TopRight, TopLeft, New, Temporal), NEW base, dx (i8), dy (i8), subpel x,
 * subpel y (Zero, PlusHalf, MinusHalf), skip.  Encode: *len = total size, frame_len[f] = each
 * frame's size, up to cap bytes copied; RIV_ERR_ENCODING_FAILED on a NEW block with a raw
 * -1/2 subpel (the reference panics).  Decode: the inverse with a fresh coder (decoder.rs);
 * RIV_ERR_FRAME on malformed data. */
riv_status riv_test_mv_encode(const uint8_t* blocks, const uint32_t* dims, uint32_t nframes, uint8_t* out, size_t cap,
                              size_t* len, uint32_t* frame_len);
/* Test hook (host only, no reference counterpart): riv_test_mv_encode with the encoder's parallel
 * form of the MV coder (the calling thread and a pool of `threads` threads; 0: the sequential
 * form).  Same bytes. */
riv_status riv_test_mv_encode_threads(const uint8_t* blocks, const uint32_t* dims, uint32_t nframes, uint32_t threads,
                                      uint8_t* out, size_t cap, size_t* len, uint32_t* frame_len);
riv_status riv_test_mv_decode(const uint8_t* data, const uint32_t* frame_len, const uint32_t* dims, uint32_t nframes,
                              uint8_t* blocks);
/* Test hook (host only, no reference counterpart): the worker-task queue of the fused search
 * launch for a frame of bw x bh MBs and w storage columns, in the order the kernel hands the
 * tasks out: 3 int32 per task (kind 0 residual pair / 1 deblock tile / 2 SAD-table MB / 3 scan
 * / 4 pack row, MB row or band, index), up to cap int32; *n = task count.  defer: the previous
 * frame's reconstruction is in the queue; deblock: its deblock level is not 0; tables: the
 * SAD table is computed in the launch; compact: its compaction is in the queue. */
riv_status riv_test_worker_queue(uint32_t bw, uint32_t bh, uint32_t w, int defer, int deblock, int tables, int compact,
                                 int32_t* out, size_t cap, size_t* n);

/* ---- Decoder (reitero_decode) up to the YUV reconstruction ---- */
/* DecodeError (dec/error.rs:4-20): Io, InvalidHeader, DecodingFailed, InvalidFrame,
 * EndOfStream, plus device failures. */
typedef enum {
    RIV_DEC_OK = 0,
    RIV_DEC_IO = 1,               /* truncated stream */
    RIV_DEC_INVALID_HEADER = 2,
    RIV_DEC_DECODING_FAILED = 3,
    RIV_DEC_INVALID_FRAME = 4,
    RIV_DEC_END_OF_STREAM = 5,
    RIV_DEC_CUDA = 6
} riv_dec_status;
typedef struct riv_decoder riv_decoder;
/* Decoder::new (dec/decoder.rs:112-171) over an in-memory .riv stream (copied): parses and
 * validates the 36-byte header; reconstruction runs on CUDA device `device`. */
riv_dec_status riv_decoder_new(const uint8_t* data, size_t len, int device, riv_decoder** out);
/* Decoder::header (dec/decoder.rs:470-473): dims5 = display w, h, storage w, h, fps. */
riv_dec_status riv_decoder_info(const riv_decoder* dec, uint32_t* dims5, uint64_t* frame_count);
/* Decoder::decode_frame (dec/decoder.rs:174-460) up to the storage-size YUV 4:2:0
 * reconstruction (the reference's final RGB conversion and crop are not on this path).
 * y/u/v (each nullable) receive the planes; the call returns once the frame is decoded.
 * RIV_DEC_END_OF_STREAM after the last frame.  Records are read up to 8 frames ahead: their
 * MVs are decoded in order on the calling thread and their coefficient streams on a pool of
 * host threads; a record that cannot be read is reported by the call for that frame (the
 * frames before it decode normally). */
riv_dec_status riv_decode_frame_yuv(riv_decoder* dec, uint8_t* y, uint8_t* u, uint8_t* v, uint32_t* frame_type,
                                    uint64_t* timestamp_ms);
/* Decoder::decode_frame's RGB output (dec/decoder.rs:445-456): the frame as display-size RGB24
 * (rgb: display w x h x 3 bytes, nullable), converted on the GPU (BT.709 limited range, this
 * library's definition: the reference uses the `yuv` crate, so byte parity with it is not
 * established).  Same read-ahead and error behaviour as riv_decode_frame_yuv. */
riv_dec_status riv_decode_frame_rgb(riv_decoder* dec, uint8_t* rgb, uint32_t* frame_type, uint64_t* timestamp_ms);
/* Decoder::current_frame (dec/decoder.rs:475-478). */
uint64_t riv_decoder_current_frame(const riv_decoder* dec);
const char* riv_decoder_last_error(const riv_decoder* dec);
void riv_decoder_free(riv_decoder* dec);

#ifdef __cplusplus
}
#endif
#endif
