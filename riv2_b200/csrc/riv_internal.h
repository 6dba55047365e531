// riv_internal.h -- shared definitions between the sm_100a kernels and the host encoder.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace riv {

// Per-macroblock output of the search/mode kernel (k_search) -- 20 bytes.
struct MbOut {
    int8_t raw[4];     // canonical search MV: dx, dy, sx, sy (enc/motion/scalar.rs:619-635)
    int8_t coded[4];   // coded_prefix (reconstructed) MV (enc/encoder.rs:667-718)
    int8_t rdelta[2];  // NEW raw delta = clamp(actual - base) (enc/encoder.rs:654-656)
    uint8_t mode;      // MvMode::as_u8 (res/mv_predictor.rs:22-32)
    uint8_t base;      // NEW base index 0..4
    uint8_t flags;     // fractional bits for NEW (0x01 x+1/2, 0x04 y+1/2), skip bit patched later
    uint8_t rdo_skip;  // RDO skip candidate (enc/rdo.rs:140-178)
    uint8_t pad[2];
    int32_t best_sad;  // half-pel refinement SAD of the chosen MV
};
static_assert(sizeof(MbOut) == 20, "MbOut layout");

// Per-macroblock record published by the search wavefront for the next MB row:
// [63:48] frame tag, [47:40] raw dx, [39:32] raw dy, [31:24] coded dx, [23:16] coded dy,
// [15:8] coded sx, [7:0] coded sy.
typedef unsigned long long MbRec;

constexpr int RIV_PROF_WORDS = 32;  // i64 phase stamps per MB in SearchParams::prof

struct ResidualParams {
    const uint8_t* cur;   // planar YUV (Y then U then V)
    const uint8_t* pred;  // planar YUV
    uint8_t* recon;       // planar YUV (pre-deblock)
    int16_t* coeffs;      // 384 per MB
    uint8_t* opt_skip;    // 1 byte per MB
    uint8_t* fmask;       // deblock mask, 1 byte per MB
    uint8_t* eobs;        // 3 per MB (last non-zero index per plane block)
    const MbOut* mb;      // nullptr for intra
    const float* qs;      // per-MB quant step (inter)
    float dead_zone;
    int W, H, BW, intra;
    const uint16_t* intra_ytab;  // 256 (intra)
    const uint16_t* intra_ctab;  // 64 (intra)
    // AQ step computed here from the ln variances and their mean (lnv != nullptr), else read qs
    const float* lnv;            // n ln variances, then the mean
    float aq_base;
    const uint32_t* expfix;
    int nexp;
    float* qs_out;               // the steps, written for inspection
    const uint8_t* ref;          // chroma prediction computed here from this reference (nullptr: read pred)
};

struct SearchParams {
    const uint8_t* ref_y;
    const uint8_t* cur_y;
    int W, H, BW, BH, sr;
    const int8_t* prev_coded;  // 4 bytes/MB from the previous P-frame, or nullptr
    long long zthr, pthr;
    double lam2;      // lambda * 2.0 (the search's bit-cost scale)
    long long c15;    // (lambda * 2.0 * 1.5) as i64
    long long c05;    // (lambda * 2.0 * 0.5) as i64
    int lambda_zero;  // lambda == 0.0
    const double* mvbits;  // 256 entries: b(0)=1, b(d)=2*log2(d)+2 (glibc log2, host-computed)
    // NEW-mode bit cost (lambda*2*(6 + b(ax) + b(ay))) as i64, for ax, ay in [0,255], host-computed
    // in f64 exactly like the reference; nullptr = evaluate in f64 on the device.
    const long long* newcost;
    // Same costs for |ax|,|ay| < 64 as a 64x64 int32 table (staged in shared memory), valid
    // when every cost is below 2^27 (small == 1); then warp argmins use 32-bit keys.
    const int* newcost32;
    int small;
    // RDO (enc/rdo.rs)
    double rdo_lambda, rdo_skip_bits, rdo_keep_bits, rdo_icpt, rdo_slope, rdo_ret, rdo_guard;
    int rdo_allow;
    const uint16_t* tab;  // exhaustive integer-SAD table (when search_use_table), tstride entries per MB
    int tstride;
    MbRec* rec;       // 2 x BW*BH wavefront records: raw MVs (search), then coded MVs (mode)
    unsigned tag;
    MbOut* out;
    int8_t* coded_out;  // coded MV (dx, dy, sx, sy) per MB: the next frame's temporal predictors
    unsigned* status;
    long long spin_limit;
    long long* prof;  // optional: RIV_PROF_WORDS words per MB (phase stamps, hexagon rounds), nullptr = off
    int nrow_ctas;    // CTAs that own MB rows (row stride); the rest of the grid are table workers
    int cta0;         // first CTA of this clip in a multi-clip launch (0 for a single clip)
    int row_helpers;  // row CTAs run worker groups before their row starts and after it ends
    unsigned* tflag;  // fused table: per-MB flag = tag once its table row is written; nullptr = precomputed
    // Prediction and AQ inside the search launch (band + table instantiations): nullptr lnv =
    // done by the separate predict / AQ kernels.
    uint8_t* pred;             // planar YUV prediction out
    uint2* varsum;             // per MB (sum, sum of squares) of the predicted luma
    float* lnv;                // BW*BH ln variances, then the mean
    unsigned* row_done;        // per MB row: tag once its ln variances are written
    const uint32_t* logfix;    // glibc logf fix-up pairs + bucket index
    int nlog;
    // Residual and deblock of the previous P-frame, run by the table workers of this launch
    // ahead of the table rows that need them (defer != 0), then (compact != 0) its compaction
    // (scan + pack, as k_scan / k_pack) at the end of the queue.  wq: [0] task counter,
    // [1 .. BH] residual MBs done per MB row, [BH+1 .. 2BH] deblock tiles done per band,
    // [2BH+1] scan done.  Launches alternate between two such arrays: each zeroes the other
    // (wq_next, wq_words words) for the next launch, its own having been zeroed by the last.
    int defer;
    ResidualParams dres;
    int db_level, db_E, db_I, db_H;
    const uint8_t* db_src;
    uint8_t* db_dst;
    const uint8_t* db_mask;
    unsigned* wq;
    unsigned* wq_next;
    int wq_words;
    int compact;
    int32_t* c_index;
    int32_t* c_offset;
    uint32_t* c_side;
    int16_t* c_packed;
    uint8_t* c_peobs;
    uint32_t* c_hdr;
};


// ---- multi-clip steps (riv_batch): one launch per stage over every clip of the step.
// One clip's frame in a step.
struct BatchClip {
    int W, H, BW, NMB;  // storage size
    int intra;          // 1 key frame, 0 P-frame
    // conversion: display-size RGB24 (nullptr: cur already holds the frame's planes)
    const uint8_t* rgb;
    int dw, dh;
    uint8_t* cur;  // planar YUV of the frame
    // P-frames: the previous frame's deblocked reconstruction, the SAD table, the search's
    // per-MB output, the prediction and the ln variances (NMB values, then their mean)
    const uint8_t* ref;
    uint16_t* tab;
    int tstride, sr;
    const MbOut* mbo;
    uint8_t* pred;
    float* lnv;
    const uint32_t* logfix;
    int nlog;
    ResidualParams rp;  // residual (steps from lnv for P-frames, intra tables for key frames)
    // deblock (db_level > 0): db_src -> db_dst
    int db_level, db_E, db_I, db_H;
    const uint8_t* db_src;
    uint8_t* db_dst;
    const uint8_t* db_mask;
    // compaction into the slot's buffers; c_hdr = mapped host words (coded MBs, coefficients,
    // status)
    int32_t* c_index;
    int32_t* c_offset;
    uint32_t* c_side;
    int16_t* c_packed;
    uint8_t* c_peobs;
    uint32_t* c_hdr;
    const unsigned* status;
};
enum BatchStage { BS_CONVERT, BS_TABLE, BS_PREDICT, BS_AQSUM, BS_RESIDUAL, BS_DEBLOCK, BS_SCAN, BS_PACK, BS_N };
// Tile shapes of a step (chosen by the batch's autotuner; the output does not depend on them).
struct BatchTune {
    int res_mbs;   // MBs per residual CTA: 2, 4 or 8
    int db_tw;     // deblock tile width in luma columns: 64, 128 or 256
    int row_ctas;  // search: percent of the device's capacity of search CTAs used by a step
    int table;     // search from an exhaustive SAD table (search ranges <= 15) or SADs computed on the way
};
struct BatchLaunch {
    const BatchClip* clips;  // device, nclips
    const int* start;        // device, BS_N x (nclips + 1) CTA prefix sums
    int nclips;
};
int batch_ctas_host(int stage, const BatchClip& k, const BatchTune& t);
int launch_batch_stage(int stage, const BatchLaunch& b, const BatchTune& t, int total_ctas, int max_sr, void* stream);
int search_multi_capacity(bool table, bool small, int max_sr, int* per_sm, size_t* smem, int* threads);
int launch_search_multi(const SearchParams* dparams, const int* dstart, int nclips, int total_ctas, bool table,
                        bool small, size_t smem, int threads, void* stream);

enum StatusBits : unsigned {
    ST_WAIT_TIMEOUT = 1u,
    ST_HEX_CAP = 2u,
};

// Launchers (riv_kernels.cu).  All are asynchronous on `stream`.
int launch_rgb_to_yuv(const uint8_t* rgb, int dw, int dh, uint8_t* yuv, int W, int H, void* stream, bool beside = false);
int launch_yuv_to_rgb(const uint8_t* yuv, int W, int H, int dw, int dh, uint8_t* rgb, void* stream);
// Launch plan of the search wavefront (chosen once per encoder).  fused: the SAD table is
// computed inside the same cooperative launch by `grid - nrow` worker CTAs.
struct SearchPlan {
    bool fast;   // band + table instantiation: loader and AQ warps (prediction and AQ in the launch)
    bool fused;
    bool helpers;  // fused: row CTAs' spare threads and finished row CTAs take worker tasks
    int grid, nrow, threads;
    size_t smem;
};
int search_plan(int sr, int W, int BH, bool table, bool small, SearchPlan* out);
int launch_search(const SearchParams& p, const SearchPlan& plan, void* stream);
bool search_use_table(int sr);
int sad_table_stride(int sr);
int launch_sad_table(const uint8_t* ref, const uint8_t* cur, int W, int H, int sr, uint16_t* tab, int tstride,
                     void* stream);
size_t search_smem_bytes(int sr);
int launch_predict(const uint8_t* ref, const MbOut* mb, uint8_t* pred, uint2* varsum, int W, int H, void* stream);
int launch_aq(const uint2* varsum, int n, float base, const uint32_t* logfix, int nlog, const uint32_t* expfix,
              int nexp, float* lnv_scratch, float* qs, void* stream);
int launch_residual(const ResidualParams& p, int nmb, void* stream);
// Decoder: dequantise + inverse-transform dense coefficients onto the prediction (inter) or
// 128 (intra); skip[mb] != 0 copies the prediction (inter).
int launch_reconstruct(const int16_t* coeffs, const uint8_t* pred, const uint8_t* skip, const float* qs, int intra,
                       const uint16_t* ytab, const uint16_t* ctab, uint8_t* recon, int W, int H, void* stream);
int launch_deblock(uint8_t* yuv, int W, int H, int E, int I, int Hev, const uint8_t* mask, void* stream);
// Out-of-place deblock of all three planes in one launch (src != dst, no overlap).
int launch_deblock_tiled(const uint8_t* src, uint8_t* dst, int W, int H, int E, int I, int Hev, const uint8_t* mask,
                         void* stream);
// Scratch of the no-allocation deblock entry point (a file-scope __device__ array of
// DEBLOCK_NOALLOC_MAX_BYTES bytes); the address is valid on the current device.
constexpr size_t DEBLOCK_NOALLOC_MAX_BYTES = (size_t)4 << 20;
int deblock_scratch_address(void** out);
// k_scan writes {coded MBs, coefficients} to hhdr (mapped host memory); k_pack fills the
// device-side side info / EOB / coefficient buffers, copied back by DMA afterwards.
int launch_compact(const uint8_t* opt_skip, const MbOut* mb, const int16_t* coeffs, const uint8_t* eobs, int nmb,
                   int intra, int32_t* index, int32_t* offset, uint32_t* dside, int16_t* dpacked, uint8_t* dpeobs,
                   uint32_t* hhdr, void* stream);
// libm device helpers exposed for the exhaustive check
int launch_libm_eval(int which, const float* in, float* out, size_t n, const uint32_t* fix, int nfix, void* stream);
// Learned-proposal form of the P-frame search and mode decision (riv_kernels.cu): lmv holds 8
// bytes per MB; counters[0] += fallbacks to the hexagon search, counters[1] += shortcuts.
// rowcnt (BH words, zero; nullable): the ln-variance mean is folded inside the search launch.
int launch_learned(const SearchParams& sp, const float* net, int margin, float skip_logit, void* lmv,
                   unsigned* counters, unsigned* rowcnt, void* stream);
int launch_libm_range(int which, uint32_t lo, uint32_t n, float* out, const uint32_t* fix, int nfix, void* stream);
int launch_wait_expiry(int which, const unsigned long long* rec, const unsigned* counter, long long limit,
                       unsigned* status, void* stream);

// ---- the worker-task queue of the fused search launch (used by the kernel and by the
// riv_test_worker_queue hook).  Step k holds, in this order: the previous frame's residual of
// MB row k (pairs of MBs), its deblock of band k - DB_LAG (tiles), the SAD-table MBs of row
// k - lag; after the last step, one scan task and one pack task per MB row (compaction).
constexpr int DB_TW = 128;  // deblock tile width (luma columns; chroma DB_TW / 2)
constexpr int DB_LAG = 3, TAB_LAG = 6;
__host__ __device__ inline int deblock_tiles_per_band(int W) {
    return (W + DB_TW - 1) / DB_TW + 2 * ((W / 2 + DB_TW / 2 - 1) / (DB_TW / 2));
}
struct QueueShape {
    int BH, nr, nd, nt, lag, steps, csteps;  // rows; residual / deblock / table tasks per row; ...
};
__host__ __device__ inline QueueShape queue_shape(int BW, int BH, int W, bool defer, bool deblock, bool tables,
                                                 bool compact) {
    QueueShape q;
    q.BH = BH;
    q.nr = defer ? (BW + 1) / 2 : 0;
    q.nd = defer && deblock ? deblock_tiles_per_band(W) : 0;
    q.nt = tables ? BW : 0;
    q.lag = defer ? TAB_LAG : 0;
    q.steps = BH + (defer ? TAB_LAG : 0);
    q.csteps = defer && compact ? 2 : 0;
    return q;
}
// every kind of task covers each MB row once
__host__ __device__ inline int queue_total(const QueueShape& q) {
    return q.BH * (q.nr + q.nd + q.nt) + (q.csteps ? 1 + q.BH : 0);
}
// task counts of step k (k < steps + csteps): R residual pairs, D deblock tiles, T table MBs
// (in the compaction steps: the scan, then the pack rows)
__host__ __device__ inline void queue_step(const QueueShape& q, int k, int& R, int& D, int& T) {
    if (k < q.steps) {
        R = k < q.BH ? q.nr : 0;
        D = k >= DB_LAG && k - DB_LAG < q.BH ? q.nd : 0;
        T = k >= q.lag && k - q.lag < q.BH ? q.nt : 0;
    } else {
        R = D = 0;
        T = k == q.steps ? 1 : q.BH;
    }
}
// task t of step k: kind 0 residual pair idx of row, 1 deblock tile idx of band row, 2 table MB
// idx of row, 3 scan, 4 pack of row
__host__ __device__ inline void queue_task(const QueueShape& q, int k, int t, int R, int D, int& kind, int& row,
                                           int& idx) {
    if (k >= q.steps) {
        kind = k == q.steps ? 3 : 4;
        row = t;
        idx = 0;
        return;
    }
    kind = t < R ? 0 : t < R + D ? 1 : 2;
    row = kind == 0 ? k : kind == 1 ? k - DB_LAG : k - q.lag;
    idx = kind == 0 ? t : kind == 1 ? t - R : t - R - D;
}

}  // namespace riv
