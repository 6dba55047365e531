// riv_entropy.h -- host-side entropy coders of the riv2 bitstream (byte-exact with the
// reference): adaptive binary rANS (com/rans.rs), the DCT-coefficient coder
// (res/rans.rs) and the motion-vector coder (res/mv_rans/encoder.rs).  They consume the
// per-MB side info and compacted coefficients produced by the GPU.
#pragma once
#include <cstdint>
#include <deque>
#include <functional>
#include <future>
#include <memory>
#include <tuple>
#include <unordered_map>
#include <vector>

namespace riv {

void entropy_init();

struct BinProb {
    uint16_t packed = 0x0101;
};

// Runs a job on another thread and returns its completion.
using BatchSubmit = std::function<std::future<void>(std::function<void()>)>;

// Binary rANS writer with the reference's buffering (BATCH = 16386 symbols per drain,
// two interleaved states, 8-bit scale, RANS_L = 2^16, u16 emission).  Every drain starts
// from fresh states, so a full batch's (probability, bit) stack is coded independently of
// the rest: with `submit` the writer hands each full batch to it and keeps modelling, and
// finish() codes the last batch itself, then appends the batches' words in order.
class RansWriter {
public:
    explicit RansWriter(std::vector<uint8_t>* sink, const BatchSubmit* submit = nullptr);
    ~RansWriter();  // waits for batches still being coded (finish() not reached)
    RansWriter(const RansWriter&) = delete;
    RansWriter& operator=(const RansWriter&) = delete;
    inline void put(bool bit, BinProb& ctx);
    inline void put_bypass(bool bit);
    void finish();
    // finish in two halves (with submit only): the last batch goes to submit as well, and
    // collect() later waits for every batch and appends the words in order
    void finish_async();
    void collect();
    bool ready();  // every handed-off batch coded (collect() would not wait)

    // The stack in a caller's registers, for symbol loops: start from stack() and depth(),
    // push downwards (stack()[--depth] = entry), call refill() at depth 0 (it hands the full
    // stack off and returns the fresh one, depth BATCH_SYMS again) and commit(depth) before any
    // other call on the writer.
    static constexpr int BATCH_SYMS = 16386;  // com/rans.rs:201
    uint16_t* stack() { return stack_.data(); }
    int depth() const { return sp_; }
    __attribute__((noinline)) uint16_t* refill();
    void commit(int depth) { sp_ = depth; }

private:
    // out of line and cold: inlined into put it costs the symbol loop its registers
    __attribute__((noinline, cold)) void drain();
    std::vector<uint8_t>* sink_;
    std::vector<uint16_t> stack_;  // entry = p | bit << 8; stack_[BATCH-1] is the oldest
    int sp_;
    const BatchSubmit* submit_;
    struct Batch {
        std::vector<uint16_t> stack;
        int sp = 0;
        std::vector<uint8_t> bytes;
        std::future<void> done;
    };
    std::deque<Batch> batches_;  // handed off, in stream order
};

// Binary rANS reader (com/rans.rs:299-354): the inverse of RansWriter.  Reads past the end
// of the data set `error` and yield zeros.
class RansReader {
public:
    RansReader(const uint8_t* data, size_t len);
    bool get(BinProb& ctx);
    bool get_bypass();
    bool error = false;

private:
    uint16_t word();
    void next_symbol();
    void advance(uint32_t& r, uint32_t start, uint32_t freq);
    const uint8_t* d_;
    size_t len_, pos_ = 0;
    uint32_t r0_ = 0, r1_ = 0;
    int count_ = 0;
};

// Inverse of encode_residual_frame for a dense layout: coeffs holds 384 int16 per MB (Y, U,
// V), zero-filled; MBs with coded[mb] == 0 are not in the stream (res/rans.rs:392-459).
// Returns false on malformed data.
bool decode_residual_frame(const uint8_t* data, size_t len, const uint8_t* coded, int nmb, bool intra,
                           int16_t* coeffs);

// Coded MBs in the GPU's compact layout: per MB, the Y, U and V blocks each truncated
// after its last non-zero coefficient (eobs = those three indices per MB).
// `submit` (optional) codes the full rANS batches on other threads; with parts > 1 as well,
// frames of 16K to 2M coded coefficients are coded by `parts` threads at once (this one and
// parts - 1 jobs given to submit, which must not run them on this thread), same bytes.
// Throws std::runtime_error where the reference encoder panics (a magnitude class above 13).
void encode_residual_frame(const int16_t* packed, const uint8_t* eobs, int nblocks, bool intra,
                           std::vector<uint8_t>& out, const BatchSubmit* submit = nullptr, int parts = 0);
// The one-thread form of encode_residual_frame with every rANS batch, the last one included,
// handed to submit: the returned writer's collect() appends the bytes to out (nullptr: no coded
// block, out empty).  The modelling thread does not wait for the batches.
std::unique_ptr<class RansWriter> encode_residual_frame_async(const int16_t* packed, const uint8_t* eobs, int nblocks,
                                                             bool intra, std::vector<uint8_t>& out,
                                                             const BatchSubmit& submit);

enum MvMode { M_ZERO = 0, M_NEAREST = 1, M_NEAR = 2, M_TOPRIGHT = 3, M_TOPLEFT = 4, M_NEW = 5, M_TEMPORAL = 6 };
enum Subpel { SP_ZERO = 0, SP_PLUS = 1, SP_MINUS = 2 };

struct MvCodedBlock {  // res/mv_rans.rs:65-78
    uint8_t mode, new_base;
    int8_t dx, dy;
    uint8_t spx, spy;
    bool skip;
};

// A frame's MV symbols in stream order (model index | bit << 15), as MvCoder::prepare lists them.
struct MvSymbols {
    std::unique_ptr<uint16_t[]> s;
    size_t n = 0, cap = 0;
};

class MvCoder {  // res/mv_rans/encoder.rs:60-412
public:
    void reset();
    // The coder in two stages that touch disjoint state, so that two threads can run them on
    // consecutive frames: prepare lists a frame's (model, bit) symbols, which depend on the
    // candidate history but on no adaptive model, then advances the history (encoder.rs:370-412);
    // code runs the adaptive models over a listed frame and codes it.  prepare and code each in
    // frame order give encode_frame's bytes.  prepare throws where encode_frame does.
    void prepare(const std::vector<MvCodedBlock>& blocks, int bw, MvSymbols& syms);
    void code(const MvSymbols& syms, std::vector<uint8_t>& out, const BatchSubmit* submit = nullptr);
    // code's modelling only, into w (its batches coded wherever w sends them; the caller
    // finishes w)
    void model(const MvSymbols& syms, RansWriter& w);
    void reset_history();  // prepare's state, as reset() leaves it
    void reset_models();   // code's state, as reset() leaves it
    // Throws std::runtime_error on a NEW block with a raw -1/2 subpel (the reference panics).
    // submit (nullable): full rANS batches are coded there while the context modelling goes on
    // (same bytes; see RansWriter).
    void encode_frame(const std::vector<MvCodedBlock>& blocks, int bw, std::vector<uint8_t>& out,
                      const BatchSubmit* submit = nullptr);
    // res/mv_rans/decoder.rs:149-283; the same context and candidate-history state as the
    // encoder, so a decoder instance follows the encoder's across frames.  false on bad data.
    bool decode_frame(const uint8_t* data, size_t len, int bw, int bh, std::vector<MvCodedBlock>& out);

    // The same bytes as encode_frame, with the context modelling split `parts` ways (this
    // thread and submit): each part lists the (model, bit) symbols of a range of MBs, each
    // model then runs over its own symbols from its state of the previous frame, and the rANS
    // batches are coded in parallel.
    void encode_frame_parallel(const std::vector<MvCodedBlock>& blocks, int bw, std::vector<uint8_t>& out,
                               const BatchSubmit& submit, int parts);

private:
    void update(const std::vector<MvCodedBlock>& blocks);
    template <class W>
    void emit(W& w, const std::vector<MvCodedBlock>& blocks, const std::vector<uint8_t>& hits, int bw, size_t b0,
              size_t b1);
    std::vector<uint8_t> hit_flags(const std::vector<MvCodedBlock>& blocks) const;
    // every adaptive model of the coder, contiguous (a model's index is its position here)
    struct Models {
        BinProb skip, m_new[4], m_nz[4], m_near[4], m_tmp[4], m_tr[4], m_tl[4], b_nearest[4], b_near[4], b_tr[4],
            b_tl[4], cls_x[4], cls_y[4], sign_x, sign_y, mag_x[10], mag_y[10], sub_x, sub_y, hit[3], cidx[4];
    } c_;
    std::vector<uint32_t> cands_;  // packed keys
    // candidate-history counts: one counter per (dx, dy, subpel x, subpel y) (allocated on first
    // use), and the keys whose counter is listed (non-zero, or decayed to zero this frame)
    std::vector<uint32_t> cnt_;
    std::vector<uint8_t> listed_;
    std::vector<uint32_t> active_;
    uint32_t total_ = 0;
};

// compute_delta_bias_for_new (enc/encoder.rs:984-1048) from per-axis histograms.
void compute_delta_bias(const std::vector<std::pair<int8_t, int8_t>>& deltas, int8_t& bx, int8_t& by);

}  // namespace riv
