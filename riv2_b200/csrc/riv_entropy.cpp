// riv_entropy.cpp -- host entropy coders (see riv_entropy.h).
#include "riv_entropy.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <exception>
#include <stdexcept>
#include <cstdlib>
#include <cstring>
#include <mutex>

namespace riv {

// ceil(2^32 / d) for d = 1 .. 510 (0 for d = 0): (zeros << 8) / (zeros + ones) of every
// BinProb state by one multiply (exact for dividends below 2^16, checked for all 65536 states
// by entropy_init)
static uint32_t g_div_m[512];
// ceil(2^64 / f) for f = 2 .. 255: floor(r / f) is the high half of r * g_rcp64[f] for every
// r < 2^32 (the rounding error r * (ceil - exact) stays below 2^64 / f); f = 1: 2^64 - 1, whose
// product's high half is r - 1 for r > 0
static uint64_t g_rcp64[256];
static std::once_flag g_once;

// BinProb update after one bit (com/rans.rs:73-84).  Computed, not tabulated: a state moves
// by 256 entries per update, so a 65536-entry table misses the L1 cache on nearly every symbol.
static inline uint16_t observe_calc(uint16_t packed, bool bit) {
    uint16_t rot = bit ? (uint16_t)((packed << 8) | (packed >> 8)) : packed;
    uint32_t sum = (uint32_t)rot + 0x100u;
    uint16_t upd = (uint16_t)sum;
    if (sum > 0xFFFFu) {
        uint16_t mask = rot == 0xff01 ? 0xff00 : 0x8100;
        upd = (uint16_t)((uint16_t)(rot + 0x101) >> 1) | mask;
    }
    return bit ? (uint16_t)((upd << 8) | (upd >> 8)) : upd;
}

static inline uint8_t prob_zero(const BinProb& b) {
    const uint32_t z = (uint32_t)b.packed >> 8, d = z + (b.packed & 0xffu);
    const uint8_t p = (uint8_t)(((uint64_t)(z << 8) * g_div_m[d]) >> 32);
    return p ? p : 1;
}
static inline void observe(BinProb& b, bool bit) { b.packed = observe_calc(b.packed, bit); }

void entropy_init() {
    std::call_once(g_once, [] {
        // BinProb zero probability (com/rans.rs:30-44): p = zeros*256/(zeros+ones) truncated
        // to u8, with 0 mapped to 1; the division by the reciprocal multiply of prob_zero
        for (uint32_t d = 1; d < 512; d++) g_div_m[d] = (uint32_t)((((uint64_t)1 << 32) + d - 1) / d);
        for (int i = 0; i < 65536; i++) {
            const int zeros = i >> 8, ones = i & 0xff;
            const uint8_t want = i == 0 ? 1 : ((uint8_t)((zeros << 8) / (zeros + ones)) ? (uint8_t)((zeros << 8) / (zeros + ones)) : 1);
            BinProb b;
            b.packed = (uint16_t)i;
            if (prob_zero(b) != want) std::abort();  // cannot happen: the reciprocals are exact here
        }
        g_rcp64[1] = ~0ull;
        for (uint32_t f = 2; f < 256; f++) {
            g_rcp64[f] = (uint64_t)((((unsigned __int128)1 << 64) + f - 1) / f);
            // spot checks at the quotient steps and the top of the range
            const uint32_t rs[6] = {0u, f - 1, f, 0xFFFFFFFFu, 0xFFFFFFFFu - 0xFFFFFFFFu % f, 0xFFFFFFFFu - 0xFFFFFFFFu % f - 1};
            for (uint32_t r : rs)
                if ((uint32_t)(((unsigned __int128)r * g_rcp64[f]) >> 64) != r / f) std::abort();
        }
    });
}


static const int BATCH = 16386;  // com/rans.rs:201
static_assert(BATCH == RansWriter::BATCH_SYMS, "the writer's stack depth is the reference's batch");
// The parallel coefficient coder takes frames of 16K to 2M coded coefficients: below, its
// fork and join cost more than they save; above, its symbol lists (up to about 26 symbols per
// coefficient) would take hundreds of MB.
static const uint32_t PARALLEL_MIN_COEFFS = 16384, PARALLEL_MAX_COEFFS = 2u << 20;
static const size_t WORK_KEEP_BYTES = 64u << 20;  // parallel coder buffers kept per thread

RansWriter::RansWriter(std::vector<uint8_t>* sink, const BatchSubmit* submit)
    : sink_(sink), stack_(BATCH), sp_(BATCH), submit_(submit) {}

inline void RansWriter::put(bool bit, BinProb& ctx) {
    uint8_t p = prob_zero(ctx);
    observe(ctx, bit);
    if (__builtin_expect(sp_ == 0, 0)) drain();
    stack_[--sp_] = (uint16_t)(p | (bit ? 0x100 : 0));
}
inline void RansWriter::put_bypass(bool bit) {
    if (__builtin_expect(sp_ == 0, 0)) drain();
    stack_[--sp_] = (uint16_t)(128 | (bit ? 0x100 : 0));
}


static inline void enc_sym(uint32_t& r, uint16_t* words, int& wp, uint16_t e) {
    uint32_t p = e & 0xff;
    p += p == 0 ? 1u : 0u;
    // bit 1: start p, frequency 256 - p; bit 0: start 0, frequency p (masks, not a branch: the
    // bits are the data)
    const uint32_t m = 0u - ((uint32_t)(e >> 8) & 1u);
    const uint32_t start = p & m, freq = (p ^ m) + (m & 257u);
    // renormalisation without a branch: the low word is stored at the next free slot either way
    // (the buffer has room for one word per symbol) and kept only when r is at or above xmax
    const uint32_t xmax = freq << 24, out = r >= xmax ? 1u : 0u;
    words[wp - 1] = (uint16_t)r;
    wp -= (int)out;
    r >>= 16 * out;
    // frequency 1: the multiplier 2^64 - 1 gives r - 1 (r > 0 here), and the comparison adds the 1
    const uint32_t q = (uint32_t)(((unsigned __int128)r * g_rcp64[freq]) >> 64) + (freq == 1 ? 1u : 0u);
    r = (q << 8) | (r - q * freq + start);
}

// RansEncoder::drain (com/rans.rs:231-269): walk the stack from the newest symbol
// back to the oldest with two interleaved states; words are pushed to the front, so
// they are written here from the end of the word buffer backwards, then appended to
// `out` as little-endian bytes.
static void code_batch(const uint16_t* stack, int sp, std::vector<uint8_t>& out) {
    thread_local std::vector<uint16_t> words(BATCH + 8);
    uint32_t r0 = 65536, r1 = 65536;
    uint16_t* w = words.data();
    int wp = (int)words.size();
    int i = sp;
    if (i & 1) {
        enc_sym(r0, w, wp, stack[i]);
        i++;
        std::swap(r0, r1);
    }
    for (; i < BATCH; i += 2) {
        enc_sym(r0, w, wp, stack[i]);
        enc_sym(r1, w, wp, stack[i + 1]);
    }
    w[--wp] = (uint16_t)(r0 >> 16);
    w[--wp] = (uint16_t)(r0 & 0xffff);
    w[--wp] = (uint16_t)(r1 >> 16);
    w[--wp] = (uint16_t)(r1 & 0xffff);
    size_t n = words.size() - wp, base = out.size();
    out.resize(base + 2 * n);
    uint8_t* o = out.data() + base;
    for (size_t k = 0; k < n; k++) {
        uint16_t v = w[wp + k];
        o[2 * k] = (uint8_t)v;
        o[2 * k + 1] = (uint8_t)(v >> 8);
    }
}

void RansWriter::drain() {
    if (submit_ == nullptr) {
        code_batch(stack_.data(), sp_, *sink_);
    } else {  // hand the full stack off and continue on a fresh one
        batches_.emplace_back();
        Batch& b = batches_.back();
        b.stack.swap(stack_);
        stack_.resize(BATCH);
        b.sp = sp_;
        b.done = (*submit_)([&b] { code_batch(b.stack.data(), b.sp, b.bytes); });
    }
    sp_ = BATCH;
}

RansWriter::~RansWriter() {
    for (Batch& b : batches_)
        if (b.done.valid()) b.done.wait();
}

void RansWriter::finish_async() {
    if (submit_ == nullptr) {
        finish();
        return;
    }
    drain();  // the partial batch as one more job
}

uint16_t* RansWriter::refill() {
    sp_ = 0;
    drain();
    return stack_.data();
}

bool RansWriter::ready() {
    for (Batch& b : batches_)
        if (b.done.wait_for(std::chrono::seconds(0)) != std::future_status::ready) return false;
    return true;
}

void RansWriter::collect() {
    for (Batch& b : batches_) {
        b.done.get();
        sink_->insert(sink_->end(), b.bytes.begin(), b.bytes.end());
    }
    batches_.clear();
}

void RansWriter::finish() {
    std::vector<uint8_t> last;
    code_batch(stack_.data(), sp_, last);  // the partial batch, here while the others finish
    sp_ = BATCH;
    for (Batch& b : batches_) {
        b.done.get();
        sink_->insert(sink_->end(), b.bytes.begin(), b.bytes.end());
    }
    batches_.clear();
    sink_->insert(sink_->end(), last.begin(), last.end());
}

// RansDecoder (com/rans.rs:299-354): two interleaved states, each symbol first takes the
// older state; a drain boundary every BATCH symbols reloads both states.
RansReader::RansReader(const uint8_t* data, size_t len) : d_(data), len_(len) {
    entropy_init();
    r0_ = word();
    r0_ |= (uint32_t)word() << 16;
    r1_ = word();
    r1_ |= (uint32_t)word() << 16;
}
uint16_t RansReader::word() {
    if (pos_ + 2 > len_) {
        error = true;
        pos_ = len_;
        return 0;
    }
    uint16_t v = (uint16_t)(d_[pos_] | (d_[pos_ + 1] << 8));
    pos_ += 2;
    return v;
}
void RansReader::next_symbol() {
    if (count_ == BATCH) {
        count_ = 0;
        r0_ = word();
        r0_ |= (uint32_t)word() << 16;
        r1_ = word();
        r1_ |= (uint32_t)word() << 16;
    }
    count_++;
}
void RansReader::advance(uint32_t& r, uint32_t start, uint32_t freq) {
    r = freq * (r >> 8) + (r & 255) - start;
    if (r < 65536) r = (r << 16) | word();
}
bool RansReader::get(BinProb& ctx) {
    next_symbol();
    uint32_t r = r0_;
    r0_ = r1_;
    const uint32_t p = prob_zero(ctx);
    const bool bit = (r & 255) >= p;
    observe(ctx, bit);
    advance(r, bit ? p : 0, bit ? 256u - p : p);
    r1_ = r;
    return bit;
}
bool RansReader::get_bypass() {
    next_symbol();
    uint32_t r = r0_;
    r0_ = r1_;
    const uint32_t start = r & 0x80;
    advance(r, start, 128);
    r1_ = r;
    return start != 0;
}

// ---------------------------------------------------------------------------------
// DCT coefficient coder (res/rans.rs:34-330)
// ---------------------------------------------------------------------------------
static inline int bit_len(unsigned v) { return v <= 1 ? (int)v : 32 - __builtin_clz(v); }
static inline int luma_band(int p) { return p == 0 ? 0 : (p < 16 ? 1 : (p < 64 ? 2 : 3)); }
static inline int chroma_band(int p) { return p == 0 ? 0 : (p < 8 ? 1 : 2); }

// The coder's adaptive models as one flat array of ids: sig_y[256], sig_c[64], mag_y[4][13],
// mag_c[3][13], eob_y[9], eob_c[7] (res/rans.rs:195-248).  CX_BYPASS marks a bypass symbol.
constexpr int CX_SIG_Y = 0, CX_SIG_C = 256, CX_MAG_Y = 320, CX_MAG_C = 372, CX_EOB_Y = 411, CX_EOB_C = 420,
              CX_COUNT = 427, CX_BYPASS = 511;

// The binary symbols of the coefficient stream, in coding order, for any sink W with
// put(bit, model id), bypass(bit) and a flag `bad`: the class/value code
// (reitero_residual/src/rans.rs:72-98, 133-159).  Class nctx is coded with nctx continue
// bits and no stop bit, as the reference does; above it the reference indexes past its
// models and panics, so the sink is marked bad and the frame fails.
template <class W>
__attribute__((always_inline)) static inline void class_value_syms(W& w, unsigned value, int cx0, int nctx) {
    int maxc = nctx - 1, cls = bit_len(value);
    if (cls > nctx) {
        w.bad = true;
        return;
    }
    for (int c = 0; c < cls; c++) w.put(true, cx0 + c);
    if (cls < maxc) w.put(false, cx0 + cls);
    if (cls >= 2) {
        unsigned off = value - (1u << (cls - 1));
        for (int b = cls - 2; b >= 0; b--) w.bypass((off >> b) & 1);
    }
}
// ... one plane block: EOB class, then per coefficient up to it the significance flag, sign
// and magnitude class (res/rans.rs:250-278); intra DC values are coded against the previous
// block's (prev_dc, per plane) ...
template <class W>
__attribute__((always_inline)) static inline void plane_syms(W& w, int16_t* prev_dc, const int16_t* pl, int last,
                                                             bool luma, int pi, bool dcp) {
    int16_t dcv = pl[0];
    if (dcp) {
        dcv = (int16_t)(pl[0] - prev_dc[pi]);
        prev_dc[pi] = pl[0];
    }
    class_value_syms(w, (unsigned)last, luma ? CX_EOB_Y : CX_EOB_C, luma ? 9 : 7);
    const int sig0 = luma ? CX_SIG_Y : CX_SIG_C;
    for (int i = 0; i <= last; i++) {
        int16_t v = i == 0 ? dcv : pl[i];
        w.put(v != 0, sig0 + i);
        if (v != 0) {
            w.bypass(v < 0);
            unsigned a = (unsigned)std::abs((int)v) - 1;
            class_value_syms(w, a, luma ? CX_MAG_Y + 13 * luma_band(i) : CX_MAG_C + 13 * chroma_band(i), 13);
        }
    }
}
// ... and blocks [b0, b1) of the compact layout starting at p (Y, U, V per MB).
template <class W>
__attribute__((always_inline)) static inline void blocks_syms(W& w, int16_t* prev_dc, const int16_t* p,
                                                              const uint8_t* eobs, int b0, int b1, bool intra) {
    for (int b = b0; b < b1; b++) {
        const uint8_t* e = eobs + 3 * b;
        plane_syms(w, prev_dc, p, e[0], true, 0, intra);
        p += e[0] + 1;
        plane_syms(w, prev_dc, p, e[1], false, 1, intra);
        p += e[1] + 1;
        plane_syms(w, prev_dc, p, e[2], false, 2, intra);
        p += e[2] + 1;
    }
}

struct DctContexts {
    BinProb sig_y[256], sig_c[64], mag_y[4][13], mag_c[3][13], eob_y[9], eob_c[7];
    int16_t prev_dc[3] = {0, 0, 0};
};

// Sequential sink: models the symbols into a RansWriter, with the writer's stack pointer and
// depth in locals (registers) between its drains, not loaded and stored per symbol; finish()
// hands the depth back to the writer.
struct ModelSink {
    RansWriter& w;
    BinProb* cx;
    bool bad = false;
    uint16_t* st;
    int sp;
    ModelSink(RansWriter& w_, BinProb* cx_) : w(w_), cx(cx_), st(w_.stack()), sp(w_.depth()) {}
    inline void push(uint16_t e) {
        if (__builtin_expect(sp == 0, 0)) {
            st = w.refill();
            sp = BATCH;
        }
        st[--sp] = e;
    }
    void put(bool bit, int id) {
        BinProb& m = cx[id];
        const uint8_t p = prob_zero(m);
        observe(m, bit);
        push((uint16_t)(p | (bit ? 0x100 : 0)));
    }
    void bypass(bool bit) { push((uint16_t)(128 | (bit ? 0x100 : 0))); }
    void finish() { w.commit(sp); }
};
// Enumerating sink: model id | bit << 15 per symbol, and how often each model is used.
struct SymList {
    std::vector<uint16_t> s;
    uint32_t cnt[CX_COUNT] = {};
    bool bad = false;
    void put(bool bit, int id) {
        s.push_back((uint16_t)(id | (bit ? 0x8000 : 0)));
        cnt[id]++;
    }
    void bypass(bool bit) { s.push_back((uint16_t)(CX_BYPASS | (bit ? 0x8000 : 0))); }
};

struct ParallelWork {
    std::vector<SymList> lists;
    std::vector<uint16_t> stacks;
    std::vector<uint32_t> occ;
    std::vector<std::vector<uint8_t>> bytes;
};

static const char* const MAG_CLASS_ERROR = "coefficient magnitude class above 13 (the reference encoder panics)";

// Runs f(0) here and f(1 .. parts-1) through submit; returns when all have ended.
static void run_parts(const BatchSubmit& submit, int parts, const std::function<void(int)>& f) {
    std::vector<std::future<void>> fs;
    std::exception_ptr err;
    try {
        for (int t = 1; t < parts; t++) fs.push_back(submit([&f, t] { f(t); }));
        f(0);
    } catch (...) {
        err = std::current_exception();
    }
    for (auto& x : fs) {
        try {
            x.get();
        } catch (...) {
            if (!err) err = std::current_exception();
        }
    }
    if (err) std::rethrow_exception(err);
}

// Stack slot of the symbol at stream position k: batch k / BATCH, whose stack holds its
// oldest symbol at the top (RansWriter::put pushes downwards).
static inline size_t stack_slot(size_t k) { return (k / BATCH) * BATCH + (BATCH - 1 - k % BATCH); }

// The same stream as the sequential coder, with the work split `parts` ways.  A model's
// probability at each of its symbols depends only on the bits it saw before, so: (1) each
// part lists the symbols (model id, bit) of a range of blocks; (2) the symbols are grouped
// by model (counting sort, positions in stream order); (3) each part runs a set of models
// over their own symbols and writes each symbol's (probability, bit) into its rANS batch
// stack; (4) the batches, which start from fresh states, are coded in parallel and
// appended in order.
static void encode_residual_parallel(const int16_t* packed, const uint8_t* eobs, int nblocks, bool intra,
                                     const std::vector<uint32_t>& off, std::vector<uint8_t>& out,
                                     const BatchSubmit& submit, int parts) {
    std::vector<int> bstart(parts + 1);
    for (int t = 0; t <= parts; t++)
        bstart[t] = (int)(std::lower_bound(off.begin(), off.end(), (uint32_t)((uint64_t)off[nblocks] * t / parts)) -
                          off.begin());
    bstart[0] = 0;
    bstart[parts] = nblocks;
    // buffers of the calling thread, kept from frame to frame (no page faults, no zeroing)
    thread_local ParallelWork ws;
    std::vector<SymList>& lists = ws.lists;
    lists.resize(parts);
    run_parts(submit, parts, [&](int t) {
        const int b0 = bstart[t], b1 = std::max(bstart[t], bstart[t + 1]);
        SymList& L = lists[t];
        L.s.clear();
        std::fill(L.cnt, L.cnt + CX_COUNT, 0u);
        L.bad = false;
        L.s.reserve((size_t)(off[b1] - off[b0]) * 2 + (size_t)(b1 - b0) * 12);
        int16_t prev_dc[3] = {0, 0, 0};
        if (intra && b0 > 0) {
            const int16_t* q = packed + off[b0 - 1];
            const uint8_t* e = eobs + 3 * (b0 - 1);
            prev_dc[0] = q[0];
            prev_dc[1] = q[e[0] + 1];
            prev_dc[2] = q[e[0] + 1 + e[1] + 1];
        }
        blocks_syms(L, prev_dc, packed + off[b0], eobs, b0, b1, intra);
    });
    std::vector<size_t> sbase(parts + 1, 0);
    for (int t = 0; t < parts; t++) {
        if (lists[t].bad) throw std::runtime_error(MAG_CLASS_ERROR);
        sbase[t + 1] = sbase[t] + lists[t].s.size();
    }
    const size_t N = sbase[parts], nb = (N + BATCH - 1) / BATCH;
    std::vector<uint32_t> cbase(CX_COUNT + 1), cstart((size_t)parts * CX_COUNT);
    uint32_t acc = 0;
    for (int c = 0; c < CX_COUNT; c++) {
        cbase[c] = acc;
        for (int t = 0; t < parts; t++) {
            cstart[(size_t)t * CX_COUNT + c] = acc;
            acc += lists[t].cnt[c];
        }
    }
    cbase[CX_COUNT] = acc;
    std::vector<uint16_t>& stacks = ws.stacks;
    std::vector<uint32_t>& occ = ws.occ;  // per model, in stream order: position | bit << 31
    if (stacks.size() < nb * BATCH) stacks.resize(nb * BATCH);
    if (occ.size() < acc) occ.resize(acc);
    run_parts(submit, parts, [&](int t) {
        uint32_t* cs = cstart.data() + (size_t)t * CX_COUNT;
        size_t k = sbase[t];
        for (uint16_t e : lists[t].s) {
            const int c = e & 0x1ff;
            const uint32_t bit = e >> 15;
            if (c == CX_BYPASS) stacks[stack_slot(k)] = (uint16_t)(128 | bit << 8);
            else occ[cs[c]++] = (uint32_t)k | bit << 31;
            k++;
        }
    });
    // models to parts, largest first onto the least loaded part
    std::vector<int> order(CX_COUNT);
    for (int c = 0; c < CX_COUNT; c++) order[c] = c;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        const uint32_t na = cbase[a + 1] - cbase[a], nb_ = cbase[b + 1] - cbase[b];
        return na != nb_ ? na > nb_ : a < b;
    });
    std::vector<std::vector<int>> groups(parts);
    std::vector<uint64_t> load(parts, 0);
    for (int c : order) {
        const uint32_t n = cbase[c + 1] - cbase[c];
        if (n == 0) break;
        const int t = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        groups[t].push_back(c);
        load[t] += n;
    }
    run_parts(submit, parts, [&](int t) {
        for (int c : groups[t]) {
            BinProb st;
            for (uint32_t i = cbase[c]; i < cbase[c + 1]; i++) {
                const uint32_t e = occ[i];
                const bool bit = (e >> 31) != 0;
                stacks[stack_slot(e & 0x7fffffffu)] = (uint16_t)(prob_zero(st) | (bit ? 0x100 : 0));
                observe(st, bit);
            }
        }
    });
    std::vector<std::vector<uint8_t>>& bytes = ws.bytes;
    if (bytes.size() < nb) bytes.resize(nb);
    for (size_t j = 0; j < nb; j++) bytes[j].clear();
    std::atomic<size_t> next{0};
    run_parts(submit, parts, [&](int) {
        for (size_t j; (j = next.fetch_add(1)) < nb;) {
            const size_t len = std::min<size_t>(BATCH, N - j * BATCH);
            code_batch(stacks.data() + j * BATCH, (int)(BATCH - len), bytes[j]);
        }
    });
    out.clear();
    for (size_t j = 0; j < nb; j++) out.insert(out.end(), bytes[j].begin(), bytes[j].end());
    // keep the buffers for the next frame only while they are small (a frame of huge
    // coefficients must not pin hundreds of MB on every thread that ever coded one)
    size_t held = ws.stacks.capacity() * 2 + ws.occ.capacity() * 4;
    for (const SymList& L : ws.lists) held += L.s.capacity() * 2;
    if (held > WORK_KEEP_BYTES) ws = ParallelWork();
}

void encode_residual_frame(const int16_t* packed, const uint8_t* eobs, int nblocks, bool intra,
                           std::vector<uint8_t>& out, const BatchSubmit* submit, int parts) {
    out.clear();
    if (nblocks == 0) return;  // the reference never instantiates the coder
    // With DC prediction the coded range ends at the last non-zero AC coefficient
    // (res/rans.rs:250-262); the GPU's last-non-zero index already equals it.  The compact
    // layout holds each plane block only up to that index.
    if (submit != nullptr && parts > 1) {
        std::vector<uint32_t> off((size_t)nblocks + 1);
        off[0] = 0;
        for (int b = 0; b < nblocks; b++)
            off[b + 1] = off[b] + eobs[3 * b] + eobs[3 * b + 1] + eobs[3 * b + 2] + 3;
        if (off[nblocks] >= PARALLEL_MIN_COEFFS && off[nblocks] <= PARALLEL_MAX_COEFFS) {
            encode_residual_parallel(packed, eobs, nblocks, intra, off, out, *submit, parts);
            return;
        }
    }
    RansWriter w(&out, submit);
    std::vector<BinProb> cx(CX_COUNT);
    int16_t prev_dc[3] = {0, 0, 0};
    ModelSink sink{w, cx.data()};
    blocks_syms(sink, prev_dc, packed, eobs, 0, nblocks, intra);
    sink.finish();
    if (sink.bad) throw std::runtime_error(MAG_CLASS_ERROR);
    w.finish();
}

std::unique_ptr<RansWriter> encode_residual_frame_async(const int16_t* packed, const uint8_t* eobs, int nblocks,
                                                       bool intra, std::vector<uint8_t>& out, const BatchSubmit& submit) {
    out.clear();
    if (nblocks == 0) return nullptr;  // the reference never instantiates the coder
    std::unique_ptr<RansWriter> w(new RansWriter(&out, &submit));
    std::vector<BinProb> cx(CX_COUNT);
    int16_t prev_dc[3] = {0, 0, 0};
    ModelSink sink{*w, cx.data()};
    blocks_syms(sink, prev_dc, packed, eobs, 0, nblocks, intra);
    sink.finish();
    if (sink.bad) throw std::runtime_error(MAG_CLASS_ERROR);
    w->finish_async();
    return w;
}

static inline unsigned get_class_value(RansReader& r, BinProb* ctx, int nctx) {
    int maxc = nctx - 1, cls = 0;
    while (cls < maxc && r.get(ctx[cls])) cls++;
    if (cls <= 1) return (unsigned)cls;
    unsigned off = 0;
    for (int k = 0; k < cls - 1; k++) off = (off << 1) | (unsigned)r.get_bypass();
    return (1u << (cls - 1)) + off;
}

static bool decode_plane(RansReader& r, DctContexts& c, int16_t* blk, int n, bool luma, int pi, bool dcp) {
    const unsigned end = luma ? get_class_value(r, c.eob_y, 9) : get_class_value(r, c.eob_c, 7);
    if ((int)end >= n) return false;
    BinProb* sig = luma ? c.sig_y : c.sig_c;
    for (unsigned i = 0; i <= end; i++) {
        if (!r.get(sig[i])) continue;
        const bool neg = r.get_bypass();
        BinProb* mc = luma ? c.mag_y[luma_band((int)i)] : c.mag_c[chroma_band((int)i)];
        const int16_t a = (int16_t)(get_class_value(r, mc, 13) + 1);
        blk[i] = neg ? (int16_t)-a : a;
    }
    if (dcp) {
        blk[0] = (int16_t)(blk[0] + c.prev_dc[pi]);
        c.prev_dc[pi] = blk[0];
    }
    return true;
}

bool decode_residual_frame(const uint8_t* data, size_t len, const uint8_t* coded, int nmb, bool intra,
                           int16_t* coeffs) {
    memset(coeffs, 0, (size_t)nmb * 384 * sizeof(int16_t));
    if (len == 0) return true;  // no coded MB: the encoder wrote nothing
    RansReader r(data, len);
    DctContexts* c = new DctContexts();
    bool ok = true;
    for (int b = 0; b < nmb && ok; b++) {
        if (!coded[b]) continue;
        int16_t* p = coeffs + (size_t)b * 384;
        ok = decode_plane(r, *c, p, 256, true, 0, intra) && decode_plane(r, *c, p + 256, 64, false, 1, intra) &&
             decode_plane(r, *c, p + 320, 64, false, 2, intra);
    }
    delete c;
    return ok && !r.error;
}

// ---------------------------------------------------------------------------------
// Motion-vector coder (res/mv_rans/encoder.rs)
// ---------------------------------------------------------------------------------
static inline uint32_t cand_key(int8_t dx, int8_t dy, uint8_t sx, uint8_t sy) {
    // Order-preserving packing of (i8, i8, Subpel, Subpel) for the tie-break sort.
    return ((uint32_t)((uint8_t)dx ^ 0x80) << 24) | ((uint32_t)((uint8_t)dy ^ 0x80) << 16) | ((uint32_t)sx << 8) | sy;
}
static inline int mv_class(unsigned mag) {  // res/mv_rans.rs:80-86
    if (mag == 0) return 0;
    return std::min(32 - __builtin_clz(mag), 10);
}

void MvCoder::reset() { *this = MvCoder(); }
void MvCoder::reset_history() {
    cands_.clear();
    cnt_.clear();
    listed_.clear();
    active_.clear();
    total_ = 0;
}
void MvCoder::reset_models() { c_ = Models(); }

template <class W>
static void enc_class(W& w, BinProb* ctx, int cls) {
    int lo = 0, hi = 10, d = 0;
    while (lo < hi) {
        int mid = (lo + hi) / 2;
        bool g = cls > mid;
        w.put(g, ctx[d]);
        if (g) lo = mid + 1; else hi = mid;
        d++;
    }
}
template <class W>
static void enc_comp(W& w, int8_t delta, BinProb* cls, BinProb& sign, BinProb* mag) {
    unsigned m = (unsigned)std::abs((int)delta);
    int c = mv_class(m);
    enc_class(w, cls, c);
    if (c == 0) return;
    w.put(delta < 0, sign);
    unsigned bits = c <= 1 ? 0 : c - 1, off = m - (1u << (c - 1));
    for (unsigned b = 0; b < bits; b++) w.put((off >> b) & 1, mag[b]);
}

// Candidate-history hit of every block (a NEW block whose MV is in the frame's candidate
// list, res/mv_rans/encoder.rs:199-230); the hit context of a block reads its left and top
// neighbours' flags.
std::vector<uint8_t> MvCoder::hit_flags(const std::vector<MvCodedBlock>& blocks) const {
    std::vector<uint8_t> hits(blocks.size(), 0);
    if (cands_.empty()) return hits;
    for (size_t i = 0; i < blocks.size(); i++) {
        const MvCodedBlock& b = blocks[i];
        if (b.mode != M_NEW) continue;
        const uint32_t key = cand_key(b.dx, b.dy, b.spx, b.spy);
        for (uint32_t k : cands_)
            if (k == key) { hits[i] = 1; break; }
    }
    return hits;
}

// The symbols of blocks b0 .. b1-1 (res/mv_rans/encoder.rs:145-255), in stream order, to w
// (w.put(bit, model)); modes and hits of the neighbours come from the whole frame.
template <class W>
void MvCoder::emit(W& w, const std::vector<MvCodedBlock>& blocks, const std::vector<uint8_t>& hits, int bw,
                   size_t b0, size_t b1) {
    for (size_t i = b0; i < b1; i++) {
        const MvCodedBlock& b = blocks[i];
        int bx = (int)(i % bw), by = (int)(i / bw);
        w.put(b.skip, c_.skip);
        // mv_mode_context (res/mv_predictor.rs:275-308)
        int score = 0;
        auto sc = [](int m) { return m == M_ZERO ? 2 : (m == M_NEW ? 0 : 1); };
        if (bx > 0) score += sc(blocks[i - 1].mode);
        if (by > 0) score += sc(blocks[i - bw].mode);
        int ctx = std::min(score, 3);
        bool is_new = b.mode == M_NEW;
        w.put(is_new, c_.m_new[ctx]);
        if (!is_new) {
            bool nz = b.mode != M_ZERO;
            w.put(nz, c_.m_nz[ctx]);
            if (nz) {
                bool nr = b.mode == M_NEAR;
                w.put(nr, c_.m_near[ctx]);
                if (!nr) {
                    bool tm = b.mode == M_TEMPORAL;
                    w.put(tm, c_.m_tmp[ctx]);
                    if (!tm) {
                        bool tr = b.mode == M_TOPRIGHT;
                        w.put(tr, c_.m_tr[ctx]);
                        if (!tr) w.put(b.mode == M_TOPLEFT, c_.m_tl[ctx]);
                    }
                }
            }
        } else {
            bool e0 = b.new_base == 0;
            w.put(e0, c_.b_nearest[ctx]);
            if (!e0) {
                bool e1 = b.new_base == 1;
                w.put(e1, c_.b_near[ctx]);
                if (!e1) {
                    bool e2 = b.new_base == 2;
                    w.put(e2, c_.b_tr[ctx]);
                    if (!e2) w.put(b.new_base == 3, c_.b_tl[ctx]);
                }
            }
            bool via = false;
            if (!cands_.empty()) {
                const bool hit = hits[i] != 0;
                int lh = bx > 0 ? hits[i - 1] : 0, th = by > 0 ? hits[i - bw] : 0;
                w.put(hit, c_.hit[lh + th]);
                if (hit) {
                    const uint32_t key = cand_key(b.dx, b.dy, b.spx, b.spy);
                    int ci = 0;
                    while (cands_[ci] != key) ci++;
                    int lo = 0, hi = 16, d = 0;
                    while (hi - lo > 1) {
                        int mid = (lo + hi) / 2;
                        bool g = ci >= mid;
                        w.put(g, c_.cidx[d]);
                        if (g) lo = mid; else hi = mid;
                        d++;
                    }
                    via = true;
                } else {
                    enc_comp(w, b.dx, c_.cls_x, c_.sign_x, c_.mag_x);
                    enc_comp(w, b.dy, c_.cls_y, c_.sign_y, c_.mag_y);
                }
            } else {
                enc_comp(w, b.dx, c_.cls_x, c_.sign_x, c_.mag_x);
                enc_comp(w, b.dy, c_.cls_y, c_.sign_y, c_.mag_y);
            }
            if (!via) {
                w.put(b.spx != SP_ZERO, c_.sub_x);
                w.put(b.spy != SP_ZERO, c_.sub_y);
            }
        }
    }
}

static void check_subpels(const std::vector<MvCodedBlock>& blocks) {
    // a NEW block with a raw -1/2 subpel: the reference panics ("raw -0.5 subpixel is
    // disallowed", res/mv_rans/encoder.rs:335-336; no candidate holds one, :379-381)
    for (const MvCodedBlock& b : blocks)
        if (b.mode == M_NEW && (b.spx == SP_MINUS || b.spy == SP_MINUS))
            throw std::runtime_error("raw -0.5 subpixel is disallowed");
}

void MvCoder::encode_frame(const std::vector<MvCodedBlock>& blocks, int bw, std::vector<uint8_t>& out,
                           const BatchSubmit* submit) {
    out.clear();
    MvSymbols syms;
    prepare(blocks, bw, syms);
    code(syms, out, submit);
}

namespace {
// Symbols of one block at most: skip, NEW, four base bits, the hit flag, then either four index
// bits or two components of at most 4 class + 1 sign + 9 magnitude bits, and two subpel flags.
constexpr size_t MV_MAX_SYMS_PER_BLOCK = 40;
struct MvRawSink {  // lists symbols into a buffer sized for the frame
    const BinProb* base;
    uint16_t* p;
    void put(bool bit, const BinProb& m) { *p++ = (uint16_t)((&m - base) | (bit ? 0x8000 : 0)); }
};
}  // namespace

void MvCoder::prepare(const std::vector<MvCodedBlock>& blocks, int bw, MvSymbols& syms) {
    check_subpels(blocks);
    const std::vector<uint8_t> hits = hit_flags(blocks);
    const size_t need = blocks.size() * MV_MAX_SYMS_PER_BLOCK;
    if (syms.cap < need) {
        syms.s.reset(new uint16_t[need]);
        syms.cap = need;
    }
    MvRawSink k{&c_.skip, syms.s.get()};
    emit(k, blocks, hits, bw, 0, blocks.size());
    syms.n = (size_t)(k.p - syms.s.get());
    update(blocks);
}

void MvCoder::model(const MvSymbols& syms, RansWriter& w) {
    ModelSink sink{w, &c_.skip};
    const uint16_t* s = syms.s.get();
    for (size_t i = 0; i < syms.n; i++) sink.put((s[i] >> 15) != 0, s[i] & 0x7fff);
    sink.finish();
}

void MvCoder::code(const MvSymbols& syms, std::vector<uint8_t>& out, const BatchSubmit* submit) {
    out.clear();
    RansWriter w(&out, submit);
    model(syms, w);
    w.finish();
}

namespace {
constexpr int MV_NMODELS = 80;  // the models of MvCoder::Models
// Lists the (model, bit) symbols of a block range without touching the models.
struct MvSymList {
    const BinProb* base;
    std::vector<uint16_t> s;  // model | bit << 15
    uint32_t cnt[MV_NMODELS];
    void put(bool bit, const BinProb& m) {
        const int id = (int)(&m - base);
        s.push_back((uint16_t)(id | (bit ? 0x8000 : 0)));
        cnt[id]++;
    }
};
}  // namespace

void MvCoder::encode_frame_parallel(const std::vector<MvCodedBlock>& blocks, int bw, std::vector<uint8_t>& out,
                                    const BatchSubmit& submit, int parts) {
    static_assert(sizeof(Models) == MV_NMODELS * sizeof(BinProb), "the models must be contiguous");
    out.clear();
    check_subpels(blocks);
    const std::vector<uint8_t> hits = hit_flags(blocks);
    const size_t nb_ = blocks.size();
    parts = std::max(1, std::min(parts, (int)std::max<size_t>(1, nb_ / 256)));
    const BinProb* base = &c_.skip;
    std::vector<MvSymList> lists(parts);
    run_parts(submit, parts, [&](int t) {
        MvSymList& L = lists[t];
        L.base = base;
        std::fill(L.cnt, L.cnt + MV_NMODELS, 0u);
        const size_t b0 = nb_ * t / parts, b1 = nb_ * (t + 1) / parts;
        L.s.reserve((b1 - b0) * 8);
        emit(L, blocks, hits, bw, b0, b1);
    });
    std::vector<size_t> sbase(parts + 1, 0);
    for (int t = 0; t < parts; t++) sbase[t + 1] = sbase[t] + lists[t].s.size();
    const size_t N = sbase[parts], nbatch = (N + BATCH - 1) / BATCH;
    if (N == 0) {
        update(blocks);
        return;
    }
    std::vector<uint32_t> cbase(MV_NMODELS + 1), cstart((size_t)parts * MV_NMODELS);
    uint32_t acc = 0;
    for (int c = 0; c < MV_NMODELS; c++) {
        cbase[c] = acc;
        for (int t = 0; t < parts; t++) {
            cstart[(size_t)t * MV_NMODELS + c] = acc;
            acc += lists[t].cnt[c];
        }
    }
    cbase[MV_NMODELS] = acc;
    std::vector<uint16_t> stacks(nbatch * BATCH);
    std::vector<uint32_t> occ(acc);  // per model, in stream order: position | bit << 31
    run_parts(submit, parts, [&](int t) {
        uint32_t* cs = cstart.data() + (size_t)t * MV_NMODELS;
        size_t k = sbase[t];
        for (uint16_t e : lists[t].s) occ[cs[e & 0x7fff]++] = (uint32_t)k++ | (uint32_t)(e >> 15) << 31;
    });
    // each model over its own symbols, from its state left by the previous frame
    BinProb* models = &c_.skip;
    std::vector<int> order;
    for (int c = 0; c < MV_NMODELS; c++)
        if (cbase[c + 1] > cbase[c]) order.push_back(c);
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        const uint32_t na = cbase[a + 1] - cbase[a], nb2 = cbase[b + 1] - cbase[b];
        return na != nb2 ? na > nb2 : a < b;
    });
    std::vector<std::vector<int>> groups(parts);
    std::vector<uint64_t> load(parts, 0);
    for (int c : order) {
        const int t = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        groups[t].push_back(c);
        load[t] += cbase[c + 1] - cbase[c];
    }
    run_parts(submit, parts, [&](int t) {
        for (int c : groups[t]) {
            BinProb st = models[c];
            for (uint32_t i = cbase[c]; i < cbase[c + 1]; i++) {
                const uint32_t e = occ[i];
                const bool bit = (e >> 31) != 0;
                stacks[stack_slot(e & 0x7fffffffu)] = (uint16_t)(prob_zero(st) | (bit ? 0x100 : 0));
                observe(st, bit);
            }
            models[c] = st;
        }
    });
    std::vector<std::vector<uint8_t>> bytes(nbatch);
    std::atomic<size_t> next{0};
    run_parts(submit, parts, [&](int) {
        for (size_t j; (j = next.fetch_add(1)) < nbatch;) {
            const size_t len = std::min<size_t>(BATCH, N - j * BATCH);
            code_batch(stacks.data() + j * BATCH, (int)(BATCH - len), bytes[j]);
        }
    });
    for (size_t j = 0; j < nbatch; j++) out.insert(out.end(), bytes[j].begin(), bytes[j].end());
    update(blocks);
}

static int dec_class(RansReader& r, BinProb* ctx) {
    int lo = 0, hi = 10, d = 0;
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (r.get(ctx[d])) lo = mid + 1;
        else hi = mid;
        d++;
    }
    return lo;
}
static int8_t dec_comp(RansReader& r, BinProb* cls, BinProb& sign, BinProb* mag) {
    const int c = dec_class(r, cls);
    if (c == 0) return 0;
    const bool neg = r.get(sign);
    const unsigned bits = c <= 1 ? 0 : c - 1;
    unsigned off = 0;
    for (unsigned b = 0; b < bits; b++)
        if (r.get(mag[b])) off |= 1u << b;
    const int v = (int)((1u << (c - 1)) + off);
    return (int8_t)std::min(std::max(neg ? -v : v, -128), 127);
}

bool MvCoder::decode_frame(const uint8_t* data, size_t len, int bw, int bh, std::vector<MvCodedBlock>& out) {
    RansReader r(data, len);
    const int n = bw * bh;
    out.assign(n, MvCodedBlock{});
    std::vector<uint8_t> modes(n), hits(n);
    for (int i = 0; i < n; i++) {
        const int bx = i % bw, by = i / bw;
        MvCodedBlock& b = out[i];
        b.skip = r.get(c_.skip);
        int score = 0;
        auto sc = [](int m) { return m == M_ZERO ? 2 : (m == M_NEW ? 0 : 1); };
        if (bx > 0) score += sc(modes[i - 1]);
        if (by > 0) score += sc(modes[i - bw]);
        const int ctx = std::min(score, 3);
        int mode;
        if (r.get(c_.m_new[ctx])) mode = M_NEW;
        else if (!r.get(c_.m_nz[ctx])) mode = M_ZERO;
        else if (r.get(c_.m_near[ctx])) mode = M_NEAR;
        else if (r.get(c_.m_tmp[ctx])) mode = M_TEMPORAL;
        else if (r.get(c_.m_tr[ctx])) mode = M_TOPRIGHT;
        else if (r.get(c_.m_tl[ctx])) mode = M_TOPLEFT;
        else mode = M_NEAREST;
        b.mode = (uint8_t)mode;
        b.new_base = 0;
        b.dx = b.dy = 0;
        b.spx = b.spy = SP_ZERO;
        hits[i] = 0;
        if (mode == M_NEW) {
            if (r.get(c_.b_nearest[ctx])) b.new_base = 0;
            else if (r.get(c_.b_near[ctx])) b.new_base = 1;
            else if (r.get(c_.b_tr[ctx])) b.new_base = 2;
            else b.new_base = r.get(c_.b_tl[ctx]) ? 3 : 4;
            bool via = false;
            if (!cands_.empty()) {
                const int lh = bx > 0 ? hits[i - 1] : 0, th = by > 0 ? hits[i - bw] : 0;
                const bool hit = r.get(c_.hit[lh + th]);
                if (hit) {
                    int lo = 0, hi = 16, d = 0;
                    while (hi - lo > 1) {
                        const int mid = (lo + hi) / 2;
                        if (r.get(c_.cidx[d])) lo = mid;
                        else hi = mid;
                        d++;
                    }
                    if (lo < (int)cands_.size()) {  // unpack cand_key
                        const uint32_t k = cands_[lo];
                        b.dx = (int8_t)(uint8_t)((k >> 24) ^ 0x80);
                        b.dy = (int8_t)(uint8_t)(((k >> 16) & 0xff) ^ 0x80);
                        b.spx = (uint8_t)((k >> 8) & 0xff);
                        b.spy = (uint8_t)(k & 0xff);
                        via = true;
                    }
                } else {
                    b.dx = dec_comp(r, c_.cls_x, c_.sign_x, c_.mag_x);
                    b.dy = dec_comp(r, c_.cls_y, c_.sign_y, c_.mag_y);
                }
                hits[i] = hit ? 1 : 0;
            } else {
                b.dx = dec_comp(r, c_.cls_x, c_.sign_x, c_.mag_x);
                b.dy = dec_comp(r, c_.cls_y, c_.sign_y, c_.mag_y);
            }
            if (!via) {
                b.spx = r.get(c_.sub_x) ? SP_PLUS : SP_ZERO;
                b.spy = r.get(c_.sub_y) ? SP_PLUS : SP_ZERO;
            }
        }
        modes[i] = (uint8_t)mode;
    }
    if (r.error) return false;
    update(out);
    return true;
}

// dense index of a candidate key (cand_key): (dx, dy) bytes and the two subpels (0..2)
static inline uint32_t key_index(uint32_t key) {
    return ((key >> 16) * 3 + ((key >> 8) & 0xff)) * 3 + (key & 0xff);
}

void MvCoder::update(const std::vector<MvCodedBlock>& blocks) {  // encoder.rs:370-412
    if (cnt_.empty()) {
        cnt_.assign(65536u * 9u, 0u);
        listed_.assign(65536u * 9u, 0);
    }
    for (uint32_t k : active_) {
        uint32_t& c = cnt_[key_index(k)];
        c = (c * 7) / 8;
    }
    total_ = (total_ * 7) / 8;
    for (auto& b : blocks)
        if (b.mode == M_NEW) {
            const uint32_t key = cand_key(b.dx, b.dy, b.spx, b.spy), i = key_index(key);
            if (!listed_[i]) {
                listed_[i] = 1;
                active_.push_back(key);
            }
            cnt_[i] += 1;
            total_++;
        }
    // drop the keys whose count decayed to zero (the reference removes them)
    size_t w = 0;
    for (uint32_t k : active_) {
        const uint32_t i = key_index(k);
        if (cnt_[i]) active_[w++] = k;
        else listed_[i] = 0;
    }
    active_.resize(w);
    cands_.clear();
    if (total_ < 100) return;
    // the 16 most frequent keys above 1 % of the total, ties to the smaller key
    const uint32_t thr = total_ / 100;
    std::vector<std::pair<uint32_t, uint32_t>> s;
    for (uint32_t k : active_) {
        const uint32_t c = cnt_[key_index(k)];
        if (c > thr) s.emplace_back(k, c);
    }
    auto better = [](const std::pair<uint32_t, uint32_t>& a, const std::pair<uint32_t, uint32_t>& b) {
        if (a.second != b.second) return a.second > b.second;
        return a.first < b.first;
    };
    const size_t take = std::min<size_t>(16, s.size());
    std::partial_sort(s.begin(), s.begin() + take, s.end(), better);
    for (size_t k = 0; k < take; k++) cands_.push_back(s[k].first);
}

void compute_delta_bias(const std::vector<std::pair<int8_t, int8_t>>& d, int8_t& bx, int8_t& by) {
    bx = by = 0;
    if (d.empty()) return;
    int64_t hx[256] = {0}, hy[256] = {0};
    for (auto& p : d) {
        hx[p.first + 128]++;
        hy[p.second + 128]++;
    }
    int vs[256], nv = 0;  // the occupied bins, in increasing order
    for (int v = 0; v < 256; v++)
        if (hx[v] || hy[v]) vs[nv++] = v;
    int64_t bzx = -1, bzy = -1, bcx = INT64_MAX, bcy = INT64_MAX;
    for (int b = -24; b <= 24; b++) {
        int64_t zx = 0, cx = 0, zy = 0, cy = 0;
        for (int k = 0; k < nv; k++) {
            const int v = vs[k];
            int a = std::min(std::max(v - 128 - b, -128), 127);
            // `adj.abs() as i32` on i8 wraps at -128 in the release build.
            int64_t ab = a == -128 ? -128 : std::abs(a);
            if (a == 0) { zx += hx[v]; zy += hy[v]; }
            cx += hx[v] * ab;
            cy += hy[v] * ab;
        }
        if (zx > bzx || (zx == bzx && cx < bcx)) { bzx = zx; bcx = cx; bx = (int8_t)b; }
        if (zy > bzy || (zy == bzy && cy < bcy)) { bzy = zy; bcy = cy; by = (int8_t)b; }
    }
}

}  // namespace riv
