// riv_entropy.cpp -- host entropy coders (see riv_entropy.h).
#include "riv_entropy.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>

namespace riv {

static uint8_t g_zero_prob[65536];
static uint64_t g_rcp_m[256];
static uint32_t g_rcp_s[256];
static std::once_flag g_once;

void entropy_init() {
    std::call_once(g_once, [] {
        // BinProb zero-probability table (com/rans.rs:30-44): p = zeros*256/(zeros+ones)
        // truncated to u8, with 0 mapped to 1.
        g_zero_prob[0] = 1;
        for (int i = 1; i < 65536; i++) {
            int zeros = i >> 8, ones = i & 0xff;
            uint8_t p = (uint8_t)((zeros << 8) / (zeros + ones));
            g_zero_prob[i] = p ? p : 1;
        }
        // Exact reciprocals for r / f, f in [1,255], r < 2^32 (round-up multiplier with
        // s = 32 + ceil(log2 f) fraction bits).
        for (uint32_t f = 1; f < 256; f++) {
            uint32_t l = 0;
            while ((1u << l) < f) l++;
            uint32_t s = 32 + l;
            unsigned __int128 one = (unsigned __int128)1 << s;
            g_rcp_m[f] = (uint64_t)((one + f - 1) / f);
            g_rcp_s[f] = s;
        }
    });
}

static inline uint8_t prob_zero(const BinProb& b) { return g_zero_prob[b.packed]; }
static inline void observe(BinProb& b, bool bit) {  // com/rans.rs:73-84
    uint16_t rot = bit ? (uint16_t)((b.packed << 8) | (b.packed >> 8)) : b.packed;
    uint32_t sum = (uint32_t)rot + 0x100u;
    uint16_t upd = (uint16_t)sum;
    if (sum > 0xFFFFu) {
        uint16_t mask = rot == 0xff01 ? 0xff00 : 0x8100;
        upd = (uint16_t)((uint16_t)(rot + 0x101) >> 1) | mask;
    }
    b.packed = bit ? (uint16_t)((upd << 8) | (upd >> 8)) : upd;
}

static const int BATCH = 16386;  // com/rans.rs:201

RansWriter::RansWriter(std::vector<uint8_t>* sink, const BatchSubmit* submit)
    : sink_(sink), stack_(BATCH), sp_(BATCH), submit_(submit) {}

inline void RansWriter::put(bool bit, BinProb& ctx) {
    uint8_t p = prob_zero(ctx);
    observe(ctx, bit);
    if (sp_ == 0) drain();
    stack_[--sp_] = (uint16_t)(p | (bit ? 0x100 : 0));
}
inline void RansWriter::put_bypass(bool bit) {
    if (sp_ == 0) drain();
    stack_[--sp_] = (uint16_t)(128 | (bit ? 0x100 : 0));
}


static inline void enc_sym(uint32_t& r, uint16_t* words, int& wp, uint16_t e) {
    uint32_t p = e & 0xff;
    if (p == 0) p = 1;
    bool bit = (e >> 8) & 1;
    uint32_t start = bit ? p : 0, freq = bit ? 256u - p : p;
    uint32_t xmax = freq << 24;
    if (r >= xmax) {
        words[--wp] = (uint16_t)r;
        r >>= 16;
    }
    uint32_t q = (uint32_t)(((unsigned __int128)r * g_rcp_m[freq]) >> g_rcp_s[freq]);
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

static inline void put_class_value(RansWriter& w, unsigned value, BinProb* ctx, int nctx) {
    int maxc = nctx - 1, cls = bit_len(value);
    for (int c = 0; c < cls; c++) w.put(true, ctx[c]);
    if (cls < maxc) w.put(false, ctx[cls]);
    if (cls >= 2) {
        unsigned off = value - (1u << (cls - 1));
        for (int b = cls - 2; b >= 0; b--) w.put_bypass((off >> b) & 1);
    }
}

struct DctContexts {
    BinProb sig_y[256], sig_c[64], mag_y[4][13], mag_c[3][13], eob_y[9], eob_c[7];
    int16_t prev_dc[3] = {0, 0, 0};
};

static void encode_plane(RansWriter& w, DctContexts& c, const int16_t* pl, int last, bool luma, int pi, bool dcp) {
    int16_t dcv = pl[0];
    if (dcp) {
        dcv = (int16_t)(pl[0] - c.prev_dc[pi]);
        c.prev_dc[pi] = pl[0];
    }
    if (luma) put_class_value(w, (unsigned)last, c.eob_y, 9);
    else put_class_value(w, (unsigned)last, c.eob_c, 7);
    BinProb* sig = luma ? c.sig_y : c.sig_c;
    for (int i = 0; i <= last; i++) {
        int16_t v = i == 0 ? dcv : pl[i];
        w.put(v != 0, sig[i]);
        if (v != 0) {
            w.put_bypass(v < 0);
            unsigned a = (unsigned)std::abs((int)v) - 1;
            BinProb* mc = luma ? c.mag_y[luma_band(i)] : c.mag_c[chroma_band(i)];
            put_class_value(w, a, mc, 13);
        }
    }
}

void encode_residual_frame(const int16_t* packed, const uint8_t* eobs, int nblocks, bool intra,
                           std::vector<uint8_t>& out, const BatchSubmit* submit) {
    out.clear();
    if (nblocks == 0) return;  // the reference never instantiates the coder
    RansWriter w(&out, submit);
    DctContexts* c = new DctContexts();
    const int16_t* p = packed;
    for (int b = 0; b < nblocks; b++) {
        const uint8_t* e = eobs + 3 * b;
        // With DC prediction the coded range ends at the last non-zero AC coefficient
        // (res/rans.rs:250-262); the GPU's last-non-zero index already equals it.  The
        // compact layout holds each plane block only up to that index.
        encode_plane(w, *c, p, e[0], true, 0, intra);
        p += e[0] + 1;
        encode_plane(w, *c, p, e[1], false, 1, intra);
        p += e[1] + 1;
        encode_plane(w, *c, p, e[2], false, 2, intra);
        p += e[2] + 1;
    }
    w.finish();
    delete c;
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

static void enc_class(RansWriter& w, BinProb* ctx, int cls) {
    int lo = 0, hi = 10, d = 0;
    while (lo < hi) {
        int mid = (lo + hi) / 2;
        bool g = cls > mid;
        w.put(g, ctx[d]);
        if (g) lo = mid + 1; else hi = mid;
        d++;
    }
}
static void enc_comp(RansWriter& w, int8_t delta, BinProb* cls, BinProb& sign, BinProb* mag) {
    unsigned m = (unsigned)std::abs((int)delta);
    int c = mv_class(m);
    enc_class(w, cls, c);
    if (c == 0) return;
    w.put(delta < 0, sign);
    unsigned bits = c <= 1 ? 0 : c - 1, off = m - (1u << (c - 1));
    for (unsigned b = 0; b < bits; b++) w.put((off >> b) & 1, mag[b]);
}

void MvCoder::encode_frame(const std::vector<MvCodedBlock>& blocks, int bw, std::vector<uint8_t>& out) {
    out.clear();
    RansWriter w(&out);
    std::vector<uint8_t> modes, hits;
    modes.reserve(blocks.size());
    hits.reserve(blocks.size());
    for (size_t i = 0; i < blocks.size(); i++) {
        const MvCodedBlock& b = blocks[i];
        int bx = (int)(i % bw), by = (int)(i / bw);
        w.put(b.skip, skip_);
        // mv_mode_context (res/mv_predictor.rs:275-308)
        int score = 0;
        auto sc = [](int m) { return m == M_ZERO ? 2 : (m == M_NEW ? 0 : 1); };
        if (bx > 0) score += sc(modes[i - 1]);
        if (by > 0) score += sc(modes[i - bw]);
        int ctx = std::min(score, 3);
        bool is_new = b.mode == M_NEW;
        w.put(is_new, m_new_[ctx]);
        if (!is_new) {
            bool nz = b.mode != M_ZERO;
            w.put(nz, m_nz_[ctx]);
            if (nz) {
                bool nr = b.mode == M_NEAR;
                w.put(nr, m_near_[ctx]);
                if (!nr) {
                    bool tm = b.mode == M_TEMPORAL;
                    w.put(tm, m_tmp_[ctx]);
                    if (!tm) {
                        bool tr = b.mode == M_TOPRIGHT;
                        w.put(tr, m_tr_[ctx]);
                        if (!tr) w.put(b.mode == M_TOPLEFT, m_tl_[ctx]);
                    }
                }
            }
            hits.push_back(0);
        } else {
            bool e0 = b.new_base == 0;
            w.put(e0, b_nearest_[ctx]);
            if (!e0) {
                bool e1 = b.new_base == 1;
                w.put(e1, b_near_[ctx]);
                if (!e1) {
                    bool e2 = b.new_base == 2;
                    w.put(e2, b_tr_[ctx]);
                    if (!e2) w.put(b.new_base == 3, b_tl_[ctx]);
                }
            }
            bool via = false;
            if (!cands_.empty()) {
                uint32_t key = cand_key(b.dx, b.dy, b.spx, b.spy);
                int ci = -1;
                for (size_t k = 0; k < cands_.size(); k++)
                    if (cands_[k] == key) { ci = (int)k; break; }
                bool hit = ci >= 0;
                int lh = bx > 0 ? hits[i - 1] : 0, th = by > 0 ? hits[i - bw] : 0;
                w.put(hit, hit_[lh + th]);
                if (hit) {
                    int lo = 0, hi = 16, d = 0;
                    while (hi - lo > 1) {
                        int mid = (lo + hi) / 2;
                        bool g = ci >= mid;
                        w.put(g, cidx_[d]);
                        if (g) lo = mid; else hi = mid;
                        d++;
                    }
                    via = true;
                } else {
                    enc_comp(w, b.dx, cls_x_, sign_x_, mag_x_);
                    enc_comp(w, b.dy, cls_y_, sign_y_, mag_y_);
                }
                hits.push_back(hit ? 1 : 0);
            } else {
                enc_comp(w, b.dx, cls_x_, sign_x_, mag_x_);
                enc_comp(w, b.dy, cls_y_, sign_y_, mag_y_);
                hits.push_back(0);
            }
            if (!via) {
                w.put(b.spx != SP_ZERO, sub_x_);
                w.put(b.spy != SP_ZERO, sub_y_);
            }
        }
        modes.push_back(b.mode);
    }
    w.finish();
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
        b.skip = r.get(skip_);
        int score = 0;
        auto sc = [](int m) { return m == M_ZERO ? 2 : (m == M_NEW ? 0 : 1); };
        if (bx > 0) score += sc(modes[i - 1]);
        if (by > 0) score += sc(modes[i - bw]);
        const int ctx = std::min(score, 3);
        int mode;
        if (r.get(m_new_[ctx])) mode = M_NEW;
        else if (!r.get(m_nz_[ctx])) mode = M_ZERO;
        else if (r.get(m_near_[ctx])) mode = M_NEAR;
        else if (r.get(m_tmp_[ctx])) mode = M_TEMPORAL;
        else if (r.get(m_tr_[ctx])) mode = M_TOPRIGHT;
        else if (r.get(m_tl_[ctx])) mode = M_TOPLEFT;
        else mode = M_NEAREST;
        b.mode = (uint8_t)mode;
        b.new_base = 0;
        b.dx = b.dy = 0;
        b.spx = b.spy = SP_ZERO;
        hits[i] = 0;
        if (mode == M_NEW) {
            if (r.get(b_nearest_[ctx])) b.new_base = 0;
            else if (r.get(b_near_[ctx])) b.new_base = 1;
            else if (r.get(b_tr_[ctx])) b.new_base = 2;
            else b.new_base = r.get(b_tl_[ctx]) ? 3 : 4;
            bool via = false;
            if (!cands_.empty()) {
                const int lh = bx > 0 ? hits[i - 1] : 0, th = by > 0 ? hits[i - bw] : 0;
                const bool hit = r.get(hit_[lh + th]);
                if (hit) {
                    int lo = 0, hi = 16, d = 0;
                    while (hi - lo > 1) {
                        const int mid = (lo + hi) / 2;
                        if (r.get(cidx_[d])) lo = mid;
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
                    b.dx = dec_comp(r, cls_x_, sign_x_, mag_x_);
                    b.dy = dec_comp(r, cls_y_, sign_y_, mag_y_);
                }
                hits[i] = hit ? 1 : 0;
            } else {
                b.dx = dec_comp(r, cls_x_, sign_x_, mag_x_);
                b.dy = dec_comp(r, cls_y_, sign_y_, mag_y_);
            }
            if (!via) {
                b.spx = r.get(sub_x_) ? SP_PLUS : SP_ZERO;
                b.spy = r.get(sub_y_) ? SP_PLUS : SP_ZERO;
            }
        }
        modes[i] = (uint8_t)mode;
    }
    if (r.error) return false;
    update(out);
    return true;
}

void MvCoder::update(const std::vector<MvCodedBlock>& blocks) {  // encoder.rs:370-412
    for (auto& kv : counts_) kv.second = (kv.second * 7) / 8;
    total_ = (total_ * 7) / 8;
    for (auto& b : blocks)
        if (b.mode == M_NEW) {
            counts_[cand_key(b.dx, b.dy, b.spx, b.spy)] += 1;
            total_++;
        }
    for (auto it = counts_.begin(); it != counts_.end();)
        if (it->second == 0) it = counts_.erase(it); else ++it;
    cands_.clear();
    if (total_ < 100) return;
    std::vector<std::pair<uint32_t, uint32_t>> s(counts_.begin(), counts_.end());
    std::sort(s.begin(), s.end(), [](const std::pair<uint32_t, uint32_t>& a, const std::pair<uint32_t, uint32_t>& b) {
        if (a.second != b.second) return a.second > b.second;
        return a.first < b.first;
    });
    uint32_t thr = total_ / 100;
    for (auto& e : s) {
        if (cands_.size() >= 16) break;
        if (e.second > thr) cands_.push_back(e.first);
    }
}

void compute_delta_bias(const std::vector<std::pair<int8_t, int8_t>>& d, int8_t& bx, int8_t& by) {
    bx = by = 0;
    if (d.empty()) return;
    int64_t hx[256] = {0}, hy[256] = {0};
    for (auto& p : d) {
        hx[p.first + 128]++;
        hy[p.second + 128]++;
    }
    int64_t bzx = -1, bzy = -1, bcx = INT64_MAX, bcy = INT64_MAX;
    for (int b = -24; b <= 24; b++) {
        int64_t zx = 0, cx = 0, zy = 0, cy = 0;
        for (int v = 0; v < 256; v++) {
            if (!hx[v] && !hy[v]) continue;
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
