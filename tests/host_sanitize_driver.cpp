// Host entropy stage under the compiler's sanitizers (built and run by
// tests/test_host_sanitizers.py with -fsanitize=address,undefined and with -fsanitize=thread).
// On seeded random coefficient frames it checks that the coefficient coder gives the same
// bytes inline, with its full rANS batches on a pool, and in its parallel form; that the
// decoder inverts it; that a magnitude class above 13 fails in every form; and that the MV
// decoder inverts the MV coder over frames with a candidate history.
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <functional>
#include <future>
#include <memory>
#include <mutex>
#include <random>
#include <stdexcept>
#include <thread>
#include <vector>

#include "riv_entropy.h"

namespace {

class Pool {
public:
    explicit Pool(unsigned n) {
        for (unsigned i = 0; i < n; i++) threads_.emplace_back([this] { run(); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : threads_) t.join();
    }
    std::future<void> submit(std::function<void()> f) {
        auto task = std::make_shared<std::packaged_task<void()>>(std::move(f));
        std::future<void> fut = task->get_future();
        {
            std::lock_guard<std::mutex> g(m_);
            q_.push_back([task] { (*task)(); });
        }
        cv_.notify_one();
        return fut;
    }

private:
    void run() {
        for (;;) {
            std::function<void()> f;
            {
                std::unique_lock<std::mutex> l(m_);
                cv_.wait(l, [this] { return stop_ || !q_.empty(); });
                if (stop_ && q_.empty()) return;
                f = std::move(q_.front());
                q_.pop_front();
            }
            f();
        }
    }
    std::vector<std::thread> threads_;
    std::deque<std::function<void()>> q_;
    std::mutex m_;
    std::condition_variable cv_;
    bool stop_ = false;
};

// Dense blocks (384 i16: Y 256, U 64, V 64) whose significance fades with the index.
std::vector<int16_t> random_blocks(std::mt19937_64& rng, int n, double density) {
    std::vector<int16_t> b((size_t)n * 384, 0);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    std::geometric_distribution<int> mag(0.4);
    static const int base[3] = {0, 256, 320}, len[3] = {256, 64, 64};
    for (int k = 0; k < n; k++)
        for (int pl = 0; pl < 3; pl++) {
            const double d = pl == 0 ? density : density / 2;
            for (int i = 0; i < len[pl]; i++)
                if (u(rng) < d * std::exp(-i / (len[pl] / 6.0))) {
                    const int v = 1 + mag(rng);
                    b[(size_t)k * 384 + base[pl] + i] = (int16_t)(u(rng) < 0.5 ? -v : v);
                }
            if (u(rng) < 0.15) b[(size_t)k * 384 + base[pl]] = (int16_t)((int)(u(rng) * 1800) - 900);
        }
    return b;
}

// The GPU compaction's layout: per plane the run up to its last non-zero coefficient (with DC
// prediction the last non-zero AC coefficient), and that index.
void compact(const std::vector<int16_t>& b, int n, bool intra, std::vector<int16_t>& packed,
             std::vector<uint8_t>& eobs) {
    static const int base[3] = {0, 256, 320}, len[3] = {256, 64, 64};
    packed.clear();
    eobs.assign((size_t)n * 3, 0);
    for (int k = 0; k < n; k++)
        for (int pl = 0; pl < 3; pl++) {
            const int16_t* p = b.data() + (size_t)k * 384 + base[pl];
            int last = 0;
            for (int i = len[pl] - 1; i >= (intra ? 1 : 0); i--)
                if (p[i] != 0) {
                    last = i;
                    break;
                }
            eobs[(size_t)k * 3 + pl] = (uint8_t)last;
            packed.insert(packed.end(), p, p + last + 1);
        }
}

int fail(const char* what, int trial) {
    std::fprintf(stderr, "FAIL %s (trial %d)\n", what, trial);
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    const int trials = argc > 1 ? std::atoi(argv[1]) : 6;
    riv::entropy_init();
    Pool pool(3);
    riv::BatchSubmit submit = [&pool](std::function<void()> f) { return pool.submit(std::move(f)); };
    std::mt19937_64 rng(20261204);
    std::vector<int16_t> packed;
    std::vector<uint8_t> eobs;
    for (int t = 0; t < trials; t++) {
        const bool intra = t % 2 == 1;
        const int n = t < 2 ? 40 : 700 + 400 * t;  // below and above the parallel form's minimum
        const std::vector<int16_t> b = random_blocks(rng, n, t < 4 ? 0.3 : 0.6);
        compact(b, n, intra, packed, eobs);
        std::vector<uint8_t> inline_bytes, pooled, parallel, async_bytes;
        riv::encode_residual_frame(packed.data(), eobs.data(), n, intra, inline_bytes);
        riv::encode_residual_frame(packed.data(), eobs.data(), n, intra, pooled, &submit);
        riv::encode_residual_frame(packed.data(), eobs.data(), n, intra, parallel, &submit, 4);
        {  // every batch handed off, joined later (the encoder joins at the record write)
            std::unique_ptr<riv::RansWriter> w =
                riv::encode_residual_frame_async(packed.data(), eobs.data(), n, intra, async_bytes, submit);
            if (w) w->collect();
        }
        if (pooled != inline_bytes) return fail("pooled batches differ from the inline coder", t);
        if (parallel != inline_bytes) return fail("parallel coder differs from the inline coder", t);
        if (async_bytes != inline_bytes) return fail("handed-off batches differ from the inline coder", t);
        std::vector<uint8_t> coded((size_t)n, 1);
        std::vector<int16_t> back((size_t)n * 384);
        if (!riv::decode_residual_frame(inline_bytes.data(), inline_bytes.size(), coded.data(), n, intra, back.data()))
            return fail("decoder reports a malformed stream", t);
        if (back != b) return fail("decoder does not invert the coder", t);
    }
    // a magnitude class above 13 fails in every form
    std::vector<int16_t> b = random_blocks(rng, 900, 0.4);
    b[(size_t)300 * 384 + 7] = 9000;
    compact(b, 900, false, packed, eobs);
    for (int form = 0; form < 4; form++) {
        std::vector<uint8_t> out;
        bool threw = false;
        try {
            if (form == 0) riv::encode_residual_frame(packed.data(), eobs.data(), 900, false, out);
            else if (form == 1) riv::encode_residual_frame(packed.data(), eobs.data(), 900, false, out, &submit);
            else if (form == 2) riv::encode_residual_frame(packed.data(), eobs.data(), 900, false, out, &submit, 4);
            else riv::encode_residual_frame_async(packed.data(), eobs.data(), 900, false, out, submit);
        } catch (const std::runtime_error&) {
            threw = true;
        }
        if (!threw) return fail("magnitude class 14 did not fail", form);
    }
    // the MV coder: frames of every mode with a candidate history, encoded by one coder and
    // decoded by another that follows it; and the same frames through the encoder's pipeline
    // (symbol listing and modelling of consecutive frames on two threads at once, every rANS
    // batch on the pool), which must give the same bytes
    {
        riv::MvCoder enc, dec, staged;
        Pool list_thread(1), model_thread(1);
        std::vector<std::vector<riv::MvCodedBlock>> frames;
        std::vector<std::vector<uint8_t>> seq_bytes;
        std::uniform_int_distribution<int> mode(0, 6), base(0, 4), delta(-128, 127), sub(0, 1), few(0, 3);
        std::bernoulli_distribution coin(0.5);
        const int bw = 24, bh = 16;
        for (int f = 0; f < 30; f++) {
            std::vector<riv::MvCodedBlock> v((size_t)bw * bh), back;
            for (riv::MvCodedBlock& b : v) {
                b = riv::MvCodedBlock{};
                b.mode = (uint8_t)mode(rng);
                b.skip = coin(rng);
                if (b.mode == riv::M_NEW) {
                    static const int8_t common[4] = {-3, 0, 2, 5};
                    b.new_base = (uint8_t)base(rng);
                    b.dx = coin(rng) ? common[few(rng)] : (int8_t)delta(rng);
                    b.dy = coin(rng) ? common[few(rng)] : (int8_t)delta(rng);
                    b.spx = (uint8_t)sub(rng);
                    b.spy = (uint8_t)sub(rng);
                }
            }
            std::vector<uint8_t> bytes;
            enc.encode_frame(v, bw, bytes);
            frames.push_back(v);
            seq_bytes.push_back(bytes);
            if (!dec.decode_frame(bytes.data(), bytes.size(), bw, bh, back)) return fail("MV decoder: malformed", f);
            for (size_t i = 0; i < v.size(); i++) {
                const riv::MvCodedBlock &a = v[i], &c = back[i];
                if (a.mode != c.mode || a.new_base != c.new_base || a.dx != c.dx || a.dy != c.dy || a.spx != c.spx ||
                    a.spy != c.spy || a.skip != c.skip)
                    return fail("MV decoder does not invert the coder", f);
            }
        }
        const size_t nf = frames.size();
        std::vector<riv::MvSymbols> syms(nf);
        std::vector<std::vector<uint8_t>> out(nf);
        std::vector<std::unique_ptr<riv::RansWriter>> writers(nf);
        std::vector<std::shared_future<void>> listed(nf);
        std::vector<std::future<void>> modelled(nf);
        for (size_t f = 0; f < nf; f++) {
            listed[f] = list_thread.submit([&, f] { staged.prepare(frames[f], bw, syms[f]); }).share();
            std::shared_future<void> lf = listed[f];
            modelled[f] = model_thread.submit([&, f, lf] {
                lf.get();
                writers[f].reset(new riv::RansWriter(&out[f], &submit));
                staged.model(syms[f], *writers[f]);
                writers[f]->finish_async();
            });
        }
        for (size_t f = 0; f < nf; f++) {
            modelled[f].get();
            writers[f]->collect();
            if (out[f] != seq_bytes[f]) return fail("pipelined MV coder differs from the sequential coder", (int)f);
        }
    }
    std::printf("host entropy sanitizer driver: ok\n");
    return 0;
}
