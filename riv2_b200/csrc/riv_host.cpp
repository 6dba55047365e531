// riv_host.cpp -- the C-ABI encoder (include/riv_gpu.h): device buffers, the per-frame
// kernel sequence, the frame pipeline and the host entropy stage.
//
// Per P-frame (one CUDA stream):  rgb->yuv -> search/mode wavefront -> predict+variance
// -> AQ -> residual/DCT/quant/recon -> deblock -> compaction; a copy stream brings the
// per-MB side info and the coded MBs' coefficients back; the host runs the motion-vector
// rANS coder (ordered, contexts persist across frames), the DCT-coefficient rANS coder
// (fresh contexts per frame, so frames code in parallel on a thread pool) and writes the
// records in frame order.  Reference: enc/encoder.rs:258-947 (enc/ =
// reitero_video/reitero_encode/src/).
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <sys/resource.h>
#include <sys/syscall.h>
#include <unistd.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <functional>
#include <future>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/riv_gpu.h"
#include "../../include/riv_nn.h"
#include "riv_entropy.h"
#include "riv_internal.h"
#include "riv_nn.h"

extern "C" int riv_upload_dct_tables(const int32_t* t16, const int32_t* t8);

namespace {

using namespace riv;

// ---------------------------------------------------------------------------------
// Small utilities
// ---------------------------------------------------------------------------------
struct CudaError {
    cudaError_t e;
    const char* where;
};
#define CK(x)                                                   \
    do {                                                        \
        cudaError_t e_ = (cudaError_t)(x);                      \
        if (e_ != cudaSuccess) throw CudaError{e_, #x};         \
    } while (0)

constexpr int BULK_NICE = 5;  // the coefficient coders' workers, below the serial stages

class ThreadPool {
public:
    // nice > 0: the workers run below the process's other threads (bulk work that must not
    // preempt the serial stages of the pipeline; a refused priority change is ignored)
    explicit ThreadPool(unsigned n, int nice = 0) {
        for (unsigned i = 0; i < n; i++)
            workers_.emplace_back([this, nice] {
                if (nice > 0) (void)setpriority(PRIO_PROCESS, (id_t)syscall(SYS_gettid), nice);
                run();
            });
    }
    ~ThreadPool() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    // urgent: ahead of every queued job (latency-critical work behind bulk work)
    std::future<void> submit(std::function<void()> f, bool urgent = false) {
        auto task = std::make_shared<std::packaged_task<void()>>(std::move(f));
        std::future<void> fut = task->get_future();
        {
            std::lock_guard<std::mutex> g(m_);
            if (urgent) q_.push_front([task] { (*task)(); });
            else q_.push_back([task] { (*task)(); });
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
    std::vector<std::thread> workers_;
    std::deque<std::function<void()>> q_;
    std::mutex m_;
    std::condition_variable cv_;
    bool stop_ = false;
};

// DCT bases from their definition: T[i][j] = round(2^18 * c_j * cos((2i+1) j pi / 2N)),
// c_0 = sqrt(1/N), c_j = sqrt(2/N) -- equal to the reference's tables
// (dct/dct16.rs:7-145, dct/dct8.rs:6-25; checked against tests/golden).
static int32_t round_half_away(double v) { return (int32_t)(v >= 0 ? floor(v + 0.5) : -floor(-v + 0.5)); }
static void dct_tables(int32_t* t16, int32_t* t8) {
    const double PI = 3.14159265358979323846;
    for (int i = 0; i < 16; i++)
        for (int j = 0; j < 16; j++)
            t16[i * 16 + j] = round_half_away(262144.0 * (j == 0 ? sqrt(1.0 / 16) : sqrt(2.0 / 16)) *
                                              cos((2 * i + 1) * j * PI / 32));
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++)
            t8[i * 8 + j] = round_half_away(262144.0 * (j == 0 ? sqrt(1.0 / 8) : 0.5) * cos((2 * i + 1) * j * PI / 16));
}

// quant_step_from_quality (res/residual.rs:13-23)
static float quant_step(uint8_t q) {
    if (q == 100) return 1.0f;
    if (q == 1) return 112.0f;
    return 1.0f + (100.0f - (float)q) / 99.0f * (112.0f - 1.0f);
}
// deblock_level_from_quant_step / thresholds (com/deblock.rs:34-58)
static int deblock_level(float qs) {
    float v = roundf(qs * 0.6f);
    v = v < 0.0f ? 0.0f : (v > 63.0f ? 63.0f : v);
    return (int)v;
}
static void deblock_thresholds(int level, bool intra, int& E, int& I, int& H) {
    I = std::max(level, 1);
    E = (level + 2) * 2 + I;
    if (intra) H = level >= 40 ? 2 : (level >= 15 ? 1 : 0);
    else H = level >= 40 ? 3 : (level >= 20 ? 2 : (level >= 15 ? 1 : 0));
}
// build_intra_{y,uv}_quant_table (res/residual.rs:58-96)
static const float JPEG_LUMA[64] = {16, 11, 10, 16, 24,  40,  51,  61,  12, 12, 14, 19, 26,  58,  60,  55,
                                    14, 13, 16, 24, 40,  57,  69,  56,  14, 17, 22, 29, 51,  87,  80,  62,
                                    18, 22, 37, 56, 68,  109, 103, 77,  24, 35, 55, 64, 81,  104, 113, 92,
                                    49, 64, 78, 87, 103, 121, 120, 101, 72, 92, 95, 98, 112, 100, 103, 99};
static const float JPEG_CHROMA[64] = {17, 18, 24, 47, 99, 99, 99, 99, 18, 21, 26, 66, 99, 99, 99, 99,
                                      24, 26, 56, 99, 99, 99, 99, 99, 47, 66, 99, 99, 99, 99, 99, 99,
                                      99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99,
                                      99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99};
static uint16_t round_max1_u16(float s) {
    float r = roundf(s);
    if (r < 1.0f) r = 1.0f;
    return r >= 65535.0f ? 65535 : (uint16_t)r;
}
static void intra_tables(float qs, uint16_t* yt, uint16_t* ct) {
    for (int v = 0; v < 16; v++)
        for (int u = 0; u < 16; u++) {
            float fx = (float)u * 7.0f / 15.0f, fy = (float)v * 7.0f / 15.0f;
            int x0 = (int)fx, y0 = (int)fy, x1 = std::min(x0 + 1, 7), y1 = std::min(y0 + 1, 7);
            float dx = fx - (float)x0, dy = fy - (float)y0;
            float val = JPEG_LUMA[y0 * 8 + x0] * (1.0f - dx) * (1.0f - dy) + JPEG_LUMA[y0 * 8 + x1] * dx * (1.0f - dy) +
                        JPEG_LUMA[y1 * 8 + x0] * (1.0f - dx) * dy + JPEG_LUMA[y1 * 8 + x1] * dx * dy;
            yt[v * 16 + u] = round_max1_u16((val / JPEG_LUMA[0]) * qs);
        }
    for (int i = 0; i < 64; i++) ct[i] = round_max1_u16((JPEG_CHROMA[i] / JPEG_CHROMA[0]) * qs);
}
// LambdaEntry::for_quality (enc/rdo.rs:23-48, 75-86)
struct Lambda {
    double lambda, ret, slope, icpt, skip_bits, keep_bits;
};
static Lambda lambda_for(uint8_t quality, double mult) {
    quality = (uint8_t)std::min(std::max((int)quality, 1), 100);
    int qp = (int)round((double)(100u - quality) * 0.6);
    qp = std::min(std::max(qp, 0), 60);
    Lambda L;
    L.lambda = mult * pow(2.0, ((double)qp - 12.0) / 3.0);
    double nq = (double)quality / 100.0, q = (double)quant_step(quality);
    L.slope = 0.5 / q;
    L.icpt = 5.0 + 0.56 * q;
    L.ret = 0.15 + ((q - 1.0) / 111.0) * 0.55;
    L.skip_bits = 0.55 - nq * 0.15;
    L.keep_bits = 1.20 + nq * 0.35;
    return L;
}
// mv_class_from_magnitude (res/mv_rans.rs:80-86): 0 for 0, else the bit length, at most 10.
static int mv_class_of(int mag) {
    if (mag == 0) return 0;
    int b = 0;
    while ((mag >> b) > 1) b++;
    return std::min(b + 1, 10);
}
static int64_t f64_as_i64(double d) {
    if (std::isnan(d)) return 0;
    if (d <= -9223372036854775808.0) return INT64_MIN;
    if (d >= 9223372036854775807.0) return INT64_MAX;
    return (int64_t)d;
}

static void put_le(std::vector<uint8_t>& b, uint64_t v, int n) {
    for (int i = 0; i < n; i++) b.push_back((uint8_t)(v >> (8 * i)));
}
// VideoHeader::to_bytes (com/format.rs:64-88)
static std::vector<uint8_t> header_bytes(const riv_config& c, uint64_t frame_count) {
    std::vector<uint8_t> b = {'R', 'I', 'V', 0};
    put_le(b, 5, 4);
    put_le(b, c.display_width, 4);
    put_le(b, c.display_height, 4);
    put_le(b, c.storage_width, 4);
    put_le(b, c.storage_height, 4);
    put_le(b, c.fps, 4);
    put_le(b, frame_count, 8);
    return b;
}

// glibc logf/exp2f fix-up tables, generated next to the library at build time.
struct LibmFix {
    std::vector<uint32_t> logf, exp2f;  // (in, out) pairs, sorted by input bits
    // device layout: the pairs, then FIX_INDEX + 1 bucket starts (first pair whose input bits
    // have top 16 bits >= the bucket number)
    std::vector<uint32_t> logf_dev, exp2f_dev;
    bool ok = false;
    std::string err;
};
static LibmFix& libm_fix() {
    static LibmFix F;
    static std::once_flag once;
    std::call_once(once, [] {
        Dl_info info;
        std::string dir = ".";
        if (dladdr((void*)&libm_fix, &info) && info.dli_fname) {
            dir = info.dli_fname;
            size_t k = dir.rfind('/');
            dir = k == std::string::npos ? "." : dir.substr(0, k);
        }
        std::string path = dir + "/libm_fixups.bin";
        FILE* f = fopen(path.c_str(), "rb");
        if (!f) { F.err = "missing " + path; return; }
        char magic[8];
        uint32_t n[2];
        if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "RIVLIBM1", 8) || fread(n, 4, 2, f) != 2) {
            F.err = "bad " + path;
            fclose(f);
            return;
        }
        F.logf.resize(2 * (size_t)n[0]);
        F.exp2f.resize(2 * (size_t)n[1]);
        bool good = fread(F.logf.data(), 4, F.logf.size(), f) == F.logf.size() &&
                    fread(F.exp2f.data(), 4, F.exp2f.size(), f) == F.exp2f.size();
        fclose(f);
        if (!good) { F.err = "short " + path; return; }
        auto with_index = [](const std::vector<uint32_t>& pairs) {
            std::vector<uint32_t> d(pairs);
            const size_t n = pairs.size() / 2;
            size_t k = 0;
            for (uint32_t h = 0; h <= 65536u; h++) {
                while (k < n && (pairs[2 * k] >> 16) < h) k++;
                d.push_back((uint32_t)k);
            }
            return d;
        };
        F.logf_dev = with_index(F.logf);
        F.exp2f_dev = with_index(F.exp2f);
        // the batched device logf search takes 9 fixed steps: every bucket must hold < 512 pairs
        for (uint32_t h = 0; h < 65536u; h++) {
            const size_t n0 = F.logf.size() / 2;
            if (F.logf_dev[n0 * 2 + h + 1] - F.logf_dev[n0 * 2 + h] >= 512u) {
                F.err = "logf fix-up bucket too large in " + path;
                return;
            }
        }
        F.ok = true;
    });
    return F;
}

struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    void alloc(size_t bytes) {
        n = bytes;
        CK(cudaMalloc(&p, bytes ? bytes : 1));
    }
    void zero(cudaStream_t s) { CK(cudaMemsetAsync(p, 0, n ? n : 1, s)); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
    }
    template <class T>
    T* as() const { return (T*)p; }
};
struct HostBuf {
    void* p = nullptr;
    void alloc(size_t bytes) { CK(cudaMallocHost(&p, bytes ? bytes : 1)); }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
    }
    template <class T>
    T* as() const { return (T*)p; }
};

// Pinned host memory mapped into the device address space: kernels write the frame's
// side info and compacted coefficients straight into it.
struct MappedBuf {
    void* h = nullptr;
    void* d = nullptr;
    void alloc(size_t bytes) {
        CK(cudaHostAlloc(&h, bytes ? bytes : 1, cudaHostAllocMapped | cudaHostAllocPortable));
        CK(cudaHostGetDevicePointer(&d, h, 0));
    }
    void release() {
        if (h) cudaFreeHost(h);
        h = d = nullptr;
    }
    template <class T>
    T* host() const { return (T*)h; }
    template <class T>
    T* dev() const { return (T*)d; }
};

// Per-frame timing events: Y = input stream, S = main chain, K = compaction stream.
constexpr int NPAR = 3;  // rotation depth of the per-frame device buffers
constexpr uint64_t TIMING_SAMPLE = 8;  // pipelined frames carry stage timing events one in this many
enum { EV_START, EV_YUV, EV_S0, EV_TABLE, EV_SEARCH, EV_PRED, EV_AQ, EV_RES, EV_DEBLOCK, EV_K0, EV_COMPACT, EV_NET0, EV_NET1, EV_N };
static const int NSTAGE = 8;  // rgb->yuv, table, search, predict, aq, residual, deblock, compact (+ total)

struct Slot {
    DevBuf rgb, dside, dpacked, dpeobs;        // compacted frame output on the device
    HostBuf side, packed, peobs;               // pinned copies (DMA on the copy stream)
    MappedBuf hdr;                             // coded MBs, coefficients, device status
    size_t prefetched = 0;                     // coefficient bytes included in the first copy
    cudaEvent_t ev_h2d = nullptr, ev_gpu = nullptr, ev_d2h = nullptr;
    cudaEvent_t ev_k[EV_N] = {};  // stage timing (recorded on timed frames only)
    cudaEvent_t ev_yuv = nullptr, ev_recon = nullptr;  // dependencies: input converted / reconstruction done
};

struct Job {
    uint64_t index = 0, ts = 0;
    int type = 0, slot = 0;
    int state = 0;  // 0 submitted, 1 entropy running
    bool tail_done = true;  // compaction and copies enqueued (false while the frame is pending)
    bool deferred = false;  // reconstructed inside the next P-frame's search launch
    bool timed = false;     // stage timing events recorded for this frame
    // multi-clip step (riv_batch): one event marks the step's GPU work and copies done, in
    // place of the slot's ev_gpu / ev_recon / ev_d2h
    cudaEvent_t xev = nullptr;
    // per-MB statistics requested for this frame: the coded MVs of the frame before (buffer
    // prev_buf when prev_valid) and the frame's search output are read back in retire
    bool want_stats = false, prev_valid = false;
    int prev_buf = 0;
    int ck = 0;             // double-buffer parity of the frame's buffers
    uint32_t count = 0;
    std::future<void> fut, fut_mv, fut_prep, fut_asm;
    std::vector<uint8_t> res_bytes, mv_bytes;
    std::vector<MvCodedBlock> mv_blocks;  // the P-frame's MV coder input
    // host timeline (milliseconds, steady clock), kept when the encoder traces: submitted; MV
    // input assembly started / done; MV listing started / done; MV coding started / done; DCT
    // coding started / done; written
    double tr[10] = {0};
    MvSymbols mv_syms;
    std::unique_ptr<RansWriter> mv_writer;  // the MV bytes' rANS batches, collected when written
    std::unique_ptr<RansWriter> res_writer;  // the coefficient bytes' rANS batches, likewise
    int8_t bias[2] = {0, 0};
    riv_frame_stats stats{};
    float times[NSTAGE + 1] = {0};
};

}  // namespace

struct riv_encoder {
    riv_config cfg;
    riv_writer_vtable wr;
    std::string err;
    bool poisoned = false;
    std::string poison_msg;  // the failure that made the encoder unusable
    uint64_t header_pos = 0, frame_count = 0, submitted = 0;
    int W = 0, H = 0, BW = 0, BH = 0, NMB = 0;
    size_t yuv_bytes = 0;
    cudaStream_t S = nullptr, C = nullptr, Hs = nullptr;  // main chain, device->host, host->device
    cudaStream_t Y = nullptr, K = nullptr;                // input conversion, compaction
    // cross-stream reuse guards: cur[k] free (its residual is done), mbout[k] and the
    // coefficient buffers free (their compaction is done)
    cudaEvent_t ev_cur_free[NPAR] = {}, ev_mbout_free[NPAR] = {}, ev_coef_free[NPAR] = {};
    // the last search launch: input conversion waits for it, so that it never holds SMs the
    // next cooperative search launch needs
    cudaEvent_t ev_search_done = nullptr;
    int fpar = 0, last_par = 0;  // rotation index of the next / last submitted frame
    // A P-frame whose residual, deblock and compaction are handed to the next P-frame's
    // search launch (pipelined encoding with the fused launch); flushed on demand.
    struct Pending {
        bool active = false;
        uint64_t index = 0;
        int ck = 0, level = 0;
        ResidualParams rp{};
        uint8_t* recon = nullptr;
    } pend;
    bool defer_ok = false;
    int wq_words = 0, wq_par = 0;  // queue words of one launch; the array the next launch uses
    // device state
    DevBuf curb[NPAR], ref[2], recon_pre, predb[NPAR], mboutb[NPAR], coded[2], rec, varsum, lnvb[NPAR], qs, coeffsb[NPAR], optskipb[NPAR],
        fmaskb[NPAR], eobsb[NPAR], status, wq;
    DevBuf cindex, coffset, sadtab;
    DevBuf lcindex, lcoffset;  // the search launch's own compaction scan (never shared with stream K's)
    DevBuf mvbits, logfix, expfix, ytab, ctab, newcost, newcost32;
    bool small_costs = false;
    bool table_ok = false;  // exhaustive SAD table + packed argmin usable (costs < 2^59)
    int ref_cur = 0, coded_cur = 0;
    bool has_ref = false, has_prev_mvs = false;
    unsigned tag = 0;
    SearchPlan splan{};
    Lambda L{};
    int inter_E = 0, inter_I = 0, inter_H = 0, inter_level = 0;
    int intra_E = 0, intra_I = 0, intra_H = 0, intra_level = 0;
    float inter_base = 0.0f;
    int nlog = 0, nexp = 0;
    std::vector<Slot> slots;
    std::deque<Job> jobs;
    MvCoder mvc;
    std::shared_ptr<ThreadPool> pool;       // coefficient modelling (shared by the clips of a batch)
    std::unique_ptr<ThreadPool> mv_exec;    // one thread: MV coding strictly in frame order
    std::unique_ptr<ThreadPool> mv_prep;    // one thread: MV symbol listing strictly in frame order
    std::unique_ptr<ThreadPool> mv_asm;     // one thread: the MV coder's input of each P-frame
    std::shared_ptr<ThreadPool> mv_pool;    // rANS batches of the MV coder (shared by the clips of a batch)
    std::shared_ptr<ThreadPool> rans_pool;  // coefficient-coder jobs (never wait)
    BatchSubmit rans_submit;
    BatchSubmit rans_submit_urgent;  // rans_pool, ahead of queued batches (a drain's last frame)
    BatchSubmit mv_submit;  // mv_pool: the MV coder is serial across frames, its batches wait for no bulk work
    int rans_parts = 1;  // threads that code one frame's coefficients: rans_pool's and the caller
    bool draining = false;  // inside drain_all: the newest frame is coded by rans_parts threads
    bool batched = false;   // a clip of a riv_batch: only the batch submits its frames
    double host_ms[6] = {0};  // submit, retire, mv coding, dct coding (summed), write, blocked
    // RIV_TRACE=<file>: every written frame's host timeline (Job::tr), appended to the file as
    // CSV when the encoder is freed
    std::string trace_path;
    std::vector<std::array<double, 11>> trace;
    std::mutex stat_mu;
    float last_times[NSTAGE + 1] = {0};
    bool have_times = false;
    riv_frame_stats last_stats{};
    double sum_times[NSTAGE + 1] = {0};
    size_t coef_guess = 0;  // bytes of coefficients copied eagerly per frame
    DevBuf prof;            // optional per-MB phase stamps of the search kernel
    DevBuf tflag;           // fused table: per-MB "table row written" flags (frame tag)
    DevBuf rowdone;         // AQ inside the search: per-row "ln variances written" flags (frame tag)
    uint64_t h2d_bytes = 0, d2h_bytes = 0, pframes = 0, launches = 0, pdeferred = 0, ptimed = 0;
    // learned / parallel forms: the proposal network's parameters (bf16 weights, f32 biases),
    // its activations, the per-MB search result and the fallback / shortcut counters
    bool learned = false, nn_loaded = false;
    DevBuf nn_w, nn_b, nn_feat, nn_a1, nn_a2, nn_a3, nn_x1, nn_h1, nn_h2, nn_o[2], lmv, lcount, lrowcnt;
    uint64_t learned_mbs = 0;
    // The network of P-frame t runs on its own stream N while frame t-1 is still searched,
    // reconstructed and deblocked: its inputs are the converted input planes of frames t and
    // t-1 and the coded MVs of frame t-2, none of which frame t-1's work changes.  Its output
    // is double-buffered (by frame parity); the search of frame t waits for ev_net_out[t & 1],
    // the network of frame t+2 for ev_net_read[t & 1] (the search that read it), and the
    // conversion into cur[k] for ev_net_cur[k] (the last network that read cur[k]).
    cudaStream_t N = nullptr;
    cudaEvent_t ev_net_out[2] = {}, ev_net_read[2] = {}, ev_net_cur[NPAR] = {};
    bool has_prev2_mvs = false;  // the frame two back was a P-frame (its coded MVs are in coded[coded_cur ^ 1])
    uint64_t nn_frames = 0;
};

namespace {

static riv_status fail(riv_encoder* e, riv_status s, const std::string& msg) {
    e->err = msg;
    if (s == RIV_ERR_CUDA || s == RIV_ERR_DEVICE_TIMEOUT) {
        e->poisoned = true;
        e->poison_msg = msg;
    }
    return s;
}
// A failure that leaves the pipeline unusable (a device failure, or an exception from a
// coder where the reference panics): later calls report it instead of running on.
static riv_status fail_poison(riv_encoder* e, riv_status s, const std::string& msg) {
    e->poisoned = true;
    e->poison_msg = msg;
    e->err = msg;
    return s;
}
static riv_status poisoned_status(riv_encoder* e) {
    e->err = "encoder unusable after an earlier failure: " + e->poison_msg;
    return RIV_ERR_ENCODING_FAILED;
}

static riv_status validate(const riv_config& c, std::string& msg) {  // enc/config.rs:129-164
    if (c.display_width == 0 || c.display_height == 0) { msg = "Width and height must be greater than 0"; return RIV_ERR_INVALID_CONFIG; }
    if (c.storage_width < c.display_width || c.storage_height < c.display_height) {
        msg = "Storage dimensions must be >= display dimensions";
        return RIV_ERR_INVALID_CONFIG;
    }
    if (c.fps == 0) { msg = "FPS must be greater than 0"; return RIV_ERR_INVALID_CONFIG; }
    if (c.search_range > 127) { msg = "search_range must be <= 127 for current MV encoding"; return RIV_ERR_INVALID_CONFIG; }
    if (c.mv_deflate_level > 10) { msg = "mv_deflate_level must be in 0..=10"; return RIV_ERR_INVALID_CONFIG; }
    if (c.keyframe_mode == RIV_KEYFRAME_FIXED && c.keyframe_interval == 0) {
        msg = "Keyframe interval must be greater than 0";
        return RIV_ERR_INVALID_CONFIG;
    }
    if (c.keyframe_mode > 2) { msg = "unknown keyframe mode"; return RIV_ERR_INVALID_CONFIG; }
    if (c.storage_width % 16 || c.storage_height % 16) { msg = "storage dimensions must be multiples of 16"; return RIV_ERR_INVALID_CONFIG; }
    if (c.encode_form > RIV_FORM_PARALLEL) { msg = "unknown encode_form"; return RIV_ERR_INVALID_CONFIG; }
    if (c.encode_form != RIV_FORM_PLAIN && c.search_range > 63) {
        msg = "the learned and parallel forms need search_range <= 63";
        return RIV_ERR_INVALID_CONFIG;
    }
    return RIV_OK;
}

static void setup_device(riv_encoder* e) {
    const riv_config& c = e->cfg;
    CK(cudaSetDevice(c.device));
    e->W = (int)c.storage_width; e->H = (int)c.storage_height;
    e->BW = e->W / 16; e->BH = e->H / 16; e->NMB = e->BW * e->BH;
    e->yuv_bytes = (size_t)e->W * e->H * 3 / 2;
    CK(cudaStreamCreateWithFlags(&e->S, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&e->C, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&e->Hs, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&e->Y, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&e->K, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&e->N, cudaStreamNonBlocking));
    for (int k = 0; k < 2; k++) {
        CK(cudaEventCreateWithFlags(&e->ev_net_out[k], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&e->ev_net_read[k], cudaEventDisableTiming));
    }
    for (int k = 0; k < NPAR; k++) CK(cudaEventCreateWithFlags(&e->ev_net_cur[k], cudaEventDisableTiming));
    for (int k = 0; k < NPAR; k++) {
        CK(cudaEventCreateWithFlags(&e->ev_cur_free[k], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&e->ev_mbout_free[k], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&e->ev_coef_free[k], cudaEventDisableTiming));
    }
    CK(cudaEventCreateWithFlags(&e->ev_search_done, cudaEventDisableTiming));
    int32_t t16[256], t8[64];
    dct_tables(t16, t8);
    CK(riv_upload_dct_tables(t16, t8));
    const int N = e->NMB;
    e->ref[0].alloc(e->yuv_bytes);
    e->ref[1].alloc(e->yuv_bytes);
    e->recon_pre.alloc(e->yuv_bytes);  // reconstruction before the (out-of-place) deblock
    e->coded[0].alloc((size_t)N * 4);
    e->coded[1].alloc((size_t)N * 4);
    e->rec.alloc((size_t)2 * N * sizeof(MbRec));  // raw-MV records, then coded-MV records
    e->varsum.alloc((size_t)N * sizeof(uint2));
    e->qs.alloc((size_t)N * sizeof(float));
    for (int k = 0; k < NPAR; k++) {  // per frame: the next frame's launch may still reconstruct this one
        e->curb[k].alloc(e->yuv_bytes);
        e->predb[k].alloc(e->yuv_bytes);
        e->mboutb[k].alloc((size_t)N * sizeof(MbOut));
        e->lnvb[k].alloc((size_t)(N + 4) * sizeof(float));
        e->coeffsb[k].alloc((size_t)N * 384 * sizeof(int16_t));
        e->optskipb[k].alloc(N);
        e->fmaskb[k].alloc(N);
        e->eobsb[k].alloc((size_t)N * 3);
    }
    e->wq_words = 2 + 2 * e->BH;
    e->wq.alloc((size_t)2 * e->wq_words * sizeof(unsigned));  // two queue arrays, alternating per launch
    e->wq.zero(e->S);
    e->status.alloc(sizeof(unsigned));
    e->rec.zero(e->S);
    e->status.zero(e->S);
    // search cost tables (enc/motion/scalar.rs:503-541): b(0)=1, b(d)=2*log2(d)+2
    double bits[256];
    bits[0] = 1.0;
    for (int d = 1; d < 256; d++) bits[d] = 2.0 * log2((double)d) + 2.0;
    e->mvbits.alloc(sizeof(bits));
    CK(cudaMemcpy(e->mvbits.p, bits, sizeof(bits), cudaMemcpyHostToDevice));
    {
        // NEW-mode cost table: (lambda * 2.0 * (6.0 + bx + by)) as i64 (enc/motion/scalar.rs:503-541)
        Lambda Lq = lambda_for(c.inter_quality, c.rdo_lambda_mult);
        std::vector<long long> nt(256 * 256);
        long long mx = 0;
        for (int a = 0; a < 256; a++)
            for (int b = 0; b < 256; b++) {
                long long v = f64_as_i64(Lq.lambda * 2.0 * (6.0 + bits[a] + bits[b]));
                nt[a * 256 + b] = v;
                mx = std::max<long long>(mx, v);
            }
        mx = std::max<long long>(mx, f64_as_i64(Lq.lambda * 2.0 * 1.5));
        e->table_ok = search_use_table(c.search_range) && mx < (1ll << 58) && Lq.lambda >= 0.0;
        e->newcost.alloc(nt.size() * sizeof(long long));
        CK(cudaMemcpy(e->newcost.p, nt.data(), nt.size() * sizeof(long long), cudaMemcpyHostToDevice));
        e->small_costs = mx < (1ll << 27) && Lq.lambda >= 0.0;
        if (const char* v = getenv("RIV_SEARCH_SMALL")) e->small_costs = e->small_costs && atoi(v) != 0;
        std::vector<int> n32(64 * 64);
        for (int a = 0; a < 64; a++)
            for (int b = 0; b < 64; b++) n32[a * 64 + b] = (int)std::min<long long>(nt[a * 256 + b], INT32_MAX);
        e->newcost32.alloc(n32.size() * sizeof(int));
        CK(cudaMemcpy(e->newcost32.p, n32.data(), n32.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    LibmFix& F = libm_fix();
    if (!F.ok) throw std::runtime_error("glibc fix-up table: " + F.err);
    e->nlog = (int)(F.logf.size() / 2);
    e->nexp = (int)(F.exp2f.size() / 2);
    e->logfix.alloc(F.logf_dev.size() * 4);
    e->expfix.alloc(F.exp2f_dev.size() * 4);
    CK(cudaMemcpy(e->logfix.p, F.logf_dev.data(), F.logf_dev.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(e->expfix.p, F.exp2f_dev.data(), F.exp2f_dev.size() * 4, cudaMemcpyHostToDevice));
    uint16_t yt[256], ct[64];
    intra_tables(quant_step(c.intra_quality), yt, ct);
    e->ytab.alloc(sizeof(yt));
    e->ctab.alloc(sizeof(ct));
    CK(cudaMemcpy(e->ytab.p, yt, sizeof(yt), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(e->ctab.p, ct, sizeof(ct), cudaMemcpyHostToDevice));
    CK(search_plan(c.search_range, (int)c.storage_width, e->BH, e->table_ok, e->small_costs, &e->splan));
    if (e->splan.grid <= 0) throw std::runtime_error("search kernel cannot be made resident");
    // P-frame reconstruction folded into the next P-frame's search launch (its worker CTAs)
    e->learned = c.encode_form != RIV_FORM_PLAIN;
    e->defer_ok = !e->learned && e->splan.fused && e->splan.fast && e->table_ok && c.pipeline_depth > 1;
    if (e->learned) {
        e->lmv.alloc((size_t)N * 8);
        e->lcount.alloc(2 * sizeof(unsigned));
        e->lcount.zero(e->S);
        e->lrowcnt.alloc((size_t)e->BH * sizeof(unsigned));
        e->lrowcnt.zero(e->S);
    }
    if (c.encode_form == RIV_FORM_LEARNED) {
        e->nn_w.alloc(nn::ParamLayout::nweights * 2);
        e->nn_b.alloc(nn::ParamLayout::nbias * 4);
        e->nn_feat.alloc((size_t)N * nn::FEAT * nn::FEAT * 2 * 2);
        e->nn_a1.alloc((size_t)N * 144 * 32 * 2);
        e->nn_a2.alloc((size_t)N * 36 * 32 * 2);
        e->nn_a3.alloc((size_t)N * 36 * 32 * 2);
        e->nn_x1.alloc((size_t)N * nn::F1 * 2);
        e->nn_h1.alloc((size_t)N * nn::HID * 2);
        e->nn_h2.alloc((size_t)N * nn::HID * 2);
        e->nn_o[0].alloc((size_t)N * nn::OUT * 4);
        e->nn_o[1].alloc((size_t)N * nn::OUT * 4);
    }
    if (e->splan.fused) {
        e->tflag.alloc((size_t)N * sizeof(unsigned));
        e->tflag.zero(e->S);
    }
    if (e->splan.fast) {
        e->rowdone.alloc((size_t)e->BH * sizeof(unsigned));
        e->rowdone.zero(e->S);
    }
    // frame constants
    e->L = lambda_for(c.inter_quality, c.rdo_lambda_mult);
    e->inter_base = quant_step(c.inter_quality);
    e->inter_level = deblock_level(quant_step(c.inter_quality));
    deblock_thresholds(e->inter_level, false, e->inter_E, e->inter_I, e->inter_H);
    e->intra_level = deblock_level(quant_step(c.intra_quality));
    deblock_thresholds(e->intra_level, true, e->intra_E, e->intra_I, e->intra_H);
    // pipeline slots
    int nslots = std::max(1u, c.pipeline_depth);
    e->slots.resize(nslots);
    size_t rgb_bytes = (size_t)c.display_width * c.display_height * 3;
    for (auto& s : e->slots) {
        s.rgb.alloc(std::max(rgb_bytes, e->yuv_bytes));
        s.dside.alloc((size_t)N * 4);
        s.dpacked.alloc((size_t)N * 384 * 2);
        s.dpeobs.alloc((size_t)N * 3);
        s.side.alloc((size_t)N * 4);
        s.packed.alloc((size_t)N * 384 * 2);
        s.peobs.alloc((size_t)N * 3);
        s.hdr.alloc(16);
        CK(cudaEventCreateWithFlags(&s.ev_h2d, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&s.ev_gpu, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&s.ev_d2h, cudaEventDisableTiming));
        for (int k = 0; k < EV_N; k++) CK(cudaEventCreate(&s.ev_k[k]));
        CK(cudaEventCreateWithFlags(&s.ev_yuv, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&s.ev_recon, cudaEventDisableTiming));
    }
    e->coef_guess = (size_t)N * 384;  // half the dense size until the first frames are seen
    if (getenv("RIV_PROFILE_SEARCH")) {
        e->prof.alloc((size_t)N * RIV_PROF_WORDS * sizeof(long long));
        e->prof.zero(e->S);
    }
    e->cindex.alloc((size_t)N * 4);
    e->coffset.alloc((size_t)N * 4);
    e->lcindex.alloc((size_t)N * 4);
    e->lcoffset.alloc((size_t)N * 4);
    if (e->table_ok)
        e->sadtab.alloc((size_t)N * sad_table_stride(c.search_range) * sizeof(uint16_t));
    // default: half the host's threads model coefficients (a frame models on one, so this is
    // several frames at once) and as many code their rANS batches; both run below the serial
    // stages (submission, MV listing and coding)
    unsigned nt = c.entropy_threads;
    if (nt == 0) nt = std::max(2u, std::min(16u, std::thread::hardware_concurrency() / 2));
    e->pool.reset(new ThreadPool(nt, BULK_NICE));
    e->mv_exec.reset(new ThreadPool(1));
    e->mv_prep.reset(new ThreadPool(1));
    e->mv_asm.reset(new ThreadPool(1));
    e->mv_pool.reset(new ThreadPool(2));
    e->rans_pool.reset(new ThreadPool(nt, BULK_NICE));
    e->rans_parts = (int)nt + 1;
    if (const char* v = getenv("RIV_TRACE")) e->trace_path = v;
    {
        ThreadPool* rp = e->rans_pool.get();
        e->rans_submit = [rp](std::function<void()> f) { return rp->submit(std::move(f)); };
        e->rans_submit_urgent = [rp](std::function<void()> f) { return rp->submit(std::move(f), true); };
        ThreadPool* mp = e->mv_pool.get();
        e->mv_submit = [mp](std::function<void()> f) { return mp->submit(std::move(f)); };
    }
    CK(cudaStreamSynchronize(e->S));
}

// Stage marks.  Timing-enabled events between back-to-back cooperative launches cost a few
// microseconds of idle GPU each, so the stage timing events are recorded on sampled frames
// only; the two marks other streams depend on also record a non-timing event every frame.
static void mark(riv_encoder* e, const Job& j, int k, cudaStream_t st) {
    Slot& s = e->slots[j.slot];
    if (j.timed) CK(cudaEventRecord(s.ev_k[k], st));
    if (k == EV_YUV) CK(cudaEventRecord(s.ev_yuv, st));
    if (k == EV_DEBLOCK) CK(cudaEventRecord(s.ev_recon, st));
}

static Job* find_job(riv_encoder* e, uint64_t index) {
    for (auto& j : e->jobs)
        if (j.index == index) return &j;
    return nullptr;
}

// Compaction of a frame whose reconstruction is enqueued (it waits for the frame's
// EV_DEBLOCK; `compacted`: the search launch that reconstructed it compacted it too), then
// the status and the device->host copies of its side info and coefficients.
static void frame_tail(riv_encoder* e, Job& j, bool compacted = false) {
    Slot& s = e->slots[j.slot];
    const int N = e->NMB, ck = j.ck;
    cudaStream_t K = e->K;
    CK(cudaStreamWaitEvent(K, s.ev_recon, 0));
    mark(e, j, EV_K0, K);
    if (!compacted) {
        e->launches += 2;  // scan + pack
        CK(launch_compact(e->optskipb[ck].as<uint8_t>(), e->mboutb[ck].as<MbOut>(), e->coeffsb[ck].as<int16_t>(),
                          e->eobsb[ck].as<uint8_t>(), N, j.type == 1 ? 1 : 0, e->cindex.as<int32_t>(),
                          e->coffset.as<int32_t>(), s.dside.as<uint32_t>(), s.dpacked.as<int16_t>(),
                          s.dpeobs.as<uint8_t>(), s.hdr.dev<uint32_t>(), K));
    }
    CK(cudaEventRecord(e->ev_coef_free[ck], K));
    CK(cudaEventRecord(e->ev_mbout_free[ck], K));
    mark(e, j, EV_COMPACT, K);
    CK(cudaMemcpyAsync(s.hdr.host<uint32_t>() + 2, e->status.p, 4, cudaMemcpyDeviceToHost, K));
    CK(cudaEventRecord(s.ev_gpu, K));
    // DMA the side info, EOBs and (a bounded prefix of) the coefficients on the copy
    // stream; the exact size is only known once the frame is done.
    CK(cudaStreamWaitEvent(e->C, s.ev_gpu, 0));
    CK(cudaMemcpyAsync(s.side.p, s.dside.p, (size_t)N * 4, cudaMemcpyDeviceToHost, e->C));
    CK(cudaMemcpyAsync(s.peobs.p, s.dpeobs.p, (size_t)N * 3, cudaMemcpyDeviceToHost, e->C));
    s.prefetched = std::min(e->coef_guess, (size_t)N * 384 * 2);
    CK(cudaMemcpyAsync(s.packed.p, s.dpacked.p, s.prefetched, cudaMemcpyDeviceToHost, e->C));
    CK(cudaEventRecord(s.ev_d2h, e->C));
    j.tail_done = true;
}

// Residual and deblock of a frame as separate kernels on S, then its tail.
static void reconstruct_now(riv_encoder* e, Job& j, const ResidualParams& rp, int level, int E, int I, int Hv,
                            const uint8_t* mask, uint8_t* recon) {
    Slot& s = e->slots[j.slot];
    cudaStream_t S = e->S;
    CK(cudaStreamWaitEvent(S, e->ev_coef_free[j.ck], 0));  // compaction of the frame NPAR back
    e->launches += 1 + (level > 0 ? 1 : 0);
    CK(launch_residual(rp, e->NMB, S));
    mark(e, j, EV_RES, S);
    CK(cudaEventRecord(e->ev_cur_free[j.ck], S));
    if (level > 0) CK(launch_deblock_tiled(e->recon_pre.as<uint8_t>(), recon, e->W, e->H, E, I, Hv, mask, S));
    mark(e, j, EV_DEBLOCK, S);
    frame_tail(e, j);
}

// Run the pending frame's reconstruction now (separate kernels), when no later launch will.
static void flush_pending(riv_encoder* e) {
    if (!e->pend.active) return;
    Job* j = find_job(e, e->pend.index);
    e->pend.active = false;
    if (!j) return;
    j->deferred = false;
    reconstruct_now(e, *j, e->pend.rp, e->pend.level, e->inter_E, e->inter_I, e->inter_H,
                    e->fmaskb[e->pend.ck].as<uint8_t>(), e->pend.recon);
}

// The proposal network over every MB of a P-frame (learned form): network input, four
// convolutions (implicit GEMM on tcgen05) and the three fully connected layers (TMA-fed
// tcgen05 GEMMs), leaving 16 outputs per MB in nn_o.  Expired device waits set bit 0 of the
// status word (RIV_ERR_DEVICE_TIMEOUT).
static void proposal_forward(riv_encoder* e, const uint8_t* cur_y, const uint8_t* ref_y, const int8_t* prev_coded,
                             void* out, cudaStream_t S) {
    using PL = nn::ParamLayout;
    const int N = e->NMB;
    const uint16_t* W = e->nn_w.as<uint16_t>();
    const float* B = e->nn_b.as<float>();
    unsigned* err = e->status.as<unsigned>();
    void *feat = e->nn_feat.p, *a1 = e->nn_a1.p, *a2 = e->nn_a2.p, *a3 = e->nn_a3.p, *x1 = e->nn_x1.p;
    // network input and conv1 in one kernel (the input stays on chip), then conv2..4 and fc1..3
    (void)feat;
    CK((cudaError_t)riv_nn_front(cur_y, ref_y, e->W, e->H, prev_coded, 0, N, W + PL::w1, B, a1, x1, S));
    CK((cudaError_t)nn_conv(2, a1, 144 * 32, W + PL::w2, B + 32, a2, 36 * 32, 32, N, err, S));
    CK((cudaError_t)nn_conv(3, a2, 36 * 32, W + PL::w3, B + 64, a3, 36 * 32, 32, N, err, S));
    CK((cudaError_t)nn_conv(4, a3, 36 * 32, W + PL::w4, B + 96, x1, nn::F1, 32, N, err, S));
    CK((cudaError_t)nn_gemm(x1, nn::F1, W + PL::f1, nn::F1, e->nn_h1.p, nn::HID, B + 128, N, nn::HID, nn::F1, 64, 2, 1,
                            1, nn::HID, err, S));
    CK((cudaError_t)nn_gemm(e->nn_h1.p, nn::HID, W + PL::f2, nn::HID, e->nn_h2.p, nn::HID, B + 256, N, nn::HID, nn::HID,
                            64, 2, 1, 1, nn::HID, err, S));
    CK((cudaError_t)nn_gemm(e->nn_h2.p, nn::HID, W + PL::f3, nn::HID, out, nn::OUT, B + 384, N, nn::OUT, nn::HID,
                            64, 0, 0, 1, nn::OUT, err, S));
}

// The search parameters of a P-frame of `e` (current planes `cur`, per-MB output `mbo`) against
// its last reconstruction, with a new frame tag; the caller sets the table, AQ, worker-queue
// and launch-shape fields.
static void frame_search_params(riv_encoder* e, const uint8_t* cur, MbOut* mbo, SearchParams& sp) {
    const riv_config& c = e->cfg;
    sp.ref_y = e->ref[e->ref_cur].as<uint8_t>();
    sp.cur_y = cur;
    sp.W = e->W; sp.H = e->H; sp.BW = e->BW; sp.BH = e->BH; sp.sr = c.search_range;
    sp.prev_coded = e->has_prev_mvs ? e->coded[e->coded_cur].as<int8_t>() : nullptr;
    sp.zthr = c.me_zero_mv_threshold;
    sp.pthr = c.me_predictor_threshold;
    double lam = e->L.lambda;
    sp.lam2 = lam * 2.0;
    sp.c15 = f64_as_i64(lam * 2.0 * 1.5);
    sp.c05 = f64_as_i64(lam * 2.0 * 0.5);
    sp.lambda_zero = lam == 0.0;
    sp.mvbits = e->mvbits.as<double>();
    sp.newcost = e->newcost.as<long long>();
    sp.newcost32 = e->newcost32.as<int>();
    sp.small = e->small_costs ? 1 : 0;
    sp.rdo_lambda = lam;
    sp.rdo_skip_bits = e->L.skip_bits;
    sp.rdo_keep_bits = e->L.keep_bits;
    sp.rdo_icpt = e->L.icpt;
    sp.rdo_slope = e->L.slope;
    sp.rdo_ret = e->L.ret;
    sp.rdo_guard = 768.0 * (double)c.skip_threshold;
    sp.rdo_allow = c.skip_threshold > 0;
    sp.rec = e->rec.as<MbRec>();
    e->tag = (e->tag + 1) & 0xffffu;
    if (e->tag == 0) e->tag = 1;
    sp.tag = e->tag;
    sp.out = mbo;
    sp.status = e->status.as<unsigned>();
    sp.spin_limit = 1ll << 22;  // ~ a few seconds, far above any legitimate wait
}

// Enqueue the GPU work of one frame.  `src` = 0 host RGB, 1 device RGB, 2 host YUV.
static void submit_gpu(riv_encoder* e, Job& j, int src, const void* a, const void* b, const void* c3) {
    const riv_config& c = e->cfg;
    Slot& s = e->slots[j.slot];
    const int W = e->W, H = e->H, N = e->NMB;
    cudaStream_t S = e->S, Y = e->Y;
    const int ck = e->fpar;  // this frame's input planes and per-MB output buffers
    j.ck = ck;
    uint8_t* cur = e->curb[ck].as<uint8_t>();
    MbOut* mbo = e->mboutb[ck].as<MbOut>();
    const bool defer_this = j.type == 2 && e->defer_ok;
    if (j.type == 1) flush_pending(e);  // key frames reconstruct immediately
    // kernels per frame: rgb->yuv, (search, predict, 3 x aq), residual, deblock, scan + pack
    const int p_launches = e->learned ? (c.encode_form == RIV_FORM_LEARNED ? 8 : 0) + 3
                                      : 1 + (e->table_ok && !e->splan.fused ? 1 : 0) + (e->splan.fast && e->table_ok ? 0 : 4);
    e->launches += (src == 2 ? 0 : 1) + (j.type == 2 ? p_launches : 0);  // + residual / deblock / compaction below
    if (src == 0) e->h2d_bytes += (uint64_t)c.display_width * c.display_height * 3;
    if (src == 2) e->h2d_bytes += e->yuv_bytes;
    // ---- input conversion on Y, overlapping the previous frame's main chain; cur[ck] is
    // free once the residual of the frame NPAR back has read it
    CK(cudaStreamWaitEvent(Y, e->ev_cur_free[ck], 0));
    if (e->learned) CK(cudaStreamWaitEvent(Y, e->ev_net_cur[ck], 0));
    // without deferral: after the previous search launch, i.e. beside that frame's residual;
    // with it the conversion runs in the gap between two launches, one frame ahead
    if (!e->defer_ok) CK(cudaStreamWaitEvent(Y, e->ev_search_done, 0));
    if (src == 0) {
        CK(cudaMemcpyAsync(s.rgb.p, a, (size_t)c.display_width * c.display_height * 3, cudaMemcpyHostToDevice, e->Hs));
        CK(cudaEventRecord(s.ev_h2d, e->Hs));
        CK(cudaStreamWaitEvent(Y, s.ev_h2d, 0));
        mark(e, j, EV_START, Y);
        CK(launch_rgb_to_yuv((const uint8_t*)s.rgb.p, (int)c.display_width, (int)c.display_height, cur, W, H, Y, e->defer_ok));
    } else if (src == 1) {
        mark(e, j, EV_START, Y);
        CK(launch_rgb_to_yuv((const uint8_t*)a, (int)c.display_width, (int)c.display_height, cur, W, H, Y, e->defer_ok));
    } else {
        uint8_t* d = s.rgb.as<uint8_t>();
        size_t ys = (size_t)W * H, cs = ys / 4;
        CK(cudaMemcpyAsync(d, a, ys, cudaMemcpyHostToDevice, e->Hs));
        CK(cudaMemcpyAsync(d + ys, b, cs, cudaMemcpyHostToDevice, e->Hs));
        CK(cudaMemcpyAsync(d + ys + cs, c3, cs, cudaMemcpyHostToDevice, e->Hs));
        CK(cudaEventRecord(s.ev_h2d, e->Hs));
        CK(cudaStreamWaitEvent(Y, s.ev_h2d, 0));
        mark(e, j, EV_START, Y);
        CK(cudaMemcpyAsync(cur, d, e->yuv_bytes, cudaMemcpyDeviceToDevice, Y));
    }
    mark(e, j, EV_YUV, Y);
    // ---- main chain on S
    CK(cudaStreamWaitEvent(S, s.ev_yuv, 0));
    mark(e, j, EV_S0, S);
    const int nxt = e->ref_cur ^ 1;
    uint8_t* recon = e->ref[nxt].as<uint8_t>();
    ResidualParams rp{};
    rp.cur = cur;
    rp.pred = e->predb[ck].as<uint8_t>();
    rp.recon = recon;  // or recon_pre when a deblock follows (set per frame type below)
    rp.coeffs = e->coeffsb[ck].as<int16_t>();
    rp.opt_skip = e->optskipb[ck].as<uint8_t>();
    rp.fmask = e->fmaskb[ck].as<uint8_t>();
    rp.eobs = e->eobsb[ck].as<uint8_t>();
    rp.dead_zone = c.inter_dead_zone;
    rp.W = W; rp.H = H; rp.BW = e->BW;
    if (j.type == 1) {
        rp.intra = 1;
        rp.intra_ytab = e->ytab.as<uint16_t>();
        rp.intra_ctab = e->ctab.as<uint16_t>();
        mark(e, j, EV_TABLE, S);
        mark(e, j, EV_SEARCH, S);
        mark(e, j, EV_PRED, S);
        mark(e, j, EV_AQ, S);
        if (e->intra_level > 0) rp.recon = e->recon_pre.as<uint8_t>();
        reconstruct_now(e, j, rp, e->intra_level, e->intra_E, e->intra_I, e->intra_H, nullptr, recon);
        e->has_prev_mvs = false;
        e->has_prev2_mvs = false;
    } else {
        SearchParams sp{};
        frame_search_params(e, cur, mbo, sp);
        sp.tab = nullptr;
        sp.tstride = 0;
        sp.tflag = nullptr;
        sp.wq = e->wq.as<unsigned>() + (size_t)e->wq_par * e->wq_words;
        sp.wq_next = e->wq.as<unsigned>() + (size_t)(e->wq_par ^ 1) * e->wq_words;
        sp.wq_words = e->wq_words;
        const int nbuf = (int)(e->nn_frames & 1);
        if (e->learned && c.encode_form == RIV_FORM_LEARNED) {
            // stage 1 of the learned form: the network, on stream N (see riv_encoder::N)
            if (!e->nn_loaded) throw std::runtime_error("learned form: no proposal network loaded (riv_encoder_set_proposal)");
            cudaStream_t Nn = e->N;
            CK(cudaStreamWaitEvent(Nn, s.ev_yuv, 0));                // this frame's planes converted
            CK(cudaStreamWaitEvent(Nn, e->ev_net_read[nbuf], 0));    // the search two frames back read nn_o[nbuf]
            if (j.timed) CK(cudaEventRecord(s.ev_k[EV_NET0], Nn));
            proposal_forward(e, cur, e->curb[e->last_par].as<uint8_t>(),
                             e->has_prev2_mvs ? e->coded[e->coded_cur ^ 1].as<int8_t>() : nullptr, e->nn_o[nbuf].p, Nn);
            if (j.timed) CK(cudaEventRecord(s.ev_k[EV_NET1], Nn));
            CK(cudaEventRecord(e->ev_net_out[nbuf], Nn));
            CK(cudaEventRecord(e->ev_net_cur[e->last_par], Nn));     // cur of the previous frame read
            CK(cudaStreamWaitEvent(S, e->ev_net_out[nbuf], 0));
        }
        if (e->table_ok && !e->learned) {
            sp.tstride = sad_table_stride(c.search_range);
            sp.tab = e->sadtab.as<uint16_t>();
            if (e->splan.fused) sp.tflag = e->tflag.as<unsigned>();  // computed inside the search launch
            else CK(launch_sad_table(sp.ref_y, sp.cur_y, W, H, c.search_range, e->sadtab.as<uint16_t>(), sp.tstride, S));
        }
        mark(e, j, EV_TABLE, S);
        sp.prof = e->prof.as<long long>();
        // coded MVs of this frame become next frame's temporal predictors
        const int cn = e->coded_cur ^ 1;
        sp.coded_out = e->coded[cn].as<int8_t>();
        // prediction, variances and ln inside the search launch (plain fused form), or inside the
        // learned forms' parallel search (their launch also folds the mean)
        const bool aq_in_search = (e->splan.fast && e->table_ok) || e->learned;
        if (aq_in_search) {  // prediction, variances and ln inside the search launch
            sp.pred = e->predb[ck].as<uint8_t>();
            sp.varsum = e->varsum.as<uint2>();
            sp.lnv = e->lnvb[ck].as<float>();
            sp.row_done = e->rowdone.as<unsigned>();
            sp.logfix = e->logfix.as<uint32_t>();
            sp.nlog = e->nlog;
        }
        // the pending frame's residual and deblock run inside this launch
        Job* pj = e->pend.active ? find_job(e, e->pend.index) : nullptr;
        if (pj) {
            sp.defer = 1;
            sp.dres = e->pend.rp;
            sp.db_level = e->pend.level;
            sp.db_E = e->inter_E; sp.db_I = e->inter_I; sp.db_H = e->inter_H;
            sp.db_src = e->recon_pre.as<uint8_t>();
            sp.db_dst = e->pend.recon;
            sp.db_mask = e->fmaskb[e->pend.ck].as<uint8_t>();
            Slot& ps = e->slots[pj->slot];  // its compaction at the end of the queue
            sp.compact = 1;
            sp.c_index = e->lcindex.as<int32_t>();
            sp.c_offset = e->lcoffset.as<int32_t>();
            sp.c_side = ps.dside.as<uint32_t>();
            sp.c_packed = ps.dpacked.as<int16_t>();
            sp.c_peobs = ps.dpeobs.as<uint8_t>();
            sp.c_hdr = ps.hdr.dev<uint32_t>();
            CK(cudaStreamWaitEvent(S, e->ev_coef_free[e->pend.ck], 0));  // compaction of the frame NPAR back
        }
        e->pend.active = false;
        CK(cudaStreamWaitEvent(S, e->ev_mbout_free[ck], 0));  // compaction of the frame NPAR back
        if (e->learned) {
            CK((cudaError_t)launch_learned(sp, c.encode_form == RIV_FORM_LEARNED ? e->nn_o[nbuf].as<float>() : nullptr,
                                           (int)c.proposal_margin, 2.2f, e->lmv.p, e->lcount.as<unsigned>(),
                                           e->lrowcnt.as<unsigned>(), S));
            CK(cudaEventRecord(e->ev_net_read[nbuf], S));
            e->nn_frames++;
            e->learned_mbs += (uint64_t)N;
        } else {
            CK(launch_search(sp, e->splan, S));
        }
        e->wq_par ^= 1;
        mark(e, j, EV_SEARCH, S);
        CK(cudaEventRecord(e->ev_search_done, S));
        if (pj) {  // the pending frame is reconstructed: its compaction and copies follow
            Slot& ps = e->slots[pj->slot];
            CK(cudaEventRecord(e->ev_cur_free[pj->ck], S));
            mark(e, *pj, EV_DEBLOCK, S);
            frame_tail(e, *pj, true);
        }
        if (!aq_in_search)
            CK(launch_predict(e->ref[e->ref_cur].as<uint8_t>(), mbo, e->predb[ck].as<uint8_t>(), e->varsum.as<uint2>(), W,
                              H, S));
        mark(e, j, EV_PRED, S);
        if (!aq_in_search)
            CK(launch_aq(e->varsum.as<uint2>(), N, e->inter_base, e->logfix.as<uint32_t>(), e->nlog, e->expfix.as<uint32_t>(),
                         e->nexp, e->lnvb[ck].as<float>(), e->qs.as<float>(), S));
        mark(e, j, EV_AQ, S);
        if (aq_in_search) {  // the residual derives the steps from the ln variances and their mean
            rp.lnv = e->lnvb[ck].as<float>();
            rp.aq_base = e->inter_base;
            rp.expfix = e->expfix.as<uint32_t>();
            rp.nexp = e->nexp;
            rp.qs_out = e->qs.as<float>();
            rp.ref = e->ref[e->ref_cur].as<uint8_t>();  // chroma prediction in the residual kernel
        }
        rp.intra = 0;
        rp.mb = mbo;
        rp.qs = e->qs.as<float>();
        if (e->inter_level > 0) rp.recon = e->recon_pre.as<uint8_t>();
        if (defer_this) {  // reconstructed by the next P-frame's launch (or a flush)
            mark(e, j, EV_RES, S);
            e->pend.active = true;
            e->pend.index = j.index;
            e->pend.ck = ck;
            e->pend.level = e->inter_level;
            e->pend.rp = rp;
            e->pend.recon = recon;
            j.tail_done = false;
            j.deferred = true;
        } else {
            reconstruct_now(e, j, rp, e->inter_level, e->inter_E, e->inter_I, e->inter_H, e->fmaskb[ck].as<uint8_t>(),
                            recon);
        }
        e->coded_cur = cn;
        e->has_prev2_mvs = e->has_prev_mvs;
        e->has_prev_mvs = true;
    }
    e->ref_cur = nxt;
    e->has_ref = true;
    e->last_par = ck;
    e->fpar = (ck + 1) % NPAR;
}

// Host part of a frame once its GPU work is done: its side info and coefficients are
// already in mapped host memory.  MV coding goes to the ordered single-thread executor
// (its contexts carry across frames), DCT-coefficient coding to the pool.
static double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
// The per-MB statistics of a P-frame that need its search output (EncodeFrameStats,
// enc/encoder.rs:436-733): RDO telemetry (RdoTelemetry, enc/rdo.rs:195-258), the number of
// distinct predictor candidates (derive_mv_predictors_with_stats, res/mv_predictor.rs:135-163),
// which raw neighbour a non-zero MV repeats (gather_mv_neighbor_set, :59-118) and the
// L1-closest NEW base.  mb: the frame's search output in raster order (raw MV, coded MV, best
// SAD); prev: the previous P-frame's coded MVs (4 bytes per MB) or nullptr.
static void search_stats(const riv_encoder* e, const MbOut* mb, const int8_t* prev, riv_frame_stats& S) {
    const riv_config& c = e->cfg;
    const int bw = e->BW, n = e->NMB;
    const Lambda& L = e->L;
    const bool allow = c.skip_threshold > 0;
    const double guard = 768.0 * (double)c.skip_threshold;
    double tot_skip = 0.0, tot_coded = 0.0;
    uint32_t umin = UINT32_MAX, umax = 0;
    typedef std::array<int, 4> Tup;
    auto coded = [&](int i) { return Tup{mb[i].coded[0], mb[i].coded[1], mb[i].coded[2], mb[i].coded[3]}; };
    for (int i = 0; i < n; i++) {
        const int bx = i % bw, by = i / bw;
        const MbOut& m = mb[i];
        // RdoContext::decide (enc/rdo.rs:140-178) as telemetry
        const double satd = (double)std::max<int32_t>(m.best_sad, 0);
        const double skip_cost = satd + L.lambda * L.skip_bits;
        double est = L.icpt + L.slope * satd;
        if (est < 0.0) est = 0.0;
        const double coded_cost = satd * L.ret + L.lambda * (L.keep_bits + est);
        const bool int_al = m.raw[2] == 0 && m.raw[3] == 0;
        if (!allow) S.rdo_forced_disabled++;
        else if (!int_al) S.rdo_forced_fractional++;
        else if (satd > guard) S.rdo_forced_threshold++;
        else if (skip_cost <= coded_cost) S.rdo_blocks_selected_skip++;
        S.rdo_blocks_evaluated++;
        tot_skip += skip_cost;
        tot_coded += coded_cost;
        // neighbours among the coded MVs of this frame and the previous one
        bool hl = bx > 0, ht = by > 0, htr = by > 0 && bx + 1 < bw, htl = by > 0 && bx > 0, htm = prev != nullptr;
        Tup l{}, t{}, tr{}, tl{}, tm{};
        if (hl) l = coded(i - 1);
        if (ht) t = coded(i - bw);
        if (htr) tr = coded(i - bw + 1);
        if (htl) tl = coded(i - bw - 1);
        if (htm) tm = Tup{prev[4 * i], prev[4 * i + 1], prev[4 * i + 2], prev[4 * i + 3]};
        Tup cand[5];
        int nc = 0;
        auto add = [&](bool has, const Tup& v) {
            if (!has) return;
            for (int k = 0; k < nc; k++)
                if (cand[k] == v) return;
            cand[nc++] = v;
        };
        add(hl, l); add(ht, t); add(htr, tr); add(htl, tl); add(htm, tm);
        const uint32_t unique = nc == 0 ? 1u : (uint32_t)nc;
        S.mv_candidate_unique_total += unique;
        S.mv_candidate_unique_samples++;
        umin = std::min(umin, unique);
        umax = std::max(umax, unique);
        const Tup zero{0, 0, 0, 0};
        const Tup nearest = nc > 0 ? cand[0] : zero, near = nc > 1 ? cand[1] : zero, temporal = htm ? tm : zero;
        const Tup actual{m.raw[0], m.raw[1], m.raw[2], m.raw[3]};
        if (actual != zero) {  // attribution of exact matches to raw neighbours
            S.mv_match_nonzero_blocks++;
            const bool ml = hl && l == actual, mt = ht && t == actual, mtr = htr && tr == actual, mtl = htl && tl == actual,
                       mtm = htm && tm == actual;
            if (ml || mt || mtr || mtl) S.mv_match_any_spatial++;
            if (mtm) S.mv_match_any_temporal++;
            S.mv_match_source_counts[ml ? 0 : mt ? 1 : mtr ? 2 : mtl ? 3 : mtm ? 4 : 5]++;
        }
        if (m.mode == M_NEW) {  // the L1-closest integer base and what it would save over nearest/near
            const int ax = m.raw[0], ay = m.raw[1];
            auto l1 = [&](const Tup& b) { return (uint32_t)(std::abs(ax - b[0]) + std::abs(ay - b[1])); };
            const uint32_t cn = l1(nearest), cr = l1(near);
            const bool has[5] = {true, true, htr, htl, true};
            const uint32_t cost[5] = {cn, cr, htr ? l1(tr) : 0u, htl ? l1(tl) : 0u, l1(temporal)};
            int best = 0;
            uint32_t bc = cn;
            for (int k = 0; k < 5; k++)
                if (has[k] && cost[k] < bc) { bc = cost[k]; best = k; }
            S.mv_new_best_ref_counts[best]++;
            const uint32_t cur = std::min(cn, cr);
            if (bc < cur) S.mv_new_best_ref_l1_saved_sum += cur - bc;
        }
    }
    S.mv_candidate_unique_min = umin == UINT32_MAX ? 0 : umin;
    S.mv_candidate_unique_max = umax;
    S.rdo_avg_skip_cost = S.rdo_blocks_evaluated ? tot_skip / (double)S.rdo_blocks_evaluated : 0.0;
    S.rdo_avg_coded_cost = S.rdo_blocks_evaluated ? tot_coded / (double)S.rdo_blocks_evaluated : 0.0;
}

// The MV coder's input of a P-frame (MvCodedBlock assembly, enc/encoder.rs:774-818) after the
// delta bias (compute_delta_bias_for_new, enc/encoder.rs:984-1048), and the frame's MV
// statistics; none of it depends on the coder's state carried across frames.
static void assemble_mv(riv_encoder* e, Job& j, const uint32_t* side, int N, const std::vector<MbOut>* mbh,
                        const std::vector<int8_t>* prevh) {
    double m0 = now_ms();
    j.tr[1] = m0;
    riv_frame_stats& S = j.stats;
    std::vector<std::pair<int8_t, int8_t>> nd;
    nd.reserve(N);
    for (int i = 0; i < N; i++)
        if ((side[i] & 7) == M_NEW) nd.emplace_back((int8_t)(side[i] >> 8), (int8_t)(side[i] >> 16));
    compute_delta_bias(nd, j.bias[0], j.bias[1]);
    // MvCodedBlock assembly (enc/encoder.rs:774-818)
    std::vector<MvCodedBlock>& blocks = j.mv_blocks;
    blocks.resize(N);
    for (int i = 0; i < N; i++) {
        uint32_t v = side[i];
        MvCodedBlock& b = blocks[i];
        b.mode = (uint8_t)(v & 7);
        b.new_base = (uint8_t)((v >> 3) & 7);
        b.skip = (v >> 24) & 1;
        b.dx = b.dy = 0;
        b.spx = b.spy = SP_ZERO;
        if (b.mode == M_NEW) {
            const int rdx = (int8_t)(v >> 8), rdy = (int8_t)(v >> 16);
            b.dx = (int8_t)std::min(std::max(rdx - j.bias[0], -128), 127);
            b.dy = (int8_t)std::min(std::max(rdy - j.bias[1], -128), 127);
            b.spx = ((v >> 6) & 1) ? SP_PLUS : SP_ZERO;
            b.spy = ((v >> 7) & 1) ? SP_PLUS : SP_ZERO;
            S.mv_new_blocks++;
            S.mv_new_base_counts[std::min<int>(b.new_base, 4)]++;
            // delta statistics before and after the bias (enc/encoder.rs:768-800, 873-884)
            if (rdx == 0 && rdy == 0) {
                S.mv_new_zero_pre_bias++;
                S.mv_zero_delta_blocks++;
            }
            const double fx = (double)b.dx, fy = (double)b.dy, mag = std::sqrt(fx * fx + fy * fy);
            S.mv_new_delta_mag_sum += mag;
            S.mv_new_delta_mag_sq_sum += mag * mag;
            S.mv_class_histogram[mv_class_of(std::abs((int)b.dx))]++;
            S.mv_class_histogram[mv_class_of(std::abs((int)b.dy))]++;
            if (b.dx == 0) S.mv_new_zero_axes_x++;
            if (b.dy == 0) S.mv_new_zero_axes_y++;
            if (b.dx == 0 && b.dy == 0) S.mv_new_zero_post_bias++;
        } else {
            S.mv_zero_delta_blocks++;
        }
        S.mv_mode_counts[b.mode]++;
        if (b.skip) S.blocks_skipped++;
    }
    S.mv_new_delta_count = S.mv_new_blocks;
    S.mv_raw_bytes = (uint32_t)(2 * N + 2 * S.mv_new_blocks);
    S.resi_raw = (int64_t)(N - (int)S.blocks_skipped) * 384 * 2;
    if (mbh) search_stats(e, mbh->data(), prevh ? prevh->data() : nullptr, S);
    S.mv_bias_dx = j.bias[0];
    S.mv_bias_dy = j.bias[1];
    S.rdo_lambda = e->L.lambda;
    j.tr[2] = now_ms();
    double dt = j.tr[2] - m0;
    std::lock_guard<std::mutex> g(e->stat_mu);
    e->host_ms[2] += dt;
}

static riv_status retire(riv_encoder* e, Job& j) {
    Slot& s = e->slots[j.slot];
    double t0 = now_ms();
    CK(cudaEventSynchronize(j.xev ? j.xev : s.ev_d2h));
    const uint32_t* hdr = s.hdr.host<uint32_t>();
    unsigned st = hdr[2];
    if (st) {
        return fail(e, (st & ST_WAIT_TIMEOUT) ? RIV_ERR_DEVICE_TIMEOUT : RIV_ERR_ENCODING_FAILED,
                    (st & ST_WAIT_TIMEOUT) ? "device-side wavefront wait timed out" : "device search iteration cap hit");
    }
    j.count = hdr[0];
    const size_t coef_bytes = (size_t)hdr[1] * 2;
    if (coef_bytes > s.prefetched) {  // the eager copy fell short: fetch the rest now
        CK(cudaMemcpyAsync((char*)s.packed.p + s.prefetched, (const char*)s.dpacked.p + s.prefetched,
                           coef_bytes - s.prefetched, cudaMemcpyDeviceToHost, e->C));
        CK(cudaStreamSynchronize(e->C));
    }
    // next frames: copy 25% + 64 KiB more than this frame needed
    e->coef_guess = coef_bytes + coef_bytes / 4 + 65536;
    e->d2h_bytes += (uint64_t)e->NMB * 7 + 12 + std::max(coef_bytes, s.prefetched);
    float t[NSTAGE + 1] = {0};
    if (!j.xev) CK(cudaEventSynchronize(s.ev_recon));  // the D2H did not wait for the deblock
    // stage 1 of the learned form is its network, on stream N
    const bool net = j.type == 2 && e->cfg.encode_form == RIV_FORM_LEARNED;
    const int spans[NSTAGE + 1][2] = {{EV_START, EV_YUV},   {net ? EV_NET0 : EV_S0, net ? EV_NET1 : EV_TABLE},
                                      {EV_TABLE, EV_SEARCH}, {EV_SEARCH, EV_PRED}, {EV_PRED, EV_AQ},   {EV_AQ, EV_RES},
                                      {EV_RES, EV_DEBLOCK}, {EV_K0, EV_COMPACT}, {EV_S0, EV_DEBLOCK}};
    if (j.timed) {
        for (int k = 0; k <= NSTAGE; k++) cudaEventElapsedTime(&t[k], s.ev_k[spans[k][0]], s.ev_k[spans[k][1]]);
        if (j.deferred) {  // residual and deblock ran inside the next launch: the chain ends with the search launch
            t[5] = t[6] = 0.0f;
            cudaEventElapsedTime(&t[NSTAGE], s.ev_k[EV_S0], s.ev_k[EV_AQ]);
        }
    }
    for (int k = 0; k <= NSTAGE; k++) j.times[k] = t[k] * 1000.0f;
    if (j.type == 2) {
        if (j.timed) {
            for (int k = 0; k <= NSTAGE; k++) e->sum_times[k] += j.times[k];
            e->ptimed++;
        }
        e->pframes++;
        if (j.deferred) e->pdeferred++;
    }
    const int N = e->NMB;
    riv_frame_stats& S = j.stats;
    memset(&S, 0, sizeof(S));
    S.frame_index = j.index;
    S.timestamp_ms = j.ts;
    S.frame_type = (uint32_t)j.type;
    S.storage_width = (uint32_t)e->W;
    S.storage_height = (uint32_t)e->H;
    S.blocks_total = (uint32_t)N;
    Job* jp = &j;
    riv_encoder* ep = e;
    const uint32_t* side = s.side.as<uint32_t>();
    std::shared_ptr<std::vector<MbOut>> mbh;
    std::shared_ptr<std::vector<int8_t>> prevh;
    if (j.type == 2 && j.want_stats) {  // the frame's search output (and the MVs it predicted from)
        mbh = std::make_shared<std::vector<MbOut>>(N);
        CK(cudaMemcpy(mbh->data(), e->mboutb[j.ck].p, (size_t)N * sizeof(MbOut), cudaMemcpyDeviceToHost));
        if (j.prev_valid) {
            prevh = std::make_shared<std::vector<int8_t>>((size_t)N * 4);
            CK(cudaMemcpy(prevh->data(), e->coded[j.prev_buf].p, (size_t)N * 4, cudaMemcpyDeviceToHost));
        }
    }
    if (j.type == 2) {
        // Three stages, each on its own thread: the coder's input (which needs nothing of the
        // coder's state), then the coder's two stages in frame order, so that frame t + 2 is
        // assembled and frame t + 1's symbols listed while frame t's are coded (same bytes as
        // one thread).
        j.fut_asm = e->mv_asm->submit([ep, jp, side, N, mbh, prevh] { assemble_mv(ep, *jp, side, N, mbh.get(), prevh.get()); });
        j.fut_prep = e->mv_prep->submit([ep, jp] {
            jp->fut_asm.get();
            double m0 = now_ms();
            jp->tr[3] = m0;
            ep->mvc.prepare(jp->mv_blocks, ep->BW, jp->mv_syms);
            jp->tr[4] = now_ms();
            double dt = jp->tr[4] - m0;
            std::lock_guard<std::mutex> g(ep->stat_mu);
            ep->host_ms[2] += dt;
        });
        j.fut_mv = e->mv_exec->submit([ep, jp] {
            jp->fut_prep.get();
            double m0 = now_ms();
            jp->tr[5] = m0;
            // modelling only on this thread; every rANS batch is coded on mv_pool and the
            // bytes are collected when the record is written
            jp->mv_bytes.clear();
            jp->mv_writer.reset(new RansWriter(&jp->mv_bytes, &ep->mv_submit));
            ep->mvc.model(jp->mv_syms, *jp->mv_writer);
            jp->mv_writer->finish_async();
            jp->tr[6] = now_ms();
            double dt = jp->tr[6] - m0;
            std::lock_guard<std::mutex> g(ep->stat_mu);
            ep->host_ms[2] += dt;
        });
    } else {
        // key frame: MV entropy contexts restart (enc/encoder.rs:335-337), in frame order on
        // both stages
        j.fut_prep = e->mv_prep->submit([ep] { ep->mvc.reset_history(); });
        j.fut_mv = e->mv_exec->submit([ep] { ep->mvc.reset_models(); });
    }
    const int16_t* packed = s.packed.as<int16_t>();
    const uint8_t* peobs = s.peobs.as<uint8_t>();
    uint32_t count = j.count;
    bool intra = j.type == 1;
    // The newest frame of a drain is coded by all of rans_pool's threads (no later frame will
    // be coded beside it); the others model on one pool thread and hand their full rANS
    // batches to rans_pool, which keeps the CPU cost per frame lowest while frames overlap
    // (splitting every drained frame measured slower on a 16-core host: the split coder's
    // extra work then competes with the frames beside it).
    const int parts = e->draining && &j == &e->jobs.back() ? e->rans_parts : 1;
    j.fut = e->pool->submit([jp, ep, packed, peobs, count, intra, parts] {
        double d0 = now_ms();
        jp->tr[7] = d0;
        if (parts > 1) encode_residual_frame(packed, peobs, (int)count, intra, jp->res_bytes, &ep->rans_submit_urgent, parts);
        else jp->res_writer = encode_residual_frame_async(packed, peobs, (int)count, intra, jp->res_bytes, ep->rans_submit);
        jp->tr[8] = now_ms();
        double dt = jp->tr[8] - d0;
        std::lock_guard<std::mutex> g(ep->stat_mu);
        ep->host_ms[3] += dt;
    });
    j.state = 1;
    e->host_ms[1] += now_ms() - t0;
    return RIV_OK;
}

// PackedFrame::to_bytes (com/format.rs:171-207) and the writer call.
static riv_status write_job(riv_encoder* e, Job& j) {
    double b0 = now_ms();
    j.fut_mv.get();
    if (j.mv_writer) {
        j.mv_writer->collect();
        j.mv_writer.reset();
    }
    j.fut.get();
    if (j.res_writer) {
        j.res_writer->collect();
        j.res_writer.reset();
    }
    double w0 = now_ms();
    e->host_ms[5] += w0 - b0;
    const riv_config& c = e->cfg;
    std::vector<uint8_t> rec;
    rec.reserve(32 + j.mv_bytes.size() + j.res_bytes.size());
    put_le(rec, j.ts, 8);
    if (j.type == 1) {
        rec.push_back(1);
        rec.push_back(c.intra_quality);
        put_le(rec, j.res_bytes.size(), 4);
        rec.insert(rec.end(), j.res_bytes.begin(), j.res_bytes.end());
    } else {
        rec.push_back(2);
        rec.push_back(c.inter_quality);
        rec.push_back((uint8_t)j.bias[0]);
        rec.push_back((uint8_t)j.bias[1]);
        rec.push_back(0);
        put_le(rec, j.mv_bytes.size(), 4);
        rec.insert(rec.end(), j.mv_bytes.begin(), j.mv_bytes.end());
        put_le(rec, j.res_bytes.size(), 4);
        rec.insert(rec.end(), j.res_bytes.begin(), j.res_bytes.end());
    }
    j.stats.total_bytes = (uint32_t)rec.size();
    j.stats.mv_bytes = (uint32_t)j.mv_bytes.size();
    j.stats.residual_bytes = (uint32_t)j.res_bytes.size();
    j.stats.resi_rans = j.type == 2 ? (int64_t)j.res_bytes.size() : -1;
    if (j.type != 2) j.stats.resi_raw = -1;
    if (e->wr.write(e->wr.user, rec.data(), rec.size()) != 0) return fail(e, RIV_ERR_IO, "writer.write failed");
    e->host_ms[4] += now_ms() - w0;
    if (!e->trace_path.empty()) {
        j.tr[9] = now_ms();
        std::array<double, 11> row;
        row[0] = (double)j.index;
        for (int k = 0; k < 10; k++) row[k + 1] = j.tr[k];
        e->trace.push_back(row);
    }
    e->frame_count++;
    if (j.timed) {
        memcpy(e->last_times, j.times, sizeof(j.times));
        e->have_times = true;
    }
    e->last_stats = j.stats;
    return RIV_OK;
}

// Advance the pipeline.  Frames are retired strictly in order (the MV coder's contexts
// carry across frames) and written strictly in order.  With `block_front` the oldest
// frame is driven to completion; everything else only advances if already possible.
static riv_status pump(riv_encoder* e, bool block_front, bool block_write);
static riv_status pump(riv_encoder* e, bool block_front) { return pump(e, block_front, block_front); }
static riv_status pump(riv_encoder* e, bool block_front, bool block_write) {
    bool block = block_front;
    for (auto& j : e->jobs) {
        if (j.state != 0) continue;
        if (!j.tail_done) {  // still waiting for the next frame's launch
            // flush only when nothing older can complete instead (a retired front frame
            // whose entropy coding the loop below waits for keeps the deferral)
            if (!block || e->jobs.front().state == 1) break;
            flush_pending(e);
        }
        if (!block) {
            cudaError_t q = cudaEventQuery(j.xev ? j.xev : e->slots[j.slot].ev_gpu);
            if (q == cudaErrorNotReady) break;
            if (q != cudaSuccess) throw CudaError{q, "cudaEventQuery"};
        }
        riv_status st = retire(e, j);
        if (st) return st;
        block = false;
    }
    block = block_write;
    while (!e->jobs.empty()) {
        Job& f = e->jobs.front();
        if (f.state != 1) break;
        if (!block && (f.fut.wait_for(std::chrono::seconds(0)) != std::future_status::ready ||
                       f.fut_mv.wait_for(std::chrono::seconds(0)) != std::future_status::ready ||
                       (f.res_writer && !f.res_writer->ready()) || (f.mv_writer && !f.mv_writer->ready())))
            break;
        riv_status st = write_job(e, f);
        // a record the writer refused is lost and not counted, as when the reference's
        // write fails (enc/encoder.rs:248-253); later frames go on
        if (st == RIV_ERR_IO) e->jobs.pop_front();
        if (st) return st;
        e->jobs.pop_front();
        block = false;
    }
    return RIV_OK;
}

static riv_status drain_all(riv_encoder* e) {
    flush_pending(e);  // no later launch is coming: reconstruct now, before the host work queued ahead of it
    struct Draining {
        riv_encoder* e;
        ~Draining() { e->draining = false; }
    } guard{e};
    e->draining = true;
    // A record the writer refuses is dropped (pump pops it) and the drain goes on, so that
    // every later record is still written and the header can be patched; the refusal is
    // reported once the queue is empty.
    // Frames are retired as soon as their GPU work is done, not after the front frame's record
    // is written, so that their host coding starts at once; the front frame's coding is
    // waited for in short slices in between.
    riv_status io = RIV_OK;
    auto retired = [e] {
        size_t n = 0;
        for (const Job& j : e->jobs) n += j.state == 1;
        return n;
    };
    while (!e->jobs.empty()) {
        const size_t n0 = e->jobs.size(), r0 = retired();
        riv_status st = pump(e, false, false);
        if (st == RIV_ERR_IO) {
            io = st;
            continue;
        }
        if (st) return st;
        if (e->jobs.empty() || e->jobs.size() != n0 || retired() != r0) continue;  // progress
        Job& f = e->jobs.front();
        const bool later_unretired = retired() < e->jobs.size();
        if (f.state == 0) st = pump(e, true, false);          // block on the front frame's GPU work
        else if (!later_unretired) st = pump(e, false, true);  // nothing else to retire: block on its record
        else if (f.fut.wait_for(std::chrono::microseconds(20)) == std::future_status::ready)
            std::this_thread::sleep_for(std::chrono::microseconds(20));  // its batches are still being coded
        if (st == RIV_ERR_IO) {
            io = st;
            continue;
        }
        if (st) return st;
    }
    if (io) e->err = "writer.write failed for at least one record; the others were written";
    return io;
}

// Frame type of the next frame (enc/encoder.rs:265-291).
static bool next_is_key(const riv_encoder* e) {
    const riv_config& c = e->cfg;
    const uint64_t n = e->submitted;
    bool intra;
    if (c.keyframe_mode == RIV_KEYFRAME_ALL_INTRA) intra = true;
    else if (c.keyframe_mode == RIV_KEYFRAME_AUTOMATIC) intra = n % 30 == 0;
    else intra = n % c.keyframe_interval == 0;
    return intra || !e->has_ref;
}

static riv_status encode_common(riv_encoder* e, int src, const void* a, const void* b, const void* c3,
                                uint64_t ts, riv_frame_stats* stats) {
    if (e->poisoned) return poisoned_status(e);
    // A record the writer refuses while this call makes room is lost (pump drops it); this
    // frame is still encoded and queued, and the refusal is reported when the call returns.
    riv_status refused = RIV_OK;
    try {
        CK(cudaSetDevice(e->cfg.device));
        size_t cap = e->slots.size();
        while (e->jobs.size() >= cap) {
            riv_status st = pump(e, true);
            if (st == RIV_ERR_IO) {
                refused = st;
                continue;
            }
            if (st) return st;
        }
        const uint64_t n = e->submitted;
        const bool intra = next_is_key(e);
        e->jobs.emplace_back();
        Job& j = e->jobs.back();
        j.index = n;
        j.ts = ts;
        if (!e->trace_path.empty()) j.tr[0] = now_ms();
        j.type = intra ? 1 : 2;
        j.slot = (int)(n % cap);
        j.timed = e->cfg.pipeline_depth == 0 || stats != nullptr || n % TIMING_SAMPLE == 0;
        j.want_stats = stats != nullptr;
        double s0 = now_ms();
        submit_gpu(e, j, src, a, b, c3);
        j.prev_valid = e->has_prev2_mvs;  // the temporal predictors this P-frame used
        j.prev_buf = e->coded_cur ^ 1;
        e->submitted++;
        e->host_ms[0] += now_ms() - s0;
        if (src == 0 || src == 2) CK(cudaEventSynchronize(e->slots[j.slot].ev_h2d));  // caller buffer reusable
        if (e->cfg.pipeline_depth == 0 || stats) {
            riv_status st = drain_all(e);
            if (st) return st;
            if (stats) *stats = e->last_stats;  // this frame was the last one written
        } else {
            riv_status st = pump(e, false);
            if (st) return st;
        }
    } catch (const CudaError& ce) {
        return fail(e, RIV_ERR_CUDA, std::string(ce.where) + ": " + cudaGetErrorString(ce.e));
    } catch (const std::exception& ex) {
        return fail_poison(e, RIV_ERR_ENCODING_FAILED, ex.what());
    }
    if (refused) e->err = "writer.write failed for an earlier frame's record; that record is lost";
    return refused;
}

}  // namespace

// =====================================================================================
// C ABI
// =====================================================================================
extern "C" {

void riv_config_default(riv_config* c, uint32_t w, uint32_t h, uint32_t fps) {
    memset(c, 0, sizeof(*c));
    c->display_width = w;
    c->display_height = h;
    c->storage_width = (w + 15) / 16 * 16;
    c->storage_height = (h + 15) / 16 * 16;
    c->fps = fps;
    c->keyframe_mode = RIV_KEYFRAME_FIXED;
    c->keyframe_interval = 30;
    c->intra_quality = 90;
    c->inter_quality = 35;
    c->search_range = 12;
    c->mv_deflate_level = 6;
    c->skip_threshold = 3;
    c->rdo_lambda_mult = 0.49;
    c->inter_dead_zone = 0.75f;
    c->device = 0;
    c->pipeline_depth = 0;
    c->entropy_threads = 0;
}

riv_status riv_encoder_new(const riv_config* cfg, const riv_writer_vtable* writer, riv_encoder** out) {
    if (!cfg || !writer || !out || !writer->write || !writer->position || !writer->seek || !writer->flush)
        return RIV_ERR_INVALID_CONFIG;
    *out = nullptr;
    std::string msg;
    riv_status st = validate(*cfg, msg);
    if (st) return st;
    entropy_init();
    riv_encoder* e = new riv_encoder();
    e->cfg = *cfg;
    e->wr = *writer;
    try {
        setup_device(e);
    } catch (const CudaError& ce) {
        std::string m = std::string(ce.where) + ": " + cudaGetErrorString(ce.e);
        fprintf(stderr, "riv_encoder_new: %s\n", m.c_str());
        riv_encoder_free(e);
        return RIV_ERR_CUDA;
    } catch (const std::exception& ex) {
        fprintf(stderr, "riv_encoder_new: %s\n", ex.what());
        riv_encoder_free(e);
        return RIV_ERR_ENCODING_FAILED;
    }
    e->header_pos = e->wr.position(e->wr.user);
    std::vector<uint8_t> h = header_bytes(e->cfg, 0);
    if (e->wr.write(e->wr.user, h.data(), h.size()) != 0) {
        riv_encoder_free(e);
        return RIV_ERR_IO;
    }
    *out = e;
    return RIV_OK;
}

riv_status riv_encoder_set_proposal(riv_encoder* e, const float* params, size_t n) {
    using PL = nn::ParamLayout;
    if (!e || !params) return RIV_ERR_INVALID_CONFIG;
    if (e->cfg.encode_form != RIV_FORM_LEARNED) return fail(e, RIV_ERR_INVALID_CONFIG, "encoder is not in the learned form");
    if (n != PL::nweights + PL::nbias) return fail(e, RIV_ERR_INVALID_CONFIG, "proposal parameters: wrong count");
    if (e->poisoned) return poisoned_status(e);
    std::vector<uint16_t> wb(PL::nweights);
    for (size_t i = 0; i < PL::nweights; i++) {  // round to the nearest bf16, ties to even
        uint32_t u;
        memcpy(&u, params + i, 4);
        wb[i] = (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
    }
    try {
        CK(cudaSetDevice(e->cfg.device));
        CK(cudaMemcpy(e->nn_w.p, wb.data(), wb.size() * 2, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(e->nn_b.p, params + PL::nweights, PL::nbias * 4, cudaMemcpyHostToDevice));
    } catch (const CudaError& ce) {
        return fail(e, RIV_ERR_CUDA, std::string(ce.where) + ": " + cudaGetErrorString(ce.e));
    }
    e->nn_loaded = true;
    return RIV_OK;
}

riv_status riv_learned_counters(riv_encoder* e, uint64_t* mbs, uint64_t* fallbacks, uint64_t* shortcuts) {
    if (!e || !mbs || !fallbacks || !shortcuts) return RIV_ERR_INVALID_CONFIG;
    *mbs = *fallbacks = *shortcuts = 0;
    if (!e->learned) return RIV_OK;
    unsigned h[2] = {0, 0};
    try {
        CK(cudaSetDevice(e->cfg.device));
        CK(cudaStreamSynchronize(e->S));
        CK(cudaMemcpy(h, e->lcount.p, sizeof(h), cudaMemcpyDeviceToHost));
    } catch (const CudaError& ce) {
        return fail(e, RIV_ERR_CUDA, std::string(ce.where) + ": " + cudaGetErrorString(ce.e));
    }
    *mbs = e->learned_mbs;
    *fallbacks = h[0];
    *shortcuts = h[1];
    return RIV_OK;
}

riv_status riv_encode_frame(riv_encoder* e, const uint8_t* rgb, uint32_t w, uint32_t h, uint64_t ts,
                            riv_frame_stats* stats) {
    if (!e) return RIV_ERR_INVALID_CONFIG;
    if (w != e->cfg.display_width || h != e->cfg.display_height) {  // enc/encoder.rs:237-242
        char buf[160];
        snprintf(buf, sizeof(buf), "Frame dimensions (%u, %u) do not match config (%u, %u)", w, h,
                 e->cfg.display_width, e->cfg.display_height);
        return fail(e, RIV_ERR_FRAME, buf);
    }
    if (!rgb) return fail(e, RIV_ERR_FRAME, "null frame data");
    riv_frame_stats tmp;
    riv_status st = encode_common(e, 0, rgb, nullptr, nullptr, ts, stats ? &tmp : nullptr);
    if (st == RIV_OK && stats) *stats = tmp;
    return st;
}

riv_status riv_encode_frame_device(riv_encoder* e, const void* d_rgb, uint64_t ts, riv_frame_stats* stats) {
    if (!e || !d_rgb) return RIV_ERR_FRAME;
    riv_frame_stats tmp;
    riv_status st = encode_common(e, 1, d_rgb, nullptr, nullptr, ts, stats ? &tmp : nullptr);
    if (st == RIV_OK && stats) *stats = tmp;
    return st;
}

riv_status riv_encode_frame_yuv(riv_encoder* e, const uint8_t* y, const uint8_t* u, const uint8_t* v, uint64_t ts,
                                riv_frame_stats* stats) {
    if (!e || !y || !u || !v) return RIV_ERR_FRAME;
    riv_frame_stats tmp;
    riv_status st = encode_common(e, 2, y, u, v, ts, stats ? &tmp : nullptr);
    if (st == RIV_OK && stats) *stats = tmp;
    return st;
}

riv_status riv_finish(riv_encoder* e) {  // enc/encoder.rs:950-961
    if (!e) return RIV_ERR_INVALID_CONFIG;
    if (e->poisoned) return poisoned_status(e);
    riv_status dropped = RIV_OK;  // RIV_ERR_IO: a record was refused, the rest were written
    try {
        CK(cudaSetDevice(e->cfg.device));
        riv_status st = drain_all(e);
        if (st && st != RIV_ERR_IO) return st;
        dropped = st;
    } catch (const CudaError& ce) {
        return fail(e, RIV_ERR_CUDA, std::string(ce.where) + ": " + cudaGetErrorString(ce.e));
    } catch (const std::exception& ex) {
        return fail_poison(e, RIV_ERR_ENCODING_FAILED, ex.what());
    }
    uint64_t end = e->wr.position(e->wr.user);
    if (e->wr.seek(e->wr.user, e->header_pos) != 0) return fail(e, RIV_ERR_IO, "writer.seek failed");
    std::vector<uint8_t> h = header_bytes(e->cfg, e->frame_count);
    if (e->wr.write(e->wr.user, h.data(), h.size()) != 0) return fail(e, RIV_ERR_IO, "writer.write failed");
    if (e->wr.seek(e->wr.user, end) != 0) return fail(e, RIV_ERR_IO, "writer.seek failed");
    if (e->wr.flush(e->wr.user) != 0) return fail(e, RIV_ERR_IO, "writer.flush failed");
    return dropped;
}

void riv_encoder_free(riv_encoder* e) {
    if (!e) return;
    cudaSetDevice(e->cfg.device);
    for (auto& j : e->jobs) {
        if (j.fut.valid()) j.fut.wait();
        if (j.fut_mv.valid()) j.fut_mv.wait();
        if (j.fut_prep.valid()) j.fut_prep.wait();
        if (j.fut_asm.valid()) j.fut_asm.wait();
    }
    if (!e->trace_path.empty() && !e->trace.empty()) {
        if (FILE* f = fopen(e->trace_path.c_str(), "a")) {
            for (const auto& r : e->trace) {
                fprintf(f, "%.0f", r[0]);
                for (int k = 1; k < 11; k++) fprintf(f, ",%.4f", r[k]);
                fprintf(f, "\n");
            }
            fclose(f);
        }
    }
    e->pool.reset();
    e->mv_exec.reset();
    e->mv_prep.reset();
    e->mv_asm.reset();
    e->mv_pool.reset();
    e->rans_pool.reset();
    if (e->S) cudaStreamSynchronize(e->S);
    if (e->C) cudaStreamSynchronize(e->C);
    if (e->Hs) cudaStreamSynchronize(e->Hs);
    if (e->Y) cudaStreamSynchronize(e->Y);
    if (e->K) cudaStreamSynchronize(e->K);
    for (auto& s : e->slots) {
        s.rgb.release(); s.dside.release(); s.dpacked.release(); s.dpeobs.release();
        s.side.release(); s.packed.release(); s.peobs.release(); s.hdr.release();
        if (s.ev_h2d) cudaEventDestroy(s.ev_h2d);
        if (s.ev_gpu) cudaEventDestroy(s.ev_gpu);
        if (s.ev_d2h) cudaEventDestroy(s.ev_d2h);
        for (int k = 0; k < EV_N; k++)
            if (s.ev_k[k]) cudaEventDestroy(s.ev_k[k]);
        if (s.ev_yuv) cudaEventDestroy(s.ev_yuv);
        if (s.ev_recon) cudaEventDestroy(s.ev_recon);
    }
    for (int k = 0; k < NPAR; k++)
        for (DevBuf* b : {&e->curb[k], &e->predb[k], &e->mboutb[k], &e->lnvb[k], &e->coeffsb[k], &e->optskipb[k], &e->fmaskb[k],
                          &e->eobsb[k]})
            b->release();
    DevBuf* bufs[] = {&e->ref[0], &e->ref[1], &e->recon_pre, &e->wq, &e->coded[0], &e->coded[1], &e->rec,
                      &e->varsum, &e->qs, &e->status,
                      &e->mvbits, &e->logfix, &e->expfix, &e->ytab, &e->ctab, &e->cindex, &e->coffset, &e->lcindex, &e->lcoffset, &e->sadtab, &e->prof, &e->tflag, &e->rowdone, &e->newcost, &e->newcost32,
                      &e->nn_w, &e->nn_b, &e->nn_feat, &e->nn_a1, &e->nn_a2, &e->nn_a3, &e->nn_x1, &e->nn_h1, &e->nn_h2,
                      &e->nn_o[0], &e->nn_o[1], &e->lmv, &e->lcount, &e->lrowcnt};
    for (DevBuf* b : bufs) b->release();
    if (e->N) cudaStreamSynchronize(e->N);
    for (int k = 0; k < 2; k++) {
        if (e->ev_net_out[k]) cudaEventDestroy(e->ev_net_out[k]);
        if (e->ev_net_read[k]) cudaEventDestroy(e->ev_net_read[k]);
    }
    for (int k = 0; k < NPAR; k++)
        if (e->ev_net_cur[k]) cudaEventDestroy(e->ev_net_cur[k]);
    if (e->N) cudaStreamDestroy(e->N);
    if (e->S) cudaStreamDestroy(e->S);
    if (e->C) cudaStreamDestroy(e->C);
    if (e->Hs) cudaStreamDestroy(e->Hs);
    if (e->Y) cudaStreamDestroy(e->Y);
    if (e->K) cudaStreamDestroy(e->K);
    for (int k = 0; k < NPAR; k++) {
        if (e->ev_cur_free[k]) cudaEventDestroy(e->ev_cur_free[k]);
        if (e->ev_mbout_free[k]) cudaEventDestroy(e->ev_mbout_free[k]);
        if (e->ev_coef_free[k]) cudaEventDestroy(e->ev_coef_free[k]);
    }
    if (e->ev_search_done) cudaEventDestroy(e->ev_search_done);
    delete e;
}

const char* riv_last_error(const riv_encoder* e) { return e ? e->err.c_str() : "null encoder"; }
uint64_t riv_frame_count(const riv_encoder* e) { return e ? e->frame_count : 0; }

riv_status riv_last_recon(riv_encoder* e, uint8_t* y, uint8_t* u, uint8_t* v) {
    if (!e || !e->has_ref) return RIV_ERR_FRAME;
    try {
        CK(cudaSetDevice(e->cfg.device));
        flush_pending(e);
        CK(cudaStreamSynchronize(e->S));
        const uint8_t* d = e->ref[e->ref_cur].as<uint8_t>();
        size_t ys = (size_t)e->W * e->H, cs = ys / 4;
        CK(cudaMemcpy(y, d, ys, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(u, d + ys, cs, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(v, d + ys + cs, cs, cudaMemcpyDeviceToHost));
    } catch (const CudaError& ce) {
        return fail(e, RIV_ERR_CUDA, std::string(ce.where) + ": " + cudaGetErrorString(ce.e));
    } catch (const std::exception& ex) {
        return fail_poison(e, RIV_ERR_ENCODING_FAILED, ex.what());
    }
    return RIV_OK;
}

riv_status riv_debug_frame_state(riv_encoder* e, int what, void* out, size_t size) {
    if (!e || !out) return RIV_ERR_FRAME;
    const DevBuf* b = nullptr;
    switch (what) {
        case 0: b = &e->mboutb[e->last_par]; break;
        case 1: b = &e->qs; break;
        case 2: b = &e->predb[e->last_par]; break;
        case 3: b = &e->curb[e->last_par]; break;
        case 4: b = &e->coeffsb[e->last_par]; break;
        case 5: b = &e->optskipb[e->last_par]; break;
        case 6: b = &e->prof; break;
        default: return RIV_ERR_FRAME;
    }
    if (size < b->n) return RIV_ERR_FRAME;
    try {
        CK(cudaSetDevice(e->cfg.device));
        flush_pending(e);
        CK(cudaStreamSynchronize(e->Y));
        CK(cudaStreamSynchronize(e->S));
        CK(cudaStreamSynchronize(e->K));
        CK(cudaMemcpy(out, b->p, b->n, cudaMemcpyDeviceToHost));
    } catch (const CudaError& ce) {
        return fail(e, RIV_ERR_CUDA, std::string(ce.where) + ": " + cudaGetErrorString(ce.e));
    } catch (const std::exception& ex) {
        return fail_poison(e, RIV_ERR_ENCODING_FAILED, ex.what());
    }
    return RIV_OK;
}

riv_status riv_host_times(riv_encoder* e, double* ms6) {
    if (!e || !ms6) return RIV_ERR_FRAME;
    std::lock_guard<std::mutex> g(e->stat_mu);
    memcpy(ms6, e->host_ms, sizeof(e->host_ms));
    return RIV_OK;
}

riv_status riv_counters(riv_encoder* e, double* us8, uint64_t* io2, uint64_t* n4) {
    if (!e) return RIV_ERR_FRAME;
    if (us8) memcpy(us8, e->sum_times, sizeof(e->sum_times));
    if (io2) { io2[0] = e->h2d_bytes; io2[1] = e->d2h_bytes; }
    if (n4) { n4[0] = e->pframes; n4[1] = e->launches; n4[2] = e->pdeferred; n4[3] = e->ptimed; }
    return RIV_OK;
}

riv_status riv_last_kernel_times(riv_encoder* e, float* us8) {
    if (!e || !e->have_times) return RIV_ERR_FRAME;
    memcpy(us8, e->last_times, sizeof(e->last_times));
    return RIV_OK;
}

// ---- in-memory writer (VecWriter semantics, enc/writer.rs:49-69) ----
struct riv_memwriter {
    std::vector<uint8_t> buf;
    uint64_t pos = 0;
};
static int mw_write(void* u, const uint8_t* d, size_t n) {
    riv_memwriter* w = (riv_memwriter*)u;
    if (w->pos + n > w->buf.size()) w->buf.resize(w->pos + n, 0);
    memcpy(w->buf.data() + w->pos, d, n);
    w->pos += n;
    return 0;
}
static uint64_t mw_position(void* u) { return ((riv_memwriter*)u)->pos; }
static int mw_seek(void* u, uint64_t p) {
    riv_memwriter* w = (riv_memwriter*)u;
    if (p > w->buf.size()) w->buf.resize(p, 0);
    w->pos = p;
    return 0;
}
static int mw_flush(void*) { return 0; }
riv_memwriter* riv_memwriter_new(void) { return new riv_memwriter(); }
void riv_memwriter_vtable(riv_memwriter* w, riv_writer_vtable* o) {
    o->write = mw_write;
    o->position = mw_position;
    o->seek = mw_seek;
    o->flush = mw_flush;
    o->user = w;
}
size_t riv_memwriter_size(const riv_memwriter* w) { return w->buf.size(); }
const uint8_t* riv_memwriter_data(const riv_memwriter* w) { return w->buf.data(); }
void riv_memwriter_free(riv_memwriter* w) { delete w; }

// ---- stage entry points ----
riv_status riv_stage_rgb_to_yuv(const uint8_t* rgb, uint32_t dw, uint32_t dh, uint32_t sw, uint32_t sh, uint8_t* out) {
    if (!rgb || !out || sw < dw || sh < dh || sw % 2 || sh % 2) return RIV_ERR_FRAME;
    void *d_rgb = nullptr, *d_yuv = nullptr;
    size_t nin = (size_t)dw * dh * 3, nout = (size_t)sw * sh * 3 / 2;
    riv_status st = RIV_OK;
    if (cudaMalloc(&d_rgb, nin) || cudaMalloc(&d_yuv, nout) || cudaMemcpy(d_rgb, rgb, nin, cudaMemcpyHostToDevice) ||
        launch_rgb_to_yuv((const uint8_t*)d_rgb, (int)dw, (int)dh, (uint8_t*)d_yuv, (int)sw, (int)sh, 0) ||
        cudaMemcpy(out, d_yuv, nout, cudaMemcpyDeviceToHost))
        st = RIV_ERR_CUDA;
    cudaFree(d_rgb);
    cudaFree(d_yuv);
    return st;
}

// Device buffers of one stage call, freed together.
struct StageBufs {
    std::vector<void*> ps;
    void* get(size_t n) {
        void* p = nullptr;
        if (cudaMalloc(&p, n ? n : 1) != cudaSuccess) throw CudaError{cudaErrorMemoryAllocation, "cudaMalloc"};
        ps.push_back(p);
        return p;
    }
    void* up(const void* h, size_t n) {
        void* p = get(n);
        CK(cudaMemcpy(p, h, n, cudaMemcpyHostToDevice));
        return p;
    }
    ~StageBufs() {
        for (void* p : ps) cudaFree(p);
    }
};

riv_status riv_stage_predict(const uint8_t* ref_yuv, const int8_t* mv4, uint32_t w, uint32_t h, uint8_t quality,
                             uint8_t* pred_yuv, float* qs) {
    if (!ref_yuv || !mv4 || !pred_yuv || w == 0 || h == 0 || w % 16 || h % 16) return RIV_ERR_FRAME;
    LibmFix& F = libm_fix();
    if (!F.ok) return RIV_ERR_ENCODING_FAILED;
    const int n = (int)((w / 16) * (h / 16));
    const size_t yuv = (size_t)w * h * 3 / 2;
    std::vector<MbOut> mb(n);
    for (int i = 0; i < n; i++) {
        memset(&mb[i], 0, sizeof(MbOut));
        memcpy(mb[i].raw, mv4 + 4 * i, 4);
        memcpy(mb[i].coded, mv4 + 4 * i, 4);
    }
    try {
        StageBufs B;
        auto* dref = (const uint8_t*)B.up(ref_yuv, yuv);
        auto* dmb = (const MbOut*)B.up(mb.data(), n * sizeof(MbOut));
        auto* dpred = (uint8_t*)B.get(yuv);
        auto* dvs = (uint2*)B.get((size_t)n * sizeof(uint2));
        auto* dlnv = (float*)B.get((size_t)(n + 1) * 4);
        auto* dqs = (float*)B.get((size_t)n * 4);
        auto* dlog = (const uint32_t*)B.up(F.logf_dev.data(), F.logf_dev.size() * 4);
        auto* dexp = (const uint32_t*)B.up(F.exp2f_dev.data(), F.exp2f_dev.size() * 4);
        CK((cudaError_t)launch_predict(dref, dmb, dpred, dvs, (int)w, (int)h, 0));
        CK((cudaError_t)launch_aq(dvs, n, quant_step(quality), dlog, (int)(F.logf.size() / 2), dexp,
                                  (int)(F.exp2f.size() / 2), dlnv, dqs, 0));
        CK(cudaMemcpy(pred_yuv, dpred, yuv, cudaMemcpyDeviceToHost));
        if (qs) CK(cudaMemcpy(qs, dqs, (size_t)n * 4, cudaMemcpyDeviceToHost));
    } catch (const CudaError&) {
        return RIV_ERR_CUDA;
    }
    return RIV_OK;
}

riv_status riv_stage_residual(const uint8_t* cur_yuv, const uint8_t* pred_yuv, const float* qs, const uint8_t* rdo_skip,
                              const int8_t* coded4, float dead_zone, uint32_t w, uint32_t h, int16_t* coeffs,
                              uint8_t* opt_skip, uint8_t* recon_yuv, uint8_t* fmask) {
    if (!cur_yuv || !pred_yuv || !qs || !rdo_skip || !coeffs || !opt_skip || !recon_yuv || w == 0 || h == 0 || w % 16 ||
        h % 16)
        return RIV_ERR_FRAME;
    const int n = (int)((w / 16) * (h / 16));
    const size_t yuv = (size_t)w * h * 3 / 2;
    std::vector<MbOut> mb(n);
    for (int i = 0; i < n; i++) {
        memset(&mb[i], 0, sizeof(MbOut));
        if (coded4) memcpy(mb[i].coded, coded4 + 4 * i, 4);
        mb[i].rdo_skip = rdo_skip[i] ? 1 : 0;
    }
    try {
        StageBufs B;
        ResidualParams rp{};
        rp.cur = (const uint8_t*)B.up(cur_yuv, yuv);
        rp.pred = (const uint8_t*)B.up(pred_yuv, yuv);
        rp.recon = (uint8_t*)B.get(yuv);
        rp.coeffs = (int16_t*)B.get((size_t)n * 384 * 2);
        rp.opt_skip = (uint8_t*)B.get(n);
        rp.fmask = (uint8_t*)B.get(n);
        rp.eobs = (uint8_t*)B.get((size_t)n * 3);
        rp.mb = (const MbOut*)B.up(mb.data(), n * sizeof(MbOut));
        rp.qs = (const float*)B.up(qs, (size_t)n * 4);
        rp.dead_zone = dead_zone;
        rp.W = (int)w;
        rp.H = (int)h;
        rp.BW = (int)w / 16;
        rp.intra = 0;
        CK((cudaError_t)launch_residual(rp, n, 0));
        CK(cudaMemcpy(coeffs, rp.coeffs, (size_t)n * 384 * 2, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(opt_skip, rp.opt_skip, n, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(recon_yuv, rp.recon, yuv, cudaMemcpyDeviceToHost));
        if (fmask) CK(cudaMemcpy(fmask, rp.fmask, n, cudaMemcpyDeviceToHost));
    } catch (const CudaError&) {
        return RIV_ERR_CUDA;
    }
    return RIV_OK;
}

riv_status riv_stage_deblock(uint8_t* yuv, uint32_t w, uint32_t h, int level, int intra, const uint8_t* mask) {
    if (!yuv || w % 16 || h % 16) return RIV_ERR_FRAME;
    if (level <= 0) return RIV_OK;
    int E, I, Hv;
    deblock_thresholds(level, intra != 0, E, I, Hv);
    size_t n = (size_t)w * h * 3 / 2, nm = (size_t)(w / 16) * (h / 16);
    void *d = nullptr, *d2 = nullptr, *dm = nullptr;
    riv_status st = RIV_OK;
    if (cudaMalloc(&d, n) || cudaMalloc(&d2, n) || cudaMemcpy(d, yuv, n, cudaMemcpyHostToDevice)) st = RIV_ERR_CUDA;
    if (!st && mask && (cudaMalloc(&dm, nm) || cudaMemcpy(dm, mask, nm, cudaMemcpyHostToDevice))) st = RIV_ERR_CUDA;
    if (!st && (launch_deblock_tiled((const uint8_t*)d, (uint8_t*)d2, (int)w, (int)h, E, I, Hv, (const uint8_t*)dm, 0) ||
                cudaMemcpy(yuv, d2, n, cudaMemcpyDeviceToHost)))
        st = RIV_ERR_CUDA;
    cudaFree(d);
    cudaFree(d2);
    cudaFree(dm);
    return st;
}

// riv_stage_deblock without device allocation: staging in the fixed device scratch.  The
// scratch address is looked up once per device, with that device current.
static_assert(DEBLOCK_NOALLOC_MAX_BYTES == RIV_DEBLOCK_NOALLOC_MAX_BYTES, "scratch size must match the header");
static std::mutex g_noalloc_mu;
static void* g_noalloc_scratch[64];

static riv_status noalloc_fail(char* errbuf, size_t len, riv_status st, const char* msg) {
    if (errbuf && len) snprintf(errbuf, len, "%s", msg);
    return st;
}

riv_status riv_stage_deblock_noalloc(uint8_t* yuv, uint32_t w, uint32_t h, int level, int intra,
                                     const uint8_t* mask, char* errbuf, size_t errbuf_len) {
    if (errbuf && errbuf_len) errbuf[0] = 0;
    if (!yuv || w == 0 || h == 0 || w % 16 || h % 16)
        return noalloc_fail(errbuf, errbuf_len, RIV_ERR_FRAME, "planes must be non-null with width and height multiples of 16");
    const size_t n = (size_t)w * h * 3 / 2, nm = (size_t)(w / 16) * (h / 16);
    const size_t need = n + (mask ? nm : 0);
    if (need > RIV_DEBLOCK_NOALLOC_MAX_BYTES) {
        char msg[160];
        snprintf(msg, sizeof msg, "%ux%u needs %zu bytes of scratch, more than the fixed %u (RIV_DEBLOCK_NOALLOC_MAX_BYTES)",
                 w, h, need, (unsigned)RIV_DEBLOCK_NOALLOC_MAX_BYTES);
        return noalloc_fail(errbuf, errbuf_len, RIV_ERR_FRAME, msg);
    }
    if (level <= 0) return RIV_OK;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return noalloc_fail(errbuf, errbuf_len, RIV_ERR_CUDA, "no usable current CUDA device");
    uint8_t* scr = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_scratch[dev]) {
            void* p = nullptr;
            if (deblock_scratch_address(&p) != 0 || !p)
                return noalloc_fail(errbuf, errbuf_len, RIV_ERR_CUDA, "cudaGetSymbolAddress of the deblock scratch failed");
            g_noalloc_scratch[dev] = p;
        }
        scr = (uint8_t*)g_noalloc_scratch[dev];
    }
    int E, I, Hv;
    deblock_thresholds(level, intra != 0, E, I, Hv);
    if (cudaMemcpy(scr, yuv, n, cudaMemcpyHostToDevice) != cudaSuccess ||
        (mask && cudaMemcpy(scr + n, mask, nm, cudaMemcpyHostToDevice) != cudaSuccess) ||
        launch_deblock(scr, (int)w, (int)h, E, I, Hv, mask ? scr + n : nullptr, 0) != 0 ||
        cudaMemcpy(yuv, scr, n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return noalloc_fail(errbuf, errbuf_len, RIV_ERR_CUDA, "CUDA copy or launch failed");
    return RIV_OK;
}

riv_status riv_stage_libm(int which, const float* in, float* out, size_t n) {
    LibmFix& F = libm_fix();
    if (!F.ok) return RIV_ERR_ENCODING_FAILED;
    const std::vector<uint32_t>& fx = which == 0 ? F.logf_dev : F.exp2f_dev;
    const int npairs = (int)((which == 0 ? F.logf : F.exp2f).size() / 2);
    void *di = nullptr, *dout = nullptr, *df = nullptr;
    riv_status st = RIV_OK;
    if (cudaMalloc(&di, n * 4) || cudaMalloc(&dout, n * 4) || cudaMalloc(&df, fx.size() * 4 + 4) ||
        cudaMemcpy(di, in, n * 4, cudaMemcpyHostToDevice) ||
        cudaMemcpy(df, fx.data(), fx.size() * 4, cudaMemcpyHostToDevice) ||
        launch_libm_eval(which, (const float*)di, (float*)dout, n, (const uint32_t*)df, npairs, 0) ||
        cudaMemcpy(out, dout, n * 4, cudaMemcpyDeviceToHost))
        st = RIV_ERR_CUDA;
    cudaFree(di);
    cudaFree(dout);
    cudaFree(df);
    return st;
}

// Exhaustive check of the device logf / exp2f against the host's glibc: every f32 with bit
// pattern in [lo_bits, hi_bits], in chunks computed on the device while the host threads
// compare the previous chunk bit for bit.
riv_status riv_test_libm_range(int which, uint32_t lo_bits, uint32_t hi_bits, uint64_t* mismatches,
                               uint32_t* first_bad_bits) {
    if (!mismatches || !first_bad_bits || which < 0 || which > 2 || hi_bits < lo_bits) return RIV_ERR_FRAME;
    *mismatches = 0;
    *first_bad_bits = 0;
    LibmFix& F = libm_fix();
    if (!F.ok) return RIV_ERR_ENCODING_FAILED;
    const std::vector<uint32_t>& fx = which == 1 ? F.exp2f_dev : F.logf_dev;
    const int npairs = (int)((which == 1 ? F.exp2f : F.logf).size() / 2);
    const uint32_t CH = 1u << 25;
    void *df = nullptr, *dout[2] = {nullptr, nullptr}, *hout[2] = {nullptr, nullptr};
    cudaStream_t st = nullptr;
    cudaEvent_t done[2] = {nullptr, nullptr};
    riv_status rs = RIV_OK;
    std::atomic<uint64_t> bad{0};
    std::atomic<uint32_t> first{0xffffffffu};
    const unsigned nthr = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    auto compare = [&](const float* got, uint32_t base, uint32_t n) {
        std::vector<std::thread> ts;
        for (unsigned t = 0; t < nthr; t++)
            ts.emplace_back([&, t] {
                const uint32_t a = (uint32_t)((uint64_t)n * t / nthr), b = (uint32_t)((uint64_t)n * (t + 1) / nthr);
                uint64_t nb = 0;
                uint32_t fb = 0xffffffffu;
                for (uint32_t i = a; i < b; i++) {
                    const uint32_t bits = base + i;
                    float x;
                    memcpy(&x, &bits, 4);
                    const float want = which == 1 ? exp2f(x) : logf(x);
                    uint32_t wb, gb;
                    memcpy(&wb, &want, 4);
                    memcpy(&gb, got + i, 4);
                    if (wb != gb && !(want != want && got[i] != got[i])) {
                        nb++;
                        fb = std::min(fb, bits);
                    }
                }
                bad += nb;
                uint32_t cur = first.load();
                while (fb < cur && !first.compare_exchange_weak(cur, fb)) {}
            });
        for (auto& t : ts) t.join();
    };
    if (cudaMalloc(&df, fx.size() * 4 + 4) || cudaMemcpy(df, fx.data(), fx.size() * 4, cudaMemcpyHostToDevice) ||
        cudaMalloc(&dout[0], (size_t)CH * 4) || cudaMalloc(&dout[1], (size_t)CH * 4) ||
        cudaMallocHost(&hout[0], (size_t)CH * 4) || cudaMallocHost(&hout[1], (size_t)CH * 4) ||
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) ||
        cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming) ||
        cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming))
        rs = RIV_ERR_CUDA;
    const uint64_t total = (uint64_t)hi_bits - lo_bits + 1;
    const uint64_t nch = (total + CH - 1) / CH;
    auto enqueue = [&](uint64_t c) {
        const int k = (int)(c & 1);
        const uint32_t base = (uint32_t)(lo_bits + c * CH);
        const uint32_t n = (uint32_t)std::min<uint64_t>(CH, total - c * CH);
        return launch_libm_range(which, base, n, (float*)dout[k], (const uint32_t*)df, npairs, st) == 0 &&
               cudaMemcpyAsync(hout[k], dout[k], (size_t)n * 4, cudaMemcpyDeviceToHost, st) == cudaSuccess &&
               cudaEventRecord(done[k], st) == cudaSuccess;
    };
    if (!rs && !enqueue(0)) rs = RIV_ERR_CUDA;
    for (uint64_t c = 0; !rs && c < nch; c++) {
        if (c + 1 < nch && !enqueue(c + 1)) { rs = RIV_ERR_CUDA; break; }
        if (cudaEventSynchronize(done[c & 1]) != cudaSuccess) { rs = RIV_ERR_CUDA; break; }
        compare((const float*)hout[c & 1], (uint32_t)(lo_bits + c * CH), (uint32_t)std::min<uint64_t>(CH, total - c * CH));
    }
    if (st) cudaStreamSynchronize(st);
    for (int k = 0; k < 2; k++) {
        cudaFree(dout[k]);
        cudaFreeHost(hout[k]);
        if (done[k]) cudaEventDestroy(done[k]);
    }
    cudaFree(df);
    if (st) cudaStreamDestroy(st);
    *mismatches = bad.load();
    *first_bad_bits = bad.load() ? first.load() : 0;
    return rs;
}

riv_status riv_test_wait_expiry(int which, int64_t spin_limit, uint32_t* status_word) {
    if (which < 0 || which > 3 || spin_limit < 1 || spin_limit > (1 << 20) || !status_word) return RIV_ERR_FRAME;
    *status_word = 0;
    try {
        StageBufs B;
        auto* rec = (unsigned long long*)B.get(4 * 8);
        auto* cnt = (unsigned*)B.get(4 * 4);
        auto* st = (unsigned*)B.get(4);
        CK(cudaMemset(rec, 0, 4 * 8));
        CK(cudaMemset(cnt, 0, 4 * 4));
        CK(cudaMemset(st, 0, 4));
        CK((cudaError_t)launch_wait_expiry(which, rec, cnt, (long long)spin_limit, st, 0));
        CK(cudaDeviceSynchronize());
        CK(cudaMemcpy(status_word, st, 4, cudaMemcpyDeviceToHost));
    } catch (const CudaError&) {
        return RIV_ERR_CUDA;
    }
    return (*status_word & ST_WAIT_TIMEOUT) ? RIV_ERR_DEVICE_TIMEOUT : RIV_OK;
}

riv_status riv_libm_fixup_counts(uint32_t* nlog, uint32_t* nexp) {
    LibmFix& F = libm_fix();
    if (!F.ok) return RIV_ERR_ENCODING_FAILED;
    *nlog = (uint32_t)(F.logf.size() / 2);
    *nexp = (uint32_t)(F.exp2f.size() / 2);
    return RIV_OK;
}

void riv_dct_tables(int32_t* t16, int32_t* t8) { dct_tables(t16, t8); }

riv_status riv_test_worker_queue(uint32_t bw, uint32_t bh, uint32_t w, int defer, int deblock, int tables, int compact,
                                 int32_t* out, size_t cap, size_t* n) {
    if (!n || bw == 0 || bh == 0) return RIV_ERR_FRAME;
    const QueueShape q = queue_shape((int)bw, (int)bh, (int)w, defer != 0, deblock != 0, tables != 0, compact != 0);
    size_t i = 0;
    for (int k = 0; k < q.steps + q.csteps; k++) {
        int R, D, T;
        queue_step(q, k, R, D, T);
        for (int t = 0; t < R + D + T; t++, i++) {
            int kind, row, idx;
            queue_task(q, k, t, R, D, kind, row, idx);
            if (out && 3 * i + 2 < cap) {
                out[3 * i] = kind;
                out[3 * i + 1] = row;
                out[3 * i + 2] = idx;
            }
        }
    }
    *n = i;
    return i == (size_t)queue_total(q) ? RIV_OK : RIV_ERR_ENCODING_FAILED;
}

riv_status riv_test_delta_bias(const int8_t* dx, const int8_t* dy, uint32_t n, int8_t* bx, int8_t* by) {
    if (!bx || !by || (n > 0 && (!dx || !dy))) return RIV_ERR_FRAME;
    std::vector<std::pair<int8_t, int8_t>> d(n);
    for (uint32_t i = 0; i < n; i++) d[i] = {dx[i], dy[i]};
    riv::compute_delta_bias(d, *bx, *by);
    return RIV_OK;
}

static riv::MvCodedBlock mv_block_from(const uint8_t* r) {
    riv::MvCodedBlock b;
    b.mode = r[0];
    b.new_base = r[1];
    b.dx = (int8_t)r[2];
    b.dy = (int8_t)r[3];
    b.spx = r[4];
    b.spy = r[5];
    b.skip = r[6] != 0;
    return b;
}

riv_status riv_test_mv_encode(const uint8_t* blocks, const uint32_t* dims, uint32_t nframes, uint8_t* out, size_t cap,
                              size_t* len, uint32_t* frame_len) {
    return riv_test_mv_encode_threads(blocks, dims, nframes, 0, out, cap, len, frame_len);
}

riv_status riv_test_mv_encode_threads(const uint8_t* blocks, const uint32_t* dims, uint32_t nframes, uint32_t threads,
                                      uint8_t* out, size_t cap, size_t* len, uint32_t* frame_len) {
    if (!len || (nframes > 0 && (!blocks || !dims || !frame_len))) return RIV_ERR_FRAME;
    entropy_init();
    riv::MvCoder coder;
    std::vector<uint8_t> all, fb;
    std::unique_ptr<ThreadPool> pool(threads > 0 ? new ThreadPool(threads) : nullptr);
    BatchSubmit submit;
    if (pool) {
        ThreadPool* tp = pool.get();
        submit = [tp](std::function<void()> f) { return tp->submit(std::move(f)); };
    }
    size_t k = 0;
    try {
        for (uint32_t f = 0; f < nframes; f++) {
            const size_t n = (size_t)dims[2 * f] * dims[2 * f + 1];
            std::vector<riv::MvCodedBlock> v(n);
            for (size_t i = 0; i < n; i++, k++) v[i] = mv_block_from(blocks + 7 * k);
            if (pool) coder.encode_frame_parallel(v, (int)dims[2 * f], fb, submit, (int)threads + 1);
            else coder.encode_frame(v, (int)dims[2 * f], fb);
            frame_len[f] = (uint32_t)fb.size();
            all.insert(all.end(), fb.begin(), fb.end());
        }
    } catch (const std::exception&) {
        return RIV_ERR_ENCODING_FAILED;
    }
    *len = all.size();
    if (out && cap) memcpy(out, all.data(), std::min(cap, all.size()));
    return RIV_OK;
}

riv_status riv_test_mv_decode(const uint8_t* data, const uint32_t* frame_len, const uint32_t* dims, uint32_t nframes,
                              uint8_t* blocks) {
    if (nframes > 0 && (!frame_len || !dims || !blocks)) return RIV_ERR_FRAME;
    entropy_init();
    riv::MvCoder coder;
    std::vector<riv::MvCodedBlock> v;
    size_t pos = 0, k = 0;
    for (uint32_t f = 0; f < nframes; f++) {
        if (frame_len[f] > 0 && !data) return RIV_ERR_FRAME;
        if (!coder.decode_frame(data + pos, frame_len[f], (int)dims[2 * f], (int)dims[2 * f + 1], v))
            return RIV_ERR_FRAME;
        pos += frame_len[f];
        for (const riv::MvCodedBlock& b : v) {
            uint8_t* r = blocks + 7 * k++;
            r[0] = b.mode;
            r[1] = b.new_base;
            r[2] = (uint8_t)b.dx;
            r[3] = (uint8_t)b.dy;
            r[4] = b.spx;
            r[5] = b.spy;
            r[6] = b.skip ? 1 : 0;
        }
    }
    return RIV_OK;
}

riv_status riv_test_dct_decode(const uint8_t* data, size_t len, const uint8_t* coded, uint32_t n, int intra,
                               int16_t* out) {
    if ((len > 0 && !data) || (n > 0 && (!coded || !out))) return RIV_ERR_FRAME;
    entropy_init();
    return decode_residual_frame(data, len, coded, (int)n, intra != 0, out) ? RIV_OK : RIV_ERR_FRAME;
}

riv_status riv_test_dct_encode(const int16_t* blocks, uint32_t n, int intra, uint32_t threads, uint8_t* out, size_t cap,
                               size_t* len) {
    if ((n > 0 && !blocks) || !len) return RIV_ERR_FRAME;
    entropy_init();
    // the GPU compaction's layout: per plane the run up to the last non-zero coefficient
    // (with DC prediction the last non-zero AC coefficient), and that index
    std::vector<int16_t> packed;
    std::vector<uint8_t> eobs((size_t)n * 3);
    static const int base[3] = {0, 256, 320}, len3[3] = {256, 64, 64};
    for (uint32_t b = 0; b < n; b++)
        for (int pl = 0; pl < 3; pl++) {
            const int16_t* p = blocks + (size_t)b * 384 + base[pl];
            int last = 0;
            for (int i = len3[pl] - 1; i >= (intra ? 1 : 0); i--)
                if (p[i] != 0) { last = i; break; }
            eobs[(size_t)b * 3 + pl] = (uint8_t)last;
            packed.insert(packed.end(), p, p + last + 1);
        }
    std::vector<uint8_t> stream;
    try {
        if (threads > 0) {
            ThreadPool pool(threads);
            BatchSubmit sub = [&pool](std::function<void()> f) { return pool.submit(std::move(f)); };
            encode_residual_frame(packed.data(), eobs.data(), (int)n, intra != 0, stream, &sub, (int)threads + 1);
        } else {
            encode_residual_frame(packed.data(), eobs.data(), (int)n, intra != 0, stream);
        }
    } catch (const std::exception&) {
        return RIV_ERR_ENCODING_FAILED;
    }
    *len = stream.size();
    if (out && cap) memcpy(out, stream.data(), std::min(cap, stream.size()));
    return RIV_OK;
}

}  // extern "C"

// =====================================================================================
// Decoder (dec/decoder.rs:112-460) up to the YUV reconstruction: host entropy decoding and
// MV reconstruction, GPU prediction, AQ, inverse transforms and deblock.
// =====================================================================================
namespace {
struct DecMv {
    int8_t dx = 0, dy = 0, sx = 0, sy = 0;
    bool operator==(const DecMv& o) const { return dx == o.dx && dy == o.dy && sx == o.sx && sy == o.sy; }
};
static int8_t sat8i(int v) { return (int8_t)std::min(std::max(v, -128), 127); }
static uint64_t get_le(const uint8_t* b, int n) {
    uint64_t v = 0;
    for (int i = n - 1; i >= 0; i--) v = (v << 8) | b[i];
    return v;
}
}  // namespace

// One record read ahead of the GPU: parsed, its MVs decoded and reconstructed (in order, on
// the calling thread: the MV coder's contexts and the temporal MVs carry across frames), its
// coefficients decoding on the pool (each frame's coefficient coder starts from fresh
// contexts, so several frames decode at once).
struct DecSlot {
    bool filled = false;
    riv_dec_status st = RIV_DEC_OK;  // a record that could not be read: reported when reached
    std::string msg;
    int type = 0;
    uint8_t q = 0;
    uint64_t ts = 0;
    HostBuf hcoeffs, hmbout, hskip, hfmask;  // pinned staging for the uploads
    std::vector<uint8_t> coded;
    bool coef_ok = false;
    std::future<void> coef;
};
constexpr int DEC_AHEAD = 8;

struct riv_decoder {
    std::vector<uint8_t> data;
    uint32_t dw = 0, dh = 0, sw = 0, sh = 0, fps = 0;
    uint64_t frame_count = 0, current = 0;
    int W = 0, H = 0, BW = 0, BH = 0, N = 0;
    int device = 0;
    std::string err;
    bool poisoned = false, has_ref = false;
    int ref_cur = 0;
    cudaStream_t S = nullptr;
    DevBuf ref[2], recon_pre, pred, coeffs, mbout, skip, fmask, varsum, lnv, qs, logfix, expfix, ytab, ctab;
    DevBuf rgbdev;  // display-size RGB24 output, allocated on first use
    int nlog = 0, nexp = 0;
    // read-ahead state (records up to DEC_AHEAD frames past `current`)
    DecSlot slots[DEC_AHEAD];
    uint64_t ahead = 0;       // next frame to read ahead
    size_t ahead_pos = 36;    // its record's offset
    bool ahead_stop = false;  // a record could not be read: nothing after it is read
    bool ahead_ref = false;   // a key frame was read (inter records have a reference)
    riv::MvCoder mvc;
    std::vector<DecMv> prev_mvs, mvs;
    std::vector<riv::MvCodedBlock> blocks;
    std::unique_ptr<ThreadPool> pool;  // coefficient decoding
};

static riv_dec_status dec_fail(riv_decoder* d, riv_dec_status s, const std::string& m) {
    d->err = m;
    if (s == RIV_DEC_CUDA) d->poisoned = true;
    return s;
}

// Read frame `d->ahead`'s record into its slot: parse it, decode and reconstruct its MVs (in
// frame order), and start its coefficient decoding on the pool.  A record that cannot be read
// is kept in the slot as an error, reported when that frame is requested; nothing after it
// is read (dec/decoder.rs:174-460).
static void dec_read_ahead(riv_decoder* d) {
    DecSlot& sl = d->slots[d->ahead % DEC_AHEAD];
    d->ahead++;
    sl.filled = true;
    sl.st = RIV_DEC_OK;
    sl.msg.clear();
    auto stop = [&](riv_dec_status st, const char* m) {
        sl.st = st;
        sl.msg = m;
        d->ahead_stop = true;
    };
    const uint8_t* b = d->data.data() + d->ahead_pos;
    const size_t left = d->data.size() - d->ahead_pos;
    if (left < 9) return stop(RIV_DEC_IO, "truncated record");
    sl.ts = get_le(b, 8);
    sl.type = b[8];
    const int N = d->N;
    const uint8_t* cdata = nullptr;
    size_t clen = 0;
    if (sl.type == 1) {  // intra (residual.rs:815-887)
        if (left < 14) return stop(RIV_DEC_IO, "truncated intra record");
        sl.q = b[9];
        clen = get_le(b + 10, 4);
        if (left < 14 + clen) return stop(RIV_DEC_IO, "truncated intra payload");
        cdata = b + 14;
        sl.coded.assign(N, 1);
        d->ahead_pos += 14 + clen;
        d->prev_mvs.clear();
        d->mvc.reset();
        d->ahead_ref = true;
    } else if (sl.type == 2) {  // inter (residual.rs:889-1079, decoder.rs:255-430)
        if (left < 17 || !d->ahead_ref) return stop(RIV_DEC_INVALID_FRAME, "inter frame without a reference");
        sl.q = b[9];
        const int biasx = (int8_t)b[10], biasy = (int8_t)b[11];
        const size_t mvs = get_le(b + 13, 4);
        if (left < 17 + mvs + 4) return stop(RIV_DEC_IO, "truncated motion data");
        const uint8_t* mvd = b + 17;
        clen = get_le(b + 17 + mvs, 4);
        if (left < 21 + mvs + clen) return stop(RIV_DEC_IO, "truncated residual data");
        cdata = b + 21 + mvs;
        if (!d->mvc.decode_frame(mvd, mvs, d->BW, d->BH, d->blocks))
            return stop(RIV_DEC_INVALID_FRAME, "malformed motion data");
        const bool tm = !d->prev_mvs.empty();
        // MV reconstruction in raster order from the decoded neighbours (mv_predictor.rs)
        const int BW = d->BW;
        d->mvs.assign(N, DecMv{});
        sl.coded.assign(N, 0);
        MbOut* mo = sl.hmbout.as<MbOut>();
        uint8_t* hs = sl.hskip.as<uint8_t>();
        uint8_t* hf = sl.hfmask.as<uint8_t>();
        for (int i = 0; i < N; i++) {
            const riv::MvCodedBlock& cb = d->blocks[i];
            const int bx = i % BW, by = i / BW;
            const bool hl = bx > 0, ht = by > 0, htr = by > 0 && bx + 1 < BW, htl = by > 0 && bx > 0;
            const DecMv L = hl ? d->mvs[i - 1] : DecMv{}, T = ht ? d->mvs[i - BW] : DecMv{};
            const DecMv TR = htr ? d->mvs[i - BW + 1] : DecMv{}, TL = htl ? d->mvs[i - BW - 1] : DecMv{};
            const DecMv TM = tm ? d->prev_mvs[i] : DecMv{};
            DecMv cand[5];
            int nc = 0;
            auto add = [&](bool has, const DecMv& m) {
                if (!has) return;
                for (int k = 0; k < nc; k++)
                    if (cand[k] == m) return;
                cand[nc++] = m;
            };
            add(hl, L); add(ht, T); add(htr, TR); add(htl, TL); add(tm, TM);
            const DecMv nearest = nc > 0 ? cand[0] : DecMv{}, nearm = nc > 1 ? cand[1] : DecMv{};
            const DecMv temporal = tm ? TM : DecMv{};
            DecMv base{};
            switch (cb.mode) {
                case riv::M_ZERO: break;
                case riv::M_NEAREST: base = nearest; break;
                case riv::M_NEAR: base = nearm; break;
                case riv::M_TOPRIGHT: base = htr ? TR : nearest; break;
                case riv::M_TOPLEFT: base = htl ? TL : nearest; break;
                case riv::M_TEMPORAL: base = temporal; break;
                default:
                    base = cb.new_base == 0 ? nearest : cb.new_base == 1 ? nearm
                           : cb.new_base == 2 ? (htr ? TR : nearest)
                           : cb.new_base == 3 ? (htl ? TL : nearest) : cb.new_base == 4 ? temporal : nearest;
            }
            DecMv m;
            if (cb.mode == riv::M_NEW) {
                m.dx = sat8i(base.dx + sat8i(cb.dx + biasx));
                m.dy = sat8i(base.dy + sat8i(cb.dy + biasy));
                m.sx = cb.spx == riv::SP_PLUS ? 1 : (cb.spx == riv::SP_MINUS ? -1 : 0);
                m.sy = cb.spy == riv::SP_PLUS ? 1 : (cb.spy == riv::SP_MINUS ? -1 : 0);
            } else {
                m = base;
            }
            d->mvs[i] = m;
            MbOut o{};
            o.raw[0] = m.dx; o.raw[1] = m.dy; o.raw[2] = m.sx; o.raw[3] = m.sy;
            mo[i] = o;
            hs[i] = cb.skip ? 1 : 0;
            hf[i] = (!cb.skip || m.dx || m.dy || m.sx || m.sy) ? 1 : 0;
            sl.coded[i] = cb.skip ? 0 : 1;
        }
        d->ahead_pos += 21 + mvs + clen;
        d->prev_mvs.swap(d->mvs);
    } else {
        return stop(RIV_DEC_INVALID_FRAME, "unknown frame type");
    }
    const bool intra = sl.type == 1;
    DecSlot* ps = &sl;
    sl.coef_ok = false;
    sl.coef = d->pool->submit([ps, cdata, clen, N, intra] {
        ps->coef_ok = riv::decode_residual_frame(cdata, clen, ps->coded.data(), N, intra, ps->hcoeffs.as<int16_t>());
    });
}


extern "C" {

riv_dec_status riv_decoder_new(const uint8_t* data, size_t len, int device, riv_decoder** out) {
    if (!out) return RIV_DEC_INVALID_HEADER;
    *out = nullptr;
    if (!data || len < 36 || memcmp(data, "RIV\0", 4) != 0 || get_le(data + 4, 4) != 5) return RIV_DEC_INVALID_HEADER;
    riv_decoder* d = nullptr;
    try {  // a large stream may not fit in host memory: no exception crosses the C ABI
        d = new riv_decoder();
        d->data.assign(data, data + len);
    } catch (const std::exception&) {
        delete d;
        return RIV_DEC_DECODING_FAILED;
    }
    d->dw = (uint32_t)get_le(data + 8, 4);
    d->dh = (uint32_t)get_le(data + 12, 4);
    d->sw = (uint32_t)get_le(data + 16, 4);
    d->sh = (uint32_t)get_le(data + 20, 4);
    d->fps = (uint32_t)get_le(data + 24, 4);
    d->frame_count = get_le(data + 28, 8);
    if (d->sw == 0 || d->sh == 0 || d->sw % 16 || d->sh % 16 || d->dw > d->sw || d->dh > d->sh || d->sw > 16384 ||
        d->sh > 16384) {
        delete d;
        return RIV_DEC_INVALID_HEADER;
    }
    d->W = (int)d->sw;
    d->H = (int)d->sh;
    d->BW = d->W / 16;
    d->BH = d->H / 16;
    d->N = d->BW * d->BH;
    d->device = device;
    LibmFix& F = libm_fix();
    if (!F.ok) {
        d->err = F.err;
        riv_decoder_free(d);
        return RIV_DEC_DECODING_FAILED;
    }
    try {
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&d->S, cudaStreamNonBlocking));
        const size_t yuv = (size_t)d->W * d->H * 3 / 2, N = (size_t)d->N;
        d->ref[0].alloc(yuv);
        d->ref[1].alloc(yuv);
        d->recon_pre.alloc(yuv);
        d->pred.alloc(yuv);
        d->coeffs.alloc(N * 384 * 2);
        d->mbout.alloc(N * sizeof(MbOut));
        d->skip.alloc(N);
        d->fmask.alloc(N);
        d->varsum.alloc(N * sizeof(uint2));
        d->lnv.alloc((N + 4) * sizeof(float));
        d->qs.alloc(N * sizeof(float));
        d->ytab.alloc(256 * 2);
        d->ctab.alloc(64 * 2);
        for (DecSlot& sl : d->slots) {
            sl.hcoeffs.alloc(N * 384 * 2);
            sl.hmbout.alloc(N * sizeof(MbOut));
            sl.hskip.alloc(N);
            sl.hfmask.alloc(N);
        }
        d->nlog = (int)(F.logf.size() / 2);
        d->nexp = (int)(F.exp2f.size() / 2);
        d->logfix.alloc(F.logf_dev.size() * 4);
        d->expfix.alloc(F.exp2f_dev.size() * 4);
        CK(cudaMemcpy(d->logfix.p, F.logf_dev.data(), F.logf_dev.size() * 4, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d->expfix.p, F.exp2f_dev.data(), F.exp2f_dev.size() * 4, cudaMemcpyHostToDevice));
        int32_t t16[256], t8[64];
        dct_tables(t16, t8);
        CK(riv_upload_dct_tables(t16, t8));
    } catch (const CudaError& ce) {
        d->err = std::string(ce.where) + ": " + cudaGetErrorString(ce.e);
        riv_decoder_free(d);
        return RIV_DEC_CUDA;
    } catch (const std::exception&) {  // host allocation failures
        riv_decoder_free(d);
        return RIV_DEC_DECODING_FAILED;
    }
    riv::entropy_init();
    const unsigned hw = std::thread::hardware_concurrency();
    d->pool.reset(new ThreadPool(std::max(1u, std::min((unsigned)DEC_AHEAD, hw > 1 ? hw - 1 : 1u))));
    *out = d;
    return RIV_DEC_OK;
}

riv_dec_status riv_decoder_info(const riv_decoder* d, uint32_t* dims5, uint64_t* frame_count) {
    if (!d) return RIV_DEC_INVALID_HEADER;
    if (dims5) {
        dims5[0] = d->dw; dims5[1] = d->dh; dims5[2] = d->sw; dims5[3] = d->sh; dims5[4] = d->fps;
    }
    if (frame_count) *frame_count = d->frame_count;
    return RIV_DEC_OK;
}

uint64_t riv_decoder_current_frame(const riv_decoder* d) { return d ? d->current : 0; }
const char* riv_decoder_last_error(const riv_decoder* d) { return d ? d->err.c_str() : "null decoder"; }

// One frame: the YUV planes and / or the display-size RGB24 (each nullable).
static riv_dec_status dec_frame(riv_decoder* d, uint8_t* y, uint8_t* u, uint8_t* v, uint8_t* rgb, uint32_t* frame_type,
                                uint64_t* timestamp_ms) {
    if (!d) return RIV_DEC_INVALID_HEADER;
    if (d->poisoned) return dec_fail(d, RIV_DEC_CUDA, "decoder unusable after a device failure");
    if (d->current >= d->frame_count) return dec_fail(d, RIV_DEC_END_OF_STREAM, "end of stream");
    auto read_ahead = [&](uint64_t upto) -> bool {  // frames before `upto`
        try {
            while (!d->ahead_stop && d->ahead < d->frame_count && d->ahead < upto) dec_read_ahead(d);
        } catch (const std::exception& ex) {
            dec_fail(d, RIV_DEC_DECODING_FAILED, ex.what());
            return false;
        }
        return true;
    };
    if (!read_ahead(d->current + 1)) return RIV_DEC_DECODING_FAILED;  // this frame; the rest while the GPU works
    DecSlot& sl = d->slots[d->current % DEC_AHEAD];
    if (!sl.filled) return dec_fail(d, RIV_DEC_IO, "truncated record");
    if (sl.st != RIV_DEC_OK) return dec_fail(d, sl.st, sl.msg);
    sl.coef.wait();
    const int type = sl.type;
    if (!sl.coef_ok)
        return dec_fail(d, RIV_DEC_INVALID_FRAME, type == 1 ? "malformed intra coefficient data" : "malformed residual data");
    const int W = d->W, H = d->H, N = d->N;
    const size_t ysz = (size_t)W * H, csz = ysz / 4;
    const int nxt = d->ref_cur ^ 1;
    uint8_t* recon = d->ref[nxt].as<uint8_t>();
    try {
        CK(cudaSetDevice(d->device));
        cudaStream_t S = d->S;
        const int level = deblock_level(quant_step(sl.q));
        uint8_t* target = level > 0 ? d->recon_pre.as<uint8_t>() : recon;
        if (type == 1) {
            uint16_t yt[256], ct[64];
            intra_tables(quant_step(sl.q), yt, ct);
            CK(cudaMemcpyAsync(d->ytab.p, yt, sizeof yt, cudaMemcpyHostToDevice, S));
            CK(cudaMemcpyAsync(d->ctab.p, ct, sizeof ct, cudaMemcpyHostToDevice, S));
            CK(cudaMemcpyAsync(d->coeffs.p, sl.hcoeffs.p, (size_t)N * 768, cudaMemcpyHostToDevice, S));
            CK(launch_reconstruct(d->coeffs.as<int16_t>(), nullptr, nullptr, nullptr, 1, d->ytab.as<uint16_t>(),
                                  d->ctab.as<uint16_t>(), target, W, H, S));
            if (level > 0) {
                int E, I, Hv;
                deblock_thresholds(level, true, E, I, Hv);
                CK(launch_deblock_tiled(target, recon, W, H, E, I, Hv, nullptr, S));
            }
        } else {
            if (!d->has_ref) return dec_fail(d, RIV_DEC_INVALID_FRAME, "inter frame without a reference");
            CK(cudaMemcpyAsync(d->mbout.p, sl.hmbout.p, (size_t)N * sizeof(MbOut), cudaMemcpyHostToDevice, S));
            CK(cudaMemcpyAsync(d->skip.p, sl.hskip.p, N, cudaMemcpyHostToDevice, S));
            CK(cudaMemcpyAsync(d->fmask.p, sl.hfmask.p, N, cudaMemcpyHostToDevice, S));
            CK(cudaMemcpyAsync(d->coeffs.p, sl.hcoeffs.p, (size_t)N * 768, cudaMemcpyHostToDevice, S));
            const uint8_t* ref = d->ref[d->ref_cur].as<uint8_t>();
            CK(launch_predict(ref, d->mbout.as<MbOut>(), d->pred.as<uint8_t>(), d->varsum.as<uint2>(), W, H, S));
            CK(launch_aq(d->varsum.as<uint2>(), N, quant_step(sl.q), d->logfix.as<uint32_t>(), d->nlog,
                         d->expfix.as<uint32_t>(), d->nexp, d->lnv.as<float>(), d->qs.as<float>(), S));
            CK(launch_reconstruct(d->coeffs.as<int16_t>(), d->pred.as<uint8_t>(), d->skip.as<uint8_t>(),
                                  d->qs.as<float>(), 0, nullptr, nullptr, target, W, H, S));
            if (level > 0) {
                int E, I, Hv;
                deblock_thresholds(level, false, E, I, Hv);
                CK(launch_deblock_tiled(target, recon, W, H, E, I, Hv, d->fmask.as<uint8_t>(), S));
            }
        }
        if (y) CK(cudaMemcpyAsync(y, recon, ysz, cudaMemcpyDeviceToHost, S));
        if (u) CK(cudaMemcpyAsync(u, recon + ysz, csz, cudaMemcpyDeviceToHost, S));
        if (v) CK(cudaMemcpyAsync(v, recon + ysz + csz, csz, cudaMemcpyDeviceToHost, S));
        if (rgb) {  // dec/decoder.rs:445-456: to RGB24, cropped to the display size
            const size_t rgb_bytes = (size_t)d->dw * d->dh * 3;
            if (!d->rgbdev.p) d->rgbdev.alloc(rgb_bytes);
            CK(launch_yuv_to_rgb(recon, W, H, (int)d->dw, (int)d->dh, d->rgbdev.as<uint8_t>(), S));
            CK(cudaMemcpyAsync(rgb, d->rgbdev.p, rgb_bytes, cudaMemcpyDeviceToHost, S));
        }
        // read the next frames while the GPU reconstructs this one (their slots are not this
        // frame's, whose staging the copies above read), then finish this frame; a failure
        // here is reported by the next call, which reads its frame first
        read_ahead(d->current + DEC_AHEAD);
        CK(cudaStreamSynchronize(S));
    } catch (const CudaError& ce) {
        return dec_fail(d, RIV_DEC_CUDA, std::string(ce.where) + ": " + cudaGetErrorString(ce.e));
    } catch (const std::exception& ex) {
        return dec_fail(d, RIV_DEC_DECODING_FAILED, ex.what());
    }
    sl.filled = false;
    d->ref_cur = nxt;
    d->has_ref = true;
    if (frame_type) *frame_type = (uint32_t)type;
    if (timestamp_ms) *timestamp_ms = sl.ts;
    d->current++;
    return RIV_DEC_OK;
}

riv_dec_status riv_decode_frame_yuv(riv_decoder* d, uint8_t* y, uint8_t* u, uint8_t* v, uint32_t* frame_type,
                                    uint64_t* timestamp_ms) {
    return dec_frame(d, y, u, v, nullptr, frame_type, timestamp_ms);
}

riv_dec_status riv_decode_frame_rgb(riv_decoder* d, uint8_t* rgb, uint32_t* frame_type, uint64_t* timestamp_ms) {
    return dec_frame(d, nullptr, nullptr, nullptr, rgb, frame_type, timestamp_ms);
}

void riv_decoder_free(riv_decoder* d) {
    if (!d) return;
    cudaSetDevice(d->device);
    if (d->S) cudaStreamSynchronize(d->S);
    DevBuf* bufs[] = {&d->ref[0], &d->ref[1], &d->recon_pre, &d->pred, &d->coeffs, &d->mbout, &d->skip, &d->fmask,
                      &d->varsum, &d->lnv, &d->qs, &d->logfix, &d->expfix, &d->ytab, &d->ctab, &d->rgbdev};
    for (DevBuf* x : bufs) x->release();
    d->pool.reset();  // finishes the coefficient decodes still queued (they write the slots)
    for (DecSlot& sl : d->slots) {
        HostBuf* hb[] = {&sl.hcoeffs, &sl.hmbout, &sl.hskip, &sl.hfmask};
        for (HostBuf* x : hb) x->release();
    }
    if (d->S) cudaStreamDestroy(d->S);
    delete d;
}

}  // extern "C"

// =====================================================================================
// Multi-clip encoding (riv_batch).  No counterpart in the reference, which encodes one
// stream per Encoder.  A batch owns one encoder per clip (its config, writer, buffers, MV
// coder and record pipeline); a step takes at most one frame per clip and runs its GPU work
// as one launch per stage over every clip of the step on one stream (riv_batch.cuh), then
// hands each clip's frame to that clip's host pipeline (retire / write_job), exactly as
// riv_encode_frame does.  Each clip's stream is therefore byte-identical to a single-clip
// encode of the clip.
// =====================================================================================
namespace {
constexpr int BT_BOUNDS = BS_N + 3;  // timing marks: start, then one after each stage
enum { TB_START, TB_CONVERT, TB_TABLE, TB_SEARCH, TB_PREDICT, TB_AQSUM, TB_RESIDUAL, TB_DEBLOCK, TB_SCAN, TB_PACK };
constexpr int BT_NSTAGE = 9;  // convert, table, search, predict, aq mean, residual, deblock, scan, pack
// Autotuner candidates (one dimension per timed stage; the streams do not depend on them).
// The search has six candidates (CTA share x SAD table or not, timed as table + search stages),
// the residual and the deblock three each (cycled twice as often).
constexpr int TUNE_NCAND = 6;
constexpr int TUNE_ROWS_PCT[TUNE_NCAND] = {100, 75, 50, 100, 75, 50};
constexpr int TUNE_TABLE[TUNE_NCAND] = {1, 1, 1, 0, 0, 0};
constexpr int TUNE_RES_MBS[3] = {4, 2, 8};
constexpr int TUNE_DB_TW[3] = {128, 64, 256};
constexpr int TUNE_ROUNDS = 2;  // all-P-frame steps measured per candidate
}  // namespace

struct riv_batch {
    int device = 0;
    std::vector<riv_encoder*> clips;
    std::shared_ptr<ThreadPool> pool, rans_pool, mv_pool;
    cudaStream_t B = nullptr, Hs = nullptr, C = nullptr;  // GPU chain, host->device, device->host
    cudaEvent_t ev_h2d = nullptr, ev_gpu = nullptr;
    std::vector<cudaEvent_t> ev_step;  // per step in flight: its GPU work and copies done
    // stage timing marks of timed steps, two sets: a step's marks are read one timed step later
    // (or at the end), so that reading them rarely waits for the GPU
    cudaEvent_t ev_t[2][BT_BOUNDS] = {};
    struct TimedStep {
        bool pending = false, tuning = false;
        int cand = 0;
        uint64_t mbs = 0, pmbs = 0;
    } tpend[2];
    int tpar = 0;
    // step descriptors: pinned staging (double-buffered), one device copy
    HostBuf hdesc[2];
    cudaEvent_t ev_desc[2] = {};
    DevBuf ddesc;
    size_t off_sp = 0, off_start = 0, off_sstart = 0, desc_bytes = 0;
    int dpar = 0;
    int max_sr = 0;
    // search capacity per variant: 0 table + small costs, 1 table, 2 no table
    int cap[3] = {0, 0, 0}, sthreads[3] = {0, 0, 0};
    size_t ssmem[3] = {0, 0, 0};
    // tile shapes and the autotuner
    BatchTune tune{4, 128, 100, 1};
    bool fixed = false, tuned = false;
    int tune_step = 0;          // tuning steps submitted (candidate = (tune_step / ROUNDS) % 3)
    double tune_us[3][TUNE_NCAND] = {};  // [dimension][candidate] summed microseconds per MB
    int tune_n[3][TUNE_NCAND] = {};      // all-P-frame steps measured per candidate
    uint64_t steps = 0, frames = 0, mbs = 0, launches = 0, timed = 0;
    double stage_us[BT_NSTAGE + 1] = {};  // sums over timed steps (last: whole step)
    uint64_t h2d_bytes = 0, d2h_bytes = 0;
    // host milliseconds: [0] making room (earlier records of a clip written before its next
    // frame), [1] descriptors and launches, [2] copies back and step bookkeeping, [3] advancing
    // the clips' pipelines after the step, [4] finish
    double host_ms[5] = {0, 0, 0, 0, 0};
    std::string err;
    bool poisoned = false;
};

namespace {

static int search_variant(const riv_encoder* e) { return e->table_ok ? (e->small_costs ? 0 : 1) : 2; }

// Row CTAs of each clip of one search launch: about proportional to its MBs, at least one, at
// most its MB rows, `total` in all (>= the number of clips).
static void spread_rows(const std::vector<int>& nmb, const std::vector<int>& bh, int total, std::vector<int>& out) {
    const size_t n = nmb.size();
    out.assign(n, 1);
    double sum = 0;
    for (size_t i = 0; i < n; i++) sum += nmb[i];
    int used = 0;
    for (size_t i = 0; i < n; i++) {
        out[i] = std::max(1, std::min(bh[i], (int)((double)total * nmb[i] / sum)));
        used += out[i];
    }
    while (used > total) {  // the minimum of one may overshoot: take from the largest
        size_t k = 0;
        for (size_t i = 1; i < n; i++)
            if (out[i] > out[k]) k = i;
        if (out[k] <= 1) break;
        out[k]--;
        used--;
    }
    while (used < total) {  // hand out what rounding left, to the clip with most MBs per CTA
        size_t k = n;
        double worst = 0;
        for (size_t i = 0; i < n; i++) {
            if (out[i] >= bh[i]) continue;
            const double load = (double)nmb[i] / out[i];
            if (k == n || load > worst) { worst = load; k = i; }
        }
        if (k == n) break;
        out[k]++;
        used++;
    }
}

static riv_status batch_fail(riv_batch* b, riv_status s, const std::string& msg) {
    b->err = msg;
    if (s == RIV_ERR_CUDA || s == RIV_ERR_DEVICE_TIMEOUT) b->poisoned = true;
    return s;
}

// The frame of clip `e` in this step: descriptor, search parameters and state updates, like
// submit_gpu but without launching anything.  src: 0 host RGB (copied on `hs`), 1 device RGB.
static void batch_collect(riv_encoder* e, Job& j, int src, const void* frame, cudaStream_t hs, BatchClip& k,
                          SearchParams& sp) {
    const riv_config& c = e->cfg;
    Slot& s = e->slots[j.slot];
    const int W = e->W, H = e->H, N = e->NMB;
    const int ck = e->fpar;
    j.ck = ck;
    uint8_t* cur = e->curb[ck].as<uint8_t>();
    MbOut* mbo = e->mboutb[ck].as<MbOut>();
    memset(&k, 0, sizeof(k));
    k.W = W; k.H = H; k.BW = e->BW; k.NMB = N;
    k.intra = j.type == 1 ? 1 : 0;
    k.dw = (int)c.display_width;
    k.dh = (int)c.display_height;
    k.cur = cur;
    if (src == 0) {
        CK(cudaMemcpyAsync(s.rgb.p, frame, (size_t)c.display_width * c.display_height * 3, cudaMemcpyHostToDevice, hs));
        k.rgb = s.rgb.as<uint8_t>();
        e->h2d_bytes += (uint64_t)c.display_width * c.display_height * 3;
    } else {
        k.rgb = (const uint8_t*)frame;
    }
    const int nxt = e->ref_cur ^ 1;
    uint8_t* recon = e->ref[nxt].as<uint8_t>();
    ResidualParams& rp = k.rp;
    rp.cur = cur;
    rp.pred = e->predb[ck].as<uint8_t>();
    rp.coeffs = e->coeffsb[ck].as<int16_t>();
    rp.opt_skip = e->optskipb[ck].as<uint8_t>();
    rp.fmask = e->fmaskb[ck].as<uint8_t>();
    rp.eobs = e->eobsb[ck].as<uint8_t>();
    rp.dead_zone = c.inter_dead_zone;
    rp.W = W; rp.H = H; rp.BW = e->BW;
    const int level = j.type == 1 ? e->intra_level : e->inter_level;
    rp.recon = level > 0 ? e->recon_pre.as<uint8_t>() : recon;
    k.db_level = level;
    k.db_src = e->recon_pre.as<uint8_t>();
    k.db_dst = recon;
    if (j.type == 1) {
        rp.intra = 1;
        rp.intra_ytab = e->ytab.as<uint16_t>();
        rp.intra_ctab = e->ctab.as<uint16_t>();
        k.db_E = e->intra_E; k.db_I = e->intra_I; k.db_H = e->intra_H;
        k.db_mask = nullptr;
        e->has_prev_mvs = false;
        e->has_prev2_mvs = false;
    } else {
        memset(&sp, 0, sizeof(sp));
        frame_search_params(e, cur, mbo, sp);
        if (e->table_ok) {
            sp.tstride = sad_table_stride(c.search_range);
            sp.tab = e->sadtab.as<uint16_t>();
        }
        const int cn = e->coded_cur ^ 1;
        sp.coded_out = e->coded[cn].as<int8_t>();
        k.ref = e->ref[e->ref_cur].as<uint8_t>();
        k.tab = e->table_ok ? e->sadtab.as<uint16_t>() : nullptr;
        k.tstride = sp.tstride;
        k.sr = c.search_range;
        k.mbo = mbo;
        k.pred = e->predb[ck].as<uint8_t>();
        k.lnv = e->lnvb[ck].as<float>();
        k.logfix = e->logfix.as<uint32_t>();
        k.nlog = e->nlog;
        rp.intra = 0;
        rp.mb = mbo;
        rp.qs = e->qs.as<float>();
        rp.lnv = k.lnv;  // the residual derives the steps from the ln variances and their mean
        rp.aq_base = e->inter_base;
        rp.expfix = e->expfix.as<uint32_t>();
        rp.nexp = e->nexp;
        rp.qs_out = e->qs.as<float>();
        k.db_E = e->inter_E; k.db_I = e->inter_I; k.db_H = e->inter_H;
        k.db_mask = rp.fmask;
        e->coded_cur = cn;
        e->has_prev2_mvs = e->has_prev_mvs;
        e->has_prev_mvs = true;
    }
    k.c_index = e->cindex.as<int32_t>();
    k.c_offset = e->coffset.as<int32_t>();
    k.c_side = s.dside.as<uint32_t>();
    k.c_packed = s.dpacked.as<int16_t>();
    k.c_peobs = s.dpeobs.as<uint8_t>();
    k.c_hdr = s.hdr.dev<uint32_t>();
    k.status = e->status.as<unsigned>();
    e->ref_cur = nxt;
    e->has_ref = true;
    e->last_par = ck;
    e->fpar = (ck + 1) % NPAR;
}

// The shapes of this step: while tuning, search candidate c = (tune_step / ROUNDS) % 6 and
// residual / deblock candidate c % 3 (each dimension is timed by its own stages).
static BatchTune batch_step_tune(riv_batch* b, bool& tuning, int& cand) {
    tuning = !b->fixed && !b->tuned;
    BatchTune t = b->tune;
    cand = (b->tune_step / TUNE_ROUNDS) % TUNE_NCAND;
    if (tuning) {
        t.row_ctas = TUNE_ROWS_PCT[cand];
        t.table = TUNE_TABLE[cand];
        t.res_mbs = TUNE_RES_MBS[cand % 3];
        t.db_tw = TUNE_DB_TW[cand % 3];
    }
    return t;
}

// Stage times of the timed step held by timing set `par` (if any): accumulated, and fed to the
// autotuner when that step ran candidate shapes.  Waits for that step's work to end.
static void batch_read_times(riv_batch* b, int par) {
    riv_batch::TimedStep& t = b->tpend[par];
    if (!t.pending) return;
    t.pending = false;
    cudaEvent_t* ev = b->ev_t[par];
    CK(cudaEventSynchronize(ev[TB_PACK]));
    float ms[BT_NSTAGE + 1] = {0};
    for (int s = 0; s < BT_NSTAGE; s++) CK(cudaEventElapsedTime(&ms[s], ev[s], ev[s + 1]));
    CK(cudaEventElapsedTime(&ms[BT_NSTAGE], ev[TB_START], ev[TB_PACK]));
    for (int s = 0; s <= BT_NSTAGE; s++) b->stage_us[s] += 1000.0 * ms[s];
    b->timed++;
    if (!t.tuning || b->tuned || b->fixed) return;
    if (t.pmbs == t.mbs && t.pmbs > 0) {  // P-frames only: comparable steps
        const int c3 = t.cand % 3;
        b->tune_us[0][t.cand] += 1000.0 * (ms[1] + ms[2]) / (double)t.pmbs;  // SAD table + search
        b->tune_us[1][c3] += 1000.0 * ms[5] / (double)t.mbs;                 // residual
        b->tune_us[2][c3] += 1000.0 * ms[6] / (double)t.mbs;                 // deblock
        b->tune_n[0][t.cand]++;
        b->tune_n[1][c3]++;
        b->tune_n[2][c3]++;
    }
    for (int q = 0; q < TUNE_NCAND; q++)
        if (b->tune_n[0][q] < TUNE_ROUNDS) return;
    auto pick = [&](int d, int nc) {
        int k = 0;
        for (int q = 1; q < nc; q++)
            if (b->tune_us[d][q] / b->tune_n[d][q] < b->tune_us[d][k] / b->tune_n[d][k]) k = q;
        return k;
    };
    const int sc = pick(0, TUNE_NCAND);
    b->tune.row_ctas = TUNE_ROWS_PCT[sc];
    b->tune.table = TUNE_TABLE[sc];
    b->tune.res_mbs = TUNE_RES_MBS[pick(1, 3)];
    b->tune.db_tw = TUNE_DB_TW[pick(2, 3)];
    b->tuned = true;
}

static riv_status batch_step(riv_batch* b, int src, const void* const* frames, const uint64_t* ts) {
    if (b->poisoned) {
        b->err = "batch unusable after an earlier failure: " + b->err;
        return RIV_ERR_ENCODING_FAILED;
    }
    const int n = (int)b->clips.size();
    riv_status refused = RIV_OK;
    try {
        CK(cudaSetDevice(b->device));
        const double h0 = now_ms();
        double room = 0.0;
        // ---- jobs, in clip order
        std::vector<int> act;
        std::vector<Job*> jobs;
        for (int i = 0; i < n; i++) {
            if (!frames[i]) continue;
            riv_encoder* e = b->clips[i];
            if (e->poisoned) return batch_fail(b, poisoned_status(e), "clip " + std::to_string(i) + ": " + e->err);
            const size_t cap = e->slots.size();
            const double r0 = now_ms();
            while (e->jobs.size() >= cap) {
                riv_status st = pump(e, true);
                if (st == RIV_ERR_IO) { refused = st; continue; }
                if (st) return batch_fail(b, st, "clip " + std::to_string(i) + ": " + e->err);
            }
            room += now_ms() - r0;
            const uint64_t idx = e->submitted;
            const bool intra = next_is_key(e);
            e->jobs.emplace_back();
            Job& j = e->jobs.back();
            j.index = idx;
            j.ts = ts[i];
            j.type = intra ? 1 : 2;
            j.slot = (int)(idx % cap);
            j.timed = false;
            act.push_back(i);
            jobs.push_back(&j);
        }
        if (act.empty()) return refused;
        const int m = (int)act.size();
        bool tuning = false;
        int cand = 0;
        BatchTune t = batch_step_tune(b, tuning, cand);
        const bool timed = tuning || b->steps % 8 == 0;
        // staging buffer of this step (its previous copy to the device is done)
        uint8_t* hd = b->hdesc[b->dpar].as<uint8_t>();
        CK(cudaEventSynchronize(b->ev_desc[b->dpar]));
        BatchClip* kc = (BatchClip*)hd;
        SearchParams* kp = (SearchParams*)(hd + b->off_sp);
        int* kst = (int*)(hd + b->off_start);
        int* kss = (int*)(hd + b->off_sstart);
        std::vector<int> pvar(m, -1);  // search variant of each P clip
        std::vector<SearchParams> sps(m);
        uint64_t step_mbs = 0, step_pmbs = 0;
        for (int a = 0; a < m; a++) {
            riv_encoder* e = b->clips[act[a]];
            batch_collect(e, *jobs[a], src, frames[act[a]], b->Hs, kc[a], sps[a]);
            step_mbs += (uint64_t)e->NMB;
            if (jobs[a]->type == 2) {
                if (!t.table) {  // SADs computed by the search itself
                    sps[a].tab = nullptr;
                    sps[a].tstride = 0;
                    kc[a].tab = nullptr;
                }
                pvar[a] = t.table ? search_variant(e) : 2;
                step_pmbs += (uint64_t)e->NMB;
            }
        }
        // stage ranges
        int tot[BS_N];
        for (int s = 0; s < BS_N; s++) {
            int* st = kst + s * (m + 1);
            st[0] = 0;
            for (int a = 0; a < m; a++) st[a + 1] = st[a] + batch_ctas_host(s, kc[a], t);
            tot[s] = st[m];
        }
        // search launches, one per variant present; each variant's parameters contiguous in kp,
        // its row CTAs spread over its clips
        int stot[3] = {0, 0, 0}, sfirst[3] = {0, 0, 0}, scount[3] = {0, 0, 0};
        int pos = 0;
        for (int v = 0; v < 3; v++) {
            std::vector<int> mem, nmb, bh, rows;
            for (int a = 0; a < m; a++)
                if (pvar[a] == v) { mem.push_back(a); nmb.push_back(kc[a].NMB); bh.push_back(kc[a].H / 16); }
            if (mem.empty()) continue;
            if ((int)mem.size() > b->cap[v]) throw std::runtime_error("more P-frame clips in one step than search CTAs fit");
            const int total = std::max((int)mem.size(), b->cap[v] * t.row_ctas / 100);
            spread_rows(nmb, bh, total, rows);
            int* ss = kss + v * (n + 1);
            ss[0] = 0;
            sfirst[v] = pos;
            scount[v] = (int)mem.size();
            for (size_t q = 0; q < mem.size(); q++) {
                SearchParams& sp = kp[pos++];
                sp = sps[mem[q]];
                sp.nrow_ctas = rows[q];
                sp.cta0 = ss[q];
                ss[q + 1] = ss[q] + rows[q];
            }
            stot[v] = ss[mem.size()];
        }
        // ---- the step's GPU work on B: the host->device copies, the descriptors, the stages
        cudaStream_t B = b->B;
        if (src == 0) {
            CK(cudaEventRecord(b->ev_h2d, b->Hs));
            CK(cudaStreamWaitEvent(B, b->ev_h2d, 0));
        }
        CK(cudaMemcpyAsync(b->ddesc.p, hd, b->desc_bytes, cudaMemcpyHostToDevice, B));
        CK(cudaEventRecord(b->ev_desc[b->dpar], B));
        b->dpar ^= 1;
        const uint8_t* dd = b->ddesc.as<uint8_t>();
        BatchLaunch L{(const BatchClip*)dd, (const int*)(dd + b->off_start), m};
        cudaEvent_t* evt = b->ev_t[b->tpar];
        auto mark = [&](int k) {
            if (timed) CK(cudaEventRecord(evt[k], B));
        };
        auto stage = [&](int s, int tb) {
            CK(launch_batch_stage(s, L, t, tot[s], b->max_sr, B));
            if (tot[s] > 0) b->launches++;
            mark(tb);
        };
        mark(TB_START);
        stage(BS_CONVERT, TB_CONVERT);
        stage(BS_TABLE, TB_TABLE);
        for (int v = 0; v < 3; v++) {
            if (!stot[v]) continue;
            const SearchParams* dps = (const SearchParams*)(dd + b->off_sp) + sfirst[v];
            const int* dss = (const int*)(dd + b->off_sstart) + v * (n + 1);
            CK(launch_search_multi(dps, dss, scount[v], stot[v], v < 2, v == 0, b->ssmem[v], b->sthreads[v], B));
            b->launches++;
        }
        mark(TB_SEARCH);
        stage(BS_PREDICT, TB_PREDICT);
        stage(BS_AQSUM, TB_AQSUM);
        stage(BS_RESIDUAL, TB_RESIDUAL);
        stage(BS_DEBLOCK, TB_DEBLOCK);
        stage(BS_SCAN, TB_SCAN);
        stage(BS_PACK, TB_PACK);
        CK(cudaEventRecord(b->ev_gpu, B));
        const double h1 = now_ms();
        b->host_ms[0] += room;
        b->host_ms[1] += h1 - h0 - room;
        // ---- copies back: side info, EOBs and a bounded prefix of the coefficients per clip
        cudaEvent_t xev = b->ev_step[b->steps % b->ev_step.size()];
        CK(cudaStreamWaitEvent(b->C, b->ev_gpu, 0));
        for (int a = 0; a < m; a++) {
            riv_encoder* e = b->clips[act[a]];
            Slot& s = e->slots[jobs[a]->slot];
            const int N = e->NMB;
            CK(cudaMemcpyAsync(s.side.p, s.dside.p, (size_t)N * 4, cudaMemcpyDeviceToHost, b->C));
            CK(cudaMemcpyAsync(s.peobs.p, s.dpeobs.p, (size_t)N * 3, cudaMemcpyDeviceToHost, b->C));
            s.prefetched = std::min(e->coef_guess, (size_t)N * 384 * 2);
            CK(cudaMemcpyAsync(s.packed.p, s.dpacked.p, s.prefetched, cudaMemcpyDeviceToHost, b->C));
            b->d2h_bytes += (uint64_t)N * 7 + s.prefetched;
        }
        CK(cudaEventRecord(xev, b->C));
        if (src == 0) {
            for (int a = 0; a < m; a++) {
                const riv_config& c = b->clips[act[a]]->cfg;
                b->h2d_bytes += (uint64_t)c.display_width * c.display_height * 3;
            }
            CK(cudaEventSynchronize(b->ev_h2d));  // the caller's buffers are reusable
        }
        for (int a = 0; a < m; a++) {
            riv_encoder* e = b->clips[act[a]];
            Job& j = *jobs[a];
            j.xev = xev;
            j.tail_done = true;
            e->submitted++;
        }
        b->steps++;
        b->frames += (uint64_t)m;
        b->mbs += step_mbs;
        if (timed) {
            riv_batch::TimedStep& tsp = b->tpend[b->tpar];
            tsp.pending = true;
            tsp.tuning = tuning;
            tsp.cand = cand;
            tsp.mbs = step_mbs;
            tsp.pmbs = step_pmbs;
            b->tpar ^= 1;
            if (tuning) b->tune_step++;
            batch_read_times(b, b->tpar);  // the other set: the previous timed step
        }
        const double h2 = now_ms();
        b->host_ms[2] += h2 - h1;
        // ---- each clip's host pipeline advances
        struct Tail {
            riv_batch* b;
            double t;
            ~Tail() { b->host_ms[3] += now_ms() - t; }
        } tail{b, h2};
        for (int a = 0; a < m; a++) {
            riv_encoder* e = b->clips[act[a]];
            riv_status st = pump(e, false);
            if (st == RIV_ERR_IO) { refused = st; continue; }
            if (st) return batch_fail(b, st, "clip " + std::to_string(act[a]) + ": " + e->err);
        }
    } catch (const CudaError& ce) {
        const std::string msg = std::string(ce.where) + ": " + cudaGetErrorString(ce.e);
        for (riv_encoder* e : b->clips) {
            e->poisoned = true;
            e->poison_msg = msg;
        }
        return batch_fail(b, RIV_ERR_CUDA, msg);
    } catch (const std::exception& ex) {
        b->poisoned = true;
        return batch_fail(b, RIV_ERR_ENCODING_FAILED, ex.what());
    }
    if (refused) b->err = "writer.write failed for a record of at least one clip; that record is lost";
    return refused;
}

}  // namespace

extern "C" {

riv_status riv_batch_new(const riv_config* cfgs, const riv_writer_vtable* writers, uint32_t n, riv_batch** out) {
    if (!cfgs || !writers || !out || n == 0 || n > RIV_BATCH_MAX_CLIPS) return RIV_ERR_INVALID_CONFIG;
    *out = nullptr;
    for (uint32_t i = 0; i < n; i++)
        if (cfgs[i].device != cfgs[0].device || cfgs[i].encode_form != RIV_FORM_PLAIN) return RIV_ERR_INVALID_CONFIG;
    riv_batch* b = new riv_batch();
    b->device = cfgs[0].device;
    try {
        CK(cudaSetDevice(b->device));
        const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
        b->pool = std::make_shared<ThreadPool>(hw - 1, BULK_NICE);
        b->rans_pool = std::make_shared<ThreadPool>(std::max(2u, hw / 2), BULK_NICE);
        b->mv_pool = std::make_shared<ThreadPool>(std::max(2u, hw / 4));
        size_t maxcap = 1;
        for (uint32_t i = 0; i < n; i++) {
            riv_config c = cfgs[i];
            c.entropy_threads = 1;  // the clips share the batch's pools (set below)
            riv_encoder* e = nullptr;
            riv_status st = riv_encoder_new(&c, &writers[i], &e);
            if (st) {
                riv_batch_free(b);
                return st;
            }
            e->cfg.entropy_threads = cfgs[i].entropy_threads;
            e->batched = true;
            e->defer_ok = false;  // each step reconstructs its frames itself
            e->pool = b->pool;
            e->rans_pool = b->rans_pool;
            e->mv_pool = b->mv_pool;
            ThreadPool* rp = b->rans_pool.get();  // both submit paths onto the shared pools
            e->rans_submit = [rp](std::function<void()> f) { return rp->submit(std::move(f)); };
            e->rans_submit_urgent = [rp](std::function<void()> f) { return rp->submit(std::move(f), true); };
            ThreadPool* mp = b->mv_pool.get();
            e->mv_submit = [mp](std::function<void()> f) { return mp->submit(std::move(f)); };
            e->rans_parts = (int)std::max(2u, hw / 2) + 1;
            b->clips.push_back(e);
            b->max_sr = std::max(b->max_sr, (int)c.search_range);
            maxcap = std::max(maxcap, e->slots.size());
        }
        CK(cudaStreamCreateWithFlags(&b->B, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&b->Hs, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&b->C, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&b->ev_h2d, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&b->ev_gpu, cudaEventDisableTiming));
        b->ev_step.resize(maxcap + 2);
        for (auto& ev : b->ev_step) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        for (int q = 0; q < 2; q++)
            for (int k = 0; k < BT_BOUNDS; k++) CK(cudaEventCreate(&b->ev_t[q][k]));
        for (int k = 0; k < 2; k++) {
            CK(cudaEventCreateWithFlags(&b->ev_desc[k], cudaEventDisableTiming));
            CK(cudaEventRecord(b->ev_desc[k], b->B));
        }
        auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
        b->off_sp = al((size_t)n * sizeof(BatchClip));
        b->off_start = b->off_sp + al((size_t)n * sizeof(SearchParams));
        b->off_sstart = b->off_start + al((size_t)BS_N * (n + 1) * sizeof(int));
        b->desc_bytes = b->off_sstart + al((size_t)3 * (n + 1) * sizeof(int));
        for (int k = 0; k < 2; k++) {
            b->hdesc[k].alloc(b->desc_bytes);
            memset(b->hdesc[k].p, 0, b->desc_bytes);
        }
        b->ddesc.alloc(b->desc_bytes);
        int dev = 0, nsm = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        for (int v = 0; v < 3; v++) {
            int per_sm = 0;
            CK(search_multi_capacity(v < 2, v == 0, b->max_sr, &per_sm, &b->ssmem[v], &b->sthreads[v]));
            b->cap[v] = per_sm * nsm;
        }
        CK(cudaStreamSynchronize(b->B));
    } catch (const CudaError& ce) {
        fprintf(stderr, "riv_batch_new: %s: %s\n", ce.where, cudaGetErrorString(ce.e));
        riv_batch_free(b);
        return RIV_ERR_CUDA;
    } catch (const std::exception& ex) {
        fprintf(stderr, "riv_batch_new: %s\n", ex.what());
        riv_batch_free(b);
        return RIV_ERR_ENCODING_FAILED;
    }
    *out = b;
    return RIV_OK;
}

riv_status riv_batch_encode(riv_batch* b, const uint8_t* const* frames, const uint64_t* ts) {
    if (!b || !frames || !ts) return RIV_ERR_FRAME;
    return batch_step(b, 0, (const void* const*)frames, ts);
}

riv_status riv_batch_encode_device(riv_batch* b, const void* const* d_frames, const uint64_t* ts) {
    if (!b || !d_frames || !ts) return RIV_ERR_FRAME;
    return batch_step(b, 1, d_frames, ts);
}

riv_status riv_batch_finish(riv_batch* b) {
    if (!b) return RIV_ERR_INVALID_CONFIG;
    try {
        CK(cudaSetDevice(b->device));
        batch_read_times(b, 0);
        batch_read_times(b, 1);
    } catch (const CudaError& ce) {
        return batch_fail(b, RIV_ERR_CUDA, std::string(ce.where) + ": " + cudaGetErrorString(ce.e));
    }
    riv_status first = RIV_OK;
    const double f0 = now_ms();
    struct Fin {
        riv_batch* b;
        double t;
        ~Fin() { b->host_ms[4] += now_ms() - t; }
    } fin{b, f0};
    for (size_t i = 0; i < b->clips.size(); i++) {
        riv_status st = riv_finish(b->clips[i]);
        if (st && !first) {
            first = st;
            b->err = "clip " + std::to_string(i) + ": " + b->clips[i]->err;
        }
    }
    return first;
}

void riv_batch_free(riv_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->B) cudaStreamSynchronize(b->B);
    if (b->C) cudaStreamSynchronize(b->C);
    if (b->Hs) cudaStreamSynchronize(b->Hs);
    for (riv_encoder* e : b->clips) riv_encoder_free(e);
    b->clips.clear();
    b->pool.reset();
    b->rans_pool.reset();
    b->mv_pool.reset();
    for (auto& ev : b->ev_step)
        if (ev) cudaEventDestroy(ev);
    for (int q = 0; q < 2; q++)
        for (int k = 0; k < BT_BOUNDS; k++)
            if (b->ev_t[q][k]) cudaEventDestroy(b->ev_t[q][k]);
    for (int k = 0; k < 2; k++) {
        if (b->ev_desc[k]) cudaEventDestroy(b->ev_desc[k]);
        b->hdesc[k].release();
    }
    if (b->ev_h2d) cudaEventDestroy(b->ev_h2d);
    if (b->ev_gpu) cudaEventDestroy(b->ev_gpu);
    b->ddesc.release();
    if (b->B) cudaStreamDestroy(b->B);
    if (b->C) cudaStreamDestroy(b->C);
    if (b->Hs) cudaStreamDestroy(b->Hs);
    delete b;
}

const char* riv_batch_last_error(const riv_batch* b) { return b ? b->err.c_str() : "null batch"; }

riv_status riv_batch_set_tune(riv_batch* b, const riv_batch_tune* t) {
    if (!b || !t) return RIV_ERR_INVALID_CONFIG;
    if ((t->res_mbs != 2 && t->res_mbs != 4 && t->res_mbs != 8) || (t->db_tw != 64 && t->db_tw != 128 && t->db_tw != 256) ||
        t->search_rows_pct < 1 || t->search_rows_pct > 100 || (t->sad_table != 0 && t->sad_table != 1))
        return RIV_ERR_INVALID_CONFIG;
    b->tune.row_ctas = t->search_rows_pct;
    b->tune.res_mbs = t->res_mbs;
    b->tune.db_tw = t->db_tw;
    b->tune.table = t->sad_table ? 1 : 0;
    b->fixed = true;
    return RIV_OK;
}

riv_status riv_batch_get_tune(const riv_batch* b, riv_batch_tune* t, int* tuned) {
    if (!b || !t) return RIV_ERR_INVALID_CONFIG;
    t->search_rows_pct = b->tune.row_ctas;
    t->res_mbs = b->tune.res_mbs;
    t->db_tw = b->tune.db_tw;
    t->sad_table = b->tune.table;
    if (tuned) *tuned = b->fixed ? 2 : (b->tuned ? 1 : 0);
    return RIV_OK;
}

riv_status riv_batch_counters(const riv_batch* b, uint64_t* c7, double* stage_us10) {
    if (!b) return RIV_ERR_INVALID_CONFIG;
    if (c7) {
        c7[0] = b->steps;
        c7[1] = b->frames;
        c7[2] = b->mbs;
        c7[3] = b->launches;
        c7[4] = b->timed;
        c7[5] = b->h2d_bytes;
        c7[6] = b->d2h_bytes;
    }
    if (stage_us10)
        for (int s = 0; s <= BT_NSTAGE; s++) stage_us10[s] = b->timed ? b->stage_us[s] / (double)b->timed : 0.0;
    return RIV_OK;
}

riv_status riv_batch_host_times(const riv_batch* b, double* ms5) {
    if (!b || !ms5) return RIV_ERR_INVALID_CONFIG;
    for (int k = 0; k < 5; k++) ms5[k] = b->host_ms[k];
    return RIV_OK;
}

riv_status riv_batch_last_recon(riv_batch* b, uint32_t clip, uint8_t* y, uint8_t* u, uint8_t* v) {
    if (!b || clip >= b->clips.size()) return RIV_ERR_INVALID_CONFIG;
    riv_encoder* e = b->clips[clip];
    if (!e->has_ref) return RIV_ERR_FRAME;
    try {
        CK(cudaSetDevice(b->device));
        CK(cudaStreamSynchronize(b->B));
        const uint8_t* d = e->ref[e->ref_cur].as<uint8_t>();
        const size_t ys = (size_t)e->W * e->H, cs = ys / 4;
        CK(cudaMemcpy(y, d, ys, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(u, d + ys, cs, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(v, d + ys + cs, cs, cudaMemcpyDeviceToHost));
    } catch (const CudaError& ce) {
        return batch_fail(b, RIV_ERR_CUDA, std::string(ce.where) + ": " + cudaGetErrorString(ce.e));
    }
    return RIV_OK;
}

riv_status riv_batch_clip_counters(const riv_batch* b, uint32_t clip, uint64_t* frames_written, double* host_ms6) {
    if (!b || clip >= b->clips.size()) return RIV_ERR_INVALID_CONFIG;
    const riv_encoder* e = b->clips[clip];
    if (frames_written) *frames_written = e->frame_count;
    if (host_ms6)
        for (int k = 0; k < 6; k++) host_ms6[k] = e->host_ms[k];
    return RIV_OK;
}

}  // extern "C"
