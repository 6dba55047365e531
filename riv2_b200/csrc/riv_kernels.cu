// riv_kernels.cu -- sm_100a kernels of the riv2 P-frame encoder hot path.
//
// Reference semantics (paths relative to the reference project root):
//   enc/ = reitero_video/reitero_encode/src/       com/ = reitero_video/reitero_video_common/src/
//   res/ = reitero_video/reitero_residual/src/     dct/ = reitero_video/reitero_dct/src/
// Floating point reproduces the reference op for op with explicit round-to-nearest
// intrinsics (__fadd_rn, __dmul_rn, ...): no FMA contraction the reference lacks.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "riv_internal.h"

namespace riv {

// ---------------------------------------------------------------------------------
// Shared tables
// ---------------------------------------------------------------------------------
// T16[i][j] = round(2^18 * c_j * cos((2i+1) j pi / 32)), T8 likewise with /16: the
// reference's fixed-point DCT bases (dct/dct16.rs:7-145, dct/dct8.rs:6-25), uploaded by
// the host (which derives them from the formula) into constant memory.
__constant__ int32_t c_T16[256];
__constant__ int32_t c_T8[64];

// ---------------------------------------------------------------------------------
// K1: RGB24 (display size) -> planar YUV 4:2:0 (storage size), pad fused.
// pad_rgb24 (enc/encoder.rs:1049-1096) == reading the display frame at clamped
// coordinates.  BT.709 limited range, 13-bit fixed point (same definition as the oracle).
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void rgb_to_yuv_quad(const uint8_t* __restrict__ rgb, int dw, int dh, uint8_t* __restrict__ Yp,
                                                uint8_t* __restrict__ Up, uint8_t* __restrict__ Vp, int W, int cx, int cy) {
    int sr = 0, sg = 0, sb = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        int x = 2 * cx + (k & 1), y = 2 * cy + (k >> 1);
        int sx = min(x, dw - 1), sy = min(y, dh - 1);
        const uint8_t* p = rgb + ((size_t)sy * dw + sx) * 3;
        int r = p[0], g = p[1], b = p[2];
        int v = (1496 * r + 5032 * g + 508 * b + (16 << 13) + (1 << 12)) >> 13;
        Yp[(size_t)y * W + x] = (uint8_t)min(max(v, 16), 235);
        sr += r; sg += g; sb += b;
    }
    int r = (sr + 2) >> 2, g = (sg + 2) >> 2, b = (sb + 2) >> 2;
    int cb = (-824 * r - 2774 * g + 3598 * b + (128 << 13) + (1 << 12)) >> 13;
    int cr = (3598 * r - 3268 * g - 330 * b + (128 << 13) + (1 << 12)) >> 13;
    size_t ci = (size_t)cy * (W / 2) + cx;
    Up[ci] = (uint8_t)min(max(cb, 16), 240);
    Vp[ci] = (uint8_t)min(max(cr, 16), 240);
}
// Grid-stride over the 2x2 quads (one chroma sample each), consecutive threads on
// consecutive quads of a row.
__global__ void k_rgb_to_yuv(const uint8_t* __restrict__ rgb, int dw, int dh, uint8_t* __restrict__ Yp,
                             uint8_t* __restrict__ Up, uint8_t* __restrict__ Vp, int W, int H) {
    const int cw = W / 2, nq = cw * (H / 2);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x)
        rgb_to_yuv_quad(rgb, dw, dh, Yp, Up, Vp, W, q % cw, q / cw);
}

// Decoder output (dec/decoder.rs:445-456: `to_rgb24` then `crop_rgb24`): storage-size YUV
// 4:2:0 to display-size RGB24, BT.709 limited range in 13-bit fixed point (the inverse of
// k_rgb_to_yuv; 8192*255/219, 8192*255/224 * 1.5748, 0.18732, 0.46812, 1.8556), each chroma
// sample covering its 2x2 luma quad.  One thread per output pixel.
__global__ void k_yuv_to_rgb(const uint8_t* __restrict__ Yp, const uint8_t* __restrict__ Up,
                             const uint8_t* __restrict__ Vp, int W, int dw, int dh, uint8_t* __restrict__ rgb) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= dw || y >= dh) return;
    const int yv = 9539 * ((int)Yp[(size_t)y * W + x] - 16);
    const size_t ci = (size_t)(y >> 1) * (W / 2) + (x >> 1);
    const int u = (int)Up[ci] - 128, v = (int)Vp[ci] - 128;
    uint8_t* p = rgb + ((size_t)y * dw + x) * 3;
    p[0] = (uint8_t)min(max((yv + 14686 * v + (1 << 12)) >> 13, 0), 255);
    p[1] = (uint8_t)min(max((yv - 1747 * u - 4366 * v + (1 << 12)) >> 13, 0), 255);
    p[2] = (uint8_t)min(max((yv + 17305 * u + (1 << 12)) >> 13, 0), 255);
}
int launch_yuv_to_rgb(const uint8_t* yuv, int W, int H, int dw, int dh, uint8_t* rgb, void* stream) {
    const uint8_t* Y = yuv;
    const uint8_t* U = yuv + (size_t)W * H;
    const uint8_t* V = U + (size_t)(W / 2) * (H / 2);
    k_yuv_to_rgb<<<dim3((dw + 127) / 128, dh), 128, 0, (cudaStream_t)stream>>>(Y, U, V, W, dw, dh, rgb);
    return (int)cudaGetLastError();
}

// `beside`: the conversion runs while a search launch holds the SMs, so one 128-thread CTA
// (4K registers) per SM at most: every SM keeps room for a search CTA (61,440 registers) and a
// search launch never waits for a conversion to drain.  Otherwise one CTA per 128 quads (the
// conversion alone on the GPU, as fast as it goes).  Either way the preferred shared-memory
// carveout is the search kernel's (maximum shared memory), so an SM that ran a conversion CTA
// needs no reconfiguration before the next search CTA.
int launch_rgb_to_yuv(const uint8_t* rgb, int dw, int dh, uint8_t* yuv, int W, int H, void* stream, bool beside) {
    static int nsm = 0;
    if (nsm == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            nsm = 1;
        cudaFuncSetAttribute(k_rgb_to_yuv, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    }
    const int nq = (W / 2) * (H / 2);
    const int blk = 128, grd = std::max(1, beside ? std::min(nsm, (nq + blk - 1) / blk) : (nq + blk - 1) / blk);
    uint8_t* Y = yuv;
    uint8_t* U = yuv + (size_t)W * H;
    uint8_t* V = U + (size_t)(W / 2) * (H / 2);
    k_rgb_to_yuv<<<grd, blk, 0, (cudaStream_t)stream>>>(rgb, dw, dh, Y, U, V, W, H);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// K4: motion search + RDO skip + MV mode decision, one warp per macroblock row.
//
// The reference processes macroblocks in raster order; each block's seeds, MV-cost
// predictors and coded-MV predictors depend on its left, top, top-right and top-left
// neighbours (enc/motion/scalar.rs:56-156, res/mv_predictor.rs:59-272).  Here CTA r
// owns MB rows r, r+grid, ...; it walks its row left to right keeping the left
// neighbour in registers and waits (bounded spin, acquire) for the top-right record
// published by the CTA of row r-1.  Critical path = (BW + 2*(BH-1)) MB steps with only
// BH-1 cross-CTA hand-offs.
//
// Within an MB every round of candidates (seeds, one hex ring, the diamond, the nine
// half-pel points) is evaluated in parallel: each lane owns 8 pixels (half a row) and
// forms partial SADs for every candidate, reduced with redux.sync.  The reference
// evaluates candidates sequentially with early-exit limits; an early exit only ever
// returns a partial SAD already above the limit (so the candidate cannot win), hence
// full SADs followed by the same in-order strict-'<' scan give identical decisions.
// ---------------------------------------------------------------------------------
// Each MB record is one 64-bit word (tag + payload), single-copy atomic, and consumers
// read nothing else the producer wrote during the kernel, so relaxed gpu-scope accesses
// suffice (no fences on the wavefront's critical path).
__device__ __forceinline__ unsigned long long ld_rec(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_rec(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned warp_sum(unsigned v) { return __reduce_add_sync(0xffffffffu, v); }

struct CostCtx {
    int nx, ny, rx, ry, mx, my;
};

// estimate_mv_cost (enc/motion/scalar.rs:453-544)
// SMALL: all costs < 2^27, |diff| < 64 entries from the shared 64x64 int32 table, the rest
// from the exact i64 table in global memory.  Otherwise the i64 table (or f64 if absent).
template <bool SMALL>
__device__ __forceinline__ long long mv_cost(int dx, int dy, const CostCtx& c, const SearchParams& p,
                                             const double* bits, const int* nc32) {
    if (p.lambda_zero) return 0;
    long long best = LLONG_MAX;
    if ((dx == c.nx && dy == c.ny) || (dx == c.rx && dy == c.ry) || (dx == c.mx && dy == c.my)) best = p.c15;
    if (dx == 0 && dy == 0) best = min(best, p.c05);
    const int ax = abs(dx - c.nx), ay = abs(dy - c.ny), bx = abs(dx - c.rx), by = abs(dy - c.ry);
    if (SMALL && ((ax | ay | bx | by) < 64)) return min(best, (long long)min(nc32[ax * 64 + ay], nc32[bx * 64 + by]));
    if (p.newcost) return min(best, min(__ldg(p.newcost + ax * 256 + ay), __ldg(p.newcost + bx * 256 + by)));
    double ba = __dadd_rn(__dadd_rn(6.0, bits[ax]), bits[ay]);
    double bb = __dadd_rn(__dadd_rn(6.0, bits[bx]), bits[by]);
    return min(best, min(__double2ll_rz(__dmul_rn(p.lam2, ba)), __double2ll_rz(__dmul_rn(p.lam2, bb))));
}

// Unaligned 32-bit read from shared memory: two aligned words and a funnel shift.  The
// reference window/band allocation carries 16 bytes of slack so the second word is
// always inside it.
__device__ __forceinline__ uint32_t lds_u32(const uint8_t* p) {
    uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
    uint32_t lo, hi;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(lo) : "r"(a & ~3u));
    asm volatile("ld.shared.u32 %0, [%1+4];" : "=r"(hi) : "r"(a & ~3u));
    return __funnelshift_r(lo, hi, (a & 3u) * 8u);
}
__device__ __forceinline__ uint32_t lds_aligned(uint32_t saddr) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(saddr));
    return v;
}
// floor((a+b)/2) per byte
__device__ __forceinline__ uint32_t favg(uint32_t a, uint32_t b) { return (a & b) + (((a ^ b) >> 1) & 0x7F7F7F7Fu); }
// floor((a+b+c+d)/4) per byte, via 16-bit lanes
__device__ __forceinline__ uint32_t favg4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    const uint32_t M = 0x00FF00FFu;
    uint32_t lo = (a & M) + (b & M) + (c & M) + (d & M);
    uint32_t hi = ((a >> 8) & M) + ((b >> 8) & M) + ((c >> 8) & M) + ((d >> 8) & M);
    return ((lo >> 2) & M) | (((hi >> 2) & M) << 8);
}

// (a+b+c+d+2)>>2 per byte (build_predicted's rounded four-tap average), via 16-bit lanes
__device__ __forceinline__ uint32_t ravg4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    const uint32_t M = 0x00FF00FFu;
    uint32_t lo = (a & M) + (b & M) + (c & M) + (d & M) + 0x00020002u;
    uint32_t hi = ((a >> 8) & M) + ((b >> 8) & M) + ((c >> 8) & M) + ((d >> 8) & M) + 0x00020002u;
    return ((lo >> 2) & M) | (((hi >> 2) & M) << 8);
}

// Reference samples of one MB: byte at frame (fx, fy) = org[(fy - wy0) * stride + fx - x0].
// Replicated borders: positions outside the frame hold the nearest frame sample.
struct RefView {
    const uint8_t* org;
    int stride, wy0;
};

// Integer SAD partial over this lane's 8 pixels, reproducing the per-4x4 sub-block
// clamped reference origin of the reference's edge path (enc/motion/satd_scalar.rs:26-97);
// for interior candidates the clamps are no-ops and this equals the plain 16x16 SAD.
__device__ __forceinline__ unsigned sad_int_part(const RefView& v, int x0, int y0, int W, int H, int dx, int dy,
                                                 int yy, int xoff, uint32_t c0, uint32_t c1) {
    int ry = min(max(y0 + (yy & ~3) + dy, 0), H - 4) + (yy & 3);
    const uint8_t* row = v.org + (ry - v.wy0) * v.stride;
    int rx0 = min(max(x0 + xoff + dx, 0), W - 4) - x0;
    int rx1 = min(max(x0 + xoff + 4 + dx, 0), W - 4) - x0;
    return __vsadu4(c0, lds_u32(row + rx0)) + __vsadu4(c1, lds_u32(row + rx1));
}

struct MvT {
    int dx, dy, sx, sy;
};
__device__ __forceinline__ bool mv_eq(const MvT& a, const MvT& b) {
    return a.dx == b.dx && a.dy == b.dy && a.sx == b.sx && a.sy == b.sy;
}
__device__ __forceinline__ int mv_class(int mag) {  // res/mv_rans.rs:80-86
    if (mag == 0) return 0;
    return min(32 - __clz(mag), 10);
}
__device__ __forceinline__ int comp_bits(int d) {  // enc/encoder.rs:142-154
    int c = mv_class(abs(d));
    return c == 0 ? 4 : 4 + c;
}
__device__ __forceinline__ int sat8(int v) { return min(max(v, -128), 127); }

__device__ __forceinline__ int median3(int a, int b, int c) {  // enc/motion/scalar.rs:24-43
    if (a > b) return b > c ? b : (a > c ? c : a);
    return a > c ? a : (b > c ? c : b);
}

__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
    uint32_t d = (uint32_t)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Band layout (BAND mode): the reference rows y0-sr-1 .. y0+16+sr of the whole MB row,
// columns -MARGIN .. W+MARGIN-1, MARGIN = round_up(sr+1, 16), filled 16-column chunk by
// chunk with cp.async one MB ahead of use.
__device__ __forceinline__ void fill_chunk(uint8_t* band, int BWB, int WS, int c, int MARGIN, int wy0,
                                          const uint8_t* __restrict__ ref, int W, int H, int lane) {
    const int fx0 = 16 * c - MARGIN;
    for (int i = lane; i < WS; i += 32) {
        int gy = min(max(wy0 + i, 0), H - 1);
        uint8_t* dst = band + (size_t)i * BWB + 16 * c;
        if (fx0 >= 0 && fx0 < W) {
            cp_async16(dst, ref + (size_t)gy * W + fx0);
        } else {
            uint32_t v = ref[(size_t)gy * W + (fx0 < 0 ? 0 : W - 1)] * 0x01010101u;
            *(uint4*)dst = make_uint4(v, v, v, v);
        }
    }
}


// ---------------------------------------------------------------------------------
// K3: exhaustive integer-SAD table of every MB over the whole search range, computed by
// the full GPU before the wavefront so its integer rounds become shared-memory lookups.
// tab[mb][(dy+sr)*(2sr+1) + dx+sr] = SAD(dx,dy) with the reference's semantics
// (per-4x4 sub-block clamped reference origin at frame edges,
// enc/motion/satd_scalar.rs:26-97; the plain 16x16 SAD elsewhere).  Values <= 65280.
// ---------------------------------------------------------------------------------
// One MB's table row by the whole CTA (at least 64 threads); `sm` holds the window and the
// current block.
// tid/nthr: this thread's index and the thread count of the group computing the MB; bar_id 0
// = the whole CTA (__syncthreads), else a named barrier of the group's nthr threads.
__device__ __forceinline__ void group_sync(int bar_id, int nthr) {
    if (bar_id == 0) __syncthreads();
    else asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthr) : "memory");
}
__device__ __forceinline__ void sad_table_mb(const uint8_t* __restrict__ ref, const uint8_t* __restrict__ cur, int W,
                                             int H, int BW, int sr, uint16_t* __restrict__ tab, int tstride, int mb,
                                             uint8_t* sm, int tid, int nthr, int bar_id) {
    const int WT = 16 + 2 * sr;                 // window side
    const int WTS = (WT + 8 + 15) & ~15;        // row stride (+ slack for the 24-byte row reads)
    uint8_t* win = sm;
    uint32_t* cw = (uint32_t*)(sm + WT * WTS + 16);  // 64 words of the current block
    const int bx = mb % BW, by = mb / BW;
    const int x0 = bx * 16, y0 = by * 16;
    const int wx0 = x0 - sr, wy0 = y0 - sr;
    for (int i = tid; i < WT * WT; i += nthr) {
        int r = i / WT, c = i - r * WT;
        int gy = min(max(wy0 + r, 0), H - 1), gx = min(max(wx0 + c, 0), W - 1);
        win[r * WTS + c] = ref[(size_t)gy * W + gx];
    }
    if (tid < 64) {
        int r = tid >> 2, g = tid & 3;
        cw[tid] = *(const uint32_t*)(cur + (size_t)(y0 + r) * W + x0 + 4 * g);
    }
    group_sync(bar_id, nthr);
    const int side = 2 * sr + 1, P = side * side;
    const bool interior = x0 - sr >= 0 && y0 - sr >= 0 && x0 + 15 + sr <= W - 1 && y0 + 15 + sr <= H - 1;
    uint16_t* out = tab + (size_t)mb * tstride;
    if (interior) {
        // Thread = 8 horizontally adjacent positions dx = 8q-sr .. 8q-sr+7 of one dy; their
        // reference rows start at window column 8q (4-byte aligned), so the shifted words
        // come from aligned loads with compile-time funnel shifts.
        const int nq = (side + 7) >> 3;
        for (int item = tid; item < side * nq; item += nthr) {
            const int dyi = item / nq, q = item - dyi * nq;
            unsigned acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 2
            for (int r = 0; r < 16; r++) {
                const uint2* rowp = (const uint2*)(win + (r + dyi) * WTS + 8 * q);
                const uint2 a = rowp[0], b = rowp[1], c = rowp[2];
                const uint32_t w[6] = {a.x, a.y, b.x, b.y, c.x, c.y};
                const uint4 cv = ((const uint4*)cw)[r];
                const uint32_t cg[4] = {cv.x, cv.y, cv.z, cv.w};
#pragma unroll
                for (int g = 0; g < 4; g++) {
#pragma unroll
                    for (int j = 0; j < 8; j++) {
                        const int k = (j >> 2) + g, sh = (j & 3) * 8;
                        const uint32_t ref = sh ? __funnelshift_r(w[k], w[k + 1], sh) : w[k];
                        acc[j] += __vsadu4(cg[g], ref);
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < 8; j++)
                if (8 * q + j < side) out[dyi * side + 8 * q + j] = (uint16_t)acc[j];
        }
    } else {
        for (int pidx = tid; pidx < P; pidx += nthr) {
            const int dy = pidx / side - sr, dx = pidx % side - sr;
            unsigned s = 0;
            for (int r = 0; r < 16; r++) {
                int ry = min(max(y0 + (r & ~3) + dy, 0), H - 4) + (r & 3) - wy0;
                const uint8_t* row = win + ry * WTS;
#pragma unroll
                for (int g = 0; g < 4; g++) {
                    int rx = min(max(x0 + 4 * g + dx, 0), W - 4) - wx0;
                    s += __vsadu4(cw[r * 4 + g], lds_u32(row + rx));
                }
            }
            out[pidx] = (uint16_t)s;
        }
    }
}

__global__ void __launch_bounds__(128) k_sad_table(const uint8_t* __restrict__ ref, const uint8_t* __restrict__ cur,
                                                   int W, int H, int BW, int sr, uint16_t* __restrict__ tab,
                                                   int tstride) {
    extern __shared__ __align__(16) uint8_t sm[];
    sad_table_mb(ref, cur, W, H, BW, sr, tab, tstride, blockIdx.x, sm, threadIdx.x, blockDim.x, 0);
}
size_t sad_table_smem(int sr) {
    int WT = 16 + 2 * sr, WTS = (WT + 8 + 15) & ~15;
    return (size_t)WT * WTS + 16 + 256;
}
int launch_sad_table(const uint8_t* ref, const uint8_t* cur, int W, int H, int sr, uint16_t* tab, int tstride,
                     void* stream) {
    int BW = W / 16, n = BW * (H / 16);
    size_t sm = sad_table_smem(sr);
    if (sm > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_sad_table, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return (int)e;
    }
    k_sad_table<<<n, 128, sm, (cudaStream_t)stream>>>(ref, cur, W, H, BW, sr, tab, tstride);
    return (int)cudaGetLastError();
}

// Warp argmin over lanes 0..7 of (total, lane) with the lowest lane winning ties; lanes
// with valid == false do not compete.  Totals are below 2^59 (the host enables the table
// path only then), so (total << 3 | lane) is an exact sort key.  Returns the winning lane
// (or -1) and the minimum total.
template <bool SMALL>
__device__ __forceinline__ int argmin8(long long total, bool valid, long long& best_total) {
    if (SMALL) {  // totals < 2^28: one redux.sync on a 32-bit key
        uint32_t k32 = valid ? ((uint32_t)total << 3) | (threadIdx.x & 7) : 0xffffffffu;
        k32 = __reduce_min_sync(0xffffffffu, k32);
        best_total = (long long)(k32 >> 3);
        return k32 == 0xffffffffu ? -1 : (int)(k32 & 7);
    }
    unsigned long long key = valid ? ((unsigned long long)total << 3) | (threadIdx.x & 7) : ~0ull;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
        unsigned long long k2 = __shfl_xor_sync(0xffffffffu, key, o);
        key = k2 < key ? k2 : key;
    }
    key = __shfl_sync(0xffffffffu, key, 0);
    best_total = (long long)(key >> 3);
    return key == ~0ull ? -1 : (int)(key & 7);
}

// Phase stamps, written when p.prof is set: RIV_PROF_WORDS i64 per MB.  Words 0-15 are SM clock
// cycles (clock64) of the search and mode warps; words 16-27 are %globaltimer nanoseconds,
// comparable across SMs: 16/17 search warp MB start / slot ready; 18/19 deferred residual of
// the MB pair starting here (of MB (r, 1): the AQ fold's end of row r's sum / loads); 30 / 31
// the mode warp's decision / the AQ warp's variance of the MB; 20/21/22 deblock tile (wait start, work start, end); 23/24/25
// SAD-table MB (wait start, work start, end); 26/27 the row loader's wait for reference bands.
__device__ __forceinline__ long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return (long long)t;
}
#define RIV_PUT(k, v)                                                      \
    do {                                                                    \
        if (p.prof != nullptr && lane == 0) p.prof[(size_t)idx * RIV_PROF_WORDS + (k)] = (v); \
    } while (0)
#define RIV_STAMP(k)                                                        \
    do {                                                                    \
        if (p.prof != nullptr && lane == 0) p.prof[(size_t)idx * RIV_PROF_WORDS + (k)] = clock64(); \
    } while (0)
#define RIV_GSTAMP(mbi, k)                                                  \
    do {                                                                    \
        if (p.prof != nullptr) p.prof[(size_t)(mbi) * RIV_PROF_WORDS + (k)] = gtimer(); \
    } while (0)

// Rounded bilinear sample at half-pel position (xh, yh) with the coordinates clamped to the
// plane (com/motion.rs:28-117).
__device__ __forceinline__ int sample_round(const uint8_t* __restrict__ pl, int w, int h, int xh, int yh) {
    xh = min(max(xh, 0), (w - 1) * 2);
    yh = min(max(yh, 0), (h - 1) * 2);
    int x0 = xh >> 1, y0 = yh >> 1;
    int xo = xh & 1, yo = yh & 1;
    int x1 = min(x0 + 1, w - 1), y1 = min(y0 + 1, h - 1);
    int a = pl[(size_t)y0 * w + x0];
    if (!xo && !yo) return a;
    int b = pl[(size_t)y0 * w + x1], d = pl[(size_t)y1 * w + x0], e = pl[(size_t)y1 * w + x1];
    if (xo && !yo) return (a + b + 1) >> 1;
    if (!xo && yo) return (a + d + 1) >> 1;
    return (a + b + d + e + 2) >> 2;
}

// fix: n (input bits, glibc result bits) pairs sorted by input bits, followed by 65537 bucket
// starts indexed by the top 16 input bits; the search runs inside one bucket.
__device__ __forceinline__ float apply_fix(float x, float y, const uint32_t* fix, int n) {
    uint32_t key = __float_as_uint(x);
    const uint32_t* idx = fix + 2 * (size_t)n;
    int lo = (int)__ldg(idx + (key >> 16)), hi = (int)__ldg(idx + (key >> 16) + 1);
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        uint32_t k = __ldg(fix + 2 * mid);
        if (k < key) lo = mid + 1; else hi = mid;
    }
    if (lo < n && __ldg(fix + 2 * lo) == key) return __uint_as_float(__ldg(fix + 2 * lo + 1));
    return y;
}
__device__ __forceinline__ float glibc_logf(float x, const uint32_t* fix, int n) {
    return apply_fix(x, __double2float_rn(log((double)x)), fix, n);
}
__device__ __forceinline__ float glibc_exp2f(float x, const uint32_t* fix, int n) {
    return apply_fix(x, __double2float_rn(exp2((double)x)), fix, n);
}
// glibc logf of FB values at once: FB independent bucket searches advance together (a fixed
// FIX_STEPS steps covers the longest bucket, 478 entries), so their dependent loads overlap.
constexpr int FIX_STEPS = 9;
template <int FB>
__device__ __forceinline__ void glibc_logf_batch(const float (&x)[FB], float (&y)[FB], const uint32_t* fix, int n) {
    const uint32_t* idx = fix + 2 * (size_t)n;
    uint32_t key[FB];
    int lo[FB], hi[FB];
#pragma unroll
    for (int j = 0; j < FB; j++) {
        key[j] = __float_as_uint(x[j]);
        y[j] = __double2float_rn(log((double)x[j]));
        lo[j] = (int)__ldg(idx + (key[j] >> 16));
        hi[j] = (int)__ldg(idx + (key[j] >> 16) + 1);
    }
#pragma unroll 1
    for (int step = 0; step < FIX_STEPS; step++) {
#pragma unroll
        for (int j = 0; j < FB; j++) {
            const int mid = (lo[j] + hi[j]) >> 1;
            const uint32_t k = lo[j] < hi[j] ? __ldg(fix + 2 * mid) : 0u;
            if (lo[j] < hi[j]) {
                if (k < key[j]) lo[j] = mid + 1;
                else hi[j] = mid;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < FB; j++)
        if (lo[j] < n && __ldg(fix + 2 * lo[j]) == key[j]) y[j] = __uint_as_float(__ldg(fix + 2 * lo[j] + 1));
}

__device__ __forceinline__ int16_t f32_to_i16_sat(float f) {
    if (f != f) return 0;
    if (f <= -32768.0f) return -32768;
    if (f >= 32767.0f) return 32767;
    return (int16_t)__float2int_rz(f);
}
__device__ __forceinline__ int32_t f32_to_i32_sat(float f) {
    if (f != f) return 0;
    if (f <= -2147483648.0f) return INT_MIN;
    if (f >= 2147483647.0f) return INT_MAX;
    return __float2int_rz(f);
}
__device__ __forceinline__ int32_t wmul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }
__device__ __forceinline__ int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
__device__ __forceinline__ int32_t wsub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }

// AAN 8-point kernel with the reference's constants (dct/fast_dct8.rs:254-330).
__device__ __forceinline__ void aan_1d(const int32_t s[8], int32_t out[8], int32_t bias, int shift) {
    int32_t p1 = wmul(wadd(s[2], s[6]), 2218);
    int32_t t2 = wadd(p1, wmul(s[6], -7572));
    int32_t t3 = wadd(p1, wmul(s[2], 3136));
    int32_t t0 = (int32_t)((uint32_t)wadd(s[0], s[4]) << 12);
    int32_t t1 = (int32_t)((uint32_t)wsub(s[0], s[4]) << 12);
    int32_t x0 = wadd(wadd(t0, t3), bias), x3 = wadd(wsub(t0, t3), bias);
    int32_t x1 = wadd(wadd(t1, t2), bias), x2 = wadd(wsub(t1, t2), bias);
    int32_t a0 = s[7], a1 = s[5], a2 = s[3], a3 = s[1];
    int32_t q3 = wadd(a0, a2), q4 = wadd(a1, a3), q1 = wadd(a0, a3), q2 = wadd(a1, a2);
    int32_t q5 = wmul(wadd(q3, q4), 4817);
    a0 = wmul(a0, 1223); a1 = wmul(a1, 8411); a2 = wmul(a2, 12595); a3 = wmul(a3, 6150);
    q1 = wadd(q5, wmul(q1, -3685));
    q2 = wadd(q5, wmul(q2, -10496));
    q3 = wmul(q3, -8035);
    q4 = wmul(q4, -1598);
    int32_t u3 = wadd(a3, wadd(q1, q4)), u2 = wadd(a2, wadd(q2, q3));
    int32_t u1 = wadd(a1, wadd(q2, q4)), u0 = wadd(a0, wadd(q1, q3));
    out[0] = wadd(x0, u3) >> shift; out[7] = wsub(x0, u3) >> shift;
    out[1] = wadd(x1, u2) >> shift; out[6] = wsub(x1, u2) >> shift;
    out[2] = wadd(x2, u1) >> shift; out[5] = wsub(x2, u1) >> shift;
    out[3] = wadd(x3, u0) >> shift; out[4] = wsub(x3, u0) >> shift;
}

// Four MBs per CTA, 64 threads (two warps) per MB.  Thread u of an MB owns luma row u >> 2,
// columns 4 * (u & 3) .. +3 in every 16x16 pass, and two adjacent chroma samples (plane
// u >> 5).  Each pass reads one basis row and one data row per term as 128-bit shared loads,
// four multiply-accumulates per pair of loads.  Per-MB named barriers (ids 1..4, 64 threads).
__device__ __forceinline__ void mb_sync(int bar) { asm volatile("bar.sync %0, 64;" ::"r"(bar) : "memory"); }
// Dequantisation and inverse transforms of one MB and its reconstruction onto the prediction
// (dct/dct16.rs:345-412, dct/fast_dct8.rs:69-174, res/residual.rs:740-752), shared by the
// encoder's residual kernel and the decoder.  64 threads per MB (named barrier bar, thread u: luma row
// yy, columns xb..xb+3; own quantised luma ql); Qc = the MB's 128 chroma coefficients and
// predc its chroma prediction in shared memory; R, RT, aant = per-MB shared scratch.
__device__ __forceinline__ void inverse_mb(int bar, int u, int yy, int xb, const int16_t (&ql)[4], float qsv, bool intra,
                                           const uint16_t* ytab, const uint16_t* ctab, uint32_t lbase, uint8_t* ry,
                                           uint8_t* rU, uint8_t* rV, int CW, int x0, int y0, const int32_t* sT16,
                                           const int32_t* sT16t, int32_t* R, int32_t* RT, int32_t* aant,
                                           const int16_t* Qc, const uint8_t* predc) {
    // dequantisation + 16x16 inverse (row pass over u, then column pass over v)
    {
        int32_t d[4];
        if (intra) {
#pragma unroll
            for (int k = 0; k < 4; k++) d[k] = (int32_t)ql[k] * max((int)ytab[yy * 16 + xb + k], 1);
        } else {
            const int32_t qfp = f32_to_i32_sat(roundf(__fmul_rn(qsv, 16384.0f)));
#pragma unroll
            for (int k = 0; k < 4; k++) d[k] = wadd(wmul((int32_t)ql[k], qfp), 8192) >> 14;
        }
        *(int4*)(R + yy * 16 + xb) = make_int4(d[0], d[1], d[2], d[3]);
    }
    mb_sync(bar);
    {  // rows[v][x] = (sum_i deq[v][i] * T[x][i] + 2^17) >> 18, wrapping   (v = yy)
        uint32_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const uint32_t r = (uint32_t)R[yy * 16 + i];
            const int4 t = *(const int4*)(sT16t + i * 16 + xb);
            a0 += r * (uint32_t)t.x; a1 += r * (uint32_t)t.y; a2 += r * (uint32_t)t.z; a3 += r * (uint32_t)t.w;
        }
        *(int4*)(RT + yy * 16 + xb) = make_int4((int32_t)(a0 + (1u << 17)) >> 18, (int32_t)(a1 + (1u << 17)) >> 18,
                                                (int32_t)(a2 + (1u << 17)) >> 18, (int32_t)(a3 + (1u << 17)) >> 18);
    }
    mb_sync(bar);
    {  // out[y][x] = (sum_v rows[v][x] * T[y][v] + 2^17) >> 18   (y = yy)
        uint32_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
        for (int v = 0; v < 16; v++) {
            const int4 r = *(const int4*)(RT + v * 16 + xb);
            const uint32_t t = (uint32_t)sT16[yy * 16 + v];
            a0 += (uint32_t)r.x * t; a1 += (uint32_t)r.y * t; a2 += (uint32_t)r.z * t; a3 += (uint32_t)r.w * t;
        }
        const uint32_t acc[4] = {a0, a1, a2, a3};
        const uint32_t bv = lbase;
        uint32_t o = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            int32_t r = (int32_t)(acc[k] + (1u << 17)) >> 18;
            r = min(max(r, -32768), 32767);
            const int base = (int)((bv >> (8 * k)) & 255u);
            o |= (uint32_t)min(max(base + r, 0), 255) << (8 * k);
        }
        *(uint32_t*)ry = o;
    }
    // chroma 8x8 AAN inverse: pass 1 over u for each (plane, v); pass 2 over v for each (plane, x)
    if (u < 16) {
        const int cp = u >> 3, v = u & 7;
        int32_t sv[8], o[8];
        int32_t qa = 0;
        if (!intra) {
            float qr = roundf(qsv);
            qr = qr < 1.0f ? 1.0f : qr;
            qa = qr >= 65535.0f ? 65535 : (int32_t)qr;
        }
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int32_t qq = intra ? max((int)ctab[v * 8 + k], 1) : qa;
            sv[k] = (int32_t)Qc[cp * 64 + v * 8 + k] * qq;
        }
        aan_1d(sv, o, 512, 10);
#pragma unroll
        for (int x = 0; x < 8; x++) aant[cp * 64 + x * 8 + v] = o[x];
    }
    mb_sync(bar);
    if (u < 16) {
        const int cp = u >> 3, x = u & 7;
        int32_t sv[8], o[8];
#pragma unroll
        for (int v = 0; v < 8; v++) sv[v] = aant[cp * 64 + x * 8 + v];
        aan_1d(sv, o, 65536, 17);
        uint8_t* Rr = cp == 0 ? rU : rV;
#pragma unroll
        for (int y = 0; y < 8; y++) {
            const int r = min(max(o[y], -32768), 32767);
            const size_t i = (size_t)(y0 / 2 + y) * CW + x0 / 2 + x;
            const int base = intra ? 128 : (int)predc[cp * 64 + y * 8 + x];
            Rr[i] = (uint8_t)min(max(base + r, 0), 255);
        }
    }
}

constexpr int RS_MB = 4;

// Per-MB shared scratch of the residual (one 64-thread group).
struct __align__(16) ResSmem {  // 16-byte rows: element k of an array must stay aligned
    int32_t res[256], rowt[256], resc[128], rowc[128];
    int16_t q[384];
    int32_t aant[2][64];
    int flags[4];  // luma eob of warp 0 / warp 1, (chroma eob << 1 | any non-zero) of warp 0 / warp 1
    float qsh;
    uint8_t predc[128];  // chroma prediction (U then V, 8x8 each)
};

// Residual, transforms, quantisation and reconstruction of MB mb by 64 threads (u = 0..63)
// synchronised on named barrier `bar`; sT16 / sT16t / sT8 hold the bases (sT16t transposed).
__device__ __forceinline__ void residual_mb(const ResidualParams& p, int nmb, int mb, int u, int bar, ResSmem& S,
                                            const int32_t* sT16, const int32_t* sT16t, const int32_t* sT8) {
    const int BW = p.BW, W = p.W, H = p.H, CW = W / 2, CH = H / 2;
    const int bx = mb % BW, by = mb / BW;
    const int x0 = bx * 16, y0 = by * 16;
    const uint8_t *cY = p.cur, *cU = p.cur + (size_t)W * H, *cV = cU + (size_t)CW * CH;
    const uint8_t *pY = p.pred, *pU = p.pred + (size_t)W * H, *pV = pU + (size_t)CW * CH;
    uint8_t *rY = p.recon, *rU = p.recon + (size_t)W * H, *rV = rU + (size_t)CW * CH;
    const int yy = u >> 2, xb = (u & 3) * 4;
    const size_t yi = (size_t)(y0 + yy) * W + x0 + xb;
    const int pl = u >> 5, ci = (u & 31) * 2, cyy = ci >> 3, cxx = ci & 7;
    const size_t cidx = (size_t)(y0 / 2 + cyy) * CW + x0 / 2 + cxx;
    const uint8_t* cC = pl == 0 ? cU : cV;
    const uint8_t* pC = pl == 0 ? pU : pV;
    uint8_t* rC = pl == 0 ? rU : rV;
    int32_t* R = S.res;
    int32_t* RT = S.rowt;
    int32_t* RC = S.resc;
    int32_t* RCT = S.rowc;
    int16_t* Q = S.q;

    // chroma prediction of this thread's two samples: computed here from the reference planes
    // (build_predicted's chroma rule, com/fast_motion.rs:264-345) or read from pred
    uint32_t pcw;
    if (!p.intra && p.ref != nullptr) {
        const MbOut m = p.mb[mb];
        const int mdx = m.raw[0] * 2 + m.raw[2], mdy = m.raw[1] * 2 + m.raw[3];
        const bool integer = ((mdx & 1) == 0) && ((mdy & 1) == 0);
        const int sx0 = x0 + (mdx >> 1), sy0 = y0 + (mdy >> 1);
        const bool copy = integer && sx0 >= 0 && sy0 >= 0 && sx0 + 15 < W && sy0 + 15 < H;
        const uint8_t* Rp = p.ref + (size_t)W * H + (pl == 0 ? 0 : (size_t)CW * CH);
        const int cyg = y0 / 2 + cyy;
        int c2[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int cxg = x0 / 2 + cxx + k;
            c2[k] = copy ? Rp[(size_t)(sy0 / 2 + cyy) * CW + sx0 / 2 + cxx + k]
                         : sample_round(Rp, CW, CH, 2 * cxg + (mdx >> 1), 2 * cyg + (mdy >> 1));
        }
        pcw = (uint32_t)c2[0] | ((uint32_t)c2[1] << 8);
    } else {
        pcw = p.intra ? 0x8080u : *(const uint16_t*)(pC + cidx);
    }
    S.predc[pl * 64 + ci] = (uint8_t)pcw;
    S.predc[pl * 64 + ci + 1] = (uint8_t)(pcw >> 8);
    auto copy_pred = [&]() {  // recon = prediction, coefficients zero
        *(uint32_t*)(rY + yi) = *(const uint32_t*)(pY + yi);
        *(uint16_t*)(rC + cidx) = (uint16_t)pcw;
        int16_t* co = p.coeffs + (size_t)mb * 384;
        *(uint2*)(co + yy * 16 + xb) = make_uint2(0u, 0u);
        *(uint32_t*)(co + 256 + pl * 64 + ci) = 0u;
        if (u == 0) {
            p.opt_skip[mb] = 1;
            const int8_t* c = p.mb[mb].coded;
            p.fmask[mb] = (c[0] | c[1] | c[2] | c[3]) != 0;
            p.eobs[3 * mb] = p.eobs[3 * mb + 1] = p.eobs[3 * mb + 2] = 0;
        }
    };
    if (!p.intra && p.lnv != nullptr) {  // AQ step (compute_aq_quant_steps, res/residual.rs:154-167)
        if (u == 0) {
            const float off = __fmul_rn(0.8f, __fsub_rn(p.lnv[mb], p.lnv[nmb]));
            const float q = __fmul_rn(p.aq_base, glibc_exp2f(__fdiv_rn(off, 6.0f), p.expfix, p.nexp));
            S.qsh = q;
            p.qs_out[mb] = q;
        }
        mb_sync(bar);
    }
    if (!p.intra && p.mb[mb].rdo_skip) {  // never transformed: residual 0, recon = prediction
        copy_pred();
        return;
    }
    {
        const uint32_t cv = *(const uint32_t*)(cY + yi);
        const uint32_t pv = p.intra ? 0x80808080u : *(const uint32_t*)(pY + yi);
#pragma unroll
        for (int k = 0; k < 4; k++) R[yy * 16 + xb + k] = (int)((cv >> (8 * k)) & 255u) - (int)((pv >> (8 * k)) & 255u);
        const uint32_t cc = *(const uint16_t*)(cC + cidx);
        const uint32_t pc = pcw;
        RC[pl * 64 + ci] = (int)(cc & 255u) - (int)(pc & 255u);
        RC[pl * 64 + ci + 1] = (int)(cc >> 8) - (int)(pc >> 8);
    }
    mb_sync(bar);
    // The reference accumulates both FDCT passes in i64 and clamps to i32.  With residuals in
    // [-255, 255] and these bases, every partial sum stays below 2^31 (16x16: row pass
    // <= 255 * 1048576 = 2.7e8, rows <= 1020, column pass <= 1020 * 1048576 + 2^17 = 1.07e9;
    // 8x8: 1.9e8, 721, 5.3e8), so exact int32 accumulation gives the same values and the
    // clamp never applies.
    {  // row pass: rowt[y][j] = sum_i res[y][i] * T[i][j]
        int32_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const int r = R[yy * 16 + i];
            const int4 t = *(const int4*)(sT16 + i * 16 + xb);
            a0 += r * t.x; a1 += r * t.y; a2 += r * t.z; a3 += r * t.w;
        }
        *(int4*)(RT + yy * 16 + xb) = make_int4((a0 + (1 << 17)) >> 18, (a1 + (1 << 17)) >> 18,
                                                (a2 + (1 << 17)) >> 18, (a3 + (1 << 17)) >> 18);
        int32_t c0 = 0, c1 = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int r = RC[pl * 64 + cyy * 8 + i];
            const int2 t = *(const int2*)(sT8 + i * 8 + cxx);
            c0 += r * t.x; c1 += r * t.y;
        }
        *(int2*)(RCT + pl * 64 + ci) = make_int2((c0 + (1 << 17)) >> 18, (c1 + (1 << 17)) >> 18);
    }
    mb_sync(bar);
    int32_t coef[4], coefc[2];
    {  // column pass: coef[v][x] = sum_i rowt[i][x] * T[i][v]   (v = yy)
        int32_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const int4 r = *(const int4*)(RT + i * 16 + xb);
            const int t = sT16[i * 16 + yy];
            a0 += r.x * t; a1 += r.y * t; a2 += r.z * t; a3 += r.w * t;
        }
        coef[0] = (a0 + (1 << 17)) >> 18; coef[1] = (a1 + (1 << 17)) >> 18;
        coef[2] = (a2 + (1 << 17)) >> 18; coef[3] = (a3 + (1 << 17)) >> 18;
        int32_t c0 = 0, c1 = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int2 r = *(const int2*)(RCT + pl * 64 + i * 8 + cxx);
            const int t = sT8[i * 8 + cyy];
            c0 += r.x * t; c1 += r.y * t;
        }
        coefc[0] = (c0 + (1 << 17)) >> 18; coefc[1] = (c1 + (1 << 17)) >> 18;
    }
    // quantisation
    float qsv = 0.0f;
    int16_t ql[4], qc[2];
    if (p.intra) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float qy = (float)max((int)p.intra_ytab[yy * 16 + xb + k], 1);
            ql[k] = f32_to_i16_sat(roundf(__fdiv_rn(__int2float_rn(coef[k]), qy)));
        }
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const float qq = (float)max((int)p.intra_ctab[ci + k], 1);
            qc[k] = f32_to_i16_sat(roundf(__fdiv_rn(__int2float_rn(coefc[k]), qq)));
        }
    } else {
        qsv = p.lnv != nullptr ? S.qsh : p.qs[mb];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float r = __fdiv_rn(__int2float_rn(coef[k]), qsv);
            ql[k] = fabsf(r) < p.dead_zone ? (int16_t)0 : f32_to_i16_sat(roundf(r));
        }
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const float r = __fdiv_rn(__int2float_rn(coefc[k]), qsv);
            qc[k] = fabsf(r) < p.dead_zone ? (int16_t)0 : f32_to_i16_sat(roundf(r));
        }
    }
    // last non-zero index per plane block (0 when all zero) and "any non-zero"
    int lz = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) lz = ql[k] != 0 ? yy * 16 + xb + k : lz;
    int lc = 0;
#pragma unroll
    for (int k = 0; k < 2; k++) lc = qc[k] != 0 ? ci + k : lc;
    const bool any = (ql[0] | ql[1] | ql[2] | ql[3] | qc[0] | qc[1]) != 0;
    lz = __reduce_max_sync(0xffffffffu, lz);
    lc = __reduce_max_sync(0xffffffffu, lc);
    const unsigned anyw = __any_sync(0xffffffffu, any);
    if ((u & 31) == 0) {
        S.flags[u >> 5] = lz;
        S.flags[2 + (u >> 5)] = (int)anyw | (lc << 1);
    }
    mb_sync(bar);
    const bool nz = ((S.flags[2] | S.flags[3]) & 1) != 0;
    if (!p.intra && !nz) {  // became all-zero after quantisation: optimized skip
        copy_pred();
        return;
    }
    {
        int16_t* co = p.coeffs + (size_t)mb * 384;
        const uint32_t w0 = (uint32_t)(uint16_t)ql[0] | ((uint32_t)(uint16_t)ql[1] << 16);
        const uint32_t w1 = (uint32_t)(uint16_t)ql[2] | ((uint32_t)(uint16_t)ql[3] << 16);
        *(uint2*)(co + yy * 16 + xb) = make_uint2(w0, w1);
        *(uint32_t*)(co + 256 + pl * 64 + ci) = (uint32_t)(uint16_t)qc[0] | ((uint32_t)(uint16_t)qc[1] << 16);
        Q[256 + pl * 64 + ci] = qc[0];
        Q[256 + pl * 64 + ci + 1] = qc[1];
        if (u == 0) {
            p.eobs[3 * mb] = (uint8_t)max(S.flags[0], S.flags[1]);
            p.eobs[3 * mb + 1] = (uint8_t)(S.flags[2] >> 1);
            p.eobs[3 * mb + 2] = (uint8_t)(S.flags[3] >> 1);
            p.opt_skip[mb] = 0;
            p.fmask[mb] = 1;
        }
    }
    const uint32_t lbase = p.intra ? 0x80808080u : *(const uint32_t*)(pY + yi);
    inverse_mb(bar, u, yy, xb, ql, qsv, p.intra != 0, p.intra_ytab, p.intra_ctab, lbase, rY + yi, rU, rV, CW, x0, y0,
               sT16, sT16t, R, RT, S.aant[0], Q + 256, S.predc);
}

__device__ __forceinline__ int c128(int x) { return min(max(x, -128), 127); }
__device__ __forceinline__ void filter_line(int* px, int E, int I, int Hv) {
    int p3 = px[0], p2 = px[1], p1 = px[2], p0 = px[3], q0 = px[4], q1 = px[5], q2 = px[6], q3 = px[7];
    bool mask = 2 * abs(p0 - q0) + abs(q1 - p1) / 2 <= E && abs(p3 - p2) <= I && abs(p2 - p1) <= I &&
                abs(p1 - p0) <= I && abs(q1 - q0) <= I && abs(q2 - q1) <= I && abs(q3 - q2) <= I;
    if (!mask) return;
    int ps2 = p2 - 128, ps1 = p1 - 128, ps0 = p0 - 128, qs0 = q0 - 128, qs1 = q1 - 128, qs2 = q2 - 128;
    bool hev = abs(p1 - p0) > Hv || abs(q1 - q0) > Hv;
    int w = c128(c128(ps1 - qs1) + 3 * (qs0 - ps0));
    if (hev) {
        int f1 = c128(w + 4) >> 3, f2 = c128(w + 3) >> 3;
        px[4] = min(max(c128(qs0 - f1) + 128, 0), 255);
        px[3] = min(max(c128(ps0 + f2) + 128, 0), 255);
    } else {
        int a = c128((27 * w + 63) >> 7);
        int nq0 = c128(qs0 - a), np0 = c128(ps0 + a);
        a = c128((18 * w + 63) >> 7);
        int nq1 = c128(qs1 - a), np1 = c128(ps1 + a);
        a = c128((9 * w + 63) >> 7);
        int nq2 = c128(qs2 - a), np2 = c128(ps2 + a);
        px[1] = min(max(np2 + 128, 0), 255);
        px[2] = min(max(np1 + 128, 0), 255);
        px[3] = min(max(np0 + 128, 0), 255);
        px[4] = min(max(nq0 + 128, 0), 255);
        px[5] = min(max(nq1 + 128, 0), 255);
        px[6] = min(max(nq2 + 128, 0), 255);
    }
}
// Out of place, all planes in one launch (src and dst must not overlap: neighbouring tiles
// read each other's pixels as halo).  A CTA owns one band of an edge grid (16 luma / 8
// chroma rows) and DB_TW luma (DB_TW/2 chroma) columns.  It loads the tile with a 4-pixel
// halo, filters every vertical edge of the halo rows in shared memory (rows are independent
// in that pass), then the horizontal edges at the band's top and bottom (their lines are 4+
// pixels apart, so they touch disjoint pixels), and stores only its own pixels.  That equals
// the reference's whole-plane vertical pass followed by the whole-plane horizontal pass.
constexpr int DB_TILE_BYTES = (16 + 8) * (DB_TW + 8);
// One tile (plane, t: band-major tile index within the plane) by nthr threads synchronised on
// group barrier `bar` (0 = the whole CTA); `tile` = DB_TILE_BYTES of shared memory.
// TW: tile width in luma columns (DB_TW everywhere but the tuned multi-clip launch), tile =
// (16 + 8) * (TW + 8) bytes.
template <int TW = DB_TW>
__device__ __forceinline__ void deblock_tile(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int W, int H,
                                             int BW, int E, int I, int Hv, const uint8_t* mask, int plane, int t,
                                             uint8_t* tile, int tid, int nthr, int bar) {
    const int w = plane ? W / 2 : W, h = plane ? H / 2 : H, g = plane ? 8 : 16, tw = plane ? TW / 2 : TW;
    const size_t poff = plane == 0 ? 0 : (size_t)W * H + (plane == 2 ? (size_t)(W / 2) * (H / 2) : 0);
    const uint8_t* pl = src + poff;
    uint8_t* po = dst + poff;
    const int tpb = (w + tw - 1) / tw;
    const int band = t / tpb, X0 = (t % tpb) * tw, X1 = min(X0 + tw, w);
    const int Y0 = band * g, Y1 = Y0 + g;
    const int ry0 = max(Y0 - 4, 0), ry1 = min(Y1 + 4, h), cx0 = max(X0 - 4, 0), cx1 = min(X1 + 4, w);
    const int TS = TW + 8, oy = Y0 - 4, ox = X0 - 4;  // tile row stride and origin
    const int nrow = ry1 - ry0, ncol = cx1 - cx0;
    // 32-bit words: cx0, cx1, w and the tile's row stride and origin are multiples of 4 (tile
    // widths and plane widths are multiples of 8), and `tile` is 16-byte aligned
    const int ncw = ncol >> 2;
    for (int i = tid; i < nrow * ncw; i += nthr) {
        const int r = i / ncw, c = i - r * ncw;
        *(uint32_t*)(tile + (ry0 + r - oy) * TS + cx0 + 4 * c - ox) =
            *(const uint32_t*)(pl + (size_t)(ry0 + r) * w + cx0 + 4 * c);
    }
    group_sync(bar, nthr);
    // vertical edges x = k*g (1 <= k < w/g) with X0 <= x <= X1, on every loaded row
    const int k0 = max(1, (X0 + g - 1) / g), k1 = min(w / g - 1, X1 / g);
    const int nk = k1 - k0 + 1;
    if (nk > 0) {
        for (int i = tid; i < nrow * nk; i += nthr) {
            const int r = i / nk, k = k0 + (i - r * nk), y = ry0 + r;
            const int by = y / g;
            if (mask && !(mask[by * BW + k - 1] | mask[by * BW + k])) continue;
            uint8_t* sp = tile + (y - oy) * TS + k * g - 4 - ox;
            int px[8];
#pragma unroll
            for (int q = 0; q < 8; q++) px[q] = sp[q];
            filter_line(px, E, I, Hv);
#pragma unroll
            for (int q = 1; q < 7; q++) sp[q] = (uint8_t)px[q];
        }
    }
    group_sync(bar, nthr);
    // horizontal edges at the band's top (Y0) and bottom (Y1), columns X0 .. X1-1
    for (int i = tid; i < 2 * (X1 - X0); i += nthr) {
        const int e = (i < X1 - X0 ? Y0 : Y1) / g, x = X0 + (i < X1 - X0 ? i : i - (X1 - X0));
        if (e < 1 || e >= h / g) continue;
        const int bxm = x / g;
        if (mask && !(mask[(e - 1) * BW + bxm] | mask[e * BW + bxm])) continue;
        uint8_t* sp = tile + (e * g - 4 - oy) * TS + x - ox;
        int px[8];
#pragma unroll
        for (int q = 0; q < 8; q++) px[q] = sp[q * TS];
        filter_line(px, E, I, Hv);
#pragma unroll
        for (int q = 1; q < 7; q++) sp[q * TS] = (uint8_t)px[q];
    }
    group_sync(bar, nthr);
    const int oww = (X1 - X0) >> 2;
    for (int i = tid; i < g * oww; i += nthr) {
        const int r = i / oww, c = i - r * oww;
        *(uint32_t*)(po + (size_t)(Y0 + r) * w + X0 + 4 * c) = *(const uint32_t*)(tile + (Y0 + r - oy) * TS + X0 + 4 * c - ox);
    }
}

// This CTA's index within its clip's part of the grid: a single-clip launch owns the whole
// grid (cta0 = 0); a multi-clip launch gives each clip a contiguous range of CTAs starting
// at cta0.
__device__ __forceinline__ int row_cta(const SearchParams& p) { return (int)blockIdx.x - p.cta0; }

// ---- search warp -> mode warp handoff through a shared-memory ring (one CTA per MB row)
// Slot word: [63:49] (n + 1) mod 2^15 for the n-th MB of the CTA, [48] failure, [47:32] best
// SAD (at most 255 * 256), [31:0] raw MV (dx, dy, sx, sy as bytes).  Tag and payload share
// one 64-bit word, so a single volatile store publishes both.
constexpr int HAND_RING = 64;
constexpr unsigned long long HAND_FAIL = 1ull << 48;

// done[0]: MBs the mode warp has taken, done[1]: MBs the AQ warp has taken (a large value
// when there is none); a slot is reused once both have taken its previous MB.
__device__ __forceinline__ bool hand_put(unsigned long long* hand, volatile int* done, int n,
                                         unsigned long long payload, long long limit) {
    long long spins = 0;
    while (n - min(done[0], done[1]) >= HAND_RING) {  // the slot's previous MB has not been taken yet
        if (++spins > limit) return false;
        __nanosleep(32);
    }
    volatile unsigned long long* h = hand + (n & (HAND_RING - 1));
    *h = ((unsigned long long)((n + 1) & 0x7fff) << 49) | payload;
    return true;
}

__device__ __forceinline__ bool hand_get(const unsigned long long* hand, int n, unsigned long long& w,
                                         long long limit) {
    const volatile unsigned long long* h = hand + (n & (HAND_RING - 1));
    const unsigned long long want = (unsigned long long)((n + 1) & 0x7fff) << 49;
    unsigned long long v = *h;
    long long spins = 0;
    while ((v & ~((1ull << 49) - 1)) != want) {
        if (++spins > limit) return false;
        if (spins > 64) __nanosleep(16);
        v = *h;
    }
    w = v;
    return true;
}

// Bounded wait for a wavefront record of this frame (tag in bits 63:48).
__device__ __forceinline__ bool rec_wait(const unsigned long long* rp, unsigned long long tagbits,
                                         unsigned long long& v, long long limit) {
    v = ld_rec(rp);
    long long spins = 0;
    while ((v & 0xffff000000000000ull) != tagbits) {
        if (++spins > limit) return false;
        __nanosleep(20);
        v = ld_rec(rp);
    }
    return true;
}

// RDO skip (enc/rdo.rs:140-178) and the MV mode decision of one MB on its coded neighbours
// (enc/encoder.rs:459-733, res/mv_predictor.rs:59-272): mode, NEW base and raw delta, flags
// and the coded (reconstructed) MV.
struct MbDecision {
    MvT coded;
    int mode, chosen, rdx, rdy;
    uint8_t flags;
    bool rdo_skip;
};
__device__ __forceinline__ MbDecision decide_mb(const SearchParams& p, const MvT& raw, long long best_sad, bool has_l,
                                                bool has_t, bool has_tr, bool has_tl, bool has_tm, const MvT& L_cod,
                                                const MvT& cT, const MvT& cTR, const MvT& cTL, const MvT& Tm_cod) {
    // ---- RDO skip decision (enc/rdo.rs:140-178)
    bool int_al = raw.sx == 0 && raw.sy == 0;
    double satd = (double)best_sad;
    double skip_cost = __dadd_rn(satd, __dmul_rn(p.rdo_lambda, p.rdo_skip_bits));
    double est = __dadd_rn(p.rdo_icpt, __dmul_rn(p.rdo_slope, satd));
    if (est < 0.0) est = 0.0;
    double coded_cost = __dadd_rn(__dmul_rn(satd, p.rdo_ret), __dmul_rn(p.rdo_lambda, __dadd_rn(p.rdo_keep_bits, est)));
    bool rdo_skip = p.rdo_allow && int_al && !(satd > p.rdo_guard) && (skip_cost <= coded_cost);

    // ---- mode decision on the coded neighbours
    const MvT zero{0, 0, 0, 0};
    MvT nearest = zero, nearm = zero;
    {
        const MvT CS[5] = {L_cod, cT, cTR, cTL, Tm_cod};
        const bool PV[5] = {has_l, has_t, has_tr, has_tl, has_tm};
        int nu = 0;
#pragma unroll
        for (int i = 0; i < 5; i++) {
            bool take = PV[i] && (nu == 0 || (nu == 1 && !mv_eq(CS[i], nearest)));
            if (take && nu == 0) nearest = CS[i];
            else if (take && nu == 1) nearm = CS[i];
            nu += take ? 1 : 0;
        }
    }
    MvT temporal = has_tm ? Tm_cod : zero;
    const int mx = raw.dx * 2 + raw.sx, my = raw.dy * 2 + raw.sy;
    auto hpeq = [&](const MvT& t) { return mx == t.dx * 2 + t.sx && my == t.dy * 2 + t.sy; };
    int mode;
    if (raw.dx == 0 && raw.dy == 0 && raw.sx == 0 && raw.sy == 0) mode = 0;  // Zero
    else if (hpeq(nearest)) mode = 1;
    else if (hpeq(nearm)) mode = 2;
    else if (has_tr && hpeq(cTR)) mode = 3;
    else if (has_tl && hpeq(cTL)) mode = 4;
    else if (hpeq(temporal)) mode = 6;
    else mode = 5;  // New
    int chosen = 0, rdx = 0, rdy = 0;
    MvT coded = raw;
    if (mode == 5) {
        const MvT bases[5] = {nearest, nearm, cTR, cTL, temporal};
        const bool hasb[5] = {true, true, has_tr, has_tl, true};
        const int selbits[5] = {1, 2, 3, 4, 4};
        unsigned best = 0xffffffffu;
        int bbx = nearest.dx, bby = nearest.dy;
#pragma unroll
        for (int k = 0; k < 5; k++) {
            if (!hasb[k]) continue;
            int ddx = sat8(raw.dx - bases[k].dx), ddy = sat8(raw.dy - bases[k].dy);
            unsigned cst = (unsigned)(selbits[k] + comp_bits(ddx) + comp_bits(ddy));
            if (cst < best) { best = cst; chosen = k; bbx = bases[k].dx; bby = bases[k].dy; }
        }
        rdx = sat8(raw.dx - bbx);
        rdy = sat8(raw.dy - bby);
        coded.dx = sat8(bbx + rdx);
        coded.dy = sat8(bby + rdy);
    } else if (mode == 1) coded = nearest;
    else if (mode == 2) coded = nearm;
    else if (mode == 3) coded = cTR;
    else if (mode == 4) coded = cTL;
    else if (mode == 6) coded = temporal;
    uint8_t flags = 0;
    if (mode == 5) flags = (raw.sx == 1 ? 0x01 : 0) | (raw.sy == 1 ? 0x04 : 0);
    if (rdo_skip) flags |= 0x40;
    return MbDecision{coded, mode, chosen, rdx, rdy, flags, rdo_skip};
}

// The second warp of each row CTA: RDO skip (enc/rdo.rs:140-178) and the MV mode decision on
// the coded (reconstructed) neighbours (enc/encoder.rs:459-733, res/mv_predictor.rs:59-272)
// for the MBs the search warp hands over, in raster order.  It publishes the coded-MV records
// the next row's mode warp reads (second half of p.rec) and the per-MB output.  None of this
// feeds the search, so it runs beside the search chain instead of on it.
__device__ __forceinline__ void mode_warp(const SearchParams& p, const unsigned long long* hand, volatile int* hand_done,
                                       unsigned long long tagbits) {
    const int lane = threadIdx.x & 31;
    MbRec* rc = p.rec + (size_t)p.BW * p.BH;
    auto rec_cod = [](unsigned long long v) {
        return MvT{(int)(int8_t)(v >> 24), (int)(int8_t)(v >> 16), (int)(int8_t)(v >> 8), (int)(int8_t)v};
    };
    const bool has_tm = p.prev_coded != nullptr;
    int n = 0;
    for (int r = row_cta(p); r < p.BH; r += p.nrow_ctas) {
        MvT L_cod{0, 0, 0, 0};
        unsigned long long vT = 0, vTL = 0;
        for (int bx = 0; bx < p.BW; bx++) {
            const int idx = r * p.BW + bx;
            unsigned long long hw = 0, vTR = 0;
            int st = 0;  // 0 ok, 1 wait expired, 2 the search warp gave up
            if (lane == 0) {
                if (!hand_get(hand, n, hw, p.spin_limit)) st = 1;
                else if (hw & HAND_FAIL) st = 2;
                if (st == 0 && r > 0) {
                    if (bx == 0 && !rec_wait(rc + (size_t)(r - 1) * p.BW, tagbits, vT, p.spin_limit)) st = 1;
                    if (st == 0 && bx + 1 < p.BW &&
                        !rec_wait(rc + (size_t)(r - 1) * p.BW + bx + 1, tagbits, vTR, p.spin_limit))
                        st = 1;
                }
                if (st == 0) *hand_done = n + 1;
            }
            st = __shfl_sync(0xffffffffu, st, 0);
            if (st != 0) {
                if (lane == 0 && st == 1) atomicOr(p.status, ST_WAIT_TIMEOUT);
                return;
            }
            n++;
            hw = __shfl_sync(0xffffffffu, hw, 0);
            vT = __shfl_sync(0xffffffffu, vT, 0);
            vTR = __shfl_sync(0xffffffffu, vTR, 0);
            const MvT raw{(int)(int8_t)hw, (int)(int8_t)(hw >> 8), (int)(int8_t)(hw >> 16), (int)(int8_t)(hw >> 24)};
            const long long best_sad = (long long)((hw >> 32) & 0xffff);
            const bool has_t = r > 0, has_l = bx > 0, has_tl = r > 0 && bx > 0, has_tr = r > 0 && bx + 1 < p.BW;
            MvT Tm_cod{0, 0, 0, 0};
            if (has_tm) {
                const char4 pc = *(const char4*)(p.prev_coded + 4 * idx);
                Tm_cod = MvT{pc.x, pc.y, pc.z, pc.w};
            }

            const MbDecision md = decide_mb(p, raw, best_sad, has_l, has_t, has_tr, has_tl, has_tm, L_cod,
                                             has_t ? rec_cod(vT) : MvT{0, 0, 0, 0},
                                             has_tr ? rec_cod(vTR) : MvT{0, 0, 0, 0},
                                             has_tl ? rec_cod(vTL) : MvT{0, 0, 0, 0}, Tm_cod);
            const MvT coded = md.coded;
            const int mode = md.mode, chosen = md.chosen, rdx = md.rdx, rdy = md.rdy;
            const uint8_t flags = md.flags;
            const bool rdo_skip = md.rdo_skip;

            RIV_STAMP(5);
            // ---- publish
            if (lane == 0) {
                unsigned long long rv = tagbits | ((unsigned long long)(uint8_t)coded.dx << 24) |
                                        ((unsigned long long)(uint8_t)coded.dy << 16) |
                                        ((unsigned long long)(uint8_t)coded.sx << 8) | (unsigned long long)(uint8_t)coded.sy;
                st_rec(rc + idx, rv);
                MbOut o;
                o.raw[0] = (int8_t)raw.dx; o.raw[1] = (int8_t)raw.dy; o.raw[2] = (int8_t)raw.sx; o.raw[3] = (int8_t)raw.sy;
                o.coded[0] = (int8_t)coded.dx; o.coded[1] = (int8_t)coded.dy;
                o.coded[2] = (int8_t)coded.sx; o.coded[3] = (int8_t)coded.sy;
                o.rdelta[0] = (int8_t)rdx; o.rdelta[1] = (int8_t)rdy;
                o.mode = (uint8_t)mode; o.base = (uint8_t)chosen; o.flags = flags; o.rdo_skip = rdo_skip ? 1 : 0;
                o.pad[0] = o.pad[1] = 0;
                o.best_sad = (int32_t)best_sad;
                p.out[idx] = o;
                *(char4*)(p.coded_out + 4 * (size_t)idx) =
                    make_char4((signed char)coded.dx, (signed char)coded.dy, (signed char)coded.sx, (signed char)coded.sy);
            }
            RIV_STAMP(6);
            if (lane == 0) RIV_GSTAMP(idx, 30);
            L_cod = coded;
            vTL = vT;
            vT = vTR;
        }
    }
}

__device__ __forceinline__ size_t sad_table_smem_dev(int sr) {
    const int WT = 16 + 2 * sr, WTS = (WT + 8 + 15) & ~15;
    return ((size_t)WT * WTS + 16 + 256 + 15) & ~(size_t)15;
}
// ---- table workers of the fused search launch: the CTAs beyond the row CTAs compute the
// SAD-table rows in raster order while the wavefront runs, and publish each MB's row with a
// flag holding the frame tag (release after the CTA's writes; the loader acquires it).
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

constexpr int TW_GROUP = 128;  // threads per worker group
constexpr int RES_HALF_BYTES = (sizeof(ResSmem) + 15) & ~15;
static_assert(sizeof(ResSmem) % 16 == 0 && offsetof(ResSmem, q) % 16 == 0 && offsetof(ResSmem, aant) % 16 == 0, "ResSmem rows");
__host__ __device__ constexpr int worker_group_bytes() {
    return 2 * RES_HALF_BYTES > DB_TILE_BYTES + 16 ? 2 * RES_HALF_BYTES : DB_TILE_BYTES + 16;
}
constexpr int WK_BASES = 2304;  // sT16, sT16t, sT8 of the deferred residual
static_assert(WK_BASES + 4 * worker_group_bytes() + 2 * 4 * 4 <= 116 * 1024, "worker CTA shared memory");

// Bounded wait until *c >= target (acquire); every thread of the group polls.
__device__ __forceinline__ bool wait_at_least(const unsigned* c, unsigned target, long long limit) {
    long long spins = 0;
    while (ld_acquire_u32(c) < target) {
        if (++spins > limit) return false;
        __nanosleep(64);
    }
    return true;
}
// The rows / bands MB row r depends on before its reference samples may be read: the
// previous frame's deblocked bands r-1 .. r+1 (or its residual rows when it has no deblock).
__device__ __forceinline__ bool wait_ref_rows(const SearchParams& p, int r, int tiles_per_band) {
    if (!p.defer) return true;
    for (int b = max(r - 1, 0); b <= min(r + 1, p.BH - 1); b++) {
        const bool ok = p.db_level > 0 ? wait_at_least(p.wq + 1 + p.BH + b, (unsigned)tiles_per_band, p.spin_limit)
                                       : wait_at_least(p.wq + 1 + b, (unsigned)p.BW, p.spin_limit);
        if (!ok) return false;
    }
    return true;
}

// ---------------------------------------------------------------------------------
// K8 helpers: per-MB side info and compaction of the coded MBs' coefficients for the host
// entropy coder.  side = mode | base<<3 | subx<<6 | suby<<7 | rdx<<8 | rdy<<16 | optskip<<24.
// Each coded MB contributes its three plane blocks truncated after the last non-zero
// coefficient (the entropy coder never reads beyond it): Y[0..eY], U[0..eU], V[0..eV].
// hdr[0] = coded MB count, hdr[1] = total coefficients written.
// ---------------------------------------------------------------------------------
// Scan by NT threads (named barrier `bar`): each thread owns IPT consecutive MBs of an
// NT * IPT chunk (all their loads are issued together), then one scan of the thread totals
// per chunk.  wsum / wsz: NT / 32 ints of shared memory each.
constexpr int SC_THREADS = 256, SC_IPT = 32;
template <int NT, int IPT>
__device__ __forceinline__ void scan_mbs(const uint8_t* opt_skip, const uint8_t* eobs, int nmb, int intra,
                                         int32_t* index, int32_t* offset, uint32_t* hdr, int tid, int bar, int* wsum,
                                         int* wsz) {
    const int lane = tid & 31, wid = tid >> 5;
    int carry = 0, carry_sz = 0;  // identical in every thread
    for (int base = 0; base < nmb; base += NT * IPT) {
        const int i0 = base + tid * IPT;
        // v = coded << 16 | coefficient count (<= 3 * 256): 32 of them sum without carry
        uint32_t v[IPT];
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            const int i = i0 + k;
            const bool f = i < nmb && (intra || !opt_skip[i]);
            v[k] = f ? (1u << 16) | (uint32_t)(eobs[3 * i] + eobs[3 * i + 1] + eobs[3 * i + 2] + 3) : 0u;
        }
        uint32_t tot = 0;
#pragma unroll
        for (int k = 0; k < IPT; k++) tot += v[k];
        const int x = (int)(tot >> 16), y = (int)(tot & 0xffffu);
        int xs = x, ys = y;  // inclusive warp scan of the thread totals
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int a2 = __shfl_up_sync(0xffffffffu, xs, o), b2 = __shfl_up_sync(0xffffffffu, ys, o);
            if (lane >= o) { xs += a2; ys += b2; }
        }
        if (lane == 31) { wsum[wid] = xs; wsz[wid] = ys; }
        group_sync(bar, NT);
        int wx = 0, wy = 0, tx = 0, ty = 0;  // exclusive prefix of this warp, chunk totals
#pragma unroll
        for (int q = 0; q < NT / 32; q++) {
            if (q < wid) { wx += wsum[q]; wy += wsz[q]; }
            tx += wsum[q];
            ty += wsz[q];
        }
        int ex = carry + wx + xs - x;
        int ez = carry_sz + wy + ys - y;
#pragma unroll
        for (int k = 0; k < IPT; k++) {
            const int i = i0 + k;
            const int f = (int)(v[k] >> 16), z = (int)(v[k] & 0xffffu);
            if (i < nmb) { index[i] = f ? ex : -1; offset[i] = ez; }
            ex += f;
            ez += z;
        }
        carry += tx;
        carry_sz += ty;
        group_sync(bar, NT);  // wsum / wsz are rewritten by the next chunk
    }
    if (tid == 0) { hdr[0] = (uint32_t)carry; hdr[1] = (uint32_t)carry_sz; }
}
// Pack MB m with one warp: side info, EOBs and the truncated coefficient blocks.
__device__ __forceinline__ void pack_mb(int m, int lane, const uint8_t* opt_skip, const MbOut* mb,
                                        const int16_t* coeffs, const uint8_t* eobs, const int32_t* index,
                                        const int32_t* offset, int intra, uint32_t* side, int16_t* packed,
                                        uint8_t* peobs) {
    const int k = index[m];
    const int e0 = eobs[3 * m], e1 = eobs[3 * m + 1], e2 = eobs[3 * m + 2];
    if (lane == 0) {
        uint32_t s = 0;
        if (!intra) {
            const MbOut o = mb[m];
            s = (uint32_t)o.mode | ((uint32_t)o.base << 3) | ((uint32_t)(o.raw[2] & 1) << 6) |
                ((uint32_t)(o.raw[3] & 1) << 7) | ((uint32_t)(uint8_t)o.rdelta[0] << 8) |
                ((uint32_t)(uint8_t)o.rdelta[1] << 16) | ((uint32_t)(opt_skip[m] & 1) << 24);
        }
        side[m] = s;
        if (k >= 0) {
            peobs[3 * k] = (uint8_t)e0;
            peobs[3 * k + 1] = (uint8_t)e1;
            peobs[3 * k + 2] = (uint8_t)e2;
        }
    }
    if (k < 0) return;
    const int n0 = e0 + 1, n1 = e1 + 1, n2 = e2 + 1;
    const int16_t* src = coeffs + (size_t)m * 384;
    int16_t* dst = packed + offset[m];
    for (int i = lane; i < n0 + n1 + n2; i += 32) {
        const int si = i < n0 ? i : (i < n0 + n1 ? 256 + (i - n0) : 320 + (i - n0 - n1));
        dst[i] = src[si];
    }
}

// The worker CTAs of the fused search launch (the CTAs beyond the row CTAs), in groups of 128
// threads that take tasks from one queue in a fixed order: for step k, the previous frame's
// residual of MB row k (pairs of MBs), its deblock of band k-DB_LAG (tiles), then the
// SAD-table MBs of row k-TAB_LAG (k when nothing is deferred).  Each task waits only for
// tasks earlier in the queue (residual rows b-1 .. b+1 for band b, deblocked bands r-1 .. r+1
// for table row r), all of which are held by running groups of this cooperative launch, so
// the waits end; the lags put two steps (more tasks than there are groups) between a task
// and what it waits for, so a group rarely holds a task whose inputs are still being made.
// One thread per group polls; the group barrier then orders the others' reads after its
// acquire.  Completion is published with release operations: per-row / per-band counters in
// wq, per-MB table flags (the frame tag) that the loaders acquire.  With p.compact the queue
// ends with the previous frame's compaction: one scan task (after every residual row), then
// one pack task per MB row (after the scan, published in wq[2BH+1]).
constexpr int WK_SCAN_IPT = 8;  // MBs per thread of the in-launch scan (registers are capped)
// Worker region: the residual bases (WK_BASES bytes), `groups` group scratch areas, then a
// task word and a status word per group.
__host__ __device__ constexpr int worker_region_bytes(int groups) {
    return WK_BASES + groups * worker_group_bytes() + 2 * groups * 4;
}
// Bases of the deferred residual into a worker region, by threads lo, lo + step, ...
__device__ __forceinline__ void load_worker_bases(const SearchParams& p, uint8_t* region, int lo, int step) {
    if (!p.defer) return;
    int32_t* sT16 = (int32_t*)region;
    int32_t* sT16t = sT16 + 256;
    int32_t* sT8 = sT16t + 256;
    for (int i = lo; i < 256; i += step) {
        sT16[i] = c_T16[i];
        sT16t[(i & 15) * 16 + (i >> 4)] = c_T16[i];
    }
    for (int i = lo; i < 64; i += step) sT8[i] = c_T8[i];
}

// The task loop of one 128-thread group: region slot g of `groups`, named barriers keyed
// by gid (the group's index in its CTA: 1 + gid for the group, 5 + 2 gid + half for the
// residual halves).  With `stop` the group takes each index only when it will run the
// task and leaves once *stop is set (no index is held early); without it, it runs until
// the queue is empty.
__device__ __forceinline__ void worker_loop(const SearchParams& p, uint8_t* region, int groups, int g, int gid,
                                            const volatile int* stop) {
    const int tid = threadIdx.x % TW_GROUP;
    const int32_t* sT16 = (const int32_t*)region;
    const int32_t* sT16t = sT16 + 256;
    const int32_t* sT8 = sT16t + 256;
    uint8_t* gsm = region + WK_BASES + (size_t)g * worker_group_bytes();
    volatile int* gtask = (volatile int*)(region + WK_BASES + (size_t)groups * worker_group_bytes()) + g;
    volatile int* gok = gtask + groups;
    const int tb = deblock_tiles_per_band(p.W);
    const QueueShape q = queue_shape(p.BW, p.BH, p.W, p.defer != 0, p.db_level > 0, p.tflag != nullptr, p.compact != 0);
    const int nmb = p.BW * p.BH;
    const int bar = 1 + gid;
    // Task indices a group takes only grow, so the step cursor (k, first task of step k) only
    // moves forward.  Thread 0 takes the next index while the group works on the current one
    // (stoppable groups do not); a group holding index n + 1 still finishes n first, so the
    // smallest unfinished task is always being worked on and the queue drains.
    int next = 0;
    if (tid == 0 && stop == nullptr) next = (int)atomicAdd(p.wq, 1u);
    int k = 0, base = 0;
    // a group that takes an index past the end leaves without walking the steps (row CTAs
    // joining late find the queue empty)
    const int total = queue_total(q);
    unsigned* scan_done = p.wq + 1 + 2 * p.BH;
    for (;;) {
        if (tid == 0) {
            if (stop == nullptr) {
                *gtask = next;
                next = (int)atomicAdd(p.wq, 1u);
            } else {
                *gtask = *stop ? -1 : (int)atomicAdd(p.wq, 1u);
            }
        }
        group_sync(bar, TW_GROUP);  // (the previous task ended with a group barrier too)
        const int task = *gtask;
        if (task < 0 || task >= total) return;  // stopped, or the queue is empty (group-uniform)
        int R = 0, D = 0, T = 0;
        for (; k < q.steps + q.csteps; k++) {
            queue_step(q, k, R, D, T);
            if (task < base + R + D + T) break;
            base += R + D + T;
        }
        if (k >= q.steps + q.csteps) return;  // the queue is empty
        int kind, row, idx;
        queue_task(q, k, task - base, R, D, kind, row, idx);
        if (kind == 0) {  // residual of MBs (row, 2 idx) and (row, 2 idx + 1)
            const int half = tid >> 6, x = 2 * idx + half;
            if (tid == 0) RIV_GSTAMP(row * p.BW + 2 * idx, 18);
            if (x < p.BW)
                residual_mb(p.dres, nmb, row * p.BW + x, tid & 63, 5 + 2 * gid + half,
                            *(ResSmem*)(gsm + half * RES_HALF_BYTES), sT16, sT16t, sT8);
            group_sync(bar, TW_GROUP);
            if (tid == 0) {
                __threadfence();
                atomicAdd(p.wq + 1 + row, (unsigned)min(2, p.BW - 2 * idx));
                RIV_GSTAMP(row * p.BW + 2 * idx, 19);
            }
        } else if (kind == 1) {  // deblock tile idx of band `row`
            if (tid == 0) {
                RIV_GSTAMP(row * p.BW + idx, 20);
                bool ok = true;
                for (int r = max(row - 1, 0); r <= min(row + 1, p.BH - 1) && ok; r++)
                    ok = wait_at_least(p.wq + 1 + r, (unsigned)p.BW, p.spin_limit);
                *gok = ok ? 1 : 0;
                if (!ok) atomicOr(p.status, ST_WAIT_TIMEOUT);
            }
            group_sync(bar, TW_GROUP);
            if (!*gok) return;
            if (tid == 0) RIV_GSTAMP(row * p.BW + idx, 21);
            const int tpy = (p.W + DB_TW - 1) / DB_TW, tpc = (p.W / 2 + DB_TW / 2 - 1) / (DB_TW / 2);
            const int plane = idx < tpy ? 0 : 1 + (idx - tpy) / tpc;
            const int tile = idx < tpy ? row * tpy + idx : row * tpc + (idx - tpy) % tpc;
            deblock_tile(p.db_src, p.db_dst, p.W, p.H, p.BW, p.db_E, p.db_I, p.db_H, p.db_mask, plane, tile, gsm, tid,
                         TW_GROUP, bar);
            group_sync(bar, TW_GROUP);
            if (tid == 0) {
                __threadfence();
                atomicAdd(p.wq + 1 + p.BH + row, 1u);
                RIV_GSTAMP(row * p.BW + idx, 22);
            }
        } else if (kind == 3) {  // scan of the previous frame's coded MBs (all residual rows done)
            if (tid == 0) {
                bool ok = true;
                for (int r = 0; r < p.BH && ok; r++) ok = wait_at_least(p.wq + 1 + r, (unsigned)p.BW, p.spin_limit);
                *gok = ok ? 1 : 0;
                if (!ok) atomicOr(p.status, ST_WAIT_TIMEOUT);
            }
            group_sync(bar, TW_GROUP);
            if (!*gok) return;
            int* ws = (int*)gsm;
            scan_mbs<TW_GROUP, WK_SCAN_IPT>(p.dres.opt_skip, p.dres.eobs, nmb, 0, p.c_index, p.c_offset, p.c_hdr, tid,
                                            bar, ws, ws + TW_GROUP / 32);
            group_sync(bar, TW_GROUP);
            if (tid == 0) {
                __threadfence();
                st_release_u32(scan_done, 1u);
            }
        } else if (kind == 4) {  // pack MB row `row` of the previous frame
            if (tid == 0) {
                const bool ok = wait_at_least(scan_done, 1u, p.spin_limit);
                *gok = ok ? 1 : 0;
                if (!ok) atomicOr(p.status, ST_WAIT_TIMEOUT);
            }
            group_sync(bar, TW_GROUP);
            if (!*gok) return;
            for (int x = tid >> 5; x < p.BW; x += TW_GROUP / 32)
                pack_mb(row * p.BW + x, tid & 31, p.dres.opt_skip, p.dres.mb, p.dres.coeffs, p.dres.eobs, p.c_index,
                        p.c_offset, 0, p.c_side, p.c_packed, p.c_peobs);
        } else {  // SAD-table row of MB (row, idx)
            if (tid == 0) {
                RIV_GSTAMP(row * p.BW + idx, 23);
                const bool ok = wait_ref_rows(p, row, tb);
                *gok = ok ? 1 : 0;
                if (!ok) atomicOr(p.status, ST_WAIT_TIMEOUT);
            }
            group_sync(bar, TW_GROUP);
            if (!*gok) return;
            const int mb = row * p.BW + idx;
            if (tid == 0) RIV_GSTAMP(mb, 24);
            sad_table_mb(p.ref_y, p.cur_y, p.W, p.H, p.BW, p.sr, const_cast<uint16_t*>(p.tab), p.tstride, mb, gsm, tid,
                         TW_GROUP, bar);
            group_sync(bar, TW_GROUP);
            if (tid == 0) {
                __threadfence();
                st_release_u32(p.tflag + mb, p.tag);
                RIV_GSTAMP(mb, 25);
            }
        }
        group_sync(bar, TW_GROUP);
    }
}

// A whole worker CTA (or a row CTA whose rows are done): bases at sm, blockDim / 128 groups.
__device__ __forceinline__ void frame_worker(const SearchParams& p, uint8_t* sm) {
    load_worker_bases(p, sm, threadIdx.x, blockDim.x);
    __syncthreads();
    const int groups = blockDim.x / TW_GROUP, g = threadIdx.x / TW_GROUP;
    worker_loop(p, sm, groups, g, g, nullptr);
}

// ---- mbarrier and bulk-copy helpers (sm_90+ PTX; no multicast)
__device__ __forceinline__ uint32_t sa32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sa32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_inval(unsigned long long* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(sa32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sa32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long* bar, unsigned tx) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sa32(bar)), "r"(tx) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(sa32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait of the whole warp for a completed phase; false when the wait gave up.
__device__ __forceinline__ bool mbar_wait_warp(unsigned long long* bar, unsigned parity, long long limit) {
    long long spins = 0;
    while (!__all_sync(0xffffffffu, mbar_test(bar, parity))) {
        if (++spins > limit) return false;
    }
    return true;
}
// Global -> shared bulk copy completing on an mbarrier (16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(sa32(dst)),
                 "l"(src), "r"(bytes), "r"(sa32(bar))
                 : "memory");
}

// Expiry of the bounded waits, on flags nothing sets (test hook).  which: 0 a wavefront record
// (rec_wait), 1 a worker-queue counter (wait_at_least), 2 a search -> mode hand-off slot
// (hand_get), 3 an mbarrier phase that never completes (mbar_wait_warp).  Each waiting warp
// gives up after `limit` polls and reports ST_WAIT_TIMEOUT in *status, as the search launch
// does; the kernel then returns normally.
__global__ void k_wait_expiry(int which, const unsigned long long* rec, const unsigned* counter, long long limit,
                              unsigned* status) {
    __shared__ unsigned long long bar;
    __shared__ unsigned long long hand[HAND_RING];
    const int lane = threadIdx.x & 31;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    for (int i = threadIdx.x; i < HAND_RING; i += blockDim.x) hand[i] = 0;
    __syncthreads();
    bool ok = true;
    if (which == 0) {
        unsigned long long v = 0;
        if (lane == 0) ok = rec_wait(rec + blockIdx.x, 0x5a5aull << 48, v, limit);
    } else if (which == 1) {
        if (lane == 0) ok = wait_at_least(counter + blockIdx.x, 1u, limit);
    } else if (which == 2) {
        unsigned long long w = 0;
        if (lane == 0) ok = hand_get(hand, 0, w, limit);
    } else {
        ok = mbar_wait_warp(&bar, 0u, limit);
    }
    if (lane == 0 && !ok) atomicOr(status, ST_WAIT_TIMEOUT);
    __syncthreads();
    if (threadIdx.x == 0) mbar_inval(&bar);
}
int launch_wait_expiry(int which, const unsigned long long* rec, const unsigned* counter, long long limit,
                       unsigned* status, void* stream) {
    k_wait_expiry<<<4, 64, 0, (cudaStream_t)stream>>>(which, rec, counter, limit, status);
    return (int)cudaGetLastError();
}

// Staging ring of the band+table search (LD_RING MBs ahead): per slot the MB's SAD-table row
// (2*tstride bytes), its 16x16 current block and the previous frame's coded MV (4 bytes).
constexpr int LD_RING = 4;
__host__ __device__ inline int ld_slot_bytes(int tstride) { return 2 * tstride + 256 + 16; }

// The third warp of each row CTA (band + table instantiations): fills the MB-row reference
// band once per row (one bulk copy per band row plus the replicated edge margins) and, up to
// LD_RING MBs ahead of the search warp, each MB's table row, current block and temporal MV,
// so that no copy is issued on the search chain.  ctl[0] = MBs the search warp has released,
// ctl[1] = rows it has finished, ctl[2] = abort.
// row_live (optional): set once the first row's reference bands are ready, which stops the
// CTA's helper worker groups from taking further tasks.
__device__ __forceinline__ void loader_warp(const SearchParams& p, unsigned long long* fullb, unsigned long long* bandb,
                                            volatile int* ctl, uint8_t* slots, uint8_t* band, volatile int* row_live) {
    const int lane = threadIdx.x & 31;
    const int sr = p.sr, WS = 18 + 2 * sr, MARGIN = (sr + 1 + 15) & ~15, BWB = p.W + 2 * MARGIN;
    const int SLOT = ld_slot_bytes(p.tstride);
    const unsigned tab_bytes = 2u * (unsigned)p.tstride;
    int n = 0, rows = 0;
    bool abort = false;
    auto wait_ctl = [&](int which, int target) {  // lane 0 polls; the answer is warp-uniform
        int ok = 1;
        if (lane == 0) {
            long long spins = 0;
            while (ctl[which] < target) {
                if (ctl[2] != 0 || ++spins > p.spin_limit) { ok = 0; break; }
                __nanosleep(64);
            }
        }
        return __shfl_sync(0xffffffffu, ok, 0) != 0;
    };
    for (int r = row_cta(p); r < p.BH && !abort; r += p.nrow_ctas) {
        const int wy0 = r * 16 - sr - 1;
        if (rows > 0 && !(wait_ctl(1, rows) && (p.lnv == nullptr || wait_ctl(3, rows)))) { abort = true; break; }
        if (p.defer) {  // the previous frame's bands r-1 .. r+1 must be deblocked (written by workers)
            int ok = 1;
            if (lane == 0) {
                RIV_GSTAMP(r * p.BW, 26);
                ok = wait_ref_rows(p, r, deblock_tiles_per_band(p.W)) ? 1 : 0;
                RIV_GSTAMP(r * p.BW, 27);
            }
            __syncwarp();  // orders every lane's copies after lane 0's acquire
            asm volatile("fence.proxy.async.global;" ::: "memory");  // generic writes -> bulk-copy reads
            if (!__shfl_sync(0xffffffffu, ok, 0)) { abort = true; break; }
        }
        if (row_live != nullptr && lane == 0) *row_live = 1;
        // ---- the band: rows wy0 .. wy0+WS-1 (edge-clamped), columns -MARGIN .. W+MARGIN-1
        for (int i = lane; i < WS; i += 32) {
            const int gy = min(max(wy0 + i, 0), p.H - 1);
            const uint8_t* src = p.ref_y + (size_t)gy * p.W;
            uint8_t* dst = band + (size_t)i * BWB;
            bulk_g2s(dst + MARGIN, src, (unsigned)p.W, bandb);
            const uint4 l = make_uint4(src[0] * 0x01010101u, 0, 0, 0), rr = make_uint4(src[p.W - 1] * 0x01010101u, 0, 0, 0);
            const uint4 lv = make_uint4(l.x, l.x, l.x, l.x), rv = make_uint4(rr.x, rr.x, rr.x, rr.x);
            for (int c = 0; c < MARGIN; c += 16) {
                *(uint4*)(dst + c) = lv;
                *(uint4*)(dst + MARGIN + p.W + c) = rv;
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive_tx(bandb, (unsigned)(WS * p.W));
        else mbar_arrive(bandb);
        // ---- per-MB staging
        for (int bx = 0; bx < p.BW; bx++) {
            const int idx = r * p.BW + bx;
            const int s = n & (LD_RING - 1);
            if (n >= LD_RING && !wait_ctl(0, n - LD_RING + 1)) { abort = true; break; }
            uint8_t* slot = slots + (size_t)s * SLOT;
            if (p.tflag != nullptr) {  // fused launch: wait until a table worker published this MB's row
                int ok = 1;
                if (lane == 0) {
                    long long spins = 0;
                    while (ld_acquire_u32(p.tflag + idx) != p.tag) {
                        if (ctl[2] != 0 || ++spins > p.spin_limit) { ok = 0; break; }
                        __nanosleep(32);
                    }
                    asm volatile("fence.proxy.async.global;" ::: "memory");  // generic writes -> bulk-copy reads
                }
                if (!__shfl_sync(0xffffffffu, ok, 0)) { abort = true; break; }
            }
            if (lane < 16)
                bulk_g2s(slot + tab_bytes + lane * 16, p.cur_y + (size_t)(r * 16 + lane) * p.W + bx * 16, 16u, fullb + s);
            if (lane == 0) {
                bulk_g2s(slot, p.tab + (size_t)idx * p.tstride, tab_bytes, fullb + s);
                const int tm = p.prev_coded ? *(const int*)(p.prev_coded + 4 * (size_t)idx) : 0;
                *(int*)(slot + tab_bytes + 256) = tm;
                mbar_arrive_tx(fullb + s, tab_bytes + 256u);
            }
            __syncwarp();
            n++;
        }
        rows++;
    }
    // never leave with copies in flight: the last use of every slot and the last band fill
    if (lane == 0) {
        for (int k = max(0, n - LD_RING); k < n; k++) {
            long long spins = 0;
            while (!mbar_test(fullb + (k & (LD_RING - 1)), (unsigned)((k / LD_RING) & 1)) && ++spins <= p.spin_limit) {}
        }
        if (rows > 0) {
            long long spins = 0;
            while (!mbar_test(bandb, (unsigned)((rows - 1) & 1)) && ++spins <= p.spin_limit) {}
        }
        if (abort && ctl[2] == 0) atomicOr(p.status, ST_WAIT_TIMEOUT);
    }
}

// The fourth warp of each row CTA (band + table instantiations, P-frames): for every MB the
// search warp hands over, in raster order, the luma motion-compensated prediction
// (build_predicted, com/fast_motion.rs:103-352) from the row's reference band, where the
// replicated edges give the same samples as the reference's clamped coordinates, and the
// predicted-luma sums (sum, sum of squares) for the MB's variance (compute_aq_quant_steps,
// res/residual.rs:116-153).  Chroma prediction is left to the residual kernel.  After each row
// it sets ctl[3] = rows it has finished (the loader refills the band only after both the search
// warp and this warp are done with it), computes the row's ln variances into lnv and publishes
// row_done[r] = tag.
__device__ __forceinline__ void aq_warp(const SearchParams& p, const unsigned long long* hand, volatile int* hand_done,
                                        volatile int* ctl, const uint8_t* band, unsigned long long* bandb) {
    const int lane = threadIdx.x & 31;
    const int sr = p.sr, MARGIN = (sr + 1 + 15) & ~15, BWB = p.W + 2 * MARGIN;
    const int W = p.W;
    uint8_t* PY = p.pred;
    const int yy = lane >> 1, xoff = (lane & 1) * 8;  // luma: row, 8-pixel half
    int n = 0, rows = 0;
    for (int r = row_cta(p); r < p.BH; r += p.nrow_ctas) {
        const int y0 = r * 16, wy0 = y0 - sr - 1;
        // observe the band fill of this row (the loader refills only after this warp is done)
        if (!mbar_wait_warp(bandb, (unsigned)(rows & 1), p.spin_limit)) {
            if (lane == 0) atomicOr(p.status, ST_WAIT_TIMEOUT);
            return;
        }
        for (int bx = 0; bx < p.BW; bx++) {
            const int idx = r * p.BW + bx, x0 = bx * 16;
            unsigned long long hw = 0;
            int st = 0;
            if (lane == 0) {
                if (!hand_get(hand, n, hw, p.spin_limit)) st = 1;
                else if (hw & HAND_FAIL) st = 2;
                else hand_done[1] = n + 1;
            }
            st = __shfl_sync(0xffffffffu, st, 0);
            if (st != 0) {
                if (lane == 0 && st == 1) atomicOr(p.status, ST_WAIT_TIMEOUT);
                return;
            }
            n++;
            hw = __shfl_sync(0xffffffffu, hw, 0);
            const int mdx = 2 * (int)(int8_t)hw + (int)(int8_t)(hw >> 16);
            const int mdy = 2 * (int)(int8_t)(hw >> 8) + (int)(int8_t)(hw >> 24);
            const int xo = mdx & 1, yo = mdy & 1;
            // luma: 8 samples of row yy from two 12-byte windows (this row and the next) of the
            // band, with packed rounded averages; the sums come from dp4a
            unsigned s = 0, s2 = 0;
            {
                const int byp = (2 * (y0 + yy) + mdy) >> 1;
                const int c0 = x0 + xoff + (mdx >> 1);  // first integer column (floor)
                const uint8_t* rp = band + (size_t)(byp - wy0) * BWB + MARGIN + c0;
                uint32_t A[2][3];  // bytes c0 .. c0+11 of rows byp, byp+1
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(rp + j * BWB);
                    const uint32_t al = sa & ~3u, sh = (sa & 3u) * 8;
                    const uint32_t q0 = lds_aligned(al), q1 = lds_aligned(al + 4), q2 = lds_aligned(al + 8),
                                   q3 = lds_aligned(al + 12);
                    A[j][0] = __funnelshift_r(q0, q1, sh);
                    A[j][1] = __funnelshift_r(q1, q2, sh);
                    A[j][2] = __funnelshift_r(q2, q3, sh);
                }
                uint32_t P[2];
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const uint32_t a = A[0][h], b = __funnelshift_r(A[0][h], A[0][h + 1], 8);
                    const uint32_t d = A[1][h], e = __funnelshift_r(A[1][h], A[1][h + 1], 8);
                    if (!xo && !yo) P[h] = a;
                    else if (xo && !yo) P[h] = (a | b) - (((a ^ b) >> 1) & 0x7F7F7F7Fu);  // (a + b + 1) >> 1
                    else if (!xo && yo) P[h] = (a | d) - (((a ^ d) >> 1) & 0x7F7F7F7Fu);
                    else {  // (a + b + d + e + 2) >> 2 in 16-bit lanes (sums <= 1022)
                        const uint32_t m = 0x00FF00FFu;
                        const uint32_t lo = ((a & m) + (b & m) + (d & m) + (e & m) + 0x00020002u) >> 2;
                        const uint32_t hi = (((a >> 8) & m) + ((b >> 8) & m) + ((d >> 8) & m) + ((e >> 8) & m) + 0x00020002u) >> 2;
                        P[h] = (lo & m) | ((hi & m) << 8);
                    }
                    s = __dp4a(P[h], 0x01010101u, s);
                    s2 = __dp4a(P[h], P[h], s2);
                }
                *(uint2*)(PY + (size_t)(y0 + yy) * W + x0 + xoff) = make_uint2(P[0], P[1]);
            }
            s = __reduce_add_sync(0xffffffffu, s);
            s2 = __reduce_add_sync(0xffffffffu, s2);
            if (lane == 0) p.varsum[idx] = make_uint2(s, s2);
            if (lane == 0) RIV_GSTAMP(idx, 31);
        }
        __syncwarp();
        if (lane == 0) ctl[3] = rows + 1;  // the band is free for the loader
        // the row's ln variances (res/residual.rs:134-153) from the sums lane 0 wrote above
        // (visible to the warp after __syncwarp), then row_done[r] for the fold
        for (int b0 = 0; b0 < p.BW; b0 += 4 * 32) {
            float v4[4], l4[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int i = b0 + j * 32 + lane;
                float var = 4.0f;
                if (i < p.BW) {
                    const uint2 vs = p.varsum[(size_t)r * p.BW + i];
                    const unsigned long long N = 256ull * vs.y - (unsigned long long)vs.x * vs.x;
                    var = __fdiv_rn(__ull2float_rn(N), 65536.0f);
                    var = var < 4.0f ? 4.0f : var;
                }
                v4[j] = var;
            }
            glibc_logf_batch<4>(v4, l4, p.logfix, p.nlog);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int i = b0 + j * 32 + lane;
                if (i < p.BW) p.lnv[(size_t)r * p.BW + i] = l4[j];
            }
        }
        __threadfence();
        __syncwarp();
        if (lane == 0) st_release_u32(p.row_done + r, p.tag);
        rows++;
    }
}

// The Iterator::sum of the per-MB ln variances, strictly left to right in raster order, while
// the rows are still being searched: one warp waits for each row's row_done flag (set by the
// row's AQ warp once the row's glibc-exact ln variances are written), stages the row's values
// in shared memory and its lane 0 folds them.  Then avg = sum / n (res/residual.rs:116-167).
__device__ __forceinline__ void aq_fold(const SearchParams& p, volatile int* ctl, float* stage) {
    const int lane = threadIdx.x & 31;
    float part = 0.0f;
    for (int r = 0; r < p.BH; r++) {
        long long spins = 0;
        bool ok = true;
        while (!__all_sync(0xffffffffu, ld_acquire_u32(p.row_done + r) == p.tag)) {
            if (ctl[2] != 0 || ++spins > p.spin_limit) { ok = false; break; }
            __nanosleep(64);
        }
        if (!ok) {
            if (lane == 0) atomicOr(p.status, ST_WAIT_TIMEOUT);
            return;
        }
        for (int c0 = 0; c0 < p.BW; c0 += 256) {
            const int m = min(256, p.BW - c0);
            for (int i = lane; i < m; i += 32) stage[i] = p.lnv[(size_t)r * p.BW + c0 + i];
            __syncwarp();
            if (lane == 0) RIV_GSTAMP((size_t)r * p.BW + 1, 19);
            if (lane == 0)
                for (int i = 0; i < m; i++) part = __fadd_rn(part, stage[i]);
            if (lane == 0) RIV_GSTAMP((size_t)r * p.BW + 1, 18);
            __syncwarp();
        }
    }
    if (lane == 0) p.lnv[(size_t)p.BW * p.BH] = __fdiv_rn(part, (float)(p.BW * p.BH));
}

template <bool BAND, bool TABLE, bool SMALL>
__device__ __forceinline__ void search_body(const SearchParams& p) {
    // FAST (band + table): three warps -- search chain, mode decision, loader.  Otherwise the
    // search warp stages its own data with cp.async and the third warp is not launched.
    constexpr bool FAST = BAND && TABLE;
    extern __shared__ __align__(16) uint8_t smem[];
    if (FAST && p.tflag != nullptr && row_cta(p) >= p.nrow_ctas) {
        frame_worker(p, smem);
        return;
    }
    double* bits = (double*)smem;                 // 256 doubles
    int* nc32s = (int*)(smem + 256 * sizeof(double));  // 64 x 64 NEW costs (small mode)
    unsigned long long* hand = (unsigned long long*)(smem + 256 * sizeof(double) + 64 * 64 * 4);  // HAND_RING
    volatile int* hand_done = (volatile int*)(hand + HAND_RING);  // MBs the mode warp has taken
    uint8_t* after_hand = (uint8_t*)(hand + HAND_RING) + 16;
    // FAST layout: LD_RING full barriers, the band barrier, loader control words, the slots
    unsigned long long* fullb = (unsigned long long*)after_hand;
    unsigned long long* bandb = fullb + LD_RING;
    volatile int* ld_ctl = (volatile int*)(bandb + 1);
    float* fold_stage = (float*)(after_hand + 64);  // 256 floats (CTA 0's ln-variance fold)
    uint8_t* slots = after_hand + 64 + 1024;
    // other layouts: double-buffered current block and table row
    uint8_t* curbuf = after_hand;  // 2 x 256 bytes
    uint16_t* tabbuf = (uint16_t*)(curbuf + 512);   // TABLE: 2 x tstride entries
    uint8_t* refmem = FAST ? slots + LD_RING * ld_slot_bytes(p.tstride)
                           : curbuf + 512 + (TABLE ? 4 * p.tstride : 0);  // band or window (+16 bytes slack)
    const int side = 2 * p.sr + 1;
    const int lane = threadIdx.x & 31;
    const int sr = p.sr;
    const int WS = 18 + 2 * sr;
    const int MARGIN = (sr + 1 + 15) & ~15;
    const int BWB = p.W + 2 * MARGIN;
    for (int i = threadIdx.x; i < 256; i += blockDim.x) bits[i] = p.mvbits[i];
    const int* nc32 = nc32s;
    if (SMALL)
        for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x) nc32s[i] = p.newcost32[i];
    for (int i = threadIdx.x; i < HAND_RING; i += blockDim.x) hand[i] = 0ull;
    // Fused launch: threads 128-511 of a row CTA are worker groups 1-3 until the row starts
    // (region after the row layout: a live flag, then a 3-group worker region), and the
    // whole CTA joins the worker queue once its rows are done.
    const bool helpers = FAST && p.tflag != nullptr && p.row_helpers;
    uint8_t* pre = smem + (((size_t)(refmem - smem) + (size_t)WS * BWB + 16 + 15) & ~(size_t)15);
    volatile int* row_live = (volatile int*)pre;
    uint8_t* preg = pre + 16;
    if (helpers) load_worker_bases(p, preg, threadIdx.x, blockDim.x);
    if (threadIdx.x == 0) {
        if (helpers) *row_live = 0;
        hand_done[0] = 0;
        hand_done[1] = FAST && p.lnv != nullptr ? 0 : 0x3fffffff;  // no AQ warp: never waited for
        if (FAST) {
            for (int i = 0; i < LD_RING; i++) mbar_init(fullb + i, 1);
            mbar_init(bandb, 32);
            ld_ctl[0] = ld_ctl[1] = ld_ctl[2] = ld_ctl[3] = 0;
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }
    __syncthreads();
    const unsigned long long tagbits = (unsigned long long)(p.tag & 0xffffu) << 48;
    auto roles = [&]() {
    if (threadIdx.x >= 64) {
        if (FAST && threadIdx.x < 96) {
            loader_warp(p, fullb, bandb, ld_ctl, slots, refmem, helpers ? row_live : nullptr);
            if (p.lnv != nullptr && row_cta(p) == 0) aq_fold(p, ld_ctl, fold_stage);
        } else if (FAST && threadIdx.x < 128 && p.lnv != nullptr) {
            aq_warp(p, hand, hand_done, ld_ctl, refmem, bandb);
        } else if (helpers && threadIdx.x >= TW_GROUP) {
            const int gid = threadIdx.x / TW_GROUP;
            worker_loop(p, preg, 3, gid - 1, gid, row_live);
        }
        return;
    }
    if (threadIdx.x >= 32) {
        mode_warp(p, hand, hand_done, tagbits);
        return;
    }
    int ln = 0;      // MBs taken from the loader (FAST)
    int lrows = 0;   // rows finished (FAST)
    auto abort_loader = [&]() {
        if (FAST && lane == 0) ld_ctl[2] = 1;
    };
    const int yy = lane >> 1;         // this lane's row inside the MB
    const int xoff = (lane & 1) * 8;  // and its 8-pixel half
    bool failed = false;
    int hn = 0;  // MBs handed to the mode warp so far

    for (int r = row_cta(p); r < p.BH; r += p.nrow_ctas) {
        const int y0 = r * 16;
        const int wy0 = y0 - sr - 1;
        __syncwarp();
        // ---- prologue: reference columns of MB 0 and its current block
        int c_done = -1;
        auto c_hi = [&](int bx) { return (16 * bx + 16 + sr + MARGIN) >> 4; };
        if (FAST) {
            if (!mbar_wait_warp(bandb, (unsigned)(lrows & 1), p.spin_limit)) {
                if (lane == 0) {
                    atomicOr(p.status, ST_WAIT_TIMEOUT);
                    hand_put(hand, hand_done, hn, HAND_FAIL, p.spin_limit);
                }
                abort_loader();
                return;
            }
        } else if (BAND) {
            for (int c = 0; c <= c_hi(0); c++) fill_chunk(refmem, BWB, WS, c, MARGIN, wy0, p.ref_y, p.W, p.H, lane);
            c_done = c_hi(0);
        }
        if (!FAST) {
            if (lane < 16) cp_async16(curbuf + lane * 16, p.cur_y + (size_t)(y0 + lane) * p.W);
            if (TABLE)
                for (int i = lane; i < p.tstride / 8; i += 32)
                    cp_async16(tabbuf + i * 8, p.tab + (size_t)(r * p.BW) * p.tstride + i * 8);
            cp_async_commit();
        }

        MvT L_raw{0, 0, 0, 0};
        unsigned long long recT = 0, recTL = 0, pref = 0;
        for (int bx = 0; bx < p.BW; bx++) {
            const int x0 = bx * 16;
            const int idx = r * p.BW + bx;
            RIV_STAMP(0);
            if (lane == 0) RIV_GSTAMP(idx, 16);
            // Refresh the prefetched top-right record now if it was not published yet when it
            // was first read: the load's latency then overlaps the slot wait below instead of
            // sitting on the chain at the wait for the row above.
            if (r > 0 && lane == 0 && (pref & 0xffff000000000000ull) != tagbits)
                pref = ld_rec(p.rec + (r - 1) * p.BW + min(bx + 1, p.BW - 1));
            // ---- FAST: wait for the loader's slot; otherwise prefetch MB bx+1 (columns, current
            // block, table row) and wait for MB bx's data
            const uint8_t* lslot = slots + (size_t)(ln & (LD_RING - 1)) * ld_slot_bytes(p.tstride);
            if (FAST) {
                if (!mbar_wait_warp(fullb + (ln & (LD_RING - 1)), (unsigned)((ln / LD_RING) & 1), p.spin_limit)) {
                    if (lane == 0) {
                        atomicOr(p.status, ST_WAIT_TIMEOUT);
                        hand_put(hand, hand_done, hn, HAND_FAIL, p.spin_limit);
                    }
                    abort_loader();
                    return;
                }
            } else if (bx + 1 < p.BW) {
                if (BAND) {
                    int hi = c_hi(bx + 1);
                    for (int c = c_done + 1; c <= hi; c++)
                        fill_chunk(refmem, BWB, WS, c, MARGIN, wy0, p.ref_y, p.W, p.H, lane);
                    c_done = hi;
                }
                RIV_STAMP(10);
                if (lane < 16)
                    cp_async16(curbuf + ((bx + 1) & 1) * 256 + lane * 16, p.cur_y + (size_t)(y0 + lane) * p.W + x0 + 16);
                if (TABLE)
                    for (int i = lane; i < p.tstride / 8; i += 32)
                        cp_async16(tabbuf + ((bx + 1) & 1) * p.tstride + i * 8,
                                   p.tab + (size_t)(idx + 1) * p.tstride + i * 8);
                RIV_STAMP(11);
            }
            if (!FAST) cp_async_commit();
            RIV_STAMP(7);
            if (lane == 0) RIV_GSTAMP(idx, 17);
            if (!FAST) cp_async_wait1();
            RefView view;
            if (BAND) {
                view.org = refmem + x0 + MARGIN;
                view.stride = BWB;
            } else {
                // per-MB window (large search ranges / very wide frames): rows wy0.., cols x0-sr-1..
                const int wx0 = x0 - sr - 1;
                __syncwarp();
                for (int i0 = 0; i0 < WS * WS; i0 += 32 * 8) {
                    uint8_t v[8];
#pragma unroll
                    for (int u = 0; u < 8; u++) {
                        int i = i0 + u * 32 + lane;
                        int wr = i / WS, wc = i - wr * WS;
                        int gy = min(max(wy0 + wr, 0), p.H - 1), gx = min(max(wx0 + wc, 0), p.W - 1);
                        v[u] = i < WS * WS ? p.ref_y[(size_t)gy * p.W + gx] : 0;
                    }
#pragma unroll
                    for (int u = 0; u < 8; u++) {
                        int i = i0 + u * 32 + lane;
                        if (i < WS * WS) refmem[i] = v[u];
                    }
                }
                view.org = refmem + (sr + 1);
                view.stride = WS;
            }
            view.wy0 = wy0;
            __syncwarp();
            const uint8_t* cb = FAST ? lslot + 2 * p.tstride : curbuf + (bx & 1) * 256;
            const uint32_t c0 = *(const uint32_t*)(cb + yy * 16 + xoff);
            const uint32_t c1 = *(const uint32_t*)(cb + yy * 16 + xoff + 4);

            RIV_STAMP(1);
            // ---- wait for the row above (top-right, or top at the last column).  The record
            // of the next MB's top-right was requested one MB earlier (pref); it is polled
            // again only if it had not been published yet.
            unsigned long long recTR = 0;
            bool has_tr = false;
            if (r > 0) {
                int wi = (r - 1) * p.BW + min(bx + 1, p.BW - 1);
                unsigned long long v = 0;
                if (lane == 0) {
                    long long spins = 0;
                    v = pref;
                    if ((v & 0xffff000000000000ull) != tagbits) v = ld_rec(p.rec + wi);
                    while ((v & 0xffff000000000000ull) != tagbits) {
                        if (++spins > p.spin_limit || failed) { failed = true; break; }
                        __nanosleep(20);
                        v = ld_rec(p.rec + wi);
                    }
                    if (bx == 0 && !failed) {  // the top record, checked like every other
                        recT = ld_rec(p.rec + (r - 1) * p.BW);
                        while ((recT & 0xffff000000000000ull) != tagbits) {
                            if (++spins > p.spin_limit) { failed = true; break; }
                            __nanosleep(20);
                            recT = ld_rec(p.rec + (r - 1) * p.BW);
                        }
                    }
                    pref = bx + 1 < p.BW ? ld_rec(p.rec + (r - 1) * p.BW + min(bx + 2, p.BW - 1)) : 0ull;
                }
                failed = __shfl_sync(0xffffffffu, (int)failed, 0) != 0;
                v = __shfl_sync(0xffffffffu, v, 0);
                recT = __shfl_sync(0xffffffffu, recT, 0);
                if (bx + 1 < p.BW) { recTR = v; has_tr = true; }
            }
            if (failed) {
                if (lane == 0) {
                    atomicOr(p.status, ST_WAIT_TIMEOUT);
                    hand_put(hand, hand_done, hn, HAND_FAIL, p.spin_limit);
                }
                abort_loader();
                if (!FAST) cp_async_wait0();
                return;
            }
            RIV_STAMP(2);
            const bool has_t = r > 0, has_l = bx > 0, has_tl = r > 0 && bx > 0;
            auto rec_raw = [](unsigned long long v, int& dx, int& dy) {
                dx = (int)(int8_t)(v >> 40); dy = (int)(int8_t)(v >> 32);
            };
            int Tx = 0, Ty = 0, TRx = 0, TRy = 0, TLx = 0, TLy = 0;
            if (has_t) rec_raw(recT, Tx, Ty);
            if (has_tr) rec_raw(recTR, TRx, TRy);
            if (has_tl) rec_raw(recTL, TLx, TLy);
            const bool has_tm = p.prev_coded != nullptr;
            int Tmx = 0, Tmy = 0;
            MvT Tm_cod{0, 0, 0, 0};
            if (has_tm) {
                const char4 pc = FAST ? *(const char4*)(lslot + 2 * p.tstride + 256) : *(const char4*)(p.prev_coded + 4 * idx);
                Tm_cod = MvT{pc.x, pc.y, pc.z, pc.w};
                Tmx = Tm_cod.dx; Tmy = Tm_cod.dy;
            }
            int sdx = 0, sdy = 0;
            if constexpr (TABLE && SMALL) {
                // ---- seeds and nearest/near/median (enc/motion/scalar.rs:56-156) in a flat form:
                // predictor slots 0..4 = left, top, top-right, top-left, temporal; lane 0 holds
                // the (0,0) seed, lane 1+i predictor i when push_candidate keeps it.
                const uint16_t* tb = FAST ? (const uint16_t*)lslot : tabbuf + (bx & 1) * p.tstride;
                const int QX[5] = {L_raw.dx, Tx, TRx, TLx, Tmx}, QY[5] = {L_raw.dy, Ty, TRy, TLy, Tmy};
                const unsigned pvm = (has_l ? 1u : 0u) | (has_t ? 2u : 0u) | (has_tr ? 4u : 0u) | (has_tl ? 8u : 0u) |
                                     (has_tm ? 16u : 0u);
                unsigned long long X5 = 0, Y5 = 0;
                unsigned okm = 0;
#pragma unroll
                for (int i = 0; i < 5; i++) {
                    X5 |= (unsigned long long)(uint8_t)QX[i] << (8 * i);
                    Y5 |= (unsigned long long)(uint8_t)QY[i] << (8 * i);
                    const bool ok = ((pvm >> i) & 1u) && abs(QX[i]) <= sr && abs(QY[i]) <= sr && (QX[i] | QY[i]) != 0;
                    okm |= ok ? (1u << i) : 0u;
                }
                auto qx = [&](int i) { return (int)(int8_t)(X5 >> (8 * i)); };
                auto qy = [&](int i) { return (int)(int8_t)(Y5 >> (8 * i)); };
                int nix = 0, niy = 0, rix = 0, riy = 0;
                if (pvm) {  // nearest = first available; near = first later one that differs
                    const int ni = __ffs(pvm) - 1;
                    nix = qx(ni);
                    niy = qy(ni);
                    unsigned dm = 0;
#pragma unroll
                    for (int i = 0; i < 5; i++) dm |= (QX[i] != nix || QY[i] != niy) ? (1u << i) : 0u;
                    const unsigned rm = pvm & dm & ~((2u << ni) - 1u);
                    if (rm) {
                        const int ri = __ffs(rm) - 1;
                        rix = qx(ri);
                        riy = qy(ri);
                    }
                }
                const int mdx = median3(L_raw.dx, Tx, has_tr ? TRx : TLx), mdy = median3(L_raw.dy, Ty, has_tr ? TRy : TLy);
                int kx = 0, ky = 0;
                bool kv = lane == 0;
                if (lane >= 1 && lane <= 5) {
                    const int ci = lane - 1;
                    kx = qx(ci);
                    ky = qy(ci);
                    unsigned eq = 0;
#pragma unroll
                    for (int j = 0; j < 5; j++) eq |= (QX[j] == kx && QY[j] == ky) ? (1u << j) : 0u;
                    kv = ((okm >> ci) & 1u) && (eq & okm & ((1u << ci) - 1u)) == 0;
                }
                const int c15i = (int)p.c15, c05i = (int)p.c05;
                // estimate_mv_cost (enc/motion/scalar.rs:453-544), every term below 2^27 here
                auto cost = [&](int cx, int cy) -> int {
                    if (p.lambda_zero) return 0;
                    int best = INT_MAX;
                    if ((cx == nix && cy == niy) || (cx == rix && cy == riy) || (cx == mdx && cy == mdy)) best = c15i;
                    if ((cx | cy) == 0) best = min(best, c05i);
                    const int ax = abs(cx - nix), ay = abs(cy - niy), bx2 = abs(cx - rix), by2 = abs(cy - riy);
                    int nc;
                    if (((ax | ay | bx2 | by2) & ~63) == 0) nc = min(nc32[ax * 64 + ay], nc32[bx2 * 64 + by2]);
                    else nc = (int)min(__ldg(p.newcost + ax * 256 + ay), __ldg(p.newcost + bx2 * 256 + by2));
                    return min(best, nc);
                };
                RIV_STAMP(12);
                // seed round: the in-order strict-'<' scan = argmin with the lowest slot winning ties
                const int t0 = kv ? (int)tb[(ky + sr) * side + kx + sr] + cost(kx, ky) : 0;
                const uint32_t k0 = __reduce_min_sync(0xffffffffu, kv ? ((uint32_t)t0 << 3) | (uint32_t)lane : 0xffffffffu);
                RIV_STAMP(13);
                const int zero_sad = (int)tb[sr * side + sr];
                if (!(p.zthr > 0 && zero_sad <= p.zthr)) {  // else stay at (0,0)
                    int scost = (int)(k0 >> 3);
                    const int w0 = (int)(k0 & 7u);
                    sdx = w0 == 0 ? 0 : qx(w0 - 1);
                    sdy = w0 == 0 ? 0 : qy(w0 - 1);
                    RIV_STAMP(9);
                    if (!(p.pthr > 0 && (int)tb[(sdy + sr) * side + sdx + sr] <= p.pthr)) {
                        // hexagon (lanes 0-5, enc/motion/scalar.rs:694-729) and the small diamond
                        // around the same centre (lanes 6-9, :731-756) in one round: the diamond
                        // result is used when the hexagon does not improve.
                        const int ol = lane < 6 ? lane : lane - 6;
                        const int ox = lane < 6 ? (int)(int8_t)(0x01FFFEFF0102ull >> (8 * ol))
                                                : (lane < 10 ? (int)(int8_t)(0x0000FF01u >> (8 * ol)) : 0);
                        const int oy = lane < 6 ? (int)(int8_t)(0xFEFE00020200ull >> (8 * ol))
                                                : (lane < 10 ? (int)(int8_t)(0xFF010000u >> (8 * ol)) : 0);
                        int iter = 0;
                        for (;;) {
                            const int cx = sdx + ox, cy = sdy + oy;
                            const bool v = lane < 10 && abs(cx) <= sr && abs(cy) <= sr;
                            const int t = v ? (int)tb[(cy + sr) * side + cx + sr] + cost(cx, cy) : 0;
                            const uint32_t kh = __reduce_min_sync(
                                0xffffffffu, v && lane < 6 ? ((uint32_t)t << 3) | (uint32_t)lane : 0xffffffffu);
                            const uint32_t kd = __reduce_min_sync(
                                0xffffffffu, v && lane >= 6 ? ((uint32_t)t << 3) | (uint32_t)(lane - 6) : 0xffffffffu);
                            if (kh != 0xffffffffu && (int)(kh >> 3) < scost) {
                                const int w = (int)(kh & 7u);
                                scost = (int)(kh >> 3);
                                sdx += (int)(int8_t)(0x01FFFEFF0102ull >> (8 * w));
                                sdy += (int)(int8_t)(0xFEFE00020200ull >> (8 * w));
                                if (++iter > 4096) {  // cost strictly decreases, so this is never reached
                                    if (lane == 0) atomicOr(p.status, ST_HEX_CAP);
                                    break;
                                }
                                continue;
                            }
                            RIV_STAMP(14);
                            RIV_PUT(8, iter);
                            if (kd != 0xffffffffu && (int)(kd >> 3) < scost) {
                                const int w = (int)(kd & 7u);
                                sdx += (int)(int8_t)(0x0000FF01u >> (8 * w));
                                sdy += (int)(int8_t)(0xFF010000u >> (8 * w));
                            }
                            break;
                        }
                    }
                }
            } else {
                // ---- seeds, nearest/near/median (enc/motion/scalar.rs:56-156).  Predictor slots in
                // the reference's order: left, top, top-right, top-left, temporal.
                const int PX[5] = {L_raw.dx, Tx, TRx, TLx, Tmx}, PY[5] = {L_raw.dy, Ty, TRy, TLy, Tmy};
                const bool PV[5] = {has_l, has_t, has_tr, has_tl, has_tm};
                CostCtx cc;
                cc.nx = cc.ny = cc.rx = cc.ry = 0;
                {
                    int nu = 0;
    #pragma unroll
                    for (int i = 0; i < 5; i++) {
                        bool take = PV[i] && (nu == 0 || (nu == 1 && !(PX[i] == cc.nx && PY[i] == cc.ny)));
                        if (take && nu == 0) { cc.nx = PX[i]; cc.ny = PY[i]; }
                        else if (take && nu == 1) { cc.rx = PX[i]; cc.ry = PY[i]; }
                        nu += take ? 1 : 0;
                    }
                    int lx = has_l ? L_raw.dx : 0, ly = has_l ? L_raw.dy : 0;
                    int tx = has_t ? Tx : 0, ty = has_t ? Ty : 0;
                    int qx = has_tr ? TRx : (has_tl ? TLx : 0), qy = has_tr ? TRy : (has_tl ? TLy : 0);
                    cc.mx = median3(lx, tx, qx);
                    cc.my = median3(ly, ty, qy);
                }
                // seed slots: 0 = (0,0), 1..5 = predictors kept if within range and not already
                // pushed (push_candidate, enc/motion/scalar.rs:46-53)
                bool SV[6];
                SV[0] = true;
    #pragma unroll
                for (int i = 0; i < 5; i++) {
                    bool ok = PV[i] && abs(PX[i]) <= sr && abs(PY[i]) <= sr && !(PX[i] == 0 && PY[i] == 0);
    #pragma unroll
                    for (int j = 0; j < i; j++) ok = ok && !(SV[j + 1] && PX[j] == PX[i] && PY[j] == PY[i]);
                    SV[i + 1] = ok;
                }
                const uint16_t* tb = FAST ? (const uint16_t*)lslot : tabbuf + (bx & 1) * p.tstride;
                if (TABLE) {
                    // ---- table-driven integer search: lane k holds candidate k of a round; the
                    // in-order strict-'<' scan of the reference equals an argmin with the lowest
                    // index winning ties.  One loop for the three round kinds (seeds, hexagon,
                    // diamond) keeps a single MV-cost evaluation site.
                    int kx = 0, ky = 0;
                    bool kv = lane == 0;
    #pragma unroll
                    for (int i = 0; i < 5; i++)
                        if (lane == i + 1) { kx = PX[i]; ky = PY[i]; kv = SV[i + 1]; }
                    const int hxl = (int)(int8_t)(0x01FFFEFF0102ull >> (8 * min(lane, 5)));
                    const int hyl = (int)(int8_t)(0xFEFE00020200ull >> (8 * min(lane, 5)));
                    const int dxl = (int)(int8_t)(0x0000FF01u >> (8 * min(lane, 3)));
                    const int dyl = (int)(int8_t)(0xFF010000u >> (8 * min(lane, 3)));
                    long long scost = 0;
                    int phase = 0, iter = 0;
                    RIV_STAMP(12);
                    for (;;) {
                        int cx, cy;
                        bool v;
                        if (phase == 0) { cx = kx; cy = ky; v = kv && lane < 6; }
                        else if (phase == 1) { cx = sdx + hxl; cy = sdy + hyl; v = lane < 6 && abs(cx) <= sr && abs(cy) <= sr; }
                        else { cx = sdx + dxl; cy = sdy + dyl; v = lane < 4 && abs(cx) <= sr && abs(cy) <= sr; }
                        long long t = v ? (long long)tb[(cy + sr) * side + cx + sr] + mv_cost<SMALL>(cx, cy, cc, p, bits, nc32) : 0;
                        long long bt;
                        const int wk = argmin8<SMALL>(t, v, bt);
                        if (phase == 0) RIV_STAMP(13);
                        if (phase == 2) RIV_STAMP(15);
                        if (phase == 0) {
                            const long long zero_sad = (long long)tb[sr * side + sr];
                            if (p.zthr > 0 && zero_sad <= p.zthr) break;  // stay at (0,0)
                            scost = bt;
                            sdx = __shfl_sync(0xffffffffu, cx, wk);
                            sdy = __shfl_sync(0xffffffffu, cy, wk);
                            if (p.pthr > 0 && (long long)tb[(sdy + sr) * side + sdx + sr] <= p.pthr) break;
                            phase = 1;
                            RIV_STAMP(9);
                        } else if (phase == 1) {  // large hexagon (enc/motion/scalar.rs:694-729)
                            if (wk < 0 || bt >= scost) { phase = 2; RIV_STAMP(14); continue; }
                            scost = bt;
                            sdx = __shfl_sync(0xffffffffu, cx, wk);
                            sdy = __shfl_sync(0xffffffffu, cy, wk);
                            if (++iter > 4096) {  // cost strictly decreases, so this is never reached
                                if (lane == 0) atomicOr(p.status, ST_HEX_CAP);
                                phase = 2;
                            }
                        } else {  // small diamond (enc/motion/scalar.rs:731-756)
                            RIV_PUT(8, iter);
                            if (wk >= 0 && bt < scost) {
                                sdx = __shfl_sync(0xffffffffu, cx, wk);
                                sdy = __shfl_sync(0xffffffffu, cy, wk);
                            }
                            break;
                        }
                    }
                } else {
                    // ---- zero SAD and the seed round; lane k evaluates the MV cost of slot k
                    long long my_cost = 0;
                    {
                        int kx = 0, ky = 0;
                        bool kv = lane == 0;
        #pragma unroll
                        for (int i = 0; i < 5; i++)
                            if (lane == i + 1) { kx = PX[i]; ky = PY[i]; kv = SV[i + 1]; }
                        if (kv) my_cost = mv_cost<SMALL>(kx, ky, cc, p, bits, nc32);
                    }
                    unsigned part[6];
                    part[0] = sad_int_part(view, x0, y0, p.W, p.H, 0, 0, yy, xoff, c0, c1);
        #pragma unroll
                    for (int i = 0; i < 5; i++)
                        part[i + 1] = SV[i + 1] ? sad_int_part(view, x0, y0, p.W, p.H, PX[i], PY[i], yy, xoff, c0, c1) : 0u;
                    long long sads[6];
        #pragma unroll
                    for (int i = 0; i < 6; i++) sads[i] = (long long)warp_sum(part[i]);
                    long long zero_sad = sads[0];
                    long long sc_cost = __shfl_sync(0xffffffffu, my_cost, 0);
                    long long scost = zero_sad + sc_cost;
                    bool skip_int = p.zthr > 0 && zero_sad <= p.zthr;
                    if (!skip_int) {
        #pragma unroll
                        for (int i = 0; i < 5; i++) {
                            long long ci = __shfl_sync(0xffffffffu, my_cost, i + 1);
                            if (!SV[i + 1]) continue;
                            long long t = sads[i + 1] + ci;
                            if (t < scost) { scost = t; sdx = PX[i]; sdy = PY[i]; sc_cost = ci; }
                        }
                        long long cur_sad = scost - sc_cost;
                        if (p.pthr > 0 && cur_sad <= p.pthr) skip_int = true;
                    }
                    if (!skip_int) {
                        // large hexagon (enc/motion/scalar.rs:694-729)
                        const int HX[6] = {2, 1, -1, -2, -1, 1}, HY[6] = {0, 2, 2, 0, -2, -2};
                        // HX/HY of lane k (k < 6) without a lane-indexed array
                        const int hxl = (int)(int8_t)(0x01FFFEFF0102ull >> (8 * min(lane, 5)));
                        const int hyl = (int)(int8_t)(0xFEFE00020200ull >> (8 * min(lane, 5)));
                        int iter = 0;
                        for (;;) {
                            int cx = sdx, cy = sdy;
                            long long lc = 0;
                            if (lane < 6) {
                                int dx = cx + hxl, dy = cy + hyl;
                                if (abs(dx) <= sr && abs(dy) <= sr) lc = mv_cost<SMALL>(dx, dy, cc, p, bits, nc32);
                            }
                            unsigned hp[6];
        #pragma unroll
                            for (int k = 0; k < 6; k++) {
                                int dx = cx + HX[k], dy = cy + HY[k];
                                hp[k] = (abs(dx) <= sr && abs(dy) <= sr)
                                            ? sad_int_part(view, x0, y0, p.W, p.H, dx, dy, yy, xoff, c0, c1) : 0u;
                            }
                            bool improved = false;
        #pragma unroll
                            for (int k = 0; k < 6; k++) {
                                long long s = (long long)warp_sum(hp[k]);
                                long long ck = __shfl_sync(0xffffffffu, lc, k);
                                int dx = cx + HX[k], dy = cy + HY[k];
                                if (abs(dx) > sr || abs(dy) > sr) continue;
                                long long t = s + ck;
                                if (t < scost) { scost = t; sdx = dx; sdy = dy; improved = true; }
                            }
                            if (!improved) break;
                            if (++iter > 4096) {  // cost strictly decreases, so this is never reached
                                if (lane == 0) atomicOr(p.status, ST_HEX_CAP);
                                break;
                            }
                        }
                        // small diamond (enc/motion/scalar.rs:731-756)
                        const int DX[4] = {1, -1, 0, 0}, DY[4] = {0, 0, 1, -1};
                        const int dxl = (int)(int8_t)(0x0000FF01u >> (8 * min(lane, 3)));
                        const int dyl = (int)(int8_t)(0xFF010000u >> (8 * min(lane, 3)));
                        int cx = sdx, cy = sdy;
                        long long lc = 0;
                        if (lane < 4) {
                            int dx = cx + dxl, dy = cy + dyl;
                            if (abs(dx) <= sr && abs(dy) <= sr) lc = mv_cost<SMALL>(dx, dy, cc, p, bits, nc32);
                        }
                        unsigned dp[4];
        #pragma unroll
                        for (int k = 0; k < 4; k++) {
                            int dx = cx + DX[k], dy = cy + DY[k];
                            dp[k] = (abs(dx) <= sr && abs(dy) <= sr)
                                        ? sad_int_part(view, x0, y0, p.W, p.H, dx, dy, yy, xoff, c0, c1) : 0u;
                        }
        #pragma unroll
                        for (int k = 0; k < 4; k++) {
                            long long s = (long long)warp_sum(dp[k]);
                            long long ck = __shfl_sync(0xffffffffu, lc, k);
                            int dx = cx + DX[k], dy = cy + DY[k];
                            if (abs(dx) > sr || abs(dy) > sr) continue;
                            long long t = s + ck;
                            if (t < scost) { scost = t; sdx = dx; sdy = dy; }
                        }
                    }
                }
            }
            if (FAST) {  // the table row, current block and temporal MV are in registers now
                __syncwarp();
                if (lane == 0) ld_ctl[0] = ln + 1;
                ln++;
            }
            RIV_STAMP(3);
            // ---- half-pel refinement (enc/motion/scalar.rs:759-839): nine floor-averaged
            // candidates around (2*sdx, 2*sdy), from a 3x3 integer neighbourhood per pixel,
            // on packed bytes.  Candidate q = (sy+1)*3 + (sx+1).
            unsigned hpart[9];
            {
                const int Yr = y0 + yy + sdy - wy0;  // band/window row of the centre samples
                const int Xr = xoff + sdx - 1;       // column (relative to x0) of the left neighbour
                uint32_t A[3][2], B[3][2], Cq[3][2];
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    const uint8_t* base = view.org + (Yr - 1 + j) * view.stride + Xr;
                    uint32_t sa = (uint32_t)__cvta_generic_to_shared(base);
                    uint32_t al = sa & ~3u, o = sa & 3u;
                    uint32_t w0 = lds_aligned(al), w1 = lds_aligned(al + 4), w2 = lds_aligned(al + 8),
                             w3 = lds_aligned(al + 12);
                    // byte offsets o, o+1, o+2 into w0..w3
                    uint32_t sh = o * 8;
                    A[j][0] = __funnelshift_r(w0, w1, sh);
                    A[j][1] = __funnelshift_r(w1, w2, sh);
                    uint32_t ob = o + 1, shb = (ob & 3) * 8;
                    B[j][0] = ob < 4 ? __funnelshift_r(w0, w1, shb) : __funnelshift_r(w1, w2, shb);
                    B[j][1] = ob < 4 ? __funnelshift_r(w1, w2, shb) : __funnelshift_r(w2, w3, shb);
                    uint32_t oc = o + 2, shc = (oc & 3) * 8;
                    Cq[j][0] = oc < 4 ? __funnelshift_r(w0, w1, shc) : __funnelshift_r(w1, w2, shc);
                    Cq[j][1] = oc < 4 ? __funnelshift_r(w1, w2, shc) : __funnelshift_r(w2, w3, shc);
                }
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const uint32_t cw = h ? c1 : c0;
                    uint32_t v[9];
                    v[0] = favg4(A[0][h], B[0][h], A[1][h], B[1][h]);
                    v[1] = favg(B[0][h], B[1][h]);
                    v[2] = favg4(B[0][h], Cq[0][h], B[1][h], Cq[1][h]);
                    v[3] = favg(A[1][h], B[1][h]);
                    v[4] = B[1][h];
                    v[5] = favg(B[1][h], Cq[1][h]);
                    v[6] = favg4(A[1][h], B[1][h], A[2][h], B[2][h]);
                    v[7] = favg(B[1][h], B[2][h]);
                    v[8] = favg4(B[1][h], Cq[1][h], B[2][h], Cq[2][h]);
#pragma unroll
                    for (int q = 0; q < 9; q++) hpart[q] = (h ? hpart[q] : 0u) + __vsadu4(cw, v[q]);
                }
            }
            long long best_sad;
            int bsx = 0, bsy = 0;
            if constexpr (SMALL) {
                // Per-lane partials are at most 8 * 255, so the warp totals (<= 65280) of two
                // candidates share one 32-bit reduction.  Then lane q < 9 holds candidate q and one
                // argmin replaces the in-order scan: the centre is the incumbent (order 0), the
                // neighbours follow in scan order (0,1,2,3,5,6,7,8), ties keep the earlier one.
                const unsigned w01 = __reduce_add_sync(0xffffffffu, hpart[0] | (hpart[1] << 16));
                const unsigned w23 = __reduce_add_sync(0xffffffffu, hpart[2] | (hpart[3] << 16));
                const unsigned w45 = __reduce_add_sync(0xffffffffu, hpart[4] | (hpart[5] << 16));
                const unsigned w67 = __reduce_add_sync(0xffffffffu, hpart[6] | (hpart[7] << 16));
                const unsigned w8 = __reduce_add_sync(0xffffffffu, hpart[8]);
                const int q = lane < 9 ? lane : 4;
                const unsigned wq = q < 2 ? w01 : q < 4 ? w23 : q < 6 ? w45 : q < 8 ? w67 : w8;
                const int hsq = (int)((wq >> ((q & 1) * 16)) & 0xffffu);
                const int sxq = q % 3 - 1, syq = q / 3 - 1;
                const bool vq = lane < 9 && !((sdx == -128 && sxq == -1) || (sdy == -128 && syq == -1));
                const int c15i = (int)p.c15;  // every neighbour is fractional in at least one axis
                const int ord = q == 4 ? 0 : (q < 4 ? q + 1 : q);
                const int tot = hsq + (q == 4 ? 0 : c15i);
                const uint32_t key = __reduce_min_sync(0xffffffffu, vq ? ((uint32_t)tot << 4) | (uint32_t)ord : 0xffffffffu);
                const int ow = (int)(key & 15u);
                const int qw = ow == 0 ? 4 : (ow <= 4 ? ow - 1 : ow);
                bsx = qw % 3 - 1;
                bsy = qw / 3 - 1;
                best_sad = (long long)((int)(key >> 4) - (qw == 4 ? 0 : c15i));
            } else {
                long long hs[9];
#pragma unroll
                for (int q = 0; q < 9; q++) hs[q] = (long long)warp_sum(hpart[q]);
                long long best_total = hs[4];
                best_sad = hs[4];
#pragma unroll
                for (int q = 0; q < 9; q++) {
                    if (q == 4) continue;
                    int sx = q % 3 - 1, sy = q / 3 - 1;
                    if ((sdx == -128 && sx == -1) || (sdy == -128 && sy == -1)) continue;
                    long long pen = p.c15;  // every neighbour is fractional in at least one axis
                    if (best_total - pen < 0) continue;
                    if (hs[q] + pen < best_total) { best_total = hs[q] + pen; best_sad = hs[q]; bsx = sx; bsy = sy; }
                }
            }
            int dxh = min(max(2 * sdx + bsx, -255), 255), dyh = min(max(2 * sdy + bsy, -255), 255);
            // MotionVector::new(dx_hp/2, dy_hp/2, dx_hp%2, dy_hp%2).as_canonicalized()
            MvT raw{sat8(dxh / 2), sat8(dyh / 2), dxh % 2, dyh % 2};
            if (raw.dx == -128 && raw.sx == -1) raw.sx = 0;
            if (raw.dy == -128 && raw.sy == -1) raw.sy = 0;
            if (raw.sx == -1) { raw.sx = 1; raw.dx = max(-128, raw.dx - 1); }
            if (raw.sy == -1) { raw.sy = 1; raw.dy = max(-128, raw.dy - 1); }

            RIV_STAMP(4);
            // ---- publish the raw MV for the next row's search; hand the MB (raw MV, best SAD)
            // to the mode warp, which runs the RDO skip and the mode decision off this chain
            if (lane == 0) {
                st_rec(p.rec + idx, tagbits | ((unsigned long long)(uint8_t)raw.dx << 40) |
                                        ((unsigned long long)(uint8_t)raw.dy << 32));
                const unsigned long long pay = ((unsigned long long)(uint16_t)best_sad << 32) |
                                               (unsigned long long)((uint32_t)(uint8_t)raw.dx | ((uint32_t)(uint8_t)raw.dy << 8) |
                                                                    ((uint32_t)(uint8_t)raw.sx << 16) |
                                                                    ((uint32_t)(uint8_t)raw.sy << 24));
                if (!hand_put(hand, hand_done, hn, pay, p.spin_limit)) failed = true;
            }
            hn++;
            failed = __shfl_sync(0xffffffffu, (int)failed, 0) != 0;
            if (failed) {
                if (lane == 0) atomicOr(p.status, ST_WAIT_TIMEOUT);
                abort_loader();
                if (!FAST) cp_async_wait0();
                return;
            }
            L_raw = MvT{raw.dx, raw.dy, 0, 0};
            recTL = recT;
            recT = recTR;
        }
        if (FAST) {  // the band of this row is no longer read
            __syncwarp();
            if (lane == 0) ld_ctl[1] = lrows + 1;
            lrows++;
        } else {
            cp_async_wait0();
        }
    }
    };
    roles();
    if (helpers) {  // the row work is done: the whole CTA takes worker tasks
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int i = 0; i < LD_RING; i++) mbar_inval(fullb + i);
            mbar_inval(bandb);
        }
        frame_worker(p, smem);
    }
}


// One CTA of 512 threads per SM, at most 120 registers a thread: 61,440 of the SM's 65,536,
// so a 128-thread CTA of the next frame's input conversion (32 registers) runs beside it.
// (An 80-register cap slows the worker tasks' residual and table code measurably.)
// Launch timeline when profiling: words 28 / 29 of ring entry (tag mod 256) get the global
// time of the first CTA's start and of the last warp's exit.
template <bool BAND, bool TABLE, bool SMALL>
__global__ void __maxnreg__(120) k_search(SearchParams p) {
    const int ring = (int)(p.tag % (unsigned)min(256, p.BW * p.BH));
    unsigned long long* tl = p.prof != nullptr ? (unsigned long long*)(p.prof + (size_t)ring * RIV_PROF_WORDS + 28) : nullptr;
    if (tl != nullptr && threadIdx.x == 0) atomicCAS(tl, 0ull, (unsigned long long)gtimer());
    if (p.wq_next != nullptr && blockIdx.x == gridDim.x - 1)  // the next launch's queue words
        for (int i = threadIdx.x; i < p.wq_words; i += blockDim.x) p.wq_next[i] = 0u;
    search_body<BAND, TABLE, SMALL>(p);
    if (tl != nullptr && (threadIdx.x & 31) == 0) atomicMax(tl + 1, (unsigned long long)gtimer());
}

// Shared memory of the search kernel; BAND when the whole MB-row band fits, TABLE when
// the exhaustive SAD table is used (search ranges up to 15).
int sad_table_stride(int sr) { return ((2 * sr + 1) * (2 * sr + 1) + 7) & ~7; }
bool search_use_table(int sr) { return sr <= 15; }
static size_t search_smem(int sr, int W, bool band, bool table) {
    size_t ws = 18 + 2 * (size_t)sr;
    size_t margin = ((size_t)sr + 1 + 15) & ~(size_t)15;
    size_t ref = band ? ws * ((size_t)W + 2 * margin) : ws * ws;
    size_t head = 256 * sizeof(double) + 64 * 64 * 4 + HAND_RING * 8 + 16;
    if (band && table) return head + 64 + 1024 + LD_RING * (size_t)ld_slot_bytes(sad_table_stride(sr)) + ref + 16;
    return head + 512 + (table ? 4 * (size_t)sad_table_stride(sr) : 0) + ref + 16;
}
static int search_threads(bool band, bool table) { return band && table ? 128 : 64; }
static const size_t SEARCH_SMEM_MAX = 200 * 1024;
static bool search_use_band(int sr, int W) {
    return search_smem(sr, W, true, search_use_table(sr)) <= SEARCH_SMEM_MAX;
}
static const void* search_fn(bool band, bool table, bool small) {
    if (table && small) return band ? (const void*)k_search<true, true, true> : (const void*)k_search<false, true, true>;
    if (table) return band ? (const void*)k_search<true, true, false> : (const void*)k_search<false, true, false>;
    return band ? (const void*)k_search<true, false, false> : (const void*)k_search<false, false, false>;
}

size_t search_smem_bytes(int sr) { return search_smem(sr, 0, false, search_use_table(sr)); }

int search_plan(int sr, int W, int BH, bool table, bool small, SearchPlan* out) {
    const bool band = search_use_band(sr, W);
    const void* fn = search_fn(band, table, table && small);
    const int threads = search_threads(band, table);
    int dev = 0, nsm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (int)e;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return (int)e;
    auto resident = [&](size_t sm, int nthreads, int* per_sm) {
        cudaError_t r = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (r == cudaSuccess) r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, fn, nthreads, sm);
        return r;
    };
    const size_t sm = search_smem(sr, W, band, table);
    SearchPlan pl{};
    pl.threads = threads;
    pl.fast = band && table;
    if (band && table) {
        // fused: one CTA per SM (the shared-memory request rules out a second), rows first,
        // table workers on the SMs the rows leave free -- used when enough of them remain
        // row CTAs' helper region (live flag + three worker groups) after the row layout,
        // where the per-CTA maximum allows it
        const size_t with_helpers = ((sm + 15) & ~(size_t)15) + 16 + (size_t)worker_region_bytes(3);
        const bool helpers = with_helpers <= (size_t)227 * 1024;
        const size_t need = helpers ? with_helpers : sm;
        const size_t smf = need > (size_t)116 * 1024 ? need : (size_t)116 * 1024;
        int per_sm = 0;
        e = resident(smf, 4 * 128, &per_sm);
        if (e != cudaSuccess) return (int)e;
        const int total = per_sm * nsm;
        const int nrow = BH < total ? BH : total;
        const size_t gsm = ((size_t)sad_table_smem(sr) + 15) & ~(size_t)15;
        if (per_sm == 1 && total - nrow >= 32 && 4 * gsm <= smf) {
            pl.fused = true;
            pl.helpers = helpers;
            pl.threads = 4 * 128;  // row CTAs use three warps; table workers four groups of 128
            pl.smem = smf;
            pl.nrow = nrow;
            pl.grid = total;
            *out = pl;
            return 0;
        }
    }
    int per_sm = 0;
    e = resident(sm, threads, &per_sm);
    if (e != cudaSuccess) return (int)e;
    pl.fused = false;
    pl.smem = sm;
    pl.grid = pl.nrow = BH < per_sm * nsm ? BH : per_sm * nsm;
    *out = pl;
    return 0;
}

int launch_search(const SearchParams& p, const SearchPlan& plan, void* stream) {
    const bool band = search_use_band(p.sr, p.W), table = p.tab != nullptr;
    SearchParams q = p;
    q.nrow_ctas = plan.nrow;
    q.row_helpers = plan.fused && plan.helpers ? 1 : 0;
    if (!plan.fused) q.tflag = nullptr;
    void* args[] = {&q};
    // Cooperative launch: every CTA of the grid is co-resident, so the row-to-row waits
    // and the waits for table rows can always make progress.
    cudaError_t e = cudaLaunchCooperativeKernel(search_fn(band, table, table && p.small), dim3(plan.grid),
                                                dim3(plan.threads), args, plan.smem, (cudaStream_t)stream);
    return (int)e;
}

// ---------------------------------------------------------------------------------
// Learned-proposal form: a parallel search seeded by the proposal network, and the mode
// decision of every MB in parallel.
//
// No MB waits for another.  Each MB's search uses, as predictors and as the basis of its MV
// cost (estimate_mv_cost, enc/motion/scalar.rs:453-544), the previous P-frame's coded MVs
// around it (left, top, top-right, top-left, co-located, zero, median of the first three)
// instead of the current frame's neighbours, so every MB can be searched at once.
//   candidates: the network's four proposals (rounded to whole pixels) and the predictors;
//   refinement: small-diamond rounds from the best candidate, then the nine half-pel
//   positions around it (floor-averaged samples, as the plain search scores them, with the
//   fractional penalty of refine_halfpel, enc/motion/scalar.rs:759-839);
//   fallback: when the best proposal's SAD exceeds the best predictor's SAD by more than
//   `margin`, the hexagon search of process_block_hex (enc/motion/scalar.rs:546-636) from
//   the best candidate instead of the short diamond;
//   shortcut: an MB whose skip probability exceeds `skip_prob` keeps its best whole-pixel
//   candidate without refinement.
// Every MV stays within +-search range (<= 63), so a NEW delta never saturates and each MB's
// coded MV equals its search MV: the mode decision then needs only the neighbours' search
// MVs, and runs for all MBs at once (k_learned_mode).
// ---------------------------------------------------------------------------------
constexpr int LS_MBS = 4;  // MBs (warps) per CTA: consecutive MBs of one row
// Width of the shared reference window of a CTA: its MBs, +-(sr + 2) columns, up to 3 more on
// the left (the left edge is rounded down to a 4-byte boundary) and 4 bytes of slack for the
// unaligned word reads; a multiple of 4.
__host__ __device__ constexpr int ls_window_width(int sr) { return ((16 * LS_MBS + 2 * (sr + 2) + 3 + 3) & ~3) + 4; }

struct LearnedMv {
    int8_t raw[4];  // dx, dy, sx, sy (canonical)
    int32_t sad;    // SAD of the chosen position (half-pel SAD when fractional)
};
static_assert(sizeof(LearnedMv) == 8, "LearnedMv layout");

struct LearnedParams {
    SearchParams sp;
    const float* net;  // per MB 16 network outputs (nullptr: predictors only, every MB refined by the hexagon search)
    int margin;
    float skip_logit;  // shortcut when the skip logit exceeds this (a probability threshold, as a logit)
    LearnedMv* out;
    unsigned* counters;  // [0] fallbacks to the hexagon search, [1] shortcuts
    // per MB row: MBs whose ln variance is written (zero between frames); non-null: the
    // launch's extra fold CTA sums the ln variances in raster order while the rows finish
    unsigned* rowcnt;
};

// The strictly sequential f32 sum of the ln variances (Iterator::sum, res/residual.rs:154-167)
// and their mean at lnv[n], by one warp of the launch's first CTA while the search CTAs run.
// Each round, lane i checks whether row r + i has published all its MBs (release: fence +
// count; acquire: the count's load), the warp takes every finished row from r on at once,
// stages their values through shared memory in chunks and lane 0 adds them left to right, so
// the L2 round trips are paid per batch of rows, not per row.  Each row's count goes back to
// zero for the next frame.  A wait past the spin limit sets ST_WAIT_TIMEOUT and ends the fold.
__device__ __forceinline__ void learned_fold(const LearnedParams& lp) {
    constexpr int CH = 1024;
    __shared__ __align__(16) float fb[CH];
    const SearchParams& p = lp.sp;
    const int lane = threadIdx.x & 31;
    float sum = 0.0f;
    long long spins = 0;
    int r = 0;
    while (r < p.BH) {
        const bool done = r + lane < p.BH && ld_acquire_u32(lp.rowcnt + r + lane) >= (unsigned)p.BW;
        const unsigned m = __ballot_sync(0xffffffffu, done);
        const int ready = m == 0xffffffffu ? 32 : __ffs(~m) - 1;  // finished rows r, r + 1, ...
        if (ready == 0) {
            if (++spins > p.spin_limit) {
                if (lane == 0) atomicOr(p.status, ST_WAIT_TIMEOUT);
                return;
            }
            __nanosleep(64);
            continue;
        }
        spins = 0;
        __syncwarp();
        const size_t base = (size_t)r * p.BW;
        const int total = ready * p.BW;
        for (int c0 = 0; c0 < total; c0 += CH) {
            const int m2 = min(CH, total - c0);
            for (int i = lane; i < m2; i += 32) fb[i] = __ldcg(p.lnv + base + c0 + i);
            __syncwarp();
            if (lane == 0) {  // eight values per pair of vector loads, the adds strictly in order
                int i = 0;
                for (; i + 8 <= m2; i += 8) {
                    const float4 a = *(const float4*)(fb + i), b = *(const float4*)(fb + i + 4);
                    sum = __fadd_rn(sum, a.x); sum = __fadd_rn(sum, a.y); sum = __fadd_rn(sum, a.z);
                    sum = __fadd_rn(sum, a.w); sum = __fadd_rn(sum, b.x); sum = __fadd_rn(sum, b.y);
                    sum = __fadd_rn(sum, b.z); sum = __fadd_rn(sum, b.w);
                }
                for (; i < m2; i++) sum = __fadd_rn(sum, fb[i]);
            }
            __syncwarp();
        }
        if (lane < ready) lp.rowcnt[r + lane] = 0u;
        r += ready;
    }
    if (lane == 0) p.lnv[p.BW * p.BH] = __fdiv_rn(sum, (float)(p.BW * p.BH));
}

// SAD of the 16x16 block at whole-pixel offset (dx, dy) over the window; lane l covers row l/2,
// eight pixels, current samples in c0, c1.
__device__ __forceinline__ unsigned ls_sad(const uint8_t* win, int ws, int ox, int oy, int dx, int dy, int lane,
                                           uint32_t c0, uint32_t c1) {
    const uint8_t* r = win + (oy + (lane >> 1) + dy) * ws + ox + (lane & 1) * 8 + dx;
    const unsigned s = __vsadu4(lds_u32(r), c0) + __vsadu4(lds_u32(r + 4), c1);
    return __reduce_add_sync(0xffffffffu, s);
}
// SAD at half-pel offset (hx, hy) with floor-averaged samples.
__device__ __forceinline__ unsigned ls_sad_hp(const uint8_t* win, int ws, int ox, int oy, int hx, int hy, int lane,
                                              uint32_t c0, uint32_t c1) {
    const int ix = hx >> 1, iy = hy >> 1, fx = hx & 1, fy = hy & 1;
    const uint8_t* r = win + (oy + (lane >> 1) + iy) * ws + ox + (lane & 1) * 8 + ix;
    uint32_t a0 = lds_u32(r), a1 = lds_u32(r + 4);
    if (fx && fy) {
        a0 = favg4(a0, lds_u32(r + 1), lds_u32(r + ws), lds_u32(r + ws + 1));
        a1 = favg4(a1, lds_u32(r + 5), lds_u32(r + ws + 4), lds_u32(r + ws + 5));
    } else if (fx) {
        a0 = favg(a0, lds_u32(r + 1));
        a1 = favg(a1, lds_u32(r + 5));
    } else if (fy) {
        a0 = favg(a0, lds_u32(r + ws));
        a1 = favg(a1, lds_u32(r + ws + 4));
    }
    const unsigned s = __vsadu4(a0, c0) + __vsadu4(a1, c1);
    return __reduce_add_sync(0xffffffffu, s);
}

// Four positions at once: lane group g (lanes 8g .. 8g + 7) scores its own position, lane i of
// the group rows 2i and 2i + 1 (16 samples each, current samples in cw: row 2i in cw[0..3], row
// 2i + 1 in cw[4..7]); the group's sum ends in every lane of the group.  Five aligned words per
// row cover the 16 unaligned bytes; `w(k, sh)` is the word at byte 4k + sh / 8 of them.
__device__ __forceinline__ uint32_t ls_word(const uint32_t (&w)[5], int k, uint32_t sh) {
    return sh >= 32u ? w[k + 1] : __funnelshift_r(w[k], w[k + 1], sh);
}
__device__ __forceinline__ void ls_row5(const uint8_t* win, int off, uint32_t (&w)[5], uint32_t& sh) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(win + off);
    const uint32_t b = a & ~3u;
    sh = (a & 3u) * 8u;
#pragma unroll
    for (int k = 0; k < 5; k++) asm volatile("ld.shared.u32 %0, [%1];" : "=r"(w[k]) : "r"(b + 4u * k));
}
__device__ __forceinline__ unsigned group_sum8(unsigned s) {
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    s += __shfl_xor_sync(0xffffffffu, s, 4);
    return s;
}
// whole-pixel offset (dx, dy)
__device__ __forceinline__ unsigned ls_sad_g(const uint8_t* win, int ws, int ox, int oy, int dx, int dy, int li,
                                             const uint32_t (&cw)[8]) {
    unsigned s = 0;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        uint32_t w[5], sh;
        ls_row5(win, (oy + 2 * li + h + dy) * ws + ox + dx, w, sh);
#pragma unroll
        for (int k = 0; k < 4; k++) s += __vsadu4(ls_word(w, k, sh), cw[4 * h + k]);
    }
    return group_sum8(s);
}
// half-pel offset (hx, hy), floor-averaged samples (the same rule as ls_sad_hp)
__device__ __forceinline__ unsigned ls_sad_hp_g(const uint8_t* win, int ws, int ox, int oy, int hx, int hy, int li,
                                                const uint32_t (&cw)[8]) {
    const int ix = hx >> 1, iy = hy >> 1, fx = hx & 1, fy = hy & 1;
    uint32_t w[3][5], sh[3];
#pragma unroll
    for (int r = 0; r < 3; r++) ls_row5(win, (oy + 2 * li + r + iy) * ws + ox + ix, w[r], sh[r]);
    unsigned s = 0;
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint32_t a = ls_word(w[h], k, sh[h]), b = ls_word(w[h], k, sh[h] + 8u);
            const uint32_t c = ls_word(w[h + 1], k, sh[h + 1]), d = ls_word(w[h + 1], k, sh[h + 1] + 8u);
            const uint32_t v = fx && fy ? favg4(a, b, c, d) : fx ? favg(a, b) : fy ? favg(a, c) : a;
            s += __vsadu4(v, cw[4 * h + k]);
        }
    return group_sum8(s);
}

__global__ void __launch_bounds__(32 * LS_MBS) k_learned_search(LearnedParams lp) {
    const SearchParams& p = lp.sp;
    extern __shared__ __align__(16) uint8_t lsm[];
    // with the fold: grid row 0 is the fold CTA (x = 0; the rest of that row returns), MB row r
    // is grid row r + 1.  The fold CTA comes first and waits only for search CTAs, which never
    // wait, so every CTA finishes.
    const int yoff = lp.rowcnt != nullptr ? 1 : 0;
    if ((int)blockIdx.y < yoff) {
        if (blockIdx.x == 0 && threadIdx.x < 32) learned_fold(lp);
        return;
    }
    const int sr = p.sr, M = sr + 2;
    const int bx0 = blockIdx.x * LS_MBS, by = (int)blockIdx.y - yoff;
    const int nmb_here = min(LS_MBS, p.BW - bx0);
    const int wx0 = (bx0 * 16 - M) & ~3, wy0 = by * 16 - M;  // left edge on a 4-byte boundary
    const int ws = ls_window_width(sr), wh = 16 + 2 * M + 1;
    // stage the window with coordinates clamped to the plane (replicated borders); word loads
    // when it lies inside the plane
    if (wx0 >= 0 && wy0 >= 0 && wx0 + ws <= p.W && wy0 + wh <= p.H) {
        const int wpr = ws / 4;
        for (int i = threadIdx.x; i < wpr * wh; i += blockDim.x) {
            const int y = i / wpr, x = i - y * wpr;
            ((uint32_t*)lsm)[i] = *(const uint32_t*)(p.ref_y + (size_t)(wy0 + y) * p.W + wx0 + 4 * x);
        }
    } else {
        for (int i = threadIdx.x; i < ws * wh; i += blockDim.x) {
            const int y = i / ws, x = i - y * ws;
            const int fy = min(max(wy0 + y, 0), p.H - 1), fx = min(max(wx0 + x, 0), p.W - 1);
            lsm[i] = p.ref_y[(size_t)fy * p.W + fx];
        }
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (w >= nmb_here) return;
    const int bx = bx0 + w, mb = by * p.BW + bx;
    const int x0 = bx * 16, y0 = by * 16;
    const int ox = x0 - wx0, oy = y0 - wy0;
    // this lane's group (g) and its place in it (li): rows 2 li, 2 li + 1 of the block
    const int g = lane >> 3, li = lane & 7;
    uint32_t cw[8];
    {
        const uint8_t* cp = p.cur_y + (size_t)(y0 + 2 * li) * p.W + x0;
        const uint4 r0 = *(const uint4*)cp, r1 = *(const uint4*)(cp + p.W);
        cw[0] = r0.x; cw[1] = r0.y; cw[2] = r0.z; cw[3] = r0.w;
        cw[4] = r1.x; cw[5] = r1.y; cw[6] = r1.z; cw[7] = r1.w;
    }
    // predictors from the previous P-frame's coded MVs (whole-pixel parts, within +-sr)
    int px[7] = {0, 0, 0, 0, 0, 0, 0}, py[7] = {0, 0, 0, 0, 0, 0, 0};
    bool av[5] = {false, false, false, false, false};
    if (p.prev_coded) {
        const int nx[5] = {bx - 1, bx, bx + 1, bx - 1, bx}, ny[5] = {by, by - 1, by - 1, by - 1, by};
#pragma unroll
        for (int k = 0; k < 5; k++) {
            if (nx[k] < 0 || ny[k] < 0 || nx[k] >= p.BW || ny[k] >= p.BH) continue;
            const char4 c = *(const char4*)(p.prev_coded + 4 * ((size_t)ny[k] * p.BW + nx[k]));
            px[k] = min(max((int)c.x, -sr), sr);
            py[k] = min(max((int)c.y, -sr), sr);
            av[k] = true;
        }
        px[6] = median3(px[0], px[1], px[2]);
        py[6] = median3(py[0], py[1], py[2]);
    }
    // cost basis: nearest / near = first two distinct available predictors, median of L, T, TR
    CostCtx cc{0, 0, 0, 0, px[6], py[6]};
    {
        int nu = 0;
#pragma unroll
        for (int k = 0; k < 5; k++) {
            if (!av[k]) continue;
            if (nu == 0) { cc.nx = px[k]; cc.ny = py[k]; nu = 1; }
            else if (nu == 1 && (px[k] != cc.nx || py[k] != cc.ny)) { cc.rx = px[k]; cc.ry = py[k]; nu = 2; }
        }
    }
    auto cost = [&](int dx, int dy, unsigned sad) { return (long long)sad + mv_cost<false>(dx, dy, cc, p, p.mvbits, nullptr); };
    // One batch: group g scores position (gx, gy) if `act` (a group-uniform flag; inactive groups
    // score a valid dummy position), and every lane then takes the group results in group order,
    // so the first strictly better position wins, as in a one-at-a-time walk.
    auto batch = [&](bool act, int gx, int gy, bool hp, unsigned& sad_out, long long& c_out) {
        const unsigned sad = hp ? ls_sad_hp_g(lsm, ws, ox, oy, gx, gy, li, cw) : ls_sad_g(lsm, ws, ox, oy, gx, gy, li, cw);
        sad_out = sad;
        c_out = act ? (hp ? (long long)sad : cost(gx, gy, sad)) : LLONG_MAX;
    };
    auto from_group = [&](int src, unsigned sad, long long c, unsigned& s2, long long& c2) {
        s2 = __shfl_sync(0xffffffffu, sad, 8 * src);
        c2 = (long long)__shfl_sync(0xffffffffu, (unsigned long long)c, 8 * src);
    };
    // candidates: 4 proposals (slots 0-3, absent without a network), then the 7 predictors
    // (slots 4-10); a position already scored in the same group (proposals / predictors) changes
    // neither that group's minimum SAD nor, with the strict `<`, the best, so the list keeps the
    // first of each (the candidates are the same in every lane)
    __shared__ int clist[LS_MBS][12];
    int cx[11] = {0, 0, 0, 0}, cy[11] = {0, 0, 0, 0};
    bool shortcut = false;
    const bool has_net = lp.net != nullptr;
    if (has_net) {
        const float4* o4 = (const float4*)(lp.net + (size_t)mb * 16);
        const float4 q0 = o4[0], q1 = o4[1], q2 = o4[2];
        const float o[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float hx = o[2 * k] * 32.0f, hy = o[2 * k + 1] * 32.0f;  // half-pel units
            cx[k] = min(max(__float2int_rn(hx * 0.5f), -sr), sr);
            cy[k] = min(max(__float2int_rn(hy * 0.5f), -sr), sr);
        }
        shortcut = q2.x > lp.skip_logit;
    }
#pragma unroll
    for (int k = 0; k < 7; k++) { cx[4 + k] = px[k]; cy[4 + k] = py[k]; }
    int nlist = 0;
#pragma unroll
    for (int k = 0; k < 11; k++) {
        if (k < 4 && !has_net) continue;
        bool seen = false;
#pragma unroll
        for (int j = 0; j < k; j++) seen |= cx[j] == cx[k] && cy[j] == cy[k] && ((j < 4) == (k < 4));
        if (seen) continue;
        if (lane == 0) clist[w][nlist] = (k << 16) | ((cy[k] & 0xFF) << 8) | (cx[k] & 0xFF);
        nlist++;
    }
    __syncwarp();
    long long best = LLONG_MAX;
    unsigned bsad = 0, bsp = 0xffffffffu, bsq = 0xffffffffu;
    int bdx = 0, bdy = 0;
    for (int b0 = 0; b0 < nlist; b0 += 4) {
        const int e = clist[w][b0 + g < nlist ? b0 + g : b0];
        unsigned sad;
        long long c;
        batch(b0 + g < nlist, (int)(int8_t)(e & 0xFF), (int)(int8_t)((e >> 8) & 0xFF), false, sad, c);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            unsigned s2;
            long long c2;
            from_group(q, sad, c, s2, c2);
            if (b0 + q >= nlist) continue;
            const int eq = clist[w][b0 + q];
            if ((eq >> 16) < 4) bsp = min(bsp, s2); else bsq = min(bsq, s2);
            if (c2 < best) { best = c2; bsad = s2; bdx = (int)(int8_t)(eq & 0xFF); bdy = (int)(int8_t)((eq >> 8) & 0xFF); }
        }
    }
    const bool fallback = !lp.net || bsp > bsq + (unsigned)lp.margin;
    if (fallback) shortcut = false;
    if (!shortcut) {
        // whole-pixel refinement: hexagon rounds (fallback) then small-diamond rounds.  After a
        // move in direction m, the points a round would evaluate again (the previous centre,
        // and for the hexagon its two neighbours of m, which are the new centre's points m + 2 ..
        // m + 4) all cost at least the new centre's cost, so under the strict `<` they can never
        // be taken: they are skipped, and the walk is unchanged.
        // hexagon directions (2,0) (1,2) (-1,2) (-2,0) (-1,-2) (1,-2); diamond (1,0) (-1,0) (0,1) (0,-1)
        // (selects, not tables: the direction is a per-lane value)
        auto HX = [](int k) { return k == 0 ? 2 : k == 1 ? 1 : k == 2 ? -1 : k == 3 ? -2 : k == 4 ? -1 : 1; };
        auto HY = [](int k) { return k == 0 || k == 3 ? 0 : k <= 2 ? 2 : -2; };
        auto DX = [](int k) { return k == 0 ? 1 : k == 1 ? -1 : 0; };
        auto DY = [](int k) { return k == 2 ? 1 : k == 3 ? -1 : 0; };
        auto in_range = [&](int dx, int dy) { return dx >= -sr && dx <= sr && dy >= -sr && dy <= sr; };
        if (fallback) {
            int moved = -1;
            for (int round = 0; round < 16; round++) {  // a bounded hexagon walk (+-32 pixels)
                // this round's directions in increasing order: all six, or m - 1, m, m + 1
                int dirs[6] = {0, 1, 2, 3, 4, 5}, nd = 6;
                if (moved >= 0) {
                    const int d0 = (moved + 5) % 6, d2 = (moved + 1) % 6;
                    const int lo = min(min(d0, moved), d2), hi = max(max(d0, moved), d2);
                    dirs[0] = lo; dirs[1] = d0 + moved + d2 - lo - hi; dirs[2] = hi;
                    nd = 3;
                }
                auto pick = [&](int i) {
                    return i == 0 ? dirs[0] : i == 1 ? dirs[1] : i == 2 ? dirs[2] : i == 3 ? dirs[3] : i == 4 ? dirs[4] : dirs[5];
                };
                int nbx = bdx, nby = bdy, nk = -1;
                long long nb = best;
                unsigned ns = bsad;
#pragma unroll
                for (int b0 = 0; b0 < 8; b0 += 4) {
                    if (b0 >= nd) break;
                    const int kg = pick(b0 + g < nd ? b0 + g : b0);
                    const int dx = bdx + HX(kg), dy = bdy + HY(kg);
                    const bool act = b0 + g < nd && in_range(dx, dy);
                    unsigned sad;
                    long long c;
                    batch(act, act ? dx : bdx, act ? dy : bdy, false, sad, c);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        unsigned s2;
                        long long c2;
                        from_group(q, sad, c, s2, c2);
                        if (b0 + q >= nd) continue;
                        const int kq = pick(b0 + q);
                        if (c2 < nb) { nb = c2; ns = s2; nbx = bdx + HX(kq); nby = bdy + HY(kq); nk = kq; }
                    }
                }
                if (nk < 0) break;
                best = nb; bsad = ns; bdx = nbx; bdy = nby; moved = nk;
            }
        }
        int moved = -1;
        for (int round = 0; round < (fallback ? 16 : 8); round++) {
            const int dx = bdx + DX(g), dy = bdy + DY(g);
            const bool act = in_range(dx, dy) && !(moved >= 0 && g == (moved ^ 1));  // not the previous centre
            unsigned sad;
            long long c;
            batch(act, act ? dx : bdx, act ? dy : bdy, false, sad, c);
            int nbx = bdx, nby = bdy, nk = -1;
            long long nb = best;
            unsigned ns = bsad;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                unsigned s2;
                long long c2;
                from_group(q, sad, c, s2, c2);
                if (c2 < nb) { nb = c2; ns = s2; nbx = bdx + DX(q); nby = bdy + DY(q); nk = q; }
            }
            if (nk < 0) break;
            best = nb; bsad = ns; bdx = nbx; bdy = nby; moved = nk;
        }
    }
    // half-pel refinement around the whole-pixel best: the centre (no penalty) first, then the
    // eight neighbours row by row, each with the fractional penalty c15
    int hx = 2 * bdx, hy = 2 * bdy;
    unsigned hsad = bsad;
    if (!shortcut) {
        long long hbest = LLONG_MAX;
        int bhx = hx, bhy = hy;
        for (int b0 = 0; b0 < 9; b0 += 4) {
            const int i = b0 + g < 9 ? b0 + g : 0;  // 0: centre, 1..8: (sy, sx) in row order without the centre
            const int n = i == 0 ? 4 : i <= 4 ? i - 1 : i;  // 3x3 index (sy + 1) * 3 + sx + 1
            const int gx = hx + n % 3 - 1, gy = hy + n / 3 - 1;
            unsigned sad;
            long long c;
            batch(true, gx, gy, true, sad, c);
            if (i != 0) c += p.c15;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                unsigned s2;
                long long c2;
                from_group(q, sad, c, s2, c2);
                if (b0 + q >= 9) continue;
                const int iq = b0 + q, nq = iq == 0 ? 4 : iq <= 4 ? iq - 1 : iq;
                if (c2 < hbest) { hbest = c2; bhx = hx + nq % 3 - 1; bhy = hy + nq / 3 - 1; hsad = s2; }
            }
        }
        hx = bhx;
        hy = bhy;
    }
    if (p.pred != nullptr) {
        // luma prediction of the chosen MV with build_predicted's rounded bilinear rule
        // (com/fast_motion.rs:103-262; the window's replicated borders equal its coordinate
        // clamps), then the MB's variance and its glibc-exact ln (compute_aq_quant_steps,
        // res/residual.rs:116-167) for the AQ fold
        const int ix = hx >> 1, iy = hy >> 1, fx = hx & 1, fy = hy & 1;
        const uint8_t* r = lsm + (oy + (lane >> 1) + iy) * ws + ox + (lane & 1) * 8 + ix;
        uint32_t q[2];
#pragma unroll
        for (int h2 = 0; h2 < 2; h2++) {
            const uint8_t* rr = r + 4 * h2;
            const uint32_t a = lds_u32(rr);
            if (fx && fy) q[h2] = ravg4(a, lds_u32(rr + 1), lds_u32(rr + ws), lds_u32(rr + ws + 1));
            else if (fx) q[h2] = __vavgu4(a, lds_u32(rr + 1));
            else if (fy) q[h2] = __vavgu4(a, lds_u32(rr + ws));
            else q[h2] = a;
        }
        *(uint2*)(p.pred + (size_t)(y0 + (lane >> 1)) * p.W + x0 + (lane & 1) * 8) = make_uint2(q[0], q[1]);
        unsigned sv = 0, sv2 = 0;
#pragma unroll
        for (int h2 = 0; h2 < 2; h2++)
#pragma unroll
            for (int b = 0; b < 4; b++) {
                const unsigned v = (q[h2] >> (8 * b)) & 255u;
                sv += v;
                sv2 += v * v;
            }
        sv = __reduce_add_sync(0xffffffffu, sv);
        sv2 = __reduce_add_sync(0xffffffffu, sv2);
        if (lane == 0) {
            const unsigned long long NN = 256ull * sv2 - (unsigned long long)sv * sv;
            float var = __fdiv_rn(__ull2float_rn(NN), 65536.0f);
            var = var < 4.0f ? 4.0f : var;
            p.lnv[mb] = glibc_logf(var, p.logfix, p.nlog);
            if (lp.rowcnt != nullptr) {  // publish for the fold CTA
                __threadfence();
                atomicAdd(lp.rowcnt + by, 1u);
            }
        }
    }
    if (lane == 0) {
        // canonical form: a -1/2 component becomes +1/2 of the whole pixel below
        LearnedMv r;
        r.raw[0] = (int8_t)(hx >> 1);
        r.raw[1] = (int8_t)(hy >> 1);
        r.raw[2] = (int8_t)(hx & 1);
        r.raw[3] = (int8_t)(hy & 1);
        r.sad = (int32_t)hsad;
        lp.out[mb] = r;
        if (fallback && lp.net) atomicAdd(lp.counters, 1u);
        if (shortcut) atomicAdd(lp.counters + 1, 1u);
    }
}

// Mode decision of every MB at once (coded MV = search MV, see above): RDO skip, mode, NEW base
// and delta through decide_mb, the same routine the wavefront's mode warp runs.
__global__ void __launch_bounds__(128) k_learned_mode(SearchParams p, const LearnedMv* __restrict__ lm) {
    const int mb = blockIdx.x * blockDim.x + threadIdx.x;
    if (mb >= p.BW * p.BH) return;
    const int bx = mb % p.BW, by = mb / p.BW;
    auto get = [&](int x, int y) {
        const LearnedMv& m = lm[(size_t)y * p.BW + x];
        return MvT{m.raw[0], m.raw[1], m.raw[2], m.raw[3]};
    };
    const MvT zero{0, 0, 0, 0};
    const bool has_t = by > 0, has_l = bx > 0, has_tl = by > 0 && bx > 0, has_tr = by > 0 && bx + 1 < p.BW;
    const bool has_tm = p.prev_coded != nullptr;
    MvT Tm{0, 0, 0, 0};
    if (has_tm) {
        const char4 pc = *(const char4*)(p.prev_coded + 4 * (size_t)mb);
        Tm = MvT{pc.x, pc.y, pc.z, pc.w};
    }
    const MvT raw = get(bx, by);
    const MbDecision md = decide_mb(p, raw, (long long)lm[mb].sad, has_l, has_t, has_tr, has_tl, has_tm,
                                    has_l ? get(bx - 1, by) : zero, has_t ? get(bx, by - 1) : zero,
                                    has_tr ? get(bx + 1, by - 1) : zero, has_tl ? get(bx - 1, by - 1) : zero, Tm);
    MbOut o;
    o.raw[0] = (int8_t)raw.dx; o.raw[1] = (int8_t)raw.dy; o.raw[2] = (int8_t)raw.sx; o.raw[3] = (int8_t)raw.sy;
    o.coded[0] = (int8_t)md.coded.dx; o.coded[1] = (int8_t)md.coded.dy;
    o.coded[2] = (int8_t)md.coded.sx; o.coded[3] = (int8_t)md.coded.sy;
    o.rdelta[0] = (int8_t)md.rdx; o.rdelta[1] = (int8_t)md.rdy;
    o.mode = (uint8_t)md.mode; o.base = (uint8_t)md.chosen; o.flags = md.flags; o.rdo_skip = md.rdo_skip ? 1 : 0;
    o.pad[0] = o.pad[1] = 0;
    o.best_sad = lm[mb].sad;
    p.out[mb] = o;
    *(char4*)(p.coded_out + 4 * (size_t)mb) =
        make_char4((signed char)md.coded.dx, (signed char)md.coded.dy, (signed char)md.coded.sx, (signed char)md.coded.sy);
    // a search MV outside +-63 would break coded == search MV for the neighbours: flag it
    if (md.coded.dx != raw.dx || md.coded.dy != raw.dy || md.coded.sx != raw.sx || md.coded.sy != raw.sy)
        atomicOr(p.status, ST_HEX_CAP);
}

__global__ void __launch_bounds__(1024) k_aq_sum(const float* __restrict__ lnv, int n, float* avg_out);

int launch_learned(const SearchParams& sp, const float* net, int margin, float skip_logit, void* lmv,
                   unsigned* counters, unsigned* rowcnt, void* stream) {
    LearnedParams lp{};
    lp.sp = sp;
    lp.net = net;
    lp.margin = margin;
    lp.skip_logit = skip_logit;
    lp.out = (LearnedMv*)lmv;
    lp.counters = counters;
    lp.rowcnt = sp.lnv != nullptr ? rowcnt : nullptr;
    const int M = sp.sr + 2;
    const int ws = ls_window_width(sp.sr), wh = 16 + 2 * M + 1;
    const size_t smem = (size_t)ws * wh + 16;
    dim3 grid((sp.BW + LS_MBS - 1) / LS_MBS, sp.BH + (lp.rowcnt != nullptr ? 1 : 0));
    k_learned_search<<<grid, 32 * LS_MBS, smem, (cudaStream_t)stream>>>(lp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    const int n = sp.BW * sp.BH;
    k_learned_mode<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(sp, (const LearnedMv*)lmv);
    e = cudaGetLastError();
    if (e != cudaSuccess || sp.lnv == nullptr || lp.rowcnt != nullptr) return (int)e;
    // the strictly sequential f32 mean of the ln variances (Iterator::sum), at lnv[n]
    k_aq_sum<<<1, 1024, 8192 * sizeof(float), (cudaStream_t)stream>>>(sp.lnv, n, sp.lnv + n);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// K6a: motion-compensated prediction (build_predicted, com/fast_motion.rs:103-352) and
// the per-MB (sum, sum of squares) of predicted luma for AQ (res/residual.rs:134-153).
// One CTA of 256 threads per MB.  Luma: per-sample clamped rounded bilinear sampling;
// chroma: copy at the truncated (x0+dx)/2 origin for in-bounds integer MVs, else
// rounded bilinear at chroma half-pel (2c + (mv_hp >> 1)).
// ---------------------------------------------------------------------------------
// MB mb by 256 threads; returns the luma (sum, sum of squares) to thread 0 (ws, ws2: 8 words
// of shared memory each).
__device__ __forceinline__ uint2 predict_mb(const uint8_t* __restrict__ ref, const MbOut* __restrict__ mbo,
                                            uint8_t* __restrict__ pred, int W, int H, int mb, unsigned* ws,
                                            unsigned* ws2) {
    const int BW = W / 16;
    const int bx = mb % BW, by = mb / BW;
    const int x0 = bx * 16, y0 = by * 16;
    const int t = threadIdx.x;
    const int CW = W / 2, CH = H / 2;
    const uint8_t* RY = ref;
    const uint8_t* RU = ref + (size_t)W * H;
    const uint8_t* RV = RU + (size_t)CW * CH;
    uint8_t* PY = pred;
    uint8_t* PU = pred + (size_t)W * H;
    uint8_t* PV = PU + (size_t)CW * CH;
    const MbOut m = mbo[mb];
    const int mdx = m.raw[0] * 2 + m.raw[2], mdy = m.raw[1] * 2 + m.raw[3];
    const bool integer = ((mdx & 1) == 0) && ((mdy & 1) == 0);
    const int sx0 = x0 + (mdx >> 1), sy0 = y0 + (mdy >> 1);
    const bool copy = integer && sx0 >= 0 && sy0 >= 0 && sx0 + 15 < W && sy0 + 15 < H;
    const int yy = t >> 4, xx = t & 15;
    int v;
    if (copy) v = RY[(size_t)(sy0 + yy) * W + sx0 + xx];
    else v = sample_round(RY, W, H, 2 * (x0 + xx) + mdx, 2 * (y0 + yy) + mdy);
    PY[(size_t)(y0 + yy) * W + x0 + xx] = (uint8_t)v;
    if (t < 128) {
        const uint8_t* R = t < 64 ? RU : RV;
        uint8_t* P = t < 64 ? PU : PV;
        int i = t & 63, cy = i >> 3, cx = i & 7;
        int cxg = x0 / 2 + cx, cyg = y0 / 2 + cy;
        int c;
        if (copy) c = R[(size_t)(sy0 / 2 + cy) * CW + sx0 / 2 + cx];
        else c = sample_round(R, CW, CH, 2 * cxg + (mdx >> 1), 2 * cyg + (mdy >> 1));
        P[(size_t)cyg * CW + cxg] = (uint8_t)c;
    }
    unsigned s = (unsigned)v, s2 = (unsigned)(v * v);
    s = __reduce_add_sync(0xffffffffu, s);
    s2 = __reduce_add_sync(0xffffffffu, s2);
    if ((t & 31) == 0) { ws[t >> 5] = s; ws2[t >> 5] = s2; }
    __syncthreads();
    unsigned a = 0, b = 0;
    if (t == 0)
        for (int i = 0; i < 8; i++) { a += ws[i]; b += ws2[i]; }
    return make_uint2(a, b);
}
__global__ void __launch_bounds__(256) k_predict(const uint8_t* __restrict__ ref, const MbOut* __restrict__ mbo,
                                                 uint8_t* __restrict__ pred, uint2* __restrict__ varsum, int W, int H) {
    __shared__ unsigned ws[8], ws2[8];
    const uint2 vs = predict_mb(ref, mbo, pred, W, H, blockIdx.x, ws, ws2);
    if (threadIdx.x == 0) varsum[blockIdx.x] = vs;
}

int launch_predict(const uint8_t* ref, const MbOut* mb, uint8_t* pred, uint2* varsum, int W, int H, void* stream) {
    int nmb = (W / 16) * (H / 16);
    k_predict<<<nmb, 256, 0, (cudaStream_t)stream>>>(ref, mb, pred, varsum, W, H);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// glibc-exact logf / exp2f.  The reference calls f32::ln / f32::exp2, i.e. glibc logf /
// exp2f, which are not correctly rounded.  Device: correctly rounded via the double
// function rounded to float, then a sorted fix-up table (input bits -> glibc output
// bits) built at build time by running glibc over the whole reachable input domain.
// ---------------------------------------------------------------------------------
__global__ void k_libm_eval(int which, const float* in, float* out, size_t n, const uint32_t* fix, int nfix) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t stride = (size_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) out[i] = which == 0 ? glibc_logf(in[i], fix, nfix) : glibc_exp2f(in[i], fix, nfix);
}
int launch_libm_eval(int which, const float* in, float* out, size_t n, const uint32_t* fix, int nfix, void* stream) {
    k_libm_eval<<<1184, 256, 0, (cudaStream_t)stream>>>(which, in, out, n, fix, nfix);
    return (int)cudaGetLastError();
}

// Every f32 whose bit pattern lies in [lo, lo + n): out[i] = f(bits lo + i).  which: 0 logf,
// 1 exp2f, 2 logf through the four-wide batched search the AQ warps use.
__global__ void k_libm_range(int which, uint32_t lo, uint32_t n, float* out, const uint32_t* fix, int nfix) {
    const uint32_t stride = gridDim.x * blockDim.x;
    if (which == 2) {
        for (uint32_t i = 4 * (blockIdx.x * blockDim.x + threadIdx.x); i < n; i += 4 * stride) {
            float x[4], y[4];
#pragma unroll
            for (int j = 0; j < 4; j++) x[j] = __uint_as_float(lo + min(i + j, n - 1));
            glibc_logf_batch<4>(x, y, fix, nfix);
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (i + j < n) out[i + j] = y[j];
        }
        return;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float x = __uint_as_float(lo + i);
        out[i] = which == 0 ? glibc_logf(x, fix, nfix) : glibc_exp2f(x, fix, nfix);
    }
}
int launch_libm_range(int which, uint32_t lo, uint32_t n, float* out, const uint32_t* fix, int nfix, void* stream) {
    k_libm_range<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(which, lo, n, out, fix, nfix);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// K_aq: compute_aq_quant_steps (res/residual.rs:116-167).  One CTA: variances and ln in
// parallel, the f32 sum strictly sequential (Iterator::sum folds left to right), then
// the per-MB steps in parallel.
// ---------------------------------------------------------------------------------
// Variance and ln(variance) of every MB in parallel.
__global__ void k_aq_log(const uint2* __restrict__ varsum, int n, const uint32_t* logfix, int nlog, float* lnv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint2 vs = varsum[i];
    unsigned long long N = 256ull * vs.y - (unsigned long long)vs.x * vs.x;
    float var = __fdiv_rn(__ull2float_rn(N), 65536.0f);
    var = var < 4.0f ? 4.0f : var;
    lnv[i] = glibc_logf(var, logfix, nlog);
}
// The strictly sequential f32 sum (Iterator::sum folds left to right): staged through
// shared memory by the whole CTA, folded by one thread.
__device__ __forceinline__ void aq_sum_cta(const float* __restrict__ lnv, int n, float* avg_out, float* sl) {
    __shared__ float part;
    if (threadIdx.x == 0) part = 0.0f;
    const int CH = 8192;
    for (int base = 0; base < n; base += CH) {
        int m = min(CH, n - base);
        __syncthreads();
        for (int i = threadIdx.x; i < m; i += blockDim.x) sl[i] = lnv[base + i];
        __syncthreads();
        if (threadIdx.x == 0) {
            float s = part;
            int i = 0;
            for (; i + 8 <= m; i += 8) {
                float4 a = *(const float4*)(sl + i), b = *(const float4*)(sl + i + 4);
                s = __fadd_rn(s, a.x); s = __fadd_rn(s, a.y); s = __fadd_rn(s, a.z); s = __fadd_rn(s, a.w);
                s = __fadd_rn(s, b.x); s = __fadd_rn(s, b.y); s = __fadd_rn(s, b.z); s = __fadd_rn(s, b.w);
            }
            for (; i < m; i++) s = __fadd_rn(s, sl[i]);
            part = s;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) *avg_out = __fdiv_rn(part, (float)n);
}
__global__ void __launch_bounds__(1024) k_aq_sum(const float* __restrict__ lnv, int n, float* avg_out) {
    extern __shared__ float sl[];
    aq_sum_cta(lnv, n, avg_out, sl);
}
__global__ void k_aq_steps(const float* __restrict__ lnv, int n, const float* avg_in, float base,
                           const uint32_t* expfix, int nexp, float* qs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float off = __fmul_rn(0.8f, __fsub_rn(lnv[i], *avg_in));
    qs[i] = __fmul_rn(base, glibc_exp2f(__fdiv_rn(off, 6.0f), expfix, nexp));
}
int launch_aq(const uint2* varsum, int n, float base, const uint32_t* logfix, int nlog, const uint32_t* expfix,
              int nexp, float* lnv_scratch, float* qs, void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    // lnv_scratch holds n floats followed by one float for the mean
    float* avg = lnv_scratch + n;
    k_aq_log<<<(n + 127) / 128, 128, 0, st>>>(varsum, n, logfix, nlog, lnv_scratch);
    k_aq_sum<<<1, 1024, 8192 * sizeof(float), st>>>(lnv_scratch, n, avg);
    k_aq_steps<<<(n + 127) / 128, 128, 0, st>>>(lnv_scratch, n, avg, base, expfix, nexp, qs);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// K6b: residual -> FDCT (i64 accumulate) -> quant -> zero test -> dequant -> IDCT
// (wrapping i32) -> recon, one CTA (256 threads) per MB.  Inter: AQ step + dead zone
// (dct/dct16.rs:274-412, dct/dct8.rs:80-135, dct/fast_dct8.rs:69-174,
// res/residual.rs:520-752).  Intra: pixel-128, JPEG-derived matrices, no dead zone
// (res/residual.rs:267-388, dct16.rs:420-560, dct8.rs:142-196).
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_residual(ResidualParams p, int nmb) {
    __shared__ __align__(16) int32_t sT16[256], sT16t[256], sT8[64];
    __shared__ __align__(16) ResSmem S[RS_MB];
    const int tid = threadIdx.x;
    sT16[tid] = c_T16[tid];
    sT16t[(tid & 15) * 16 + (tid >> 4)] = c_T16[tid];  // sT16t[i][x] = T[x][i]
    if (tid < 64) sT8[tid] = c_T8[tid];
    __syncthreads();
    const int g = tid >> 6, u = tid & 63;
    const int mb = blockIdx.x * RS_MB + g;
    if (mb >= nmb) return;
    residual_mb(p, nmb, mb, u, g + 1, S[g], sT16, sT16t, sT8);
}

// Decoder reconstruction (res/residual.rs:815-887 intra, :889-1079 inter): the decoded
// coefficients (384 per MB, dense) dequantised, inverse-transformed and added to the
// prediction (inter) or to 128 (intra); skipped inter MBs copy the prediction.  Same thread
// layout and arithmetic as the encoder's reconstruction (inverse_mb).
__global__ void __launch_bounds__(256) k_reconstruct(const int16_t* __restrict__ coeffs, const uint8_t* __restrict__ pred,
                                                     const uint8_t* __restrict__ skip, const float* __restrict__ qs,
                                                     int intra, const uint16_t* ytab, const uint16_t* ctab,
                                                     uint8_t* __restrict__ recon, int W, int H, int BW, int nmb) {
    __shared__ __align__(16) int32_t sT16[256], sT16t[256];
    __shared__ __align__(16) int32_t res[RS_MB][256], rowt[RS_MB][256];
    __shared__ __align__(16) int16_t qc[RS_MB][128];
    __shared__ int32_t aant[RS_MB][2][64];
    __shared__ uint8_t predc[RS_MB][128];
    const int tid = threadIdx.x;
    sT16[tid] = c_T16[tid];
    sT16t[(tid & 15) * 16 + (tid >> 4)] = c_T16[tid];
    __syncthreads();
    const int g = tid >> 6, u = tid & 63;
    const int mb = blockIdx.x * RS_MB + g;
    if (mb >= nmb) return;
    const int CW = W / 2, CH = H / 2;
    const int bx = mb % BW, by = mb / BW, x0 = bx * 16, y0 = by * 16;
    const int yy = u >> 2, xb = (u & 3) * 4;
    const size_t yi = (size_t)(y0 + yy) * W + x0 + xb;
    const int pl = u >> 5, ci = (u & 31) * 2, cyy = ci >> 3, cxx = ci & 7;
    const size_t cidx = (size_t)(y0 / 2 + cyy) * CW + x0 / 2 + cxx;
    const size_t coff = (size_t)W * H + (pl == 0 ? 0 : (size_t)CW * CH);
    uint8_t *rY = recon, *rU = recon + (size_t)W * H, *rV = rU + (size_t)CW * CH;
    if (!intra && skip[mb]) {
        *(uint32_t*)(rY + yi) = *(const uint32_t*)(pred + yi);
        *(uint16_t*)(recon + coff + cidx) = *(const uint16_t*)(pred + coff + cidx);
        return;
    }
    const int16_t* co = coeffs + (size_t)mb * 384;
    const uint2 lw = *(const uint2*)(co + yy * 16 + xb);
    const int16_t ql[4] = {(int16_t)(lw.x & 0xffff), (int16_t)(lw.x >> 16), (int16_t)(lw.y & 0xffff), (int16_t)(lw.y >> 16)};
    const uint32_t cw = *(const uint32_t*)(co + 256 + pl * 64 + ci);
    qc[g][pl * 64 + ci] = (int16_t)(cw & 0xffff);
    qc[g][pl * 64 + ci + 1] = (int16_t)(cw >> 16);
    const uint32_t pcw = intra ? 0x8080u : *(const uint16_t*)(pred + coff + cidx);
    predc[g][pl * 64 + ci] = (uint8_t)pcw;
    predc[g][pl * 64 + ci + 1] = (uint8_t)(pcw >> 8);
    const uint32_t lbase = intra ? 0x80808080u : *(const uint32_t*)(pred + yi);
    const float qsv = intra ? 0.0f : qs[mb];
    inverse_mb(g + 1, u, yy, xb, ql, qsv, intra != 0, ytab, ctab, lbase, rY + yi, rU, rV, CW, x0, y0, sT16, sT16t, res[g],
               rowt[g], aant[g][0], qc[g], predc[g]);
}

int launch_reconstruct(const int16_t* coeffs, const uint8_t* pred, const uint8_t* skip, const float* qs, int intra,
                       const uint16_t* ytab, const uint16_t* ctab, uint8_t* recon, int W, int H, void* stream) {
    const int BW = W / 16, n = BW * (H / 16);
    k_reconstruct<<<(n + RS_MB - 1) / RS_MB, 64 * RS_MB, 0, (cudaStream_t)stream>>>(coeffs, pred, skip, qs, intra, ytab,
                                                                                   ctab, recon, W, H, BW, n);
    return (int)cudaGetLastError();
}

int launch_residual(const ResidualParams& p, int nmb, void* stream) {
    k_residual<<<(nmb + RS_MB - 1) / RS_MB, 64 * RS_MB, 0, (cudaStream_t)stream>>>(p, nmb);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// K7: in-loop deblock (com/deblock.rs:60-202).  Vertical edges, then horizontal edges,
// each pass in place: lines of one pass touch disjoint pixels (an edge line reads
// x-4..x+3 and writes x-3..x+2, edges are >= 8 px apart), so a thread per edge line
// reproduces the reference's sequential loops exactly.
// ---------------------------------------------------------------------------------
// TW: luma tile width (256 for this standalone launch: fewer, wider tiles measured faster than
// the worker tasks' DB_TW; the output does not depend on it).
constexpr int DB_TW_STANDALONE = 256;
template <int TW>
__global__ void __launch_bounds__(128) k_deblock_tiled(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int W,
                                                       int H, int BW, int E, int I, int Hv, const uint8_t* mask,
                                                       int ntiles_y) {
    __shared__ __align__(16) uint8_t tile[(16 + 8) * (TW + 8)];
    int t = blockIdx.x;
    int plane = t < ntiles_y ? 0 : (t - ntiles_y) % 2 + 1;
    if (plane > 0) t = (t - ntiles_y) / 2;
    deblock_tile<TW>(src, dst, W, H, BW, E, I, Hv, mask, plane, t, tile, threadIdx.x, blockDim.x, 0);
}

int launch_deblock_tiled(const uint8_t* src, uint8_t* dst, int W, int H, int E, int I, int Hv, const uint8_t* mask,
                         void* stream) {
    constexpr int TW = DB_TW_STANDALONE;
    const int BW = W / 16;
    const int ty = (H / 16) * ((W + TW - 1) / TW);
    const int tc = ((H / 2) / 8) * ((W / 2 + TW / 2 - 1) / (TW / 2));
    k_deblock_tiled<TW><<<ty + 2 * tc, 128, 0, (cudaStream_t)stream>>>(src, dst, W, H, BW, E, I, Hv, mask, ty);
    return (int)cudaGetLastError();
}

// In place, two passes over each plane (vertical edges, then horizontal edges).
// Vertical edges of one plane: thread per (row y, edge e >= 1).
__global__ void k_deblock_v(uint8_t* pl, int w, int h, int grid, int BW, int E, int I, int Hv, const uint8_t* mask) {
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    int e = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (y >= h || e >= w / grid) return;
    int by = y / grid;
    if (mask && !(mask[by * BW + e - 1] | mask[by * BW + e])) return;
    uint8_t* s = pl + (size_t)y * w + e * grid - 4;
    int px[8];
#pragma unroll
    for (int k = 0; k < 8; k++) px[k] = s[k];
    filter_line(px, E, I, Hv);
#pragma unroll
    for (int k = 1; k < 7; k++) s[k] = (uint8_t)px[k];
}
// Horizontal edges of one plane: thread per (column x, edge e >= 1).
__global__ void k_deblock_h(uint8_t* pl, int w, int h, int grid, int BW, int E, int I, int Hv, const uint8_t* mask) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int e = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (x >= w || e >= h / grid) return;
    int bxm = x / grid;
    if (mask && !(mask[(e - 1) * BW + bxm] | mask[e * BW + bxm])) return;
    uint8_t* s = pl + (size_t)(e * grid - 4) * w + x;
    int px[8];
#pragma unroll
    for (int k = 0; k < 8; k++) px[k] = s[(size_t)k * w];
    filter_line(px, E, I, Hv);
#pragma unroll
    for (int k = 1; k < 7; k++) s[(size_t)k * w] = (uint8_t)px[k];
}

int launch_deblock(uint8_t* yuv, int W, int H, int E, int I, int Hv, const uint8_t* mask, void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    const int BW = W / 16;
    uint8_t* planes[3] = {yuv, yuv + (size_t)W * H, yuv + (size_t)W * H + (size_t)(W / 2) * (H / 2)};
    for (int k = 0; k < 3; k++) {
        int w = k == 0 ? W : W / 2, h = k == 0 ? H : H / 2, g = k == 0 ? 16 : 8;
        int ne = w / g - 1;
        if (ne > 0) {
            dim3 b(32, 8), gr((ne + 31) / 32, (h + 7) / 8);
            k_deblock_v<<<gr, b, 0, st>>>(planes[k], w, h, g, BW, E, I, Hv, mask);
        }
    }
    for (int k = 0; k < 3; k++) {
        int w = k == 0 ? W : W / 2, h = k == 0 ? H : H / 2, g = k == 0 ? 16 : 8;
        int ne = h / g - 1;
        if (ne > 0) {
            dim3 b(128, 1), gr((w + 127) / 128, ne);
            k_deblock_h<<<gr, b, 0, st>>>(planes[k], w, h, g, BW, E, I, Hv, mask);
        }
    }
    return (int)cudaGetLastError();
}

// Fixed device scratch of the no-allocation deblock entry point: the YUV planes and the
// optional per-MB mask of one call are staged here instead of in memory allocated per
// call.  Nothing in it has to start at zero (each call writes every byte it reads), and
// calls that overlap on one device share it.
static __device__ __align__(256) uint8_t g_deblock_scratch[DEBLOCK_NOALLOC_MAX_BYTES];

int deblock_scratch_address(void** out) { return (int)cudaGetSymbolAddress(out, g_deblock_scratch); }

// ---------------------------------------------------------------------------------
// K8 kernels (compaction of a frame reconstructed outside a search launch; the layout is
// described at scan_mbs / pack_mb).
// ---------------------------------------------------------------------------------
// Scan: one CTA of SC_THREADS threads (scan_mbs), small enough to run beside the search kernel.
__global__ void __launch_bounds__(SC_THREADS) k_scan(const uint8_t* opt_skip, const uint8_t* eobs, int nmb, int intra,
                                                     int32_t* index, int32_t* offset, uint32_t* hdr) {
    __shared__ int wsum[SC_THREADS / 32], wsz[SC_THREADS / 32];
    scan_mbs<SC_THREADS, SC_IPT>(opt_skip, eobs, nmb, intra, index, offset, hdr, threadIdx.x, 1, wsum, wsz);
}
// Pack: one warp per MB.
__global__ void __launch_bounds__(256) k_pack(const uint8_t* opt_skip, const MbOut* mb, const int16_t* coeffs,
                                              const uint8_t* eobs, const int32_t* index, const int32_t* offset,
                                              int intra, int nmb, uint32_t* side, int16_t* packed, uint8_t* peobs) {
    const int m = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (m < nmb) pack_mb(m, threadIdx.x & 31, opt_skip, mb, coeffs, eobs, index, offset, intra, side, packed, peobs);
}

int launch_compact(const uint8_t* opt_skip, const MbOut* mb, const int16_t* coeffs, const uint8_t* eobs, int nmb,
                   int intra, int32_t* index, int32_t* offset, uint32_t* dside, int16_t* dpacked, uint8_t* dpeobs,
                   uint32_t* hhdr, void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    k_scan<<<1, SC_THREADS, 0, st>>>(opt_skip, eobs, nmb, intra, index, offset, hhdr);
    k_pack<<<(nmb + 7) / 8, 256, 0, st>>>(opt_skip, mb, coeffs, eobs, index, offset, intra, nmb, dside, dpacked, dpeobs);
    return (int)cudaGetLastError();
}

// Multi-clip launches of the stages above (riv_batch).
#include "riv_batch.cuh"

}  // namespace riv

// Table upload helper (host side of the constant tables).
extern "C" int riv_upload_dct_tables(const int32_t* t16, const int32_t* t8) {
    cudaError_t e = cudaMemcpyToSymbol(riv::c_T16, t16, 256 * sizeof(int32_t));
    if (e != cudaSuccess) return (int)e;
    return (int)cudaMemcpyToSymbol(riv::c_T8, t8, 64 * sizeof(int32_t));
}
