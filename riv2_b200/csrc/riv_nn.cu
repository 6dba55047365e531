// riv_nn.cu -- tensor-core kernels of the motion-proposal network (sm_100a).
//
// Both kernels accumulate bf16 x bf16 products in f32 tensor memory with tcgen05.mma, issued
// by one thread of the CTA, operands read from shared memory through 64-bit matrix
// descriptors (K-major, 128-byte or 64-byte swizzle), completion tracked by tcgen05.commit on
// mbarriers, the accumulator read back with tcgen05.ld for the epilogue.
//
//  * k_nn_gemm: D = A . B^T with both operands staged by TMA (cp.async.bulk.tensor) through a
//    four-deep ring: warp 0 issues the copies, warp 1 the MMAs, all four warps run the
//    epilogue (warp w owns accumulator rows 32w .. 32w+31, the TMEM lanes it may read).
//  * k_nn_conv_i2c: implicit-GEMM 3x3 convolution (32 input channels: conv2-4).  The weights
//    come in once by TMA and stay in shared memory; each 128-row tile of output positions is
//    loaded by the TMA's im2col mode, one 128 x 32-channel load per filter tap, while the
//    tensor core consumes earlier taps.  Persistent CTAs, two per SM.
//  * k_nn_conv: the same GEMM with the operand gathered by the CTA's threads (cp.async straight
//    into the swizzled layout): conv1 of the training path, and conv2-4 when RIV_CONV_GATHER=1.
//
// Every wait is bounded; an expired wait sets bit 0 of *err and the kernel runs to its end
// without waiting again (tensor memory is always released).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "../../include/riv_nn.h"
#include "riv_nn.h"

namespace {

constexpr long long NN_SPIN = 1ll << 22;  // polls of mbarrier.try_wait (a few seconds at most)

__device__ __forceinline__ uint32_t s32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// ---- mbarriers
__device__ __forceinline__ void mb_init(uint64_t* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mb_expect_tx(uint64_t* b, unsigned tx) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(s32(b)), "r"(tx) : "memory");
}
__device__ __forceinline__ bool mb_try(uint64_t* b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(s32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the completion of the phase with the given parity.  `dead` short-cuts all
// later waits once one has expired.
__device__ __forceinline__ bool mb_wait(uint64_t* b, unsigned parity, unsigned* err, bool& dead) {
    if (dead) return false;
    long long n = 0;
    while (!mb_try(b, parity)) {
        if (++n > NN_SPIN) {
            atomicOr(err, 1u);
            dead = true;
            return false;
        }
    }
    return true;
}

// ---- TMA
__device__ __forceinline__ void tma_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            s32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(s32(bar))
        : "memory");
}

// ---- tensor memory and tcgen05
__device__ __forceinline__ void tm_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s32(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tm_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// K-major shared-memory matrix descriptor: rows of 128 (or 64) bytes, 16-byte chunks XOR
// swizzled by the row within 8-row groups that lie 1024 (512) bytes apart.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, int swz) {
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;                                   // leading offset: unused when swizzled
    d |= (uint64_t)((swz == 128 ? 1024u : 512u) >> 4) << 32;  // stride between 8-row groups
    d |= (uint64_t)1 << 46;                                   // descriptor version of sm_100
    d |= (uint64_t)(swz == 128 ? 2u : 4u) << 61;              // swizzle mode
    return d;
}
// Instruction descriptor: bf16 A and B (K-major), f32 accumulator, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma(uint32_t dtm, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtm),
        "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(s32(bar))
                 : "memory");
}
__device__ __forceinline__ void tm_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *(uint32_t*)&h;
}

// =====================================================================================
// GEMM
// =====================================================================================
constexpr int GEMM_STAGES = 4;

struct GemmArgs {
    int M, N, nkb_total, kb_per_cta, ntile;
    float* d;
    __nv_bfloat16* dh;
    int ldd;
    const float* bias;
    int relu, mode;
    unsigned* err;
};

template <int BK>
__global__ void __launch_bounds__(128, 1)
    k_nn_gemm(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, GemmArgs g) {
    constexpr int SWZ = BK * 2;  // bytes per operand row
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sm = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int BN = g.ntile;
    const int a_bytes = 128 * SWZ, b_bytes = BN * SWZ;
    const int stage_bytes = (a_bytes + b_bytes + 1023) & ~1023;
    uint64_t* full = (uint64_t*)(sm + GEMM_STAGES * stage_bytes);
    uint64_t* empty = full + GEMM_STAGES;
    uint64_t* accum = empty + GEMM_STAGES;
    uint32_t* slot = (uint32_t*)(accum + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * 128, n0 = blockIdx.z * BN;
    const int kb0 = blockIdx.y * g.kb_per_cta;
    const int nkb = min(g.kb_per_cta, g.nkb_total - kb0);
    uint32_t ncols = 32;
    while ((int)ncols < BN) ncols <<= 1;
    if (threadIdx.x == 0) {
        for (int s = 0; s < GEMM_STAGES; s++) {
            mb_init(&full[s], 1);
            mb_init(&empty[s], 1);
        }
        mb_init(accum, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tm_alloc(slot, ncols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tacc = *slot;
    bool dead = false;
    if (nkb > 0) {
        if (warp == 0 && lane == 0) {  // TMA producer
            for (int i = 0; i < nkb && !dead; i++) {
                const int s = i % GEMM_STAGES;
                if (i >= GEMM_STAGES) mb_wait(&empty[s], ((i / GEMM_STAGES) - 1) & 1, g.err, dead);
                if (dead) break;
                uint8_t* st = sm + s * stage_bytes;
                mb_expect_tx(&full[s], (unsigned)(a_bytes + b_bytes));
                tma_2d(st, &ta, (kb0 + i) * BK, m0, &full[s]);
                tma_2d(st + a_bytes, &tb, (kb0 + i) * BK, n0, &full[s]);
            }
        } else if (warp == 1 && lane == 0) {  // MMA issuer
            const uint32_t idesc = idesc_bf16(128, BN);
            for (int i = 0; i < nkb && !dead; i++) {
                const int s = i % GEMM_STAGES;
                if (!mb_wait(&full[s], (i / GEMM_STAGES) & 1, g.err, dead)) break;
                tc_fence_after();
                const uint32_t sa = s32(sm + s * stage_bytes);
                const uint64_t ad = sdesc(sa, SWZ), bd = sdesc(sa + a_bytes, SWZ);
#pragma unroll
                for (int k = 0; k < BK / 16; k++) umma(tacc, ad + 2 * k, bd + 2 * k, idesc, (i | k) != 0);
                umma_commit(&empty[s]);
            }
            umma_commit(accum);  // arrives once every MMA issued above is complete
        }
        __syncwarp();
        // epilogue: warp w reads accumulator rows 32w + lane
        mb_wait(accum, 0, g.err, dead);
        __syncwarp();
        tc_fence_after();
        const int row = m0 + warp * 32 + lane;
        for (int c = 0; c < BN; c += 16) {
            __syncwarp();  // tcgen05.ld is warp-collective
            uint32_t r[16];
            tm_ld16(tacc + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, r);
            if (row >= g.M || dead) continue;
            float v[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
                v[j] = __uint_as_float(r[j]);
                if (g.bias) v[j] += g.bias[n0 + c + j];
                if (g.relu) v[j] = fmaxf(v[j], 0.0f);
            }
            const size_t o = (size_t)row * g.ldd + n0 + c;
            if (g.mode == 0) {
#pragma unroll
                for (int j = 0; j < 16; j += 4) *(float4*)(g.d + o + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
            } else if (g.mode == 1) {
#pragma unroll
                for (int j = 0; j < 16; j++) atomicAdd(g.d + o + j, v[j]);
            } else {
                uint4 p0 = make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]),
                                      pack_bf16(v[6], v[7]));
                uint4 p1 = make_uint4(pack_bf16(v[8], v[9]), pack_bf16(v[10], v[11]), pack_bf16(v[12], v[13]),
                                      pack_bf16(v[14], v[15]));
                *(uint4*)(g.dh + o) = p0;
                *(uint4*)(g.dh + o + 8) = p1;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tm_dealloc(tacc, ncols);
}

// =====================================================================================
// Implicit-GEMM convolution
// =====================================================================================
// Warp roles (288 threads): warps 0-3 gather the operand (one output position per thread,
// cp.async straight into the swizzled K-major layout, zero-filled padding taps) into a ring of
// CV_STAGES k-blocks and mark each stage full on an mbarrier once their copies have landed;
// warp 4 holds the tensor memory and its lane 0 issues the MMAs; warps 5-8 run the epilogue
// (warp w reads TMEM lanes 32 (w % 4) .. +31).  The accumulator is double-buffered (2 x 32
// columns), so a tile's epilogue overlaps the next tile's MMAs and gathers.
constexpr int CV_THREADS = 288;
constexpr int CV_LAG = 2;  // k-blocks a gathering thread keeps in flight before marking one full

struct ConvArgs {
    const __nv_bfloat16* in;
    __nv_bfloat16* out;
    const float* bias;
    int in_mb, out_mb, out_ld;
    int nmb, hin, hout, stride;
    unsigned* err;
};

template <int CIN>
struct ConvCfg {
    static constexpr int BK = CIN == 2 ? 32 : 64;      // k-block width (elements)
    static constexpr int SWZ = BK * 2;                 // bytes per operand row
    static constexpr int NKB = CIN == 2 ? 1 : 5;       // k-blocks per tile
    static constexpr int STAGES = CIN == 2 ? 8 : 5;    // operand ring depth
    static constexpr int W_TILE = 32 * SWZ;
    static constexpr int A_TILE = 128 * SWZ;
    static constexpr size_t smem() {
        return 1024 + ((NKB * W_TILE + 1023) & ~1023) + (size_t)STAGES * A_TILE + 512;
    }
};

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, unsigned bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src, unsigned bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void mb_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(s32(b)) : "memory");
}

template <int CIN>
__global__ void __launch_bounds__(CV_THREADS, 2) k_nn_conv(const __grid_constant__ CUtensorMap tw, ConvArgs a) {
    using CF = ConvCfg<CIN>;
    constexpr int BK = CF::BK, SWZ = CF::SWZ, NKB = CF::NKB, S = CF::STAGES;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sm = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sw = sm;                                        // NKB weight tiles
    uint8_t* sa = sm + ((NKB * CF::W_TILE + 1023) & ~1023);  // S operand stages
    uint64_t* wfull = (uint64_t*)(sa + S * CF::A_TILE);
    uint64_t* full = wfull + 1;
    uint64_t* empty = full + S;
    uint64_t* accf = empty + S;
    uint64_t* acce = accf + 2;
    uint32_t* slot = (uint32_t*)(acce + 2);
    float* sbias = (float*)(slot + 4);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        mb_init(wfull, 1);
        for (int k = 0; k < S; k++) {
            mb_init(&full[k], 128);
            mb_init(&empty[k], 1);
        }
        for (int k = 0; k < 2; k++) {
            mb_init(&accf[k], 1);
            mb_init(&acce[k], 128);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (tid < 32) sbias[tid] = a.bias[tid];
    if (warp == 4) tm_alloc(slot, 64);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tacc = *slot;
    bool dead = false;
    const int pos = a.hout * a.hout;
    const long long rows = (long long)a.nmb * pos;
    const int ntiles = (int)((rows + 127) / 128);

    if (warp < 4) {
        // ---- gather: row `tid` of every tile, one ring stage per k-block
        const uint32_t sa0 = s32(sa);
        int it = 0;
        for (int tile = blockIdx.x; tile < ntiles && !dead; tile += gridDim.x) {
            const long long m = (long long)tile * 128 + tid;
            const bool valid = m < rows;
            const int b = valid ? (int)(m / pos) : 0, p = valid ? (int)(m % pos) : 0;
            const int oy = p / a.hout, ox = p % a.hout;
            const __nv_bfloat16* inb = a.in + (size_t)b * a.in_mb;
            for (int kb = 0; kb < NKB; kb++, it++) {
                const int s = it % S;
                if (it >= S && !mb_wait(&empty[s], ((it / S) - 1) & 1, a.err, dead)) break;
                const uint32_t row = sa0 + (uint32_t)(s * CF::A_TILE + tid * SWZ);
                if (CIN == 2) {  // k = tap * 2 + channel: taps 0..8, zeros from tap 9
                    const int x = (tid >> 1) & 3;
#pragma unroll
                    for (int t = 0; t < 16; t++) {
                        const int iy = oy * a.stride + t / 3 - 1, ix = ox * a.stride + t % 3 - 1;
                        const bool in = valid && t < 9 && iy >= 0 && iy < a.hin && ix >= 0 && ix < a.hin;
                        const __nv_bfloat16* src = in ? inb + ((size_t)iy * a.hin + ix) * 2 : a.in;
                        cp_async4(row + ((((t >> 2) ^ x)) << 4) + (t & 3) * 4, src, in ? 4u : 0u);
                    }
                } else {  // two taps of 32 channels per k-block
                    const int x = tid & 7;
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const int t = 2 * kb + h;
                        const int iy = oy * a.stride + t / 3 - 1, ix = ox * a.stride + t % 3 - 1;
                        const bool in = valid && t < 9 && iy >= 0 && iy < a.hin && ix >= 0 && ix < a.hin;
                        const __nv_bfloat16* src = in ? inb + ((size_t)iy * a.hin + ix) * 32 : a.in;
#pragma unroll
                        for (int c = 0; c < 4; c++)
                            cp_async16(row + ((((4 * h + c) ^ x)) << 4), in ? src + 8 * c : src, in ? 16u : 0u);
                    }
                }
                cp_commit();
                if (it >= CV_LAG) {  // the stage of CV_LAG k-blocks ago has landed: hand it over
                    cp_wait<CV_LAG>();
                    fence_async_smem();
                    mb_arrive(&full[(it - CV_LAG) % S]);
                }
            }
        }
        cp_wait<0>();
        fence_async_smem();
        for (int k = it - CV_LAG < 0 ? 0 : it - CV_LAG; k < it; k++) mb_arrive(&full[k % S]);
    } else if (warp == 4) {
        // ---- MMA issue (lane 0); the weights by TMA first
        if (lane == 0) {
            mb_expect_tx(wfull, (unsigned)(NKB * CF::W_TILE));
            for (int kb = 0; kb < NKB; kb++) tma_2d(sw + kb * CF::W_TILE, &tw, kb * BK, 0, wfull);
            mb_wait(wfull, 0, a.err, dead);
            const uint32_t idesc = idesc_bf16(128, 32);
            int it = 0, nt = 0;
            for (int tile = blockIdx.x; tile < ntiles && !dead; tile += gridDim.x, nt++) {
                const int buf = nt & 1;
                if (nt >= 2 && !mb_wait(&acce[buf], ((nt >> 1) - 1) & 1, a.err, dead)) break;
                tc_fence_after();
                for (int kb = 0; kb < NKB; kb++, it++) {
                    const int s = it % S;
                    if (!mb_wait(&full[s], (it / S) & 1, a.err, dead)) break;
                    tc_fence_after();
                    const uint64_t ad = sdesc(s32(sa + s * CF::A_TILE), SWZ), bd = sdesc(s32(sw + kb * CF::W_TILE), SWZ);
#pragma unroll
                    for (int k = 0; k < BK / 16; k++)
                        umma(tacc + (uint32_t)(buf * 32), ad + 2 * k, bd + 2 * k, idesc, (kb | k) != 0);
                    umma_commit(&empty[s]);
                }
                umma_commit(&accf[buf]);
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue: bias, ReLU, bf16, one 64-byte output row per thread
        const int g = warp & 3, r = g * 32 + lane;
        int nt = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, nt++) {
            const int buf = nt & 1;
            const bool ok = mb_wait(&accf[buf], (nt >> 1) & 1, a.err, dead);
            if (!__all_sync(0xffffffffu, ok)) {  // warp-uniform: tcgen05.ld is warp-collective
                dead = true;
                break;
            }
            tc_fence_after();
            uint32_t r0[16], r1[16];
            tm_ld16(tacc + ((uint32_t)(g * 32) << 16) + (uint32_t)(buf * 32), r0);
            tm_ld16(tacc + ((uint32_t)(g * 32) << 16) + (uint32_t)(buf * 32 + 16), r1);
            tc_fence_before();
            mb_arrive(&acce[buf]);
            const long long m = (long long)tile * 128 + r;
            if (m < rows && !dead) {
                const int b = (int)(m / pos), p = (int)(m % pos);
                uint32_t o[16];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    o[j] = pack_bf16(fmaxf(__uint_as_float(r0[2 * j]) + sbias[2 * j], 0.0f),
                                     fmaxf(__uint_as_float(r0[2 * j + 1]) + sbias[2 * j + 1], 0.0f));
                    o[8 + j] = pack_bf16(fmaxf(__uint_as_float(r1[2 * j]) + sbias[16 + 2 * j], 0.0f),
                                         fmaxf(__uint_as_float(r1[2 * j + 1]) + sbias[16 + 2 * j + 1], 0.0f));
                }
                uint4* dst = (uint4*)(a.out + (size_t)b * a.out_mb + (size_t)p * a.out_ld);
#pragma unroll
                for (int c = 0; c < 4; c++) dst[c] = make_uint4(o[4 * c], o[4 * c + 1], o[4 * c + 2], o[4 * c + 3]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 4) tm_dealloc(tacc, 64);
}

// =====================================================================================
// Implicit-GEMM convolution with the operand loaded by the TMA's im2col mode (32 channels in)
// =====================================================================================
// The input is a 4-D tensor {C = 32, W = hin, H = hin, N = MBs} (NHWC per MB, MBs back to
// back).  Its im2col tensor map walks output positions in (MB, y, x) order: the bounding box of
// a layer with padding 1 and a 3x3 filter spans base positions -1 .. hin - 2 in x and y
// (corners -1, -1), stepped by the layer's stride, and wraps to the next MB at its end.  One
// load fetches the 32 channels of 128 consecutive output positions for one tap (im2col
// offsets kx, ky added to every base position; positions outside the MB read zeros) as a
// 128 x 64-byte K-major tile in the 64-byte swizzle, so a tile's operand is nine such loads
// and nothing is gathered by threads.  The MMA for tap t reads that tile as A (K = 32: two
// instructions) and the weights' columns 32t .. 32t + 31 as B, in the same K order as the
// k-block kernel above, so both kernels accumulate identically.
// Warp roles (192 threads): warp 0 lane 0 issues the loads (weights first), warp 1 holds the
// tensor memory and its lane 0 the MMAs, warps 2-5 run the epilogue of k_nn_conv.
constexpr int CI_THREADS = 192;
constexpr int CI_STAGES = 10;       // ring of tap tiles
constexpr int CI_TAP = 128 * 64;    // one tap tile: 128 positions x 32 channels bf16
constexpr int CI_WKB = 32 * 128;    // one weight k-block: 32 rows x 64 elements, 128-byte swizzle
constexpr size_t ci_smem() { return 1024 + 5 * (size_t)CI_WKB + (size_t)CI_STAGES * CI_TAP + 512; }

__device__ __forceinline__ void tma_im2col_4d(void* dst, const CUtensorMap* map, int c, int w, int h, int n,
                                              uint16_t off_w, uint16_t off_h, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.im2col.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6], {%7, %8};" ::"r"(s32(dst)),
        "l"((uint64_t)map), "r"(c), "r"(w), "r"(h), "r"(n), "r"(s32(bar)), "h"(off_w), "h"(off_h)
        : "memory");
}

__global__ void __launch_bounds__(CI_THREADS, 2)
    k_nn_conv_i2c(const __grid_constant__ CUtensorMap tw, const __grid_constant__ CUtensorMap tin, ConvArgs a) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sm = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sw = sm;                 // 5 weight k-blocks
    uint8_t* sa = sm + 5 * CI_WKB;    // CI_STAGES tap tiles
    uint64_t* wfull = (uint64_t*)(sa + CI_STAGES * CI_TAP);
    uint64_t* full = wfull + 1;
    uint64_t* empty = full + CI_STAGES;
    uint64_t* accf = empty + CI_STAGES;
    uint64_t* acce = accf + 2;
    uint32_t* slot = (uint32_t*)(acce + 2);
    float* sbias = (float*)(slot + 4);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        mb_init(wfull, 1);
        for (int k = 0; k < CI_STAGES; k++) {
            mb_init(&full[k], 1);
            mb_init(&empty[k], 1);
        }
        for (int k = 0; k < 2; k++) {
            mb_init(&accf[k], 1);
            mb_init(&acce[k], 128);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (tid < 32) sbias[tid] = a.bias[tid];
    if (warp == 1) tm_alloc(slot, 64);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tacc = *slot;
    bool dead = false;
    const int pos = a.hout * a.hout;
    const long long rows = (long long)a.nmb * pos;
    const int ntiles = (int)((rows + 127) / 128);

    if (warp == 0) {
        // ---- loads: the weights, then nine tap tiles per output tile
        if (lane == 0) {
            mb_expect_tx(wfull, (unsigned)(5 * CI_WKB));
            for (int kb = 0; kb < 5; kb++) tma_2d(sw + kb * CI_WKB, &tw, kb * 64, 0, wfull);
            int it = 0;
            for (int tile = blockIdx.x; tile < ntiles && !dead; tile += gridDim.x) {
                const long long m0 = (long long)tile * 128;
                const int n = (int)(m0 / pos), p = (int)(m0 % pos);
                const int w0 = (p % a.hout) * a.stride - 1, h0 = (p / a.hout) * a.stride - 1;
                for (int t = 0; t < 9; t++, it++) {
                    const int s = it % CI_STAGES;
                    if (it >= CI_STAGES && !mb_wait(&empty[s], ((it / CI_STAGES) - 1) & 1, a.err, dead)) break;
                    mb_expect_tx(&full[s], (unsigned)CI_TAP);
                    tma_im2col_4d(sa + s * CI_TAP, &tin, 0, w0, h0, n, (uint16_t)(t % 3), (uint16_t)(t / 3), &full[s]);
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---- MMA issue
        if (lane == 0 && mb_wait(wfull, 0, a.err, dead)) {
            const uint32_t idesc = idesc_bf16(128, 32);
            int it = 0, nt = 0;
            for (int tile = blockIdx.x; tile < ntiles && !dead; tile += gridDim.x, nt++) {
                const int buf = nt & 1;
                if (nt >= 2 && !mb_wait(&acce[buf], ((nt >> 1) - 1) & 1, a.err, dead)) break;
                tc_fence_after();
                for (int t = 0; t < 9; t++, it++) {
                    const int s = it % CI_STAGES;
                    if (!mb_wait(&full[s], (it / CI_STAGES) & 1, a.err, dead)) break;
                    tc_fence_after();
                    const uint64_t ad = sdesc(s32(sa + s * CI_TAP), 64);
                    const uint64_t bd = sdesc(s32(sw + (t >> 1) * CI_WKB), 128) + (uint64_t)((t & 1) * 4);
                    umma(tacc + (uint32_t)(buf * 32), ad, bd, idesc, t != 0);
                    umma(tacc + (uint32_t)(buf * 32), ad + 2, bd + 2, idesc, 1);
                    umma_commit(&empty[s]);
                }
                umma_commit(&accf[buf]);
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue: bias, ReLU, bf16, one 64-byte output row per thread
        const int g = warp & 3, r = g * 32 + lane;
        int nt = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, nt++) {
            const int buf = nt & 1;
            const bool ok = mb_wait(&accf[buf], (nt >> 1) & 1, a.err, dead);
            if (!__all_sync(0xffffffffu, ok)) {  // warp-uniform: tcgen05.ld is warp-collective
                dead = true;
                break;
            }
            tc_fence_after();
            uint32_t r0[16], r1[16];
            tm_ld16(tacc + ((uint32_t)(g * 32) << 16) + (uint32_t)(buf * 32), r0);
            tm_ld16(tacc + ((uint32_t)(g * 32) << 16) + (uint32_t)(buf * 32 + 16), r1);
            tc_fence_before();
            mb_arrive(&acce[buf]);
            const long long m = (long long)tile * 128 + r;
            if (m < rows && !dead) {
                const int b = (int)(m / pos), p = (int)(m % pos);
                uint32_t o[16];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    o[j] = pack_bf16(fmaxf(__uint_as_float(r0[2 * j]) + sbias[2 * j], 0.0f),
                                     fmaxf(__uint_as_float(r0[2 * j + 1]) + sbias[2 * j + 1], 0.0f));
                    o[8 + j] = pack_bf16(fmaxf(__uint_as_float(r1[2 * j]) + sbias[16 + 2 * j], 0.0f),
                                         fmaxf(__uint_as_float(r1[2 * j + 1]) + sbias[16 + 2 * j + 1], 0.0f));
                }
                uint4* dst = (uint4*)(a.out + (size_t)b * a.out_mb + (size_t)p * a.out_ld);
#pragma unroll
                for (int c = 0; c < 4; c++) dst[c] = make_uint4(o[4 * c], o[4 * c + 1], o[4 * c + 2], o[4 * c + 3]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) tm_dealloc(tacc, 64);
}

// ---- host side: tensor maps
PFN_cuTensorMapEncodeIm2col_v12000 encode_im2col_fn() {
    static PFN_cuTensorMapEncodeIm2col_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeIm2col", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeIm2col_v12000)p;
    });
    return fn;
}

// im2col map over nmb MBs of hin x hin x 32 bf16 (in_mb elements apart): 128 positions x 32
// channels per load, 64-byte swizzle, base positions -1 .. hin - 2 stepped by `stride`.
bool make_im2col_map(CUtensorMap* m, const void* base, int hin, int in_mb, int nmb, int stride) {
    auto fn = encode_im2col_fn();
    if (!fn || ((uintptr_t)base & 15) || (in_mb * 2) % 16) return false;
    cuuint64_t dims[4] = {32, (cuuint64_t)hin, (cuuint64_t)hin, (cuuint64_t)nmb};
    cuuint64_t strides[3] = {64, (cuuint64_t)hin * 64, (cuuint64_t)in_mb * 2};
    int lower[2] = {-1, -1}, upper[2] = {-1, -1};
    cuuint32_t es[4] = {1, (cuuint32_t)stride, (cuuint32_t)stride, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, lower, upper, 32, 128, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

// 2-D bf16 map over rows x cols (row pitch ld elements), box of `box_rows` rows x bk columns.
bool make_map(CUtensorMap* m, const void* base, uint64_t rows, uint64_t cols, uint64_t ld, uint32_t box_rows,
              uint32_t bk) {
    auto fn = encode_fn();
    if (!fn || ((uintptr_t)base & 15) || (ld * 2) % 16) return false;
    cuuint64_t dims[2] = {cols, rows};
    cuuint64_t strides[1] = {ld * 2};
    cuuint32_t box[2] = {bk, box_rows};
    cuuint32_t es[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, bk == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int num_sms() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

}  // namespace

int nn_gemm(const void* A, int lda, const void* B, int ldb, void* D, int ldd, const float* bias, int M, int N, int K,
            int bk, int mode, int relu, int ksplit, int ntile, unsigned* err, void* stream) {
    if (M <= 0 || N <= 0 || K <= 0 || N % 16 || (bk != 64 && bk != 32) || ksplit < 1 || ntile < 16 || ntile > 256 ||
        ntile % 16 || N % ntile || mode < 0 || mode > 2)
        return (int)cudaErrorInvalidValue;
    CUtensorMap ta, tb;
    if (!make_map(&ta, A, (uint64_t)M, (uint64_t)K, (uint64_t)lda, 128, (uint32_t)bk) ||
        !make_map(&tb, B, (uint64_t)N, (uint64_t)K, (uint64_t)ldb, (uint32_t)ntile, (uint32_t)bk))
        return (int)cudaErrorInvalidValue;
    GemmArgs g{};
    g.M = M;
    g.N = N;
    g.nkb_total = (K + bk - 1) / bk;
    g.kb_per_cta = (g.nkb_total + ksplit - 1) / ksplit;
    const int splits = (g.nkb_total + g.kb_per_cta - 1) / g.kb_per_cta;  // every CTA gets >= 1 k-block
    g.ntile = ntile;
    g.d = (float*)D;
    g.dh = (__nv_bfloat16*)D;
    g.ldd = ldd;
    g.bias = bias;
    g.relu = relu;
    g.mode = mode;
    g.err = err;
    const int stage = (128 * bk * 2 + ntile * bk * 2 + 1023) & ~1023;
    const size_t smem = 1024 + (size_t)GEMM_STAGES * stage + 256;
    const void* fn = bk == 64 ? (const void*)k_nn_gemm<64> : (const void*)k_nn_gemm<32>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    dim3 grid((M + 127) / 128, splits, N / ntile);
    if (bk == 64)
        k_nn_gemm<64><<<grid, 128, smem, (cudaStream_t)stream>>>(ta, tb, g);
    else
        k_nn_gemm<32><<<grid, 128, smem, (cudaStream_t)stream>>>(ta, tb, g);
    return (int)cudaGetLastError();
}

int nn_conv(int layer, const void* in, int in_mb, const void* W, const float* bias, void* out, int out_mb, int out_ld,
            int nmb, unsigned* err, void* stream) {
    static const int HIN[5] = {0, 24, 12, 6, 6}, HOUT[5] = {0, 12, 6, 6, 3}, STRIDE[5] = {0, 2, 2, 1, 2};
    if (layer < 1 || layer > 4 || nmb <= 0 || ((uintptr_t)in & 15) || ((uintptr_t)out & 15) || out_ld % 8 || in_mb % 8 ||
        out_mb % 8)
        return (int)cudaErrorInvalidValue;
    const int cin = layer == 1 ? 2 : 32, bk = layer == 1 ? 32 : 64, k = layer == 1 ? nn::K1 : nn::KC;
    CUtensorMap tw;
    if (!make_map(&tw, W, 32, (uint64_t)k, (uint64_t)k, 32, (uint32_t)bk)) return (int)cudaErrorInvalidValue;
    ConvArgs a{};
    a.in = (const __nv_bfloat16*)in;
    a.out = (__nv_bfloat16*)out;
    a.bias = bias;
    a.in_mb = in_mb;
    a.out_mb = out_mb;
    a.out_ld = out_ld;
    a.nmb = nmb;
    a.hin = HIN[layer];
    a.hout = HOUT[layer];
    a.stride = STRIDE[layer];
    a.err = err;
    const long long rows = (long long)nmb * a.hout * a.hout;
    const int ntiles = (int)((rows + 127) / 128);
    const char* gv = getenv("RIV_CONV_GATHER");  // read per call: a test switches it between calls
    if (cin == 32 && !(gv && gv[0] == '1')) {
        CUtensorMap tin;
        if (!make_im2col_map(&tin, in, a.hin, in_mb, nmb, a.stride)) return (int)cudaErrorInvalidValue;
        const size_t smem = ci_smem();
        cudaError_t e = cudaFuncSetAttribute(k_nn_conv_i2c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        const int cap = num_sms() * 2;
        const int grid = ntiles < cap ? ntiles : cap;
        k_nn_conv_i2c<<<grid, CI_THREADS, smem, (cudaStream_t)stream>>>(tw, tin, a);
        return (int)cudaGetLastError();
    }
    const size_t smem = cin == 2 ? ConvCfg<2>::smem() : ConvCfg<32>::smem();
    const void* fn = cin == 2 ? (const void*)k_nn_conv<2> : (const void*)k_nn_conv<32>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    // persistent CTAs: as many per SM as shared memory allows (64 TMEM columns each), at most 2
    // (288 threads of at most 96 registers each)
    int per_sm = (int)((227 * 1024) / (smem + 1024));
    per_sm = per_sm < 1 ? 1 : (per_sm > 2 ? 2 : per_sm);
    const int cap = num_sms() * per_sm;
    const int grid = ntiles < cap ? ntiles : cap;
    if (cin == 2)
        k_nn_conv<2><<<grid, CV_THREADS, smem, (cudaStream_t)stream>>>(tw, a);
    else
        k_nn_conv<32><<<grid, CV_THREADS, smem, (cudaStream_t)stream>>>(tw, a);
    return (int)cudaGetLastError();
}

// =====================================================================================
// Network input: correlation volume, predictor prior map and predictor values
// =====================================================================================
// Per MB (one 128-thread CTA): the 64x64 reference window at (x0 - 24, y0 - 24) and the 16x16
// current block, both averaged over 2x2 (rounded), coordinates clamped to the plane; the sum of
// absolute differences of the 8x8 current block against the 32x32 window at the 24x24 offsets
// (u, v) = half-resolution displacement (u - 12, v - 12) becomes channel 0, 1 - min(V, 2048) / 1024;
// channel 1 marks the offsets the seven predictor MVs round to.  The predictor MVs come from the
// previous P-frame's coded MVs around the MB (left, top, top-right, top-left, co-located, zero,
// median of the first three; absent neighbours count as zero), in half-pel units / 64, written
// to fc1's input row (columns 288 .. 303; 304 .. 319 zero).
__device__ __forceinline__ int med3(int a, int b, int c) { return max(min(a, b), min(max(a, b), c)); }

constexpr int PF_MBS = 4;               // MBs of a row per CTA
constexpr int PF_WARPS = 6, PF_THREADS = 32 * PF_WARPS;
constexpr int PF_WW = 16 * PF_MBS + 48;  // window width shared by them (full resolution)

// bf16 tensor-core product of one 16x16 A fragment and one 16x8 B fragment, f32 accumulate
// (mma.sync m16n8k16; register layouts of the PTX ISA).
__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// FRONT = false: the network input to global memory (feat, x1).  FRONT = true: the input stays
// in shared memory and conv1 (+ bias, ReLU) runs on it at once, writing its output a1
// (nmb x 144 positions x 32 channels bf16) and x1's predictor columns: the 24x24x2 input never
// goes to global memory.  conv1's reduction is 9 taps x 2 channels (k = 2 tap + channel, zero
// from k = 18), too small for a tcgen05 tile of its own, so each warp runs it with mma.sync on
// 16 output positions at a time: A rows = positions, the fragment's k pairs = one tap's two
// channels (one 32-bit word of the shared input), B = W1 (32 x 32, bf16), f32 accumulation.
template <bool FRONT>
__global__ void __launch_bounds__(PF_THREADS, 5) k_prop_input(const uint8_t* __restrict__ cur, const uint8_t* __restrict__ ref,
                                                    int W, int H, const int8_t* __restrict__ prev_coded, int mb0,
                                                    int nmb, __nv_bfloat16* __restrict__ feat,
                                                    __nv_bfloat16* __restrict__ x1,
                                                    const __nv_bfloat16* __restrict__ w1, const float* __restrict__ b1,
                                                    __nv_bfloat16* __restrict__ a1) {
    // the input, one word per pixel, behind a leading row and column of zeros (conv1's padding)
    constexpr int FP = nn::FEAT + 1, NF = FP * FP;
    __shared__ __align__(16) uint32_t F[FRONT ? PF_MBS * NF : 1];
    __shared__ __align__(16) uint32_t O[FRONT ? PF_WARPS * 16 * 16 : 1];  // per warp: 16 output rows of 64 bytes
    __shared__ __align__(16) uint32_t win[64][PF_WW / 4];   // reference window, 4 MBs wide
    __shared__ __align__(16) uint32_t R[32][PF_WW / 8 + 1];  // its 2x2 averages (+ a word of slack)
    __shared__ __align__(16) uint32_t Cb[PF_MBS][8][2];     // the current blocks' 2x2 averages
    __shared__ uint32_t mark[PF_MBS][nn::FEAT];              // per volume row: bit u = a predictor's offset
    __shared__ int ph[PF_MBS][2 * nn::NPRED];
    const int BW = W / 16, BH = H / 16;
    const int t = threadIdx.x;
    // the CTA's MBs: PF_MBS consecutive MBs of one row, starting at raster index first
    const int rows_groups = (BW + PF_MBS - 1) / PF_MBS;
    const int gi = blockIdx.x, by = gi / rows_groups, bx0 = (gi % rows_groups) * PF_MBS;
    const int nhere = min(PF_MBS, BW - bx0);
    const int first = by * BW + bx0;
    if (first + nhere <= mb0 || first >= mb0 + nmb) return;
    const int wx = bx0 * 16 - nn::WIN_OFF, wy = by * 16 - nn::WIN_OFF;
    if (wx >= 0 && wy >= 0 && wx + PF_WW <= W && wy + 64 <= H) {  // inside the frame: word loads
        for (int k = t; k < 64 * (PF_WW / 4); k += PF_THREADS) {
            const int r = k / (PF_WW / 4), c = k % (PF_WW / 4);
            win[r][c] = *(const uint32_t*)(ref + (size_t)(wy + r) * W + wx + 4 * c);
        }
    } else {  // at a border: coordinates clamped per sample
        for (int k = t; k < 64 * (PF_WW / 4); k += PF_THREADS) {
            const int r = k / (PF_WW / 4), c = k % (PF_WW / 4);
            const int yy = min(max(wy + r, 0), H - 1);
            uint32_t v = 0;
#pragma unroll
            for (int b = 0; b < 4; b++) {
                const int xx = min(max(wx + 4 * c + b, 0), W - 1);
                v |= (uint32_t)ref[(size_t)yy * W + xx] << (8 * b);
            }
            win[r][c] = v;
        }
    }
    for (int k = t; k < 64 * nhere; k += PF_THREADS) {
        const int m = k >> 6, j = (k >> 3) & 7, c = k & 7;
        const uint8_t* p = cur + (size_t)(by * 16 + 2 * j) * W + (bx0 + m) * 16 + 2 * c;
        ((uint8_t*)Cb[m])[j * 8 + c] = (uint8_t)((p[0] + p[1] + p[W] + p[W + 1] + 2) >> 2);
    }
    if (t < PF_MBS * nn::FEAT) mark[t / nn::FEAT][t % nn::FEAT] = 0u;
    __syncthreads();
    if (t < nhere) {
        const int bx = bx0 + t;
        int px[nn::NPRED] = {0}, py[nn::NPRED] = {0};
        if (prev_coded) {
            auto get = [&](int xx, int yy, int& hx, int& hy) {
                if (xx < 0 || yy < 0 || xx >= BW || yy >= BH) { hx = hy = 0; return; }
                const int8_t* c = prev_coded + 4 * ((size_t)yy * BW + xx);
                hx = 2 * c[0] + c[2];
                hy = 2 * c[1] + c[3];
            };
            get(bx - 1, by, px[0], py[0]);
            get(bx, by - 1, px[1], py[1]);
            get(bx + 1, by - 1, px[2], py[2]);
            get(bx - 1, by - 1, px[3], py[3]);
            get(bx, by, px[4], py[4]);
            px[6] = med3(px[0], px[1], px[2]);
            py[6] = med3(py[0], py[1], py[2]);
        }
        for (int k = 0; k < nn::NPRED; k++) {
            // nearest half-resolution offset of the MV (half-pel units / 4, rounded half up)
            const int u = ((px[k] + 2) >> 2) + 12, v = ((py[k] + 2) >> 2) + 12;
            if (u >= 0 && u < nn::FEAT && v >= 0 && v < nn::FEAT) atomicOr(&mark[t][v], 1u << u);
            ph[t][2 * k] = px[k];
            ph[t][2 * k + 1] = py[k];
        }
    }
    // 2x2 rounded averages of the window, four output bytes per step
    for (int k = t; k < 32 * (PF_WW / 8); k += PF_THREADS) {
        const int j = k / (PF_WW / 8), c = k % (PF_WW / 8);  // output row j, output word c
        const uint32_t a0 = win[2 * j][2 * c], a1 = win[2 * j][2 * c + 1];
        const uint32_t b0 = win[2 * j + 1][2 * c], b1 = win[2 * j + 1][2 * c + 1];
        const uint32_t M = 0x00FF00FFu;
        // pair sums of adjacent bytes in 16-bit lanes: lane 0 = bytes 0+1, lane 1 = bytes 2+3
        const uint32_t s0 = (a0 & M) + ((a0 >> 8) & M) + (b0 & M) + ((b0 >> 8) & M) + 0x00020002u;
        const uint32_t s1 = (a1 & M) + ((a1 >> 8) & M) + (b1 & M) + ((b1 >> 8) & M) + 0x00020002u;
        R[j][c] = ((s0 >> 2) & 0xFFu) | (((s0 >> 18) & 0xFFu) << 8) | (((s1 >> 2) & 0xFFu) << 16) |
                  (((s1 >> 18) & 0xFFu) << 24);
    }
    if (t < 32) R[t][PF_WW / 8] = 0u;
    if (FRONT)  // the padding row and column of each MB's input
        for (int k = t; k < PF_MBS * (2 * FP - 1); k += PF_THREADS) {
            const int m = k / (2 * FP - 1), j = k % (2 * FP - 1);
            F[m * NF + (j < FP ? j : (j - FP + 1) * FP)] = 0u;
        }
    __syncthreads();
    // the volume in blocks of 4 horizontally adjacent x 3 vertically adjacent offsets per item:
    // each reference row's words and their byte shifts (0, 8, 16, 24 bits) are loaded once and
    // serve the three offset rows that use them; the current block stays in registers
    constexpr int UB = 4, VB = 3, NUG = nn::FEAT / UB, NVG = nn::FEAT / VB;
    for (int k = t; k < nhere * NUG * NVG; k += PF_THREADS) {
        const int m = k / (NUG * NVG), kg = k % (NUG * NVG);
        const int mb = first + m;
        if (mb < mb0 || mb >= mb0 + nmb) continue;
        const int v0 = VB * (kg / NUG), u0 = UB * (kg % NUG);
        const int wq = (8 * m + u0) >> 2;  // 8 m + u0 is a multiple of 4
        uint32_t cw[8][2];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const uint2 c = *(const uint2*)Cb[m][j];
            cw[j][0] = c.x;
            cw[j][1] = c.y;
        }
        unsigned sad[VB][UB];
#pragma unroll
        for (int dv = 0; dv < VB; dv++)
#pragma unroll
            for (int q = 0; q < UB; q++) sad[dv][q] = 0u;
#pragma unroll
        for (int rr = 0; rr < 8 + VB - 1; rr++) {
            const uint32_t* row = R[v0 + rr];
            const uint32_t w0 = row[wq], w1 = row[wq + 1], w2 = row[wq + 2];
            uint32_t lo[UB], hi[UB];
            lo[0] = w0;
            hi[0] = w1;
#pragma unroll
            for (int q = 1; q < UB; q++) {
                lo[q] = __funnelshift_r(w0, w1, 8 * q);
                hi[q] = __funnelshift_r(w1, w2, 8 * q);
            }
#pragma unroll
            for (int dv = 0; dv < VB; dv++) {
                const int j = rr - dv;  // row of the current block against this reference row
                if (j < 0 || j >= 8) continue;
#pragma unroll
                for (int q = 0; q < UB; q++) sad[dv][q] += __vsadu4(lo[q], cw[j][0]) + __vsadu4(hi[q], cw[j][1]);
            }
        }
#pragma unroll
        for (int dv = 0; dv < VB; dv++) {
            const int v = v0 + dv;
            const uint32_t mk = mark[m][v] >> u0;
            uint32_t o[UB];
#pragma unroll
            for (int q = 0; q < UB; q++) {
                const float f0 = 1.0f - (float)min((int)sad[dv][q], 2048) * (1.0f / 1024.0f);
                o[q] = pack_bf16(f0, ((mk >> q) & 1u) ? 1.0f : 0.0f);
            }
            if (FRONT) {
                uint32_t* f = F + m * NF + (v + 1) * FP + u0 + 1;
#pragma unroll
                for (int q = 0; q < UB; q++) f[q] = o[q];
            } else {
                const int kk = v * nn::FEAT + u0;  // 16-byte aligned word index
                *(uint4*)(feat + (size_t)(mb - mb0) * (nn::FEAT * nn::FEAT * 2) + 2 * kk) = make_uint4(o[0], o[1], o[2], o[3]);
            }
        }
    }
    if (t < 16 * nhere) {
        const int m = t >> 4, q = t & 15, mb = first + m;
        if (mb >= mb0 && mb < mb0 + nmb) {
            const float v = q < 2 * nn::NPRED ? (float)ph[m][q] * (1.0f / 64.0f) : 0.0f;
            x1[(size_t)(mb - mb0) * nn::F1 + 288 + q] = __float2bfloat16_rn(v);
            x1[(size_t)(mb - mb0) * nn::F1 + 304 + q] = __float2bfloat16_rn(0.0f);
        }
    }
    if constexpr (FRONT) {
        __syncthreads();
        const int warp = t >> 5, lane = t & 31, g = lane >> 2, tig = lane & 3;
        // B fragments of W1 ([32 out][32 k]): k-step s, n-tile nt: (k = 16 s + 2 tig (+8), n = 8 nt + g)
        uint32_t bw[2][4][2];
#pragma unroll
        for (int ks = 0; ks < 2; ks++)
#pragma unroll
            for (int nt = 0; nt < 4; nt++) {
                const __nv_bfloat16* wr = w1 + (size_t)(8 * nt + g) * nn::K1 + 16 * ks + 2 * tig;
                bw[ks][nt][0] = __ldg((const unsigned int*)wr);
                bw[ks][nt][1] = __ldg((const unsigned int*)(wr + 8));
            }
        float bias[4][2];
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            bias[nt][0] = __ldg(b1 + 8 * nt + 2 * tig);
            bias[nt][1] = __ldg(b1 + 8 * nt + 2 * tig + 1);
        }
        uint32_t* ob = O + warp * 256;  // 16 rows x 16 words
        // the word of output position (oy, ox) at tap (ky, kx) is F[(2 oy + ky) * FP + 2 ox + kx]
        // (stride 2: only the leading padding row and column are ever read); this thread's
        // taps are tig, tig + 4 and, for tig 0, tap 8
        const int oa = (tig / 3) * FP + tig % 3, ob4 = ((tig + 4) / 3) * FP + (tig + 4) % 3, o8 = 2 * FP + 2;
        // 9 tiles of 16 positions per MB; warp w takes tiles w, w + PF_WARPS, ...
        for (int tile = warp; tile < nhere * 9; tile += PF_WARPS) {
            const int m = tile / 9, p0 = (tile % 9) * 16, mb = first + m;
            if (mb < mb0 || mb >= mb0 + nmb) continue;  // warp-uniform
            const int r0 = p0 + g, r1 = p0 + g + 8;
            const uint32_t* f0 = F + m * NF + 2 * (r0 / 12) * FP + 2 * (r0 % 12);
            const uint32_t* f1 = F + m * NF + 2 * (r1 / 12) * FP + 2 * (r1 % 12);
            const uint32_t a0[4] = {f0[oa], f1[oa], f0[ob4], f1[ob4]};
            const uint32_t a1f[4] = {tig == 0 ? f0[o8] : 0u, tig == 0 ? f1[o8] : 0u, 0u, 0u};
#pragma unroll
            for (int nt = 0; nt < 4; nt++) {
                float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                mma_bf16_16816(d, a0, bw[0][nt][0], bw[0][nt][1]);
                mma_bf16_16816(d, a1f, bw[1][nt][0], bw[1][nt][1]);
                // rows g and g + 8, channels 8 nt + 2 tig (+1): one 32-bit word each
                ob[g * 16 + 4 * nt + tig] = pack_bf16(fmaxf(d[0] + bias[nt][0], 0.0f), fmaxf(d[1] + bias[nt][1], 0.0f));
                ob[(g + 8) * 16 + 4 * nt + tig] =
                    pack_bf16(fmaxf(d[2] + bias[nt][0], 0.0f), fmaxf(d[3] + bias[nt][1], 0.0f));
            }
            __syncwarp();
            // the tile's 16 rows are 1 KB contiguous in a1: two 16-byte stores per lane
            uint4* dst = (uint4*)(a1 + ((size_t)(mb - mb0) * 144 + p0) * 32);
            const uint4* src = (const uint4*)ob;
            dst[lane] = src[lane];
            dst[lane + 32] = src[lane + 32];
            __syncwarp();
        }
    }
}

// =====================================================================================
// Training kernels
// =====================================================================================
// im2col^T of a 3x3 convolution: out[k][m] (k = tap * cin + channel, m = MB * hout^2 + position)
// for k < 9 * cin; rows 9 * cin .. kpad - 1 are zero.  One thread per (k, m) pair, m fastest.
__global__ void k_nn_im2col_t(const __nv_bfloat16* __restrict__ in, int in_mb, int cin, int hin, int hout, int stride,
                              int nmb, int kpad, __nv_bfloat16* __restrict__ out) {
    const long long M = (long long)nmb * hout * hout;
    const long long n = M * kpad;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(idx / M);
        const long long m = idx - (long long)k * M;
        __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
        if (k < 9 * cin) {
            const int tap = k / cin, c = k % cin;
            const int b = (int)(m / (hout * hout)), p = (int)(m % (hout * hout));
            const int iy = (p / hout) * stride + tap / 3 - 1, ix = (p % hout) * stride + tap % 3 - 1;
            if (iy >= 0 && iy < hin && ix >= 0 && ix < hin) v = in[(size_t)b * in_mb + ((size_t)iy * hin + ix) * cin + c];
        }
        out[idx] = v;
    }
}

// col2im of the input gradient of a 3x3 convolution (dcol: [m][kpad] f32, k = tap * 32 + channel),
// times the ReLU derivative of the input activation (act, NHWC bf16 with per-MB stride act_mb),
// written as bf16 in two layouts: dz[mi][32] (mi = MB * hin^2 + position) and dzt[32][Mi].
__global__ void k_nn_col2im(const float* __restrict__ dcol, int kpad, int hin, int hout, int stride, int nmb,
                            const __nv_bfloat16* __restrict__ act, int act_mb, __nv_bfloat16* __restrict__ dz,
                            __nv_bfloat16* __restrict__ dzt) {
    const long long Mi = (long long)nmb * hin * hin;
    const long long n = Mi * 32;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const long long mi = idx >> 5;
        const int c = (int)(idx & 31);
        const int b = (int)(mi / (hin * hin)), p = (int)(mi % (hin * hin));
        const int iy = p / hin, ix = p % hin;
        float g = 0.0f;
        for (int tap = 0; tap < 9; tap++) {
            const int ny = iy + 1 - tap / 3, nx = ix + 1 - tap % 3;  // = o * stride
            if (ny < 0 || nx < 0 || ny % stride || nx % stride) continue;
            const int oy = ny / stride, ox = nx / stride;
            if (oy >= hout || ox >= hout) continue;
            const long long m = (long long)b * hout * hout + oy * hout + ox;
            g += dcol[m * kpad + tap * 32 + c];
        }
        const float a = __bfloat162float(act[(size_t)b * act_mb + (size_t)p * 32 + c]);
        const float d = a > 0.0f ? g : 0.0f;
        dz[idx] = __float2bfloat16_rn(d);
        dzt[(size_t)c * Mi + mi] = __float2bfloat16_rn(d);
    }
}

// ReLU derivative of a layer's output: d (f32) times (act > 0) (act bf16), as bf16 rows x n (dz)
// and n x rows (dzt).  Rows come in groups of grp: row r, column c lies at
// (r / grp) * ld + (r % grp) * n + c, with ld = ldd for d and lda for act (grp = 1: plain rows).
__global__ void k_nn_relu_bwd(const float* __restrict__ d, int ldd, const __nv_bfloat16* __restrict__ act, int lda,
                              int rows, int n, int grp, __nv_bfloat16* __restrict__ dz, __nv_bfloat16* __restrict__ dzt) {
    const long long total = (long long)rows * n;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(idx / n), c = (int)(idx % n);
        const int g = r / grp, q = r - g * grp;
        const float a = __bfloat162float(act[(size_t)g * lda + (size_t)q * n + c]);
        const float v = a > 0.0f ? d[(size_t)g * ldd + (size_t)q * n + c] : 0.0f;
        dz[idx] = __float2bfloat16_rn(v);
        dzt[(size_t)c * rows + r] = __float2bfloat16_rn(v);
    }
}

// bf16 transpose: in rows x cols (pitch ld) -> out cols x rows.
__global__ void k_nn_transpose(const __nv_bfloat16* __restrict__ in, int ld, int rows, int cols,
                               __nv_bfloat16* __restrict__ out) {
    __shared__ __nv_bfloat16 tile[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int j = ty; j < 32; j += 8) {
        const int r = r0 + j, c = c0 + tx;
        if (r < rows && c < cols) tile[j][tx] = in[(size_t)r * ld + c];
    }
    __syncthreads();
    for (int j = ty; j < 32; j += 8) {
        const int c = c0 + j, r = r0 + tx;
        if (r < rows && c < cols) out[(size_t)c * rows + r] = tile[tx][j];
    }
}

// Column sums of a bf16 matrix (rows x n, pitch ld) added into out[n] (bias gradients).
__global__ void k_nn_colsum(const __nv_bfloat16* __restrict__ z, int ld, long long rows, int n, float* __restrict__ out) {
    const int c = threadIdx.x % n, lanes = blockDim.x / n;
    float acc = 0.0f;
    for (long long r = (long long)blockIdx.x * lanes + threadIdx.x / n; r < rows; r += (long long)gridDim.x * lanes)
        acc += __bfloat162float(z[r * ld + c]);
    if ((int)threadIdx.x < lanes * n) atomicAdd(out + c, acc);
}

// Loss of the head and its gradient.  o: rows x 16 f32 (fc3 output); target MV (half-pel) and
// skip flag per row.  Candidates k = 0..3 are (o[2k], o[2k+1]) * 32 half-pel; each axis error is
// a Huber loss with a one-half-pel knee; the closest candidate takes weight 1, the others 0.05;
// the skip logit o[8] a logistic loss with weight 0.5.  Mean over the rows.  dout: rows x 32
// bf16 (columns 16 .. 31 zero), doutt: 16 x rows bf16; loss_sum accumulates the summed loss.
__global__ void k_nn_head_loss(const float* __restrict__ o, const int16_t* __restrict__ tmv,
                               const uint8_t* __restrict__ tskip, int rows, __nv_bfloat16* __restrict__ dout,
                               __nv_bfloat16* __restrict__ doutt, float* __restrict__ loss_sum) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (r < rows) {
        const float* q = o + (size_t)r * 16;
        const float tx = tmv[2 * r] * (1.0f / 32.0f), ty = tmv[2 * r + 1] * (1.0f / 32.0f);
        const float dl = 1.0f / 32.0f;
        float h[4], gx[4], gy[4];
        int best = 0;
        for (int k = 0; k < 4; k++) {
            const float ex = q[2 * k] - tx, ey = q[2 * k + 1] - ty;
            const float hx = fabsf(ex) < dl ? 0.5f * ex * ex / dl : fabsf(ex) - 0.5f * dl;
            const float hy = fabsf(ey) < dl ? 0.5f * ey * ey / dl : fabsf(ey) - 0.5f * dl;
            h[k] = hx + hy;
            gx[k] = fabsf(ex) < dl ? ex / dl : (ex > 0.0f ? 1.0f : -1.0f);
            gy[k] = fabsf(ey) < dl ? ey / dl : (ey > 0.0f ? 1.0f : -1.0f);
            if (h[k] < h[best]) best = k;
        }
        const float z = q[8], y = tskip[r] ? 1.0f : 0.0f;
        const float sg = 1.0f / (1.0f + __expf(-z));
        const float bce = fmaxf(z, 0.0f) - z * y + log1pf(__expf(-fabsf(z)));
        const float inv = 1.0f / (float)rows;
        float g[16];
        for (int k = 0; k < 16; k++) g[k] = 0.0f;
        for (int k = 0; k < 4; k++) {
            const float w = k == best ? 1.0f : 0.05f;
            l += w * h[k];
            g[2 * k] = w * gx[k] * inv;
            g[2 * k + 1] = w * gy[k] * inv;
        }
        l += 0.5f * bce;
        g[8] = 0.5f * (sg - y) * inv;
        for (int k = 0; k < 16; k++) {
            dout[(size_t)r * 32 + k] = __float2bfloat16_rn(g[k]);
            dout[(size_t)r * 32 + 16 + k] = __float2bfloat16_rn(0.0f);
            doutt[(size_t)k * rows + r] = __float2bfloat16_rn(g[k]);
        }
    }
    for (int off = 16; off; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss_sum, l);
}

// AdamW over n parameters: f32 master weights p, gradients g (scaled by gscale), moments m, v;
// bf16 copy pb (nullable).  Decoupled weight decay wd (applied where decay != 0).
__global__ void k_nn_adamw(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, __nv_bfloat16* __restrict__ pb, long long n, float lr, float b1,
                           float b2, float eps, float wd, float c1, float c2, int decay) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        float w = p[i];
        if (decay) w -= lr * wd * w;
        w -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = w;
        if (pb) pb[i] = __float2bfloat16_rn(w);
    }
}

// =====================================================================================
// C ABI (device pointers; the network's training driver and tests call these)
// =====================================================================================
extern "C" {

int riv_nn_gemm(const void* A, int lda, const void* B, int ldb, void* D, int ldd, const float* bias, int M, int N,
                int K, int bk, int mode, int relu, int ksplit, int ntile, unsigned* err, void* stream) {
    return nn_gemm(A, lda, B, ldb, D, ldd, bias, M, N, K, bk, mode, relu, ksplit, ntile, err, stream);
}

int riv_nn_conv(int layer, const void* in, int in_mb, const void* W, const float* bias, void* out, int out_mb,
                int out_ld, int nmb, unsigned* err, void* stream) {
    return nn_conv(layer, in, in_mb, W, bias, out, out_mb, out_ld, nmb, err, stream);
}

static int grid_for(long long n, int per = 256) {
    long long g = (n + per - 1) / per;
    return (int)(g < 148 * 32 ? (g < 1 ? 1 : g) : 148 * 32);
}

int riv_nn_features(const uint8_t* cur_y, const uint8_t* ref_y, int W, int H, const int8_t* prev_coded, int mb0,
                    int nmb, void* feat, void* x1, void* stream) {
    if (W <= 0 || H <= 0 || W % 16 || H % 16 || nmb <= 0 || mb0 < 0 || mb0 + nmb > (W / 16) * (H / 16))
        return (int)cudaErrorInvalidValue;
    // CTAs over groups of PF_MBS MBs of a row; those outside mb0 .. mb0+nmb-1 return at once
    const int BW = W / 16, groups = (BW + PF_MBS - 1) / PF_MBS * (H / 16);
    k_prop_input<false><<<groups, PF_THREADS, 0, (cudaStream_t)stream>>>(cur_y, ref_y, W, H, prev_coded, mb0, nmb,
                                                                  (__nv_bfloat16*)feat, (__nv_bfloat16*)x1, nullptr,
                                                                  nullptr, nullptr);
    return (int)cudaGetLastError();
}

int riv_nn_front(const uint8_t* cur_y, const uint8_t* ref_y, int W, int H, const int8_t* prev_coded, int mb0, int nmb,
                 const void* w1, const float* b1, void* a1, void* x1, void* stream) {
    if (W <= 0 || H <= 0 || W % 16 || H % 16 || nmb <= 0 || mb0 < 0 || mb0 + nmb > (W / 16) * (H / 16) ||
        ((uintptr_t)a1 & 15) || ((uintptr_t)w1 & 3))
        return (int)cudaErrorInvalidValue;
    const int BW = W / 16, groups = (BW + PF_MBS - 1) / PF_MBS * (H / 16);
    k_prop_input<true><<<groups, PF_THREADS, 0, (cudaStream_t)stream>>>(cur_y, ref_y, W, H, prev_coded, mb0, nmb, nullptr,
                                                                 (__nv_bfloat16*)x1, (const __nv_bfloat16*)w1, b1,
                                                                 (__nv_bfloat16*)a1);
    return (int)cudaGetLastError();
}

int riv_nn_im2col_t(int layer, const void* in, int in_mb, int nmb, void* out, void* stream) {
    static const int HIN[5] = {0, 24, 12, 6, 6}, HOUT[5] = {0, 12, 6, 6, 3}, STRIDE[5] = {0, 2, 2, 1, 2};
    if (layer < 1 || layer > 4 || nmb <= 0) return (int)cudaErrorInvalidValue;
    const int cin = layer == 1 ? 2 : 32, kpad = layer == 1 ? nn::K1 : nn::KC;
    const long long n = (long long)nmb * HOUT[layer] * HOUT[layer] * kpad;
    k_nn_im2col_t<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)in, in_mb, cin, HIN[layer],
                                                                 HOUT[layer], STRIDE[layer], nmb, kpad,
                                                                 (__nv_bfloat16*)out);
    return (int)cudaGetLastError();
}

int riv_nn_col2im(int layer, const float* dcol, int nmb, const void* act, int act_mb, void* dz, void* dzt,
                  void* stream) {
    static const int HIN[5] = {0, 24, 12, 6, 6}, HOUT[5] = {0, 12, 6, 6, 3}, STRIDE[5] = {0, 2, 2, 1, 2};
    if (layer < 2 || layer > 4 || nmb <= 0) return (int)cudaErrorInvalidValue;
    const long long n = (long long)nmb * HIN[layer] * HIN[layer] * 32;
    k_nn_col2im<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(dcol, nn::KC, HIN[layer], HOUT[layer], STRIDE[layer], nmb,
                                                               (const __nv_bfloat16*)act, act_mb, (__nv_bfloat16*)dz,
                                                               (__nv_bfloat16*)dzt);
    return (int)cudaGetLastError();
}

int riv_nn_relu_bwd(const float* d, int ldd, const void* act, int lda, int rows, int n, int grp, void* dz, void* dzt,
                    void* stream) {
    if (grp < 1 || n <= 0 || rows <= 0) return (int)cudaErrorInvalidValue;
    k_nn_relu_bwd<<<grid_for((long long)rows * n), 256, 0, (cudaStream_t)stream>>>(
        d, ldd, (const __nv_bfloat16*)act, lda, rows, n, grp, (__nv_bfloat16*)dz, (__nv_bfloat16*)dzt);
    return (int)cudaGetLastError();
}

int riv_nn_transpose(const void* in, int ld, int rows, int cols, void* out, void* stream) {
    dim3 grid((cols + 31) / 32, (rows + 31) / 32);
    k_nn_transpose<<<grid, 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)in, ld, rows, cols,
                                                          (__nv_bfloat16*)out);
    return (int)cudaGetLastError();
}

int riv_nn_colsum(const void* z, int ld, long long rows, int n, float* out, void* stream) {
    if (n <= 0 || n > 256) return (int)cudaErrorInvalidValue;
    const int per = 256 / n * n;
    k_nn_colsum<<<grid_for(rows, per / n), per, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)z, ld, rows, n, out);
    return (int)cudaGetLastError();
}

int riv_nn_head_loss(const float* o, const int16_t* tmv, const uint8_t* tskip, int rows, void* dout, void* doutt,
                     float* loss_sum, void* stream) {
    k_nn_head_loss<<<(rows + 127) / 128, 128, 0, (cudaStream_t)stream>>>(o, tmv, tskip, rows, (__nv_bfloat16*)dout,
                                                                         (__nv_bfloat16*)doutt, loss_sum);
    return (int)cudaGetLastError();
}

int riv_nn_adamw(float* p, const float* g, float* m, float* v, void* pb, long long n, float lr, float b1, float b2,
                 float eps, float wd, int step, int decay, void* stream) {
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_nn_adamw<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, (__nv_bfloat16*)pb, n, lr, b1, b2, eps, wd,
                                                             c1, c2, decay);
    return (int)cudaGetLastError();
}

}  // extern "C"
