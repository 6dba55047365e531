// riv_nn.h -- the motion-proposal network of the learned encode form (host-side view).
//
// Shapes (per 16x16 macroblock, NHWC bf16 activations, f32 accumulation):
//   input   24x24x2   correlation volume of the 2x-downsampled current block (8x8) against the
//                     2x-downsampled 64x64 reference window (32x32), and a predictor prior map
//   conv1   3x3 s2 p1  2 -> 32, ReLU   12x12x32
//   conv2   3x3 s2 p1 32 -> 32, ReLU    6x6x32
//   conv3   3x3 s1 p1 32 -> 32, ReLU    6x6x32
//   conv4   3x3 s2 p1 32 -> 32, ReLU    3x3x32
//   fc1     (288 + 16 predictor values + 16 zeros) = 320 -> 128, ReLU
//   fc2     128 -> 128, ReLU
//   fc3     128 -> 16: four candidate MVs (x, y; half-pel units / 32) and a skip logit
#pragma once
#include <cstddef>
#include <cstdint>

namespace nn {

constexpr int FEAT = 24;     // correlation volume side
constexpr int WIN = 64;      // reference window side (full resolution)
constexpr int WIN_OFF = 24;  // window origin relative to the MB origin (both axes)
constexpr int NPRED = 7;     // predictor MVs: left, top, top-right, top-left, temporal, zero, median
constexpr int CH = 32;       // conv channels
constexpr int K1 = 32;       // conv1 reduction (9 taps x 2 channels = 18, zero padded)
constexpr int KC = 320;      // conv2..4 reduction (9 taps x 32 channels = 288, zero padded)
constexpr int F1 = 320;      // fc1 input: conv4 output (288) + predictor values (16) + zeros (16)
constexpr int HID = 128;
constexpr int OUT = 16;

// Parameter blob (bf16 weights, f32 biases), in this order; each weight is [out][in] (K-major).
struct ParamLayout {
    static constexpr size_t w1 = 0, nw1 = (size_t)CH * K1;
    static constexpr size_t w2 = w1 + nw1, nw2 = (size_t)CH * KC;
    static constexpr size_t w3 = w2 + nw2, nw3 = (size_t)CH * KC;
    static constexpr size_t w4 = w3 + nw3, nw4 = (size_t)CH * KC;
    static constexpr size_t f1 = w4 + nw4, nf1 = (size_t)HID * F1;
    static constexpr size_t f2 = f1 + nf1, nf2 = (size_t)HID * HID;
    static constexpr size_t f3 = f2 + nf2, nf3 = (size_t)OUT * HID;
    static constexpr size_t nweights = f3 + nf3;  // bf16 elements
    // biases (f32): conv1..4 (32 each), fc1 (128), fc2 (128), fc3 (16)
    static constexpr size_t nbias = 4 * CH + 2 * HID + OUT;
};

}  // namespace nn

// Launchers (riv_nn.cu).  All pointers are device pointers; `stream` is a cudaStream_t.
// GEMM: D[M, N] = A[M, K] . B[N, K]^T, A and B bf16 row-major with K contiguous (lda, ldb in
// elements, multiples of 8), f32 accumulation in tensor memory.  bk: 64 (128-byte rows) or 32.
// mode 0: D f32 (+ bias, relu); 1: atomicAdd into D f32 (split over the reduction: ksplit
// CTAs along it); 2: D bf16 (+ bias, relu).  N a multiple of 16; ntile columns per CTA (<= 256).
int nn_gemm(const void* A, int lda, const void* B, int ldb, void* D, int ldd, const float* bias, int M, int N, int K,
            int bk, int mode, int relu, int ksplit, int ntile, unsigned* err, void* stream);
// Implicit-GEMM 3x3 convolution + bias + ReLU over nmb MBs (layer 1..4 geometry above): in and
// out NHWC bf16 with per-MB strides in_mb / out_mb elements and out_ld elements between output
// positions; W [32][K] bf16.
int nn_conv(int layer, const void* in, int in_mb, const void* W, const float* bias, void* out, int out_mb, int out_ld,
            int nmb, unsigned* err, void* stream);
