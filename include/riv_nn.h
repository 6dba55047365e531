/*
 * riv_nn.h -- C ABI of the motion-proposal network's device kernels (sm_100a).
 *
 * No counterpart in the reference: the reference encoder's motion search
 * (process_block_hex, reitero_encode/src/motion/scalar.rs:546-636) has no learned part.
 * These entry points let a host driver (this library's Python trainer, or any caller that
 * owns device memory) run the network's forward pass, backward pass and optimizer on its
 * own buffers.  Every pointer is a device pointer; `stream` is a cudaStream_t (NULL: the
 * legacy default stream).  They return 0 or a cudaError_t value and never synchronise.
 * `err` (device, one u32) gets bit 0 set when a bounded device wait expired.
 *
 * Network (per 16x16 macroblock, NHWC bf16 activations, f32 accumulation in tensor memory):
 *   input 24x24x2 -> conv 3x3/2 (32) -> conv 3x3/2 (32) -> conv 3x3/1 (32) -> conv 3x3/2 (32)
 *   -> fc 320->128 -> fc 128->128 -> fc 128->16 (4 candidate MVs in half-pel/32, skip logit).
 */
#ifndef RIV_NN_H
#define RIV_NN_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* D[M,N] = A[M,K] . B[N,K]^T (+ bias[N], ReLU): A, B bf16 with K contiguous (lda, ldb
 * elements, multiples of 8, 16-byte aligned bases), f32 accumulation by tcgen05.mma with
 * operands staged by TMA.  bk 64 or 32 (k-block width); mode 0: D f32, 1: atomicAdd into D
 * f32 over ksplit CTAs along K, 2: D bf16.  N a multiple of 16, ntile (<= 256) divides N. */
int riv_nn_gemm(const void* A, int lda, const void* B, int ldb, void* D, int ldd, const float* bias, int M, int N,
                int K, int bk, int mode, int relu, int ksplit, int ntile, unsigned* err, void* stream);
/* Convolution layer 1..4 (+ bias, ReLU) over nmb MBs as an implicit GEMM on tcgen05: in/out
 * NHWC bf16 with in_mb / out_mb elements per MB and out_ld elements per output position;
 * W [32][K] bf16 (K = 32 for layer 1, 320 otherwise; k = tap * channels + channel). */
int riv_nn_conv(int layer, const void* in, int in_mb, const void* W, const float* bias, void* out, int out_mb,
                int out_ld, int nmb, unsigned* err, void* stream);
/* Network input of MBs mb0 .. mb0+nmb-1 of a W x H luma frame: correlation volume and predictor
 * prior map (feat: nmb x 24 x 24 x 2 bf16) and the predictor values (columns 288..319 of the
 * nmb x 320 bf16 fc1 input x1), from the current and reference luma planes and the previous
 * P-frame's coded MVs (4 x i8 per MB, NULL when there is none). */
int riv_nn_features(const uint8_t* cur_y, const uint8_t* ref_y, int W, int H, const int8_t* prev_coded, int mb0,
                    int nmb, void* feat, void* x1, void* stream);
/* Inference front end: the network input of riv_nn_features kept on chip and conv1 (+ bias b1,
 * ReLU) applied to it at once: a1 = nmb x 144 x 32 bf16 (conv1's output, 16-byte aligned), x1's
 * predictor columns as riv_nn_features writes them; w1 = conv1's [32][32] bf16 weights.  The
 * same function as riv_nn_features followed by riv_nn_conv(1, ...) up to the order of the f32
 * accumulation. */
int riv_nn_front(const uint8_t* cur_y, const uint8_t* ref_y, int W, int H, const int8_t* prev_coded, int mb0, int nmb,
                 const void* w1, const float* b1, void* a1, void* x1, void* stream);
/* Training: im2col^T of layer `layer`'s input (K x nmb*positions bf16). */
int riv_nn_im2col_t(int layer, const void* in, int in_mb, int nmb, void* out, void* stream);
/* Training: col2im of layer `layer`'s input gradient (f32 [positions][320]) times the ReLU
 * derivative of that input (act), as bf16 in row (dz) and transposed (dzt) layout. */
int riv_nn_col2im(int layer, const float* dcol, int nmb, const void* act, int act_mb, void* dz, void* dzt,
                  void* stream);
/* Training: d (f32) times (act > 0) as bf16 rows x n (dz) and n x rows (dzt); rows in groups of
 * grp at pitches ldd / lda. */
int riv_nn_relu_bwd(const float* d, int ldd, const void* act, int lda, int rows, int n, int grp, void* dz, void* dzt,
                    void* stream);
/* bf16 transpose rows x cols (pitch ld) -> cols x rows. */
int riv_nn_transpose(const void* in, int ld, int rows, int cols, void* out, void* stream);
/* Column sums of a bf16 matrix added into out[n] (bias gradients). */
int riv_nn_colsum(const void* z, int ld, long long rows, int n, float* out, void* stream);
/* Training: the head's loss (summed into *loss_sum) and its gradient (dout rows x 32 bf16,
 * doutt 16 x rows bf16) from the fc3 output o (rows x 16 f32), target MVs (half-pel, i16
 * pairs) and target skip flags. */
int riv_nn_head_loss(const float* o, const int16_t* tmv, const uint8_t* tskip, int rows, void* dout, void* doutt,
                     float* loss_sum, void* stream);
/* AdamW step `step` (1-based) over n f32 parameters with decoupled weight decay (decay != 0);
 * pb (nullable) receives their bf16 copy. */
int riv_nn_adamw(float* p, const float* g, float* m, float* v, void* pb, long long n, float lr, float b1, float b2,
                 float eps, float wd, int step, int decay, void* stream);

#ifdef __cplusplus
}
#endif
#endif
