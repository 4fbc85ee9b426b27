/* eemd_surrogate.h -- C ABI of the learned ensemble surrogate's kernels
 * (libeemd_surrogate.so, sm_100a).
 *
 * The surrogate maps the 8-trial ensemble-mean IMFs of a signal to its
 * 256-trial ensemble mean with a dilated 1-D convolution network.  The
 * reference has no learned component: these entry points have no counterpart
 * in it.  The plain full-ensemble EEMD (eemd_b200.h) produces the training
 * pairs and remains the fallback and the judge of the surrogate's output.
 *
 * Tensors are device pointers.  Activations are bfloat16, channels-last
 * ([batch][time][C], C = 16 or 64).  Packed weights are the bfloat16 image of
 * a K-major tensor-core operand (see eemd_sg_pack).  All calls are
 * asynchronous on `stream`.
 */
#ifndef EEMD_SURROGATE_H
#define EEMD_SURROGATE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EEMD_SG_ABI_VERSION 1

#define EEMD_SG_OK 0
#define EEMD_SG_E_BADARG -1
#define EEMD_SG_E_CUDA -5
#define EEMD_SG_E_TIMEOUT -4 /* a bounded device wait gave up (written to *err) */

int32_t eemd_sg_version(void);

/* y[b][t][n] = act(bias[n] + sum_{tap,c} x[b][t + dir*(tap-1)*dil][c] * W[n][tap][c])
 * (zero outside [0, T)).  (cin, cout) in {(16,64), (64,64), (64,16)}.
 * dir = 1: forward convolution; dir = -1 with transposed packed weights: the
 * gradient with respect to the input.  relu != 0 applies max(., 0); a
 * non-null mask ([b][t][cout] bf16) zeroes entries whose mask is not > 0
 * (the ReLU derivative).  tensor_cores = 1 runs the tcgen05 implicit GEMM,
 * 0 a CUDA-core reference kernel with identical semantics.  *err (device,
 * may be null) receives EEMD_SG_E_TIMEOUT if a tensor-core wait gives up
 * after spin_limit polls (0: default). */
int32_t eemd_sg_conv(const void* x, const void* w_packed, const float* bias, void* y, int32_t B, int32_t T,
                     int32_t cin, int32_t cout, int32_t dil, int32_t dir, int32_t relu, const void* mask,
                     int32_t tensor_cores, int32_t* err, int64_t spin_limit, void* stream);

/* Packs f32 weights w[nv][3][cv] (transpose = 0) or w[cv][3][nv]
 * (transpose = 1, the input-gradient operand) into the bf16 operand image of
 * n_rows x (3*c) (n_rows, c multiples of 16; zero padding beyond nv, cv). */
int32_t eemd_sg_pack(const float* w, void* w_packed, int32_t n_rows, int32_t c, int32_t nv, int32_t cv,
                     int32_t transpose, void* stream);

/* Accumulates dw[n][tap][c] += sum_t dy[b][t][n] * x[b][t+(tap-1)*dil][c]
 * (n < nv, c < cv) and db[n] += sum_t dy[b][t][n]; dy is [B][T][n_rows],
 * x is [B][T][c] (both bf16, n_rows, c <= 64). */
int32_t eemd_sg_wgrad(const void* dy, const void* x, float* dw, float* db, int32_t B, int32_t T, int32_t n_rows,
                      int32_t c, int32_t nv, int32_t cv, int32_t dil, void* stream);

/* Mean squared error of base + out against target over channels < cv and
 * time [margin, T - margin): adds the loss to *loss (device f32) and writes
 * d loss / d out (bf16, zero elsewhere). */
int32_t eemd_sg_loss(const void* out, const void* base, const void* target, void* dout, float* loss, int32_t B,
                     int32_t T, int32_t c, int32_t cv, int32_t margin, void* stream);

/* One Adam step (bias-corrected, step >= 1) on n f32 parameters. */
int32_t eemd_sg_adam(float* p, const float* g, float* m, float* v, int32_t n, float lr, float b1, float b2,
                     float eps, int32_t step, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* EEMD_SURROGATE_H */
