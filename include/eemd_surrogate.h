/* eemd_surrogate.h -- C ABI of the learned ensemble surrogate's kernels
 * (libeemd_surrogate.so, sm_100a).
 *
 * The surrogate maps the 8-trial ensemble-mean IMFs of a signal to its
 * 256-trial ensemble mean with a dilated 1-D convolution network.  The
 * reference has no learned component: these entry points have no counterpart
 * in it.  The plain full-ensemble EEMD (eemd_b200.h) produces the training
 * pairs and remains both the fallback and the yardstick of the surrogate's output.
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

#define EEMD_SG_ABI_VERSION 2

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
 * 2 its double-buffered form (the next tile's copies and the previous tile's
 * epilogue overlap the MMA), 3 the double-buffered form fed by bulk-tensor
 * (TMA) copies of a 3-D tensor map over x (x must be 16-byte aligned), 4
 * a warp-specialised form: a copy warp, an MMA warp and eight epilogue warps
 * on their own barriers, swizzled operands (one bulk-tensor box per tap) and
 * bulk-tensor stores of y (x, y, the packed weights and mask 16-byte
 * aligned); all four give the same results bit for bit.  0 runs a CUDA-core reference
 * kernel with identical semantics.  *err (device,
 * may be null) receives EEMD_SG_E_TIMEOUT if a tensor-core wait gives up
 * after spin_limit polls (0: default). */
int32_t eemd_sg_conv(const void* x, const void* w_packed, const float* bias, void* y, int32_t B, int32_t T,
                     int32_t cin, int32_t cout, int32_t dil, int32_t dir, int32_t relu, const void* mask,
                     int32_t tensor_cores, int32_t* err, int64_t spin_limit, void* stream);

/* Packs f32 weights w[nv][3][cv] (transpose = 0) or w[cv][3][nv]
 * (transpose = 1, the input-gradient operand) into the bf16 operand image of
 * n_rows x (3*c) (n_rows, c multiples of 16; zero padding beyond nv, cv).
 * project = 1 subtracts from each weight its mean over the forward layer's
 * output channels, so that the layer's outputs sum to zero over them. */
int32_t eemd_sg_pack(const float* w, void* w_packed, int32_t n_rows, int32_t c, int32_t nv, int32_t cv,
                     int32_t transpose, int32_t project, void* stream);

/* bias[n] = b[n] for n < nv (minus the mean of b[0..nv) when project), 0 for
 * nv <= n < n_rows (n_rows <= 1024). */
int32_t eemd_sg_bias(const float* b, float* bias, int32_t n_rows, int32_t nv, int32_t project, void* stream);

/* Accumulates dw[n][tap][c] += sum_t dy[b][t][n] * x[b][t+(tap-1)*dil][c]
 * (n < nv, c < cv) and db[n] += sum_t dy[b][t][n]; dy is [B][T][n_rows],
 * x is [B][T][c] (both bf16, n_rows, c <= 64).  tensor_cores != 0 (and n_rows
 * 16 or 64): an implicit GEMM over time on tcgen05 (accumulators in tensor
 * memory; a wait that gives up after spin_limit polls -- 0 = default -- sets
 * *err to EEMD_SG_E_TIMEOUT); otherwise the CUDA-core kernel. */
int32_t eemd_sg_wgrad(const void* dy, const void* x, float* dw, float* db, int32_t B, int32_t T, int32_t n_rows,
                      int32_t c, int32_t nv, int32_t cv, int32_t dil, int32_t tensor_cores, int32_t* err,
                      int64_t spin_limit, void* stream);

/* Mean error of base + out (base may be null) against target over channels
 * < cv and time [margin, T - margin): squared (delta <= 0) or Huber with
 * threshold delta, each channel times channel_weight[ch] (device f32 [cv],
 * may be null).  Adds the loss to *loss (device f32) and writes
 * d loss / d out (bf16, zero elsewhere).  project = 1 (c = 16) removes each
 * sample's mean over the cv channels from the gradient (the output layer is
 * packed with project = 1). */
int32_t eemd_sg_loss(const void* out, const void* base, const void* target, void* dout, float* loss, int32_t B,
                     int32_t T, int32_t c, int32_t cv, int32_t margin, int32_t project, float delta,
                     const float* channel_weight, void* stream);

/* One Adam step (bias-corrected, step >= 1) on n f32 parameters.  With
 * max_norm > 0 the gradient is first scaled to a Euclidean norm of at most
 * max_norm (work: one device float of scratch), and a step whose gradient
 * norm is not finite leaves p, m and v unchanged. */
int32_t eemd_sg_adam(float* p, const float* g, float* m, float* v, int32_t n, float lr, float b1, float b2,
                     float eps, int32_t step, float max_norm, float* work, void* stream);

/* Surrogate input and output stages over a batch of S signals of N samples
 * x[s][t] (float32).  imf_sum [S][K][N] float64 and mode_count [S][K] int32
 * are the engine's ensemble sums (eemd_run) of the small ensemble.
 *
 * eemd_sg_scale: scale[s] = RMS of x[s] (1 for a zero signal).
 * eemd_sg_prepare: network input out[s][t][C] (bf16) = (mean_0..mean_{K-1},
 *   x - sum(mean), 0...) / scale[s], mean_m = imf_sum / max(mode_count, 1),
 *   the residual summed in mode order as eemd_finalize does (K + 1 <= C <= 32,
 *   C a multiple of 8).  With imf_sum2 / mode_count2 (else null), the
 *   channels of the first decomposition minus those of the second, formed in
 *   float64 before the rounding (the training target: large-ensemble minus
 *   small-ensemble channels).
 * eemd_sg_combine: the served decomposition from the network output
 *   net_out[s][t][C], the corrections of the first P modes (P <= 6):
 *   imfs_out[s][m][t] = mean_m + scale * net_out[.., m] for m < P and mean_m
 *   beyond, resid_out[s][t] = x - sum(mean) - scale * sum_{m<P} net_out[.., m]
 *   (float64; the IMFs and the residual still sum to x), then the gate:
 *   metrics[s][4] = {||x - sum(imfs) - resid|| / ||x||, orthogonality index
 *   of the P corrected modes, orthogonality index of all K IMFs and the
 *   residual, orthogonality index of the first P small-ensemble means}
 *   (Huang et al. 1998: sum of <c_j, c_k> over pairs j != k of the
 *   components, over ||x||^2); fallback[s] = 1 when the first exceeds
 *   recon_bound or the second exceeds io_bound in magnitude (io_relative = 0)
 *   or in magnitude less the magnitude of the fourth (io_relative = 1), or
 *   any of these is not finite.  partial is device scratch of
 *   S * chunks * eemd_sg_stat_count() doubles; the chunk sums are added in a
 *   fixed order.  K must be 10. */
int32_t eemd_sg_scale(const float* x, float* scale, int32_t S, int32_t N, void* stream);
int32_t eemd_sg_prepare(const double* imf_sum, const int32_t* mode_count, const double* imf_sum2,
                        const int32_t* mode_count2, const float* x, const float* scale, void* out, int32_t S,
                        int32_t N, int32_t K, int32_t C, void* stream);
int32_t eemd_sg_combine(const double* imf_sum, const int32_t* mode_count, const float* x, const float* scale,
                        const void* net_out, double* imfs_out, double* resid_out, double* partial, int32_t chunks,
                        int32_t S, int32_t N, int32_t K, int32_t C, int32_t P, double recon_bound,
                        double io_bound, int32_t io_relative, double* metrics, int32_t* fallback,
                        void* stream);
int32_t eemd_sg_stat_count(void);

#ifdef __cplusplus
}
#endif

#endif /* EEMD_SURROGATE_H */
