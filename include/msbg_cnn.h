/* Learned 3D CNN of the B200 pressure solver: a small per-tile network that
 * predicts the pressure (initial guess) and a per-V-cycle correction.  It has
 * no counterpart in the reference; it is judged against the FP64 CPU oracle
 * (oracle/cnn_oracle.py) and by the solves it speeds up or not.
 *
 * Network, per 16^3 tile of MG level 0 with a 1-cell halo (18^3 inputs):
 *   conv 4->16 (valid on the 18^3 box) ReLU, conv 16->16 ReLU,
 *   conv 16->16 ReLU, conv 16->1; 3^3 kernels, no biases.
 * Input channels: value / s (right-hand side or residual, s = max |value| in
 * the tile), solid mask, air (p = 0) mask, resolution level / (levels - 1).
 * The output times s / mean(a_ii over the tile's liquid cells) is the
 * pressure (or correction) of the tile's cells.
 *
 * Arithmetic: BF16 weights and activations, FP32 accumulation, on tcgen05
 * tensor cores (implicit GEMM, M = 128 cells, N = 16 channels, K = 16 per
 * kernel tap); weight gradients in FP32 on CUDA cores.  Training is Adam on
 * FP32 master weights.
 *
 * Weights: NPARAM FP32 values, layer after layer, each in [cout][cin][kz][ky][kx]
 * order (the layout of torch.nn.Conv3d weights).
 *
 * Tensors passed to the network are DEVICE pointers:
 *   feat   [n][4][18][18][18] FP32 (channel planes of the padded box, z slowest)
 *   out, target, mask  [n][16][16][16] FP32 (mask 1 = liquid cell, else 0)
 */
#ifndef MSBG_CNN_H
#define MSBG_CNN_H

#include <stdint.h>

#include "msbg_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct msbg_cnn msbg_cnn;

/* Number of weights (15984). */
int msbg_cnn_num_params(void);

/* A network on `device` with He-uniform weights from a fixed seed. */
int msbg_cnn_create(int device, msbg_cnn** out);
int msbg_cnn_destroy(msbg_cnn* net);
const char* msbg_cnn_last_error(msbg_cnn* net);

/* Host copies of the FP32 master weights (n = msbg_cnn_num_params()).  Setting
 * the weights resets the optimiser state. */
int msbg_cnn_set_weights(msbg_cnn* net, const float* w, int64_t n);
int msbg_cnn_get_weights(msbg_cnn* net, float* w, int64_t n);

/* out = net(feat) for n tiles. */
int msbg_cnn_forward(msbg_cnn* net, const float* feat, float* out, int n);

/* Loss  sum(mask * (net(feat) - target)^2) / count  and its gradient with
 * respect to the weights (kept on the device for msbg_cnn_adam_step; copied
 * to gradHost when it is not NULL). */
int msbg_cnn_loss_grad(msbg_cnn* net, const float* feat, const float* target,
                       const float* mask, int n, double count, double* loss,
                       float* gradHost);

/* One Adam step with the gradient of the last msbg_cnn_loss_grad. */
int msbg_cnn_adam_step(msbg_cnn* net, float lr, float beta1, float beta2, float eps);

/* Use `net` (NULL: none) in the pressure solves of ctx with
 * msbg_gpu_solve_params.learned > 0.  The network must outlive its use.
 * The network runs on the 16^3 tiles of MG level 0 (tiles of other sizes
 * get no prediction). */
int msbg_gpu_pressure_set_cnn(msbg_gpu_ctx* ctx, msbg_cnn* net);

/* The network's prediction of the pressure of the prepared problem (the
 * initial guess of a learned solve; 0 off the liquid and on tiles the network
 * does not cover), in the layout of msbg_gpu_pressure_download. */
int msbg_gpu_pressure_learned_guess(msbg_gpu_ctx* ctx, float* packed, int64_t n);

/* Training pairs from the last refined solve of ctx (maxRefine > 0): for up
 * to maxPairs level-0 16^3 tiles spread evenly over the grid, the features of
 * the right-hand side, the normalised FP64 solution as target and the liquid
 * mask, written to the device arrays feat / target / mask (layouts above).
 * *nPairs = pairs written. */
int msbg_gpu_pressure_training_pairs(msbg_gpu_ctx* ctx, float* feat, float* target,
                                     float* mask, int maxPairs, int* nPairs);

/* Attaches (or with NULL detaches) the network used as the per-V-cycle
 * correction of solves with (msbg_gpu_solve_params.learned & 2): from the
 * residual r' the V-cycle leaves it estimates the remaining error c, and the
 * preconditioner returns V r + omega c with the energy-optimal
 * omega = (c.r')/(c.Ac). */
int msbg_gpu_pressure_set_correction_cnn(msbg_gpu_ctx* ctx, msbg_cnn* net);

/* Training pairs of the correction network, from the last refined solve of
 * ctx: after pcgIters iterations of plain MGPCG from zero (V-cycle of p),
 * y = x_k + V(b - A x_k); features of r' = b - A y, target the normalised
 * error x* - y (x* = the refined solution, kept), liquid mask.  Same layouts
 * and tile choice as msbg_gpu_pressure_training_pairs. */
int msbg_gpu_pressure_correction_pairs(msbg_gpu_ctx* ctx, const msbg_gpu_solve_params* p,
                                       int pcgIters, float* feat, float* target, float* mask,
                                       int maxPairs, int* nPairs);

#ifdef __cplusplus
}
#endif

#endif /* MSBG_CNN_H */
