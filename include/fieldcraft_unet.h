/* fieldcraft_unet.h — the learned preconditioner and flexible CG (no reference counterpart).
 *
 * The reference solves K u = f by direct Cholesky only ("no iterative solver",
 * docs/linear-solvers.md:375-376). This adds the other way to reach the same relative residual:
 * flexible conjugate gradients (FCG) preconditioned by a small 3D-convolution U-Net that maps a
 * residual r to an approximation of K^-1 r, trained on the GPU on pairs (r, K^-1 r) that the
 * Cholesky solve itself produces, with the Cholesky factor as the fallback when FCG does not
 * converge. All device pointers; the network's kernels are this library's own (BF16 operands,
 * FP32 accumulation on the tensor pipe); FCG's vectors and scalars are FP64.
 *
 * The network works on the hex8 mesh's node grid (nx + 1) x (ny + 1) x (nz + 1): input channels
 * are the residual's three components at each node (zero where held) and a fixed per-node feature
 * (the log of the Young's modulus around the node, normalised); the output's first three channels
 * are the correction at each node. Architecture: a U-Net of `levels` levels (three by default;
 * 2x2x2 average pooling, nearest upsampling, additive skips), two 3x3x3 convolutions of 32
 * channels with leaky ReLU per level and side, a first convolution from 16 (4 used) channels and
 * a last one to 16 (3 used): 4 levels - 1 convolutions in all. With the operator set
 * (fc_unet_set_operator) the preconditioner is M(r) = B r + net(r), B the nodal 3 x 3 block-Jacobi
 * inverse of K, and the network learns the rest of K^-1 r. */
#ifndef FIELDCRAFT_UNET_H
#define FIELDCRAFT_UNET_H

#include <stdint.h>

#include "fieldcraft_chol.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fc_unet fc_unet;

/* A network for the node grid of an nx x ny x nz element box with n equations: eq[3 v + a] is
 * the equation of DOF a of node v (-1 when held), feat[v] the node feature; kref scales the output
 * (the ratio ||r|| / ||K^-1 r|| of typical pairs). Weights are He-initialised from `seed`, the last
 * layer's to zero. Host arrays. */
int fc_unet_create(int32_t nx, int32_t ny, int32_t nz, int64_t n, const int64_t *eq, const float *feat, double kref,
                   uint64_t seed, int32_t device, fc_unet **out, fc_status *status);
/* The same with `levels` levels (1..8); fc_unet_create is levels = 3. A deeper network reaches
 * farther across the grid (its coarsest convolutions see 2^(levels-1) times as far). */
int fc_unet_create_levels(int32_t nx, int32_t ny, int32_t nz, int64_t n, const int64_t *eq, const float *feat,
                          double kref, int32_t levels, uint64_t seed, int32_t device, fc_unet **out,
                          fc_status *status);
void fc_unet_destroy(fc_unet *net);
/* K by rows on the device (as fc_csr_spmv_device; the pointers are read here only): adds the
 * nodal block-Jacobi part B r to the preconditioner (equations node by node, three a node: n must
 * be a multiple of 3). d_ptr null removes it. FC_NOT_POSITIVE_DEFINITE when a 3 x 3 block is not. */
int fc_unet_set_operator(fc_unet *net, const int64_t *d_ptr, const int32_t *d_idx, const double *d_val);
/* odd != 0 (the default): the network part of M is (net(r) - net(-r)) / 2, two passes, so that
 * M(-r) = -M(r) and M(0) = 0 as for a linear preconditioner (a part of the output that does not
 * depend on r, from the biases and the modulus channel, cancels; training sees the same form);
 * odd = 0: net(r), one pass. */
int fc_unet_set_odd(fc_unet *net, int32_t odd);
/* on = 0: the preconditioner is the block-Jacobi part alone (the network is not run; needs the
 * operator set); on = 1 (the default): B r + net(r); on = 2: the same without FCG's safeguard. */
int fc_unet_enable(fc_unet *net, int32_t on);
/* The network's numbers: 0 levels, 1 iterations of the last fc_fcg_solve that used the network,
 * 2 whether its safeguard dropped the network, 3 whether the block-Jacobi part is set. */
int64_t fc_unet_stat(const fc_unet *net, int32_t what);
int fc_unet_set_stream(fc_unet *net, void *stream);
/* Parameters (FP32, per layer: weights [27][cout][cin] then biases [cout]) and their gradients
 * after the last backward pass, as host arrays of fc_unet_param_count values. */
int64_t fc_unet_param_count(const fc_unet *net);
int fc_unet_get_params(fc_unet *net, float *host);
int fc_unet_set_params(fc_unet *net, const float *host);
int fc_unet_get_grads(fc_unet *net, float *host);
/* The network on a grid directly (for checks against a reference implementation): x and y are
 * device FP32 arrays of voxels x 16 channels (channels last); backward takes dL/dy and leaves the
 * parameters' gradients. */
int fc_unet_forward_grid(fc_unet *net, const float *d_x, float *d_y);
int fc_unet_backward_grid(fc_unet *net, const float *d_dy);
/* z = M(r): the network applied to an equation vector (scaled by ||r|| so that M(a r) = a M(r)),
 * plus B r when the operator is set; B r alone while the network is switched off. */
int fc_unet_apply(fc_unet *net, const double *d_r, double *d_z);
/* One Adam step on one pair (r, e = K^-1 r): loss = ||M(r) - e||^2 / ||e||^2, or with K given by
 * rows (d_ptr non-null) the energy norm (M(r) - e)^T K (M(r) - e) / e^T r; written to *d_loss (a
 * device double) when not null. `step` counts from 1. */
int fc_unet_train_step(fc_unet *net, const double *d_r, const double *d_e, const int64_t *d_ptr, const int32_t *d_idx,
                       const double *d_val, float lr, int32_t step, double *d_loss);

/* One Adam step on the mean gradient of `count` pairs (column q of d_r and d_e at q * ld, ld >= n):
 * the losses as fc_unet_train_step; *d_loss gets their sum. */
int fc_unet_train_batch(fc_unet *net, const double *d_r, const double *d_e, int32_t count, int64_t ld,
                        const int64_t *d_ptr, const int32_t *d_idx, const double *d_val, float lr, int32_t step,
                        double *d_loss);
/* Flexible CG on A x = b (A by rows on the device, as fc_csr_spmv_device), x from zero, with the
 * network as preconditioner (net null: plain CG), keeping `keep` (1..8) earlier directions
 * A-orthogonal. A safeguard drops the network for the rest of the solve when, from iteration 50 on,
 * 25 iterations with it lower ||r||^2 by less than a factor 4 (the block-Jacobi part, if set,
 * stays; fc_unet_stat says whether and when) and restarts from the true residual b - A x with no
 * kept directions. Stops when ||b - A x|| <= tol ||b|| or after max_iter
 * iterations (the host reads the residuals every 8 iterations, so up to 7 more may run past the
 * one that reached it); when the recurrence's residual reaches the tolerance but b - A x itself
 * does not (rounding has let them drift apart), FCG goes on from the true residual, at most 8
 * times. Then, when not
 * converged and `fallback` (a factor of A) is given, x is the Cholesky solution and *used_fallback
 * is 1. *relres is the relative residual of the x returned (recomputed for the fallback). Returns
 * FC_TIMEOUT when neither reached the tolerance. */
int fc_fcg_solve(fc_unet *net, fc_chol *fallback, int64_t n, const int64_t *d_ptr, const int32_t *d_idx,
                 const double *d_val, const double *d_b, double *d_x, double tol, int32_t max_iter, int32_t keep,
                 int32_t *iterations, double *relres, int32_t *used_fallback, fc_status *status);

#ifdef __cplusplus
}
#endif

#endif
