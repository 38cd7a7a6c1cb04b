// Kernels of the learned preconditioner: a 3-level, 32-channel 3D-convolution U-Net on the node
// grid of a hex8 mesh, BF16 activations and weights with FP32 accumulation on the tensor pipe,
// and the vector kernels of flexible CG.
//
// Activations are channels-last: voxel v = x + X (y + Y z) holds C consecutive BF16 channels.
// Weights of a 3x3x3 convolution are [tap][cout][cin] BF16 (tap = dx+1 + 3 (dy+1 + 3 (dz+1))).
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace fc {
namespace unet {

struct Grid {
  int X, Y, Z;
  __host__ __device__ int64_t voxels() const { return (int64_t)X * Y * Z; }
};

// out = act(conv3x3x3(in, w) + bias) on grid g; CIN, COUT in {16, 32}. relu: the leaky ReLU
// (x for x > 0, 0.05 x otherwise). mask (optional, COUT channels): out *= (mask > 0 ? 1 : 0.05),
// the derivative of the leaky ReLU whose output is `mask`, applied to a gradient. bias may be null.
void conv3(const Grid &g, int cin, int cout, const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias,
           bool relu, const __nv_bfloat16 *mask, __nv_bfloat16 *out, cudaStream_t st);
// Weight gradient of conv3: part[chunk][tap][cout][cin] = sum over the chunk's voxels of
// dy[v][cout] in[v + tap][cin]; then gw[tap][cout][cin] = sum of the chunks in order, and
// gb[cout] = sum_v dy[v][cout]. part must hold dw_chunks(g) * 27 * cin * cout floats.
int dw_chunks(const Grid &g);
void conv3_dw(const Grid &g, int cin, int cout, const __nv_bfloat16 *in, const __nv_bfloat16 *dy, float *part,
              float *gw, float *gb, cudaStream_t st);
// Weights for the transposed convolution (the input gradient): wt[26 - tap][cin][cout] = w[tap][cout][cin].
void flip_weights(int cin, int cout, const __nv_bfloat16 *w, __nv_bfloat16 *wt, cudaStream_t st);
// FP32 master weights -> BF16 copies (n values).
void to_bf16(int64_t n, const float *src, __nv_bfloat16 *dst, cudaStream_t st);

// 2x2x2 average (sum / 8) onto the coarse grid gc (ceil halves); C = 32.
void pool(const Grid &gf, const Grid &gc, const __nv_bfloat16 *fine, __nv_bfloat16 *coarse, cudaStream_t st);
// fine = coarse(x/2, y/2, z/2) + skip; C = 32.
void up_add(const Grid &gf, const Grid &gc, const __nv_bfloat16 *coarse, const __nv_bfloat16 *skip,
            __nv_bfloat16 *fine, cudaStream_t st);
// The adjoints, times the leaky ReLU's derivative at `mask` (1 where mask > 0, else 0.05):
// coarse = sum of the 8 children of dfine (nearest upsampling); fine = dcoarse(parent) / 8 + dskip
// (average pooling plus the skip path).
void up_adjoint(const Grid &gf, const Grid &gc, const __nv_bfloat16 *dfine, const __nv_bfloat16 *mask,
                __nv_bfloat16 *dcoarse, cudaStream_t st);
void pool_adjoint(const Grid &gf, const Grid &gc, const __nv_bfloat16 *dcoarse, const __nv_bfloat16 *dskip,
                  const __nv_bfloat16 *mask, __nv_bfloat16 *dfine, cudaStream_t st);

// Between the equations' vectors and the grid: the 16 input channels of voxel v are
// (r_x, r_y, r_z) * scale[0] at the node's free DOFs (0 where held), feat[v] (a fixed feature:
// the node's log Young's modulus), and zeros. eq[3 v + a] is the equation of DOF a of node v, -1
// when held. Out: z[eq] = y[v][a] * scale[1].
void scatter_input(const Grid &g, const int64_t *eq, const double *r, const float *feat, const double *scale,
                   __nv_bfloat16 *x, cudaStream_t st);
void gather_output(const Grid &g, const int64_t *eq, const __nv_bfloat16 *y, const double *scale, double *z,
                   cudaStream_t st);
// dy[v][a] = dz[eq[3v + a]] * scale (a < 3; the other 13 channels zero), BF16.
void scatter_grad(const Grid &g, const int64_t *eq, const double *dz, const double *scale, __nv_bfloat16 *dy,
                  cudaStream_t st);

// Adam on n FP32 parameters: m = b1 m + (1 - b1) g, v = b2 v + (1 - b2) g^2,
// p -= lr (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps).
void adam(int64_t n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2, float eps, int t,
          cudaStream_t st);

// ---- vector kernels (FP64) of flexible CG, scalars on the device --------------------------------
// out[k] = sum_i a_k[i] b_k[i] for the pairs (a, b) given; a fixed-order two-pass reduction
// (partials per CTA, then one CTA), so results are the same on every run.
void dots(int64_t n, int pairs, const double *const *a, const double *const *b, double *partial, double *out,
          cudaStream_t st);
// y += alpha[0] * x (alpha on the device, sign s: y += s alpha x)
void axpy_dev(int64_t n, const double *alpha, double sign, const double *x, double *y, cudaStream_t st);
// p = z - sum_j beta_j p_j with beta_j = num[j] / den[slot[j]] (device scalars), q = A p done by
// the caller
void fcg_direction(int64_t n, int m, const double *z, const double *const *pj, const int *slot, const double *num,
                   const double *den, double *p, cudaStream_t st);
// alpha = s[0] / s[1] (0 when s[1] is 0), *den = s[1], x += alpha p, r -= alpha q
void fcg_update(int64_t n, const double *s, double *den, const double *p, const double *q, double *x, double *r,
                cudaStream_t st);
// The norms' scalars for the input scaling of the network: s[0] = sqrt(n) / ||r||,
// s[1] = ||r|| / (sqrt(n) kref); nrm2 = ||r||^2 from dots.
void input_scales(int64_t n, const double *nrm2, double kref, double *s, cudaStream_t st);

}  // namespace unet
}  // namespace fc
