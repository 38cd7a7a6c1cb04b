// The learned preconditioner's network (forward, backward, Adam) and flexible CG, behind the C ABI
// of include/fieldcraft_unet.h. The network's layers run on this library's own kernels
// (cuda/unet_kernels.cu); this file holds its buffers and the order of the passes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "../../include/fieldcraft_unet.h"
#include "cuda/kernels.cuh"
#include "cuda/unet_kernels.cuh"
#include "device_buf.hpp"

using fc::host::DeviceBuf;
using fc::host::set_status;
using fc::unet::Grid;
using bf16 = __nv_bfloat16;

namespace {

constexpr int C = 32, CIO = 16;
constexpr int MAX_LEVELS = 8;
constexpr int MAX_LAYERS = 4 * MAX_LEVELS - 1;

__global__ void f32_to_bf16_kernel(int64_t n, const float *__restrict__ a, bf16 *__restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = __float2bfloat16_rn(a[i]);
}
__global__ void bf16_to_f32_kernel(int64_t n, const bf16 *__restrict__ a, float *__restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = __bfloat162float(a[i]);
}
// d = z - e
__global__ void sub_kernel(int64_t n, const double *__restrict__ z, const double *__restrict__ e, double *__restrict__ d) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = z[i] - e[i];
}
// d *= 2 / s[1]; loss = s[0] / s[1] (s = {d.d, e.e}, or {d.Kd, e.r} in the energy norm)
__global__ void loss_grad_kernel(int64_t n, const double *__restrict__ s, double *__restrict__ d, double *loss) {
  const double ee = s[1] > 0.0 ? s[1] : 1.0;
  if (blockIdx.x == 0 && threadIdx.x == 0 && loss) *loss = s[0] / ee;
  const double c = 2.0 / ee;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] *= c;
}
__global__ void copy_kernel(int64_t n, const double *__restrict__ a, double *__restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = a[i];
}
// t = b - t (t holds A x)
__global__ void residual_from_kernel(int64_t n, const double *__restrict__ b, double *__restrict__ t) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    t[i] = b[i] - t[i];
}
__global__ void residual_inplace_kernel(int64_t n, const double *__restrict__ b, double *__restrict__ r) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    r[i] = b[i] - r[i];
}
// Nodal block-Jacobi: per node k (equations 3k..3k+2) the inverse of K's 3 x 3 diagonal block,
// from the rows of K (columns sorted); ok[0] is cleared for a block that is not positive definite.
__global__ void block_jacobi_kernel(int64_t nodes, const int64_t *__restrict__ ptr, const int32_t *__restrict__ idx,
                                    const double *__restrict__ val, double *__restrict__ inv, int *ok) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nodes; k += (int64_t)gridDim.x * blockDim.x) {
    double a[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int i = 0; i < 3; ++i) {
      const int64_t row = 3 * k + i;
      for (int64_t q = ptr[row]; q < ptr[row + 1]; ++q) {
        const int64_t c = idx[q] - 3 * k;
        if (c >= 0 && c < 3) a[i][c] = val[q];
      }
    }
    // the inverse by cofactors (a symmetric 3 x 3)
    const double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1], c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2],
                 c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    const double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
    double *o = inv + 9 * k;
    if (!(det > 0.0) || !(a[0][0] > 0.0)) {
      *ok = 0;
      for (int q = 0; q < 9; ++q) o[q] = 0.0;
      continue;
    }
    const double d = 1.0 / det;
    o[0] = c00 * d;
    o[1] = c01 * d;
    o[2] = c02 * d;
    o[3] = c01 * d;
    o[4] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * d;
    o[5] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) * d;
    o[6] = c02 * d;
    o[7] = o[5];
    o[8] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * d;
  }
}
// z += B r, B the nodal block-Jacobi inverse
__global__ void block_jacobi_add_kernel(int64_t nodes, const double *__restrict__ inv, const double *__restrict__ r,
                                        double *__restrict__ z) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nodes; k += (int64_t)gridDim.x * blockDim.x) {
    const double *o = inv + 9 * k;
    const double r0 = r[3 * k], r1 = r[3 * k + 1], r2 = r[3 * k + 2];
    z[3 * k] += o[0] * r0 + o[1] * r1 + o[2] * r2;
    z[3 * k + 1] += o[3] * r0 + o[4] * r1 + o[5] * r2;
    z[3 * k + 2] += o[6] * r0 + o[7] * r1 + o[8] * r2;
  }
}
// acc = first ? g s : acc + g s (FP32 gradients of a minibatch)
__global__ void accumulate_kernel(int64_t n, const float *__restrict__ g, float s, bool first, float *__restrict__ acc) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    acc[i] = first ? g[i] * s : acc[i] + g[i] * s;
}
__global__ void add_scalar_kernel(const double *__restrict__ a, double *__restrict__ acc, bool first) {
  acc[0] = first ? a[0] : acc[0] + a[0];
}

// the odd network's two passes: P = (s0, s1 / 2), M = (-s0, -s1 / 2) from s = (s0, s1)
__global__ void odd_scales_kernel(const double *__restrict__ s, double *__restrict__ P, double *__restrict__ M) {
  P[0] = s[0], P[1] = 0.5 * s[1];
  M[0] = -s[0], M[1] = -0.5 * s[1];
}
__global__ void add_kernel(int64_t n, const double *__restrict__ a, double *__restrict__ z) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    z[i] += a[i];
}
__global__ void add_f32_kernel(int64_t n, const float *__restrict__ a, float *__restrict__ z) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    z[i] += a[i];
}

int blocks(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)); }

Grid coarser(const Grid &g) { return Grid{(g.X + 1) / 2, (g.Y + 1) / 2, (g.Z + 1) / 2}; }

}  // namespace

struct fc_unet {
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t n = 0;
  double kref = 1.0;
  int levels = 3, layers = 11;
  Grid g[MAX_LEVELS];
  int lcin[MAX_LAYERS], lcout[MAX_LAYERS], llevel[MAX_LAYERS];
  int64_t w_off[MAX_LAYERS], b_off[MAX_LAYERS], wb_off[MAX_LAYERS];
  int64_t params = 0, wcount = 0;
  DeviceBuf p, grad, m, v;   // FP32 parameters, gradients and Adam moments
  DeviceBuf gacc;            // a minibatch's summed gradients
  DeviceBuf wb, wt;          // BF16 weights and their flipped transposes
  DeviceBuf eq, feat;
  // activations (BF16, channels last), per level: the (pooled) input, the two convolutions of the
  // way down (s = the skip), the way up: u = upsampled + skip, its two convolutions b, d
  DeviceBuf x, y, pin[MAX_LEVELS], a[MAX_LEVELS], s[MAX_LEVELS], u[MAX_LEVELS], b[MAX_LEVELS], d[MAX_LEVELS];
  // gradients per level
  DeviceBuf dy, ga[MAX_LEVELS], gb[MAX_LEVELS], gs[MAX_LEVELS];
  DeviceBuf part;            // weight-gradient partials
  DeviceBuf scal, dotpart;   // device scalars: [0,1] input scales, [2..] dots; dot partials
  DeviceBuf tz, td, tf;      // training: network output and its difference; FP32 grid copies
  DeviceBuf bj;              // nodal block-Jacobi inverses (9 doubles a node), added to the output
  bool has_bj = false;
  bool net_on = true;         // false: the preconditioner is the block-Jacobi part alone
  bool safeguard = true;      // FCG drops a stalling network (fc_unet_enable 2: it never does)
  // odd: M(r) = B r + (net(r) - net(-r)) / 2, so that M(-r) = -M(r) and M(0) = 0 (a part of the
  // output that does not depend on r, from the biases and the modulus channel, cancels)
  bool odd = true;
  DeviceBuf tz2, gtmp;        // the second pass's output and gradients
  int64_t last_net_iterations = 0, last_dropped = 0;
  bool weights_stale = true;
  std::mutex lock;
};

namespace {

bf16 *B(const DeviceBuf &b) { return b.as<bf16>(); }

cudaError_t alloc_bf16(DeviceBuf &b, const Grid &g, int c) { return b.alloc(sizeof(bf16) * (size_t)g.voxels() * c); }

// BF16 copies of the weights (and the flipped ones for the input gradients) after a change.
void refresh_weights(fc_unet *u) {
  if (!u->weights_stale) return;
  cudaStream_t st = u->stream;
  for (int l = 0; l < u->layers; ++l) {
    const int64_t nw = (int64_t)27 * u->lcin[l] * u->lcout[l];
    fc::unet::to_bf16(nw, u->p.as<float>() + u->w_off[l], B(u->wb) + u->wb_off[l], st);
    fc::unet::flip_weights(u->lcin[l], u->lcout[l], B(u->wb) + u->wb_off[l], B(u->wt) + u->wb_off[l], st);
  }
  u->weights_stale = false;
}

const Grid &G(const fc_unet *u, int level) { return u->g[level]; }

void conv(fc_unet *u, int l, const DeviceBuf &in, DeviceBuf &out, bool relu) {
  fc::unet::conv3(G(u, u->llevel[l]), u->lcin[l], u->lcout[l], B(in), B(u->wb) + u->wb_off[l],
                  u->p.as<float>() + u->b_off[l], relu, nullptr, B(out), u->stream);
}
// the input gradient of layer l from its output gradient: conv with the flipped weights, then
// the ReLU mask of the layer's input (mask null: no ReLU there)
void conv_t(fc_unet *u, int l, const DeviceBuf &dout, const DeviceBuf *mask, DeviceBuf &din) {
  fc::unet::conv3(G(u, u->llevel[l]), u->lcout[l], u->lcin[l], B(dout), B(u->wt) + u->wb_off[l], nullptr, false,
                  mask ? B(*mask) : nullptr, B(din), u->stream);
}
void conv_dw(fc_unet *u, int l, const DeviceBuf &in, const DeviceBuf &dout) {
  fc::unet::conv3_dw(G(u, u->llevel[l]), u->lcin[l], u->lcout[l], B(in), B(dout), u->part.as<float>(),
                     u->grad.as<float>() + u->w_off[l], u->grad.as<float>() + u->b_off[l], u->stream);
}

// the level's input on the way down: x at the top, the pooled skip of the level above below it
const DeviceBuf &input_of(const fc_unet *u, int lv) { return lv == 0 ? u->x : u->pin[lv]; }
// what the level returns upwards: the bottom's second convolution, or the way up's last one
const DeviceBuf &low_of(const fc_unet *u, int lv) { return lv == u->levels - 1 ? u->s[lv] : u->d[lv]; }
DeviceBuf &low_of(fc_unet *u, int lv) { return lv == u->levels - 1 ? u->s[lv] : u->d[lv]; }

// y = net(x): per level on the way down two convolutions (the second's output is the skip) and a
// 2x2x2 average pooling, two at the bottom, per level on the way up nearest upsampling plus the
// skip and two convolutions, then the output convolution (layers in this order).
void forward(fc_unet *u) {
  refresh_weights(u);
  cudaStream_t st = u->stream;
  const int D = u->levels;
  int l = 0;
  for (int lv = 0; lv < D; ++lv) {
    conv(u, l++, input_of(u, lv), u->a[lv], true);
    conv(u, l++, u->a[lv], u->s[lv], true);
    if (lv < D - 1) fc::unet::pool(u->g[lv], u->g[lv + 1], B(u->s[lv]), B(u->pin[lv + 1]), st);
  }
  for (int lv = D - 2; lv >= 0; --lv) {
    fc::unet::up_add(u->g[lv], u->g[lv + 1], B(low_of(u, lv + 1)), B(u->s[lv]), B(u->u[lv]), st);
    conv(u, l++, u->u[lv], u->b[lv], true);
    conv(u, l++, u->b[lv], u->d[lv], true);
  }
  conv(u, l, low_of(u, 0), u->y, false);
}

// parameters' gradients from dL/dy (in u->dy), after forward() on the same input
void backward(fc_unet *u) {
  cudaStream_t st = u->stream;
  const int D = u->levels;
  int l = u->layers - 1;
  conv_dw(u, l, low_of(u, 0), u->dy);
  conv_t(u, l, u->dy, &low_of(u, 0), u->ga[0]);  // dL/d(top output), through its activation
  for (int lv = 0; lv < D - 1; ++lv) {  // the way up, from the top level to the coarsest
    l -= 2;
    conv_dw(u, l + 1, u->b[lv], u->ga[lv]);
    conv_t(u, l + 1, u->ga[lv], &u->b[lv], u->gb[lv]);
    conv_dw(u, l, u->u[lv], u->gb[lv]);
    conv_t(u, l, u->gb[lv], nullptr, u->gs[lv]);  // dL/du: to the skip and, upsampled, below
    fc::unet::up_adjoint(u->g[lv], u->g[lv + 1], B(u->gs[lv]), B(low_of(u, lv + 1)), B(u->ga[lv + 1]), st);
  }
  for (int lv = D - 1; lv >= 0; --lv) {  // the way down, from the bottom up
    l -= 2;
    conv_dw(u, l + 1, u->a[lv], u->ga[lv]);
    conv_t(u, l + 1, u->ga[lv], &u->a[lv], u->gb[lv]);
    conv_dw(u, l, input_of(u, lv), u->gb[lv]);
    if (lv == 0) break;
    conv_t(u, l, u->gb[lv], nullptr, u->ga[lv]);  // dL/d(pooled input)
    fc::unet::pool_adjoint(u->g[lv - 1], u->g[lv], B(u->ga[lv]), B(u->gs[lv - 1]), B(u->s[lv - 1]),
                           B(u->ga[lv - 1]), st);  // dL/d(skip of the level above), masked
  }
}

double *scal(fc_unet *u, int k) { return u->scal.as<double>() + k; }

// z = M(r) on u's stream. The odd network runs twice, on +r then on -r (the second pass's
// activations stay for a backward pass: scales at scal 12..13, the first's at 10..11).
void apply(fc_unet *u, const double *r, double *z) {
  cudaStream_t st = u->stream;
  const double *a[1] = {r}, *b[1] = {r};
  const int64_t *eq = u->eq.as<int64_t>();
  fc::unet::dots(u->n, 1, a, b, u->dotpart.as<double>(), scal(u, 2), st);
  fc::unet::input_scales(u->n, scal(u, 2), u->kref, scal(u, 0), st);
  cudaMemsetAsync(z, 0, sizeof(double) * (size_t)u->n, st);
  if (u->odd) {
    odd_scales_kernel<<<1, 1, 0, st>>>(scal(u, 0), scal(u, 10), scal(u, 12));
    fc::unet::scatter_input(u->g[0], eq, r, u->feat.as<float>(), scal(u, 10), B(u->x), st);
    forward(u);
    fc::unet::gather_output(u->g[0], eq, B(u->y), scal(u, 10), z, st);
    double *z2 = u->tz2.as<double>();
    cudaMemsetAsync(z2, 0, sizeof(double) * (size_t)u->n, st);
    fc::unet::scatter_input(u->g[0], eq, r, u->feat.as<float>(), scal(u, 12), B(u->x), st);
    forward(u);
    fc::unet::gather_output(u->g[0], eq, B(u->y), scal(u, 12), z2, st);
    add_kernel<<<blocks(u->n), 256, 0, st>>>(u->n, z2, z);
  } else {
    fc::unet::scatter_input(u->g[0], eq, r, u->feat.as<float>(), scal(u, 0), B(u->x), st);
    forward(u);
    fc::unet::gather_output(u->g[0], eq, B(u->y), scal(u, 0), z, st);
  }
  if (u->has_bj) block_jacobi_add_kernel<<<blocks(u->n / 3), 256, 0, st>>>(u->n / 3, u->bj.as<double>(), r, z);
}

// z = B r alone (the network left out)
void apply_jacobi(fc_unet *u, const double *r, double *z) {
  cudaMemsetAsync(z, 0, sizeof(double) * (size_t)u->n, u->stream);
  block_jacobi_add_kernel<<<blocks(u->n / 3), 256, 0, u->stream>>>(u->n / 3, u->bj.as<double>(), r, z);
}

// The loss of the pair (r, e) and its gradient into u->grad (forward and backward of the network).
void pair_gradient(fc_unet *u, const double *d_r, const double *d_e, const int64_t *d_ptr, const int32_t *d_idx,
                   const double *d_val, double *d_loss) {
  cudaStream_t st = u->stream;
  double *z = u->tz.as<double>(), *d = u->td.as<double>();
  apply(u, d_r, z);
  sub_kernel<<<blocks(u->n), 256, 0, st>>>(u->n, z, d_e, d);
  if (d_ptr) {
    // energy norm: loss = d.Kd / e.r (e.r = e.K e), dL/dz = 2 Kd / e.r
    fc::launch_spmv(u->n, d_ptr, d_idx, d_val, d, u->n, z, u->n, 1, st);
    const double *a[2] = {d, d_e}, *b[2] = {z, d_r};
    fc::unet::dots(u->n, 2, a, b, u->dotpart.as<double>(), scal(u, 4), st);
    loss_grad_kernel<<<blocks(u->n), 256, 0, st>>>(u->n, scal(u, 4), z, d_loss);
    d = z;
  } else {
    const double *a[2] = {d, d_e}, *b[2] = {d, d_e};
    fc::unet::dots(u->n, 2, a, b, u->dotpart.as<double>(), scal(u, 4), st);
    loss_grad_kernel<<<blocks(u->n), 256, 0, st>>>(u->n, scal(u, 4), d, d_loss);
  }
  const int64_t *eq = u->eq.as<int64_t>();
  if (!u->odd) {
    fc::unet::scatter_grad(u->g[0], eq, d, scal(u, 0), B(u->dy), st);
    backward(u);
    return;
  }
  // the second pass (-r) is the one whose activations are live: its gradients first, kept aside;
  // then the first pass (+r) again, forward and backward, and the two added
  fc::unet::scatter_grad(u->g[0], eq, d, scal(u, 12), B(u->dy), st);
  backward(u);
  cudaMemcpyAsync(u->gtmp.p, u->grad.p, sizeof(float) * (size_t)u->params, cudaMemcpyDeviceToDevice, st);
  fc::unet::scatter_input(u->g[0], eq, d_r, u->feat.as<float>(), scal(u, 10), B(u->x), st);
  forward(u);
  fc::unet::scatter_grad(u->g[0], eq, d, scal(u, 10), B(u->dy), st);
  backward(u);
  add_f32_kernel<<<blocks(u->params), 256, 0, st>>>(u->params, u->gtmp.as<float>(), u->grad.as<float>());
}

int cuda_fail(fc_status *st, cudaError_t e, const char *where) {
  set_status(st, FC_CUDA_ERROR, -1, 0, 0, std::string(where) + ": " + cudaGetErrorString(e));
  return FC_CUDA_ERROR;
}

}  // namespace

extern "C" {

int fc_unet_create_levels(int32_t nx, int32_t ny, int32_t nz, int64_t n, const int64_t *eq, const float *feat,
                          double kref, int32_t levels, uint64_t seed, int32_t device, fc_unet **out,
                          fc_status *status) {
  if (!out || nx < 1 || ny < 1 || nz < 1 || n < 1 || !eq || !feat || !(kref > 0) || levels < 1 ||
      levels > MAX_LEVELS) {
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "bad network arguments");
    return FC_INVALID_ARGUMENT;
  }
  *out = nullptr;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(status, e, "device");
  fc_unet *u = new fc_unet();
  u->device = device;
  u->n = n;
  u->kref = kref;
  u->levels = levels;
  u->g[0] = Grid{nx + 1, ny + 1, nz + 1};
  for (int lv = 1; lv < levels; ++lv) u->g[lv] = coarser(u->g[lv - 1]);
  // the layers in forward order: (cin, cout, level)
  int L = 0;
  for (int lv = 0; lv < levels; ++lv)
    for (int q = 0; q < 2; ++q) u->lcin[L] = (lv == 0 && q == 0) ? CIO : C, u->lcout[L] = C, u->llevel[L++] = lv;
  for (int lv = levels - 2; lv >= 0; --lv)
    for (int q = 0; q < 2; ++q) u->lcin[L] = C, u->lcout[L] = C, u->llevel[L++] = lv;
  u->lcin[L] = C, u->lcout[L] = CIO, u->llevel[L++] = 0;
  u->layers = L;
  int64_t off = 0, woff = 0;
  size_t part = 8192;
  for (int l = 0; l < L; ++l) {
    const int64_t nw = (int64_t)27 * u->lcin[l] * u->lcout[l];
    u->w_off[l] = off;
    off += nw;
    u->b_off[l] = off;
    off += u->lcout[l];
    u->wb_off[l] = woff;
    woff += nw;
    part = std::max(part, (size_t)fc::unet::dw_chunks(u->g[u->llevel[l]]) * (size_t)nw);
  }
  u->params = off;
  u->wcount = woff;
  const int64_t nodes = u->g[0].voxels();
  std::vector<float> host(off, 0.f);
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> normal(0.f, 1.f);
  for (int l = 0; l < L - 1; ++l) {  // the last layer starts at zero: M(r) = 0, a loss of one
    const float sd = std::sqrt(2.f / (27.f * (l == 0 ? 4 : u->lcin[l])));
    const int64_t nw = (int64_t)27 * u->lcin[l] * u->lcout[l];
    for (int64_t q = 0; q < nw; ++q) host[u->w_off[l] + q] = sd * normal(rng);
  }
  bool ok = u->p.alloc(sizeof(float) * off) == cudaSuccess && u->grad.alloc(sizeof(float) * off) == cudaSuccess &&
            u->m.alloc(sizeof(float) * off) == cudaSuccess && u->v.alloc(sizeof(float) * off) == cudaSuccess &&
            u->gacc.alloc(sizeof(float) * off) == cudaSuccess &&
            u->wb.alloc(sizeof(bf16) * woff) == cudaSuccess && u->wt.alloc(sizeof(bf16) * woff) == cudaSuccess &&
            u->eq.alloc(sizeof(int64_t) * 3 * nodes) == cudaSuccess &&
            u->feat.alloc(sizeof(float) * nodes) == cudaSuccess && u->part.alloc(sizeof(float) * part) == cudaSuccess &&
            u->scal.alloc(sizeof(double) * 64) == cudaSuccess &&
            u->dotpart.alloc(sizeof(double) * 8 * 512) == cudaSuccess &&
            u->tz.alloc(sizeof(double) * n) == cudaSuccess && u->td.alloc(sizeof(double) * n) == cudaSuccess &&
            u->tz2.alloc(sizeof(double) * n) == cudaSuccess && u->gtmp.alloc(sizeof(float) * off) == cudaSuccess;
  ok = ok && alloc_bf16(u->x, u->g[0], CIO) == cudaSuccess && alloc_bf16(u->y, u->g[0], CIO) == cudaSuccess &&
       alloc_bf16(u->dy, u->g[0], CIO) == cudaSuccess;
  for (int lv = 0; lv < levels && ok; ++lv) {
    const Grid &g = u->g[lv];
    for (DeviceBuf *b : {&u->a[lv], &u->s[lv], &u->ga[lv], &u->gb[lv]}) ok = ok && alloc_bf16(*b, g, C) == cudaSuccess;
    if (lv > 0) ok = ok && alloc_bf16(u->pin[lv], g, C) == cudaSuccess;
    if (lv < levels - 1)
      for (DeviceBuf *b : {&u->u[lv], &u->b[lv], &u->d[lv], &u->gs[lv]}) ok = ok && alloc_bf16(*b, g, C) == cudaSuccess;
  }
  ok = ok && u->tf.alloc(sizeof(float) * (size_t)u->g[0].voxels() * CIO) == cudaSuccess;
  if (!ok) {
    delete u;
    set_status(status, FC_OUT_OF_MEMORY, -1, 0, 0, "device memory for the network");
    return FC_OUT_OF_MEMORY;
  }
  cudaMemcpy(u->p.p, host.data(), sizeof(float) * off, cudaMemcpyHostToDevice);
  cudaMemset(u->m.p, 0, sizeof(float) * off);
  cudaMemset(u->v.p, 0, sizeof(float) * off);
  cudaMemset(u->grad.p, 0, sizeof(float) * off);
  cudaMemcpy(u->eq.p, eq, sizeof(int64_t) * 3 * nodes, cudaMemcpyHostToDevice);
  cudaMemcpy(u->feat.p, feat, sizeof(float) * nodes, cudaMemcpyHostToDevice);
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    delete u;
    return cuda_fail(status, e, "network set-up");
  }
  *out = u;
  set_status(status, FC_OK);
  return FC_OK;
}

int fc_unet_create(int32_t nx, int32_t ny, int32_t nz, int64_t n, const int64_t *eq, const float *feat, double kref,
                   uint64_t seed, int32_t device, fc_unet **out, fc_status *status) {
  return fc_unet_create_levels(nx, ny, nz, n, eq, feat, kref, 3, seed, device, out, status);
}

int fc_unet_set_operator(fc_unet *u, const int64_t *d_ptr, const int32_t *d_idx, const double *d_val) {
  if (!u || u->n % 3 != 0) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(u->lock);
  cudaSetDevice(u->device);
  if (!d_ptr) {
    u->has_bj = false;
    return FC_OK;
  }
  if (!d_idx || !d_val) return FC_INVALID_ARGUMENT;
  const int64_t nodes = u->n / 3;
  if (!u->bj.p && u->bj.alloc(sizeof(double) * 9 * (size_t)nodes) != cudaSuccess) return FC_OUT_OF_MEMORY;
  int *ok = u->scal.as<int>() + 2 * 60;  // a flag in the last scalar slots
  int one = 1;
  cudaMemcpyAsync(ok, &one, sizeof(int), cudaMemcpyHostToDevice, u->stream);
  block_jacobi_kernel<<<blocks(nodes), 256, 0, u->stream>>>(nodes, d_ptr, d_idx, d_val, u->bj.as<double>(), ok);
  cudaMemcpyAsync(&one, ok, sizeof(int), cudaMemcpyDeviceToHost, u->stream);
  if (cudaStreamSynchronize(u->stream) != cudaSuccess) return FC_CUDA_ERROR;
  u->has_bj = one != 0;
  return one ? FC_OK : FC_NOT_POSITIVE_DEFINITE;
}

int fc_unet_set_odd(fc_unet *u, int32_t odd) {
  if (!u) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(u->lock);
  u->odd = odd != 0;
  return FC_OK;
}

int fc_unet_enable(fc_unet *u, int32_t on) {
  if (!u || on < 0 || on > 2 || (!on && !u->has_bj)) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(u->lock);
  u->net_on = on != 0;
  u->safeguard = on != 2;
  return FC_OK;
}

int64_t fc_unet_stat(const fc_unet *u, int32_t what) {
  if (!u) return -1;
  switch (what) {
    case 0: return u->levels;
    case 1: return u->last_net_iterations;
    case 2: return u->last_dropped;
    case 3: return u->has_bj ? 1 : 0;
    default: return -1;
  }
}

void fc_unet_destroy(fc_unet *u) {
  if (!u) return;
  cudaSetDevice(u->device);
  if (u->stream) cudaStreamSynchronize(u->stream);
  delete u;
}

int fc_unet_set_stream(fc_unet *u, void *stream) {
  if (!u) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(u->lock);
  u->stream = static_cast<cudaStream_t>(stream);
  return FC_OK;
}

int64_t fc_unet_param_count(const fc_unet *u) { return u ? u->params : -1; }

int fc_unet_get_params(fc_unet *u, float *host) {
  if (!u || !host) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(u->lock);
  cudaSetDevice(u->device);
  cudaStreamSynchronize(u->stream);
  return cudaMemcpy(host, u->p.p, sizeof(float) * u->params, cudaMemcpyDeviceToHost) == cudaSuccess ? FC_OK
                                                                                                    : FC_CUDA_ERROR;
}

int fc_unet_set_params(fc_unet *u, const float *host) {
  if (!u || !host) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(u->lock);
  cudaSetDevice(u->device);
  cudaStreamSynchronize(u->stream);
  u->weights_stale = true;
  return cudaMemcpy(u->p.p, host, sizeof(float) * u->params, cudaMemcpyHostToDevice) == cudaSuccess ? FC_OK
                                                                                                    : FC_CUDA_ERROR;
}

int fc_unet_get_grads(fc_unet *u, float *host) {
  if (!u || !host) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(u->lock);
  cudaSetDevice(u->device);
  cudaStreamSynchronize(u->stream);
  return cudaMemcpy(host, u->grad.p, sizeof(float) * u->params, cudaMemcpyDeviceToHost) == cudaSuccess
             ? FC_OK
             : FC_CUDA_ERROR;
}

int fc_unet_forward_grid(fc_unet *u, const float *d_x, float *d_y) {
  if (!u || !d_x || !d_y) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(u->lock);
  cudaSetDevice(u->device);
  const int64_t nv = u->g[0].voxels() * CIO;
  f32_to_bf16_kernel<<<blocks(nv), 256, 0, u->stream>>>(nv, d_x, B(u->x));
  forward(u);
  bf16_to_f32_kernel<<<blocks(nv), 256, 0, u->stream>>>(nv, B(u->y), d_y);
  const cudaError_t e = cudaStreamSynchronize(u->stream);
  return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? FC_OK : FC_CUDA_ERROR;
}

int fc_unet_backward_grid(fc_unet *u, const float *d_dy) {
  if (!u || !d_dy) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(u->lock);
  cudaSetDevice(u->device);
  const int64_t nv = u->g[0].voxels() * CIO;
  f32_to_bf16_kernel<<<blocks(nv), 256, 0, u->stream>>>(nv, d_dy, B(u->dy));
  backward(u);
  const cudaError_t e = cudaStreamSynchronize(u->stream);
  return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? FC_OK : FC_CUDA_ERROR;
}

int fc_unet_apply(fc_unet *u, const double *d_r, double *d_z) {
  if (!u || !d_r || !d_z) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(u->lock);
  cudaSetDevice(u->device);
  if (u->net_on)
    apply(u, d_r, d_z);
  else
    apply_jacobi(u, d_r, d_z);
  return cudaGetLastError() == cudaSuccess ? FC_OK : FC_CUDA_ERROR;
}

int fc_unet_train_step(fc_unet *u, const double *d_r, const double *d_e, const int64_t *d_ptr, const int32_t *d_idx,
                       const double *d_val, float lr, int32_t step, double *d_loss) {
  if (!u || !d_r || !d_e || step < 1 || (d_ptr && (!d_idx || !d_val))) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(u->lock);
  cudaSetDevice(u->device);
  pair_gradient(u, d_r, d_e, d_ptr, d_idx, d_val, d_loss);
  fc::unet::adam(u->params, u->p.as<float>(), u->grad.as<float>(), u->m.as<float>(), u->v.as<float>(), lr, 0.9f,
                 0.999f, 1e-8f, step, u->stream);
  u->weights_stale = true;
  return cudaGetLastError() == cudaSuccess ? FC_OK : FC_CUDA_ERROR;
}

int fc_unet_train_batch(fc_unet *u, const double *d_r, const double *d_e, int32_t count, int64_t ld,
                        const int64_t *d_ptr, const int32_t *d_idx, const double *d_val, float lr, int32_t step,
                        double *d_loss) {
  if (!u || !d_r || !d_e || count < 1 || ld < u->n || step < 1 || (d_ptr && (!d_idx || !d_val)))
    return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(u->lock);
  cudaSetDevice(u->device);
  cudaStream_t st = u->stream;
  double *one = scal(u, 8);
  for (int32_t q = 0; q < count; ++q) {
    pair_gradient(u, d_r + (int64_t)q * ld, d_e + (int64_t)q * ld, d_ptr, d_idx, d_val, one);
    accumulate_kernel<<<blocks(u->params), 256, 0, st>>>(u->params, u->grad.as<float>(), 1.f / (float)count, q == 0,
                                                         u->gacc.as<float>());
    if (d_loss) add_scalar_kernel<<<1, 1, 0, st>>>(one, d_loss, q == 0);
  }
  fc::unet::adam(u->params, u->p.as<float>(), u->gacc.as<float>(), u->m.as<float>(), u->v.as<float>(), lr, 0.9f,
                 0.999f, 1e-8f, step, st);
  u->weights_stale = true;
  return cudaGetLastError() == cudaSuccess ? FC_OK : FC_CUDA_ERROR;
}

int fc_fcg_solve(fc_unet *net, fc_chol *fallback, int64_t n, const int64_t *d_ptr, const int32_t *d_idx,
                 const double *d_val, const double *d_b, double *d_x, double tol, int32_t max_iter, int32_t keep,
                 int32_t *iterations, double *relres, int32_t *used_fallback, fc_status *status) {
  if (iterations) *iterations = 0;
  if (used_fallback) *used_fallback = 0;
  if (n < 1 || !d_ptr || !d_idx || !d_val || !d_b || !d_x || keep < 1 || keep > 8 || max_iter < 0 ||
      (net && net->n != n)) {
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "bad solver arguments");
    return FC_INVALID_ARGUMENT;
  }
  std::unique_lock<std::mutex> guard;
  if (net) {
    guard = std::unique_lock<std::mutex>(net->lock);
    cudaSetDevice(net->device);
  }
  cudaStream_t st = net ? net->stream : nullptr;
  // vectors: r, z, q and the ring of `keep` directions p_j and A p_j
  DeviceBuf vec, sc, part;
  const int ring = keep;
  if (vec.alloc(sizeof(double) * (size_t)n * (3 + 2 * ring)) != cudaSuccess ||
      sc.alloc(sizeof(double) * 64) != cudaSuccess || part.alloc(sizeof(double) * 8 * 512) != cudaSuccess) {
    set_status(status, FC_OUT_OF_MEMORY, -1, 0, 0, "device memory for FCG");
    return FC_OUT_OF_MEMORY;
  }
  double *r = vec.as<double>(), *z = r + n, *tmp = z + n;
  std::vector<double *> P(ring), Q(ring);
  for (int j = 0; j < ring; ++j) P[j] = tmp + n * (1 + 2 * j), Q[j] = P[j] + n;
  // [0] b.b [1] r.r [2] p.r [3] p.q [5] b - A x squared [8..8+ring) z.q_j [16..16+ring) p_j.q_j
  // [32..32+CHECK) the last iterations' r.r
  double *s = sc.as<double>();
  cudaMemsetAsync(d_x, 0, sizeof(double) * n, st);
  copy_kernel<<<blocks(n), 256, 0, st>>>(n, d_b, r);
  {
    const double *a[1] = {d_b}, *b[1] = {d_b};
    fc::unet::dots(n, 1, a, b, part.as<double>(), s + 0, st);
  }
  double bb = 0.0, rr = 0.0;
  cudaMemcpyAsync(&bb, s, sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(status, e, "FCG set-up");
  const double target = tol * tol * bb;
  int it = 0, stored = 0;
  bool converged = bb == 0.0;
  // The safeguard: while the network is in use, from iteration 2 SAFE_WINDOW on, a window of
  // SAFE_WINDOW iterations that does not lower ||r||^2 by SAFE_DROP drops it for the rest of the
  // solve (the block-Jacobi part, when set, stays) and restarts from the true residual b - A x with
  // no kept directions: directions made with the network's outputs slow the rest of the solve
  // down (measured: more than 1 500 iterations after a drop at 50, against 864 for block Jacobi
  // from zero), while after a restart the rest is block-Jacobi PCG from the current x.
  constexpr int SAFE_WINDOW = 25;
  constexpr int MAX_REPLACEMENTS = 8;  // residual replacements at most (see below)
  int replacements = 0;
  constexpr double SAFE_DROP = 0.25;
  bool use_net = net != nullptr && net->net_on;
  std::vector<double> history;
  if (net) net->last_dropped = 0, net->last_net_iterations = 0;
  // ||r||^2 of each iteration lands in a ring of device scalars (s + 32 + it % CHECK); the host
  // reads them every CHECK iterations (one synchronisation per CHECK iterations), then decides on
  // convergence, the safeguard and a residual replacement in iteration order.
  constexpr int CHECK = 8;
  int since = 0;
  double ring_rr[CHECK];
  while (!converged && it < max_iter) {
    // z = M(r)
    if (use_net)
      apply(net, r, z);
    else if (net && net->has_bj)
      apply_jacobi(net, r, z);
    else
      copy_kernel<<<blocks(n), 256, 0, st>>>(n, r, z);
    // p = z - sum_j (z.q_j / p_j.q_j) p_j over the stored directions (the denominators were kept
    // in s + 16 + slot when each direction was made)
    double *p = P[it % ring], *q = Q[it % ring];
    const int m = std::min(stored, ring);
    std::vector<const double *> pj, qj, zz;
    std::vector<int> slot;
    for (int j = 0; j < m; ++j) {
      const int k = (it - 1 - j) % ring;  // the most recent first
      if (k < 0) continue;
      slot.push_back(k);
      pj.push_back(P[k]);
      qj.push_back(Q[k]);
      zz.push_back(z);
    }
    if (!slot.empty()) {
      fc::unet::dots(n, (int)slot.size(), zz.data(), qj.data(), part.as<double>(), s + 8, st);
      fc::unet::fcg_direction(n, (int)slot.size(), z, pj.data(), slot.data(), s + 8, s + 16, p, st);
    } else {
      copy_kernel<<<blocks(n), 256, 0, st>>>(n, z, p);
    }
    fc::launch_spmv(n, d_ptr, d_idx, d_val, p, n, q, n, 1, st);
    {
      const double *a[2] = {p, p}, *b[2] = {r, q};
      fc::unet::dots(n, 2, a, b, part.as<double>(), s + 2, st);
    }
    // alpha = p.r / p.q (kept as this direction's denominator), x += alpha p, r -= alpha q
    fc::unet::fcg_update(n, s + 2, s + 16 + (it % ring), p, q, d_x, r, st);
    {
      const double *a[1] = {r}, *b[1] = {r};
      fc::unet::dots(n, 1, a, b, part.as<double>(), s + 32 + (it % CHECK), st);
    }
    ++it;
    stored = std::min(stored + 1, ring);
    if (++since < CHECK && it < max_iter) continue;
    cudaMemcpyAsync(ring_rr, s + 32, sizeof(double) * CHECK, cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(status, e, "FCG");
    bool nan = false, dropped = false;
    for (int k = it - since; k < it && !converged; ++k) {
      rr = ring_rr[k % CHECK];
      if (!(rr == rr)) {
        nan = true;
        break;
      }
      converged = rr <= target;
      history.push_back(rr);
      if (use_net) {
        net->last_net_iterations = k + 1;
        const size_t h = history.size();
        if (net->safeguard && h >= 2 * SAFE_WINDOW && rr > SAFE_DROP * history[h - 1 - SAFE_WINDOW]) {
          use_net = false;
          net->last_dropped = 1;
          dropped = true;
        }
      }
    }
    since = 0;
    if (nan) break;  // NaN: give up on FCG
    if (dropped && !converged) {
      // the network is dropped: go on from the true residual with no kept directions
      fc::launch_spmv(n, d_ptr, d_idx, d_val, d_x, n, tmp, n, 1, st);
      residual_from_kernel<<<blocks(n), 256, 0, st>>>(n, d_b, tmp);
      copy_kernel<<<blocks(n), 256, 0, st>>>(n, tmp, r);
      stored = 0;
    }
    if (converged && replacements < MAX_REPLACEMENTS) {
      // the recurrence says converged: check b - A x itself; when rounding has let the two drift
      // apart, go on from the true residual (the kept directions restart)
      fc::launch_spmv(n, d_ptr, d_idx, d_val, d_x, n, tmp, n, 1, st);
      residual_from_kernel<<<blocks(n), 256, 0, st>>>(n, d_b, tmp);
      const double *a[1] = {tmp}, *b2[1] = {tmp};
      fc::unet::dots(n, 1, a, b2, part.as<double>(), s + 5, st);
      double tr = 0.0;
      cudaMemcpyAsync(&tr, s + 5, sizeof(double), cudaMemcpyDeviceToHost, st);
      e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return cuda_fail(status, e, "FCG");
      if (!(tr <= target)) {
        copy_kernel<<<blocks(n), 256, 0, st>>>(n, tmp, r);
        stored = 0;
        converged = false;
        ++replacements;
      }
    }
  }
  if (iterations) *iterations = it;
  // the true residual of the returned x
  auto true_relres = [&]() {
    fc::launch_spmv(n, d_ptr, d_idx, d_val, d_x, n, r, n, 1, st);
    residual_inplace_kernel<<<blocks(n), 256, 0, st>>>(n, d_b, r);
    const double *a[1] = {r}, *b[1] = {r};
    fc::unet::dots(n, 1, a, b, part.as<double>(), s + 1, st);
    cudaMemcpyAsync(&rr, s + 1, sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return bb > 0.0 ? std::sqrt(rr / bb) : std::sqrt(rr);
  };
  double rel = true_relres();
  if (!(rel <= tol) && fallback) {
    cudaMemcpyAsync(d_x, d_b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    cudaStreamSynchronize(st);
    fc_status cs{};
    const int rc = fc_chol_solve_device(fallback, d_x, 1, n, &cs);
    if (rc != FC_OK) {
      if (status) *status = cs;
      return rc;
    }
    if (used_fallback) *used_fallback = 1;
    rel = true_relres();
  }
  if (relres) *relres = rel;
  if (!(rel <= tol)) {
    set_status(status, FC_TIMEOUT, -1, 0, 0, "FCG did not reach the tolerance");
    return FC_TIMEOUT;
  }
  set_status(status, FC_OK);
  return FC_OK;
}

}  // extern "C"
