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

constexpr int C = 32, CIO = 16, LAYERS = 11;
// (cin, cout, level) of each convolution, in forward order
constexpr int LAYER_CIN[LAYERS] = {CIO, C, C, C, C, C, C, C, C, C, C};
constexpr int LAYER_COUT[LAYERS] = {C, C, C, C, C, C, C, C, C, C, CIO};
constexpr int LAYER_LEVEL[LAYERS] = {0, 0, 1, 1, 2, 2, 1, 1, 0, 0, 0};

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
// alpha = s[0] / s[1] (p.r / p.q)
__global__ void ratio_kernel(const double *__restrict__ s, double *__restrict__ alpha) {
  alpha[0] = s[1] != 0.0 ? s[0] / s[1] : 0.0;
}
__global__ void copy_kernel(int64_t n, const double *__restrict__ a, double *__restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = a[i];
}
__global__ void residual_inplace_kernel(int64_t n, const double *__restrict__ b, double *__restrict__ r) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    r[i] = b[i] - r[i];
}
int blocks(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)); }

Grid coarser(const Grid &g) { return Grid{(g.X + 1) / 2, (g.Y + 1) / 2, (g.Z + 1) / 2}; }

}  // namespace

struct fc_unet {
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t n = 0;
  double kref = 1.0;
  Grid g[3];
  int64_t w_off[LAYERS], b_off[LAYERS], wb_off[LAYERS];
  int64_t params = 0, wcount = 0;
  DeviceBuf p, grad, m, v;   // FP32 parameters, gradients and Adam moments
  DeviceBuf wb, wt;          // BF16 weights and their flipped transposes
  DeviceBuf eq, feat;
  // activations (BF16, channels last)
  DeviceBuf x, a0, s0, p1, a1, s1, p2, a2, m2, u1, a3, d1, u0, a4, d0, y;
  // gradients
  DeviceBuf dy, g0a, g0b, gs0, g1a, g1b, gs1, g2a, g2b;
  DeviceBuf part;            // weight-gradient partials
  DeviceBuf scal, dotpart;   // device scalars: [0,1] input scales, [2..] dots; dot partials
  DeviceBuf tz, td, tf;      // training: network output and its difference; FP32 grid copies
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
  for (int l = 0; l < LAYERS; ++l) {
    const int64_t nw = (int64_t)27 * LAYER_CIN[l] * LAYER_COUT[l];
    fc::unet::to_bf16(nw, u->p.as<float>() + u->w_off[l], B(u->wb) + u->wb_off[l], st);
    fc::unet::flip_weights(LAYER_CIN[l], LAYER_COUT[l], B(u->wb) + u->wb_off[l], B(u->wt) + u->wb_off[l], st);
  }
  u->weights_stale = false;
}

const Grid &G(const fc_unet *u, int level) { return u->g[level]; }

void conv(fc_unet *u, int l, const DeviceBuf &in, DeviceBuf &out, bool relu) {
  fc::unet::conv3(G(u, LAYER_LEVEL[l]), LAYER_CIN[l], LAYER_COUT[l], B(in), B(u->wb) + u->wb_off[l],
                  u->p.as<float>() + u->b_off[l], relu, nullptr, B(out), u->stream);
}
// the input gradient of layer l from its output gradient: conv with the flipped weights, then
// the ReLU mask of the layer's input (mask null: no ReLU there)
void conv_t(fc_unet *u, int l, const DeviceBuf &dout, const DeviceBuf *mask, DeviceBuf &din) {
  fc::unet::conv3(G(u, LAYER_LEVEL[l]), LAYER_COUT[l], LAYER_CIN[l], B(dout), B(u->wt) + u->wb_off[l], nullptr, false,
                  mask ? B(*mask) : nullptr, B(din), u->stream);
}
void conv_dw(fc_unet *u, int l, const DeviceBuf &in, const DeviceBuf &dout) {
  fc::unet::conv3_dw(G(u, LAYER_LEVEL[l]), LAYER_CIN[l], LAYER_COUT[l], B(in), B(dout), u->part.as<float>(),
                     u->grad.as<float>() + u->w_off[l], u->grad.as<float>() + u->b_off[l], u->stream);
}

// y = net(x)
void forward(fc_unet *u) {
  refresh_weights(u);
  cudaStream_t st = u->stream;
  conv(u, 0, u->x, u->a0, true);
  conv(u, 1, u->a0, u->s0, true);
  fc::unet::pool(u->g[0], u->g[1], B(u->s0), B(u->p1), st);
  conv(u, 2, u->p1, u->a1, true);
  conv(u, 3, u->a1, u->s1, true);
  fc::unet::pool(u->g[1], u->g[2], B(u->s1), B(u->p2), st);
  conv(u, 4, u->p2, u->a2, true);
  conv(u, 5, u->a2, u->m2, true);
  fc::unet::up_add(u->g[1], u->g[2], B(u->m2), B(u->s1), B(u->u1), st);
  conv(u, 6, u->u1, u->a3, true);
  conv(u, 7, u->a3, u->d1, true);
  fc::unet::up_add(u->g[0], u->g[1], B(u->d1), B(u->s0), B(u->u0), st);
  conv(u, 8, u->u0, u->a4, true);
  conv(u, 9, u->a4, u->d0, true);
  conv(u, 10, u->d0, u->y, false);
}

// parameters' gradients from dL/dy (in u->dy), after forward() on the same input
void backward(fc_unet *u) {
  cudaStream_t st = u->stream;
  conv_dw(u, 10, u->d0, u->dy);
  conv_t(u, 10, u->dy, &u->d0, u->g0a);
  conv_dw(u, 9, u->a4, u->g0a);
  conv_t(u, 9, u->g0a, &u->a4, u->g0b);
  conv_dw(u, 8, u->u0, u->g0b);
  conv_t(u, 8, u->g0b, nullptr, u->gs0);  // dL/du0: to d1 (upsampled) and to s0 (skip)
  fc::unet::up_adjoint(u->g[0], u->g[1], B(u->gs0), B(u->d1), B(u->g1a), st);
  conv_dw(u, 7, u->a3, u->g1a);
  conv_t(u, 7, u->g1a, &u->a3, u->g1b);
  conv_dw(u, 6, u->u1, u->g1b);
  conv_t(u, 6, u->g1b, nullptr, u->gs1);  // dL/du1: to m2 and to s1
  fc::unet::up_adjoint(u->g[1], u->g[2], B(u->gs1), B(u->m2), B(u->g2a), st);
  conv_dw(u, 5, u->a2, u->g2a);
  conv_t(u, 5, u->g2a, &u->a2, u->g2b);
  conv_dw(u, 4, u->p2, u->g2b);
  conv_t(u, 4, u->g2b, nullptr, u->g2a);  // dL/dp2
  fc::unet::pool_adjoint(u->g[1], u->g[2], B(u->g2a), B(u->gs1), B(u->s1), B(u->g1a), st);  // dL/ds1
  conv_dw(u, 3, u->a1, u->g1a);
  conv_t(u, 3, u->g1a, &u->a1, u->g1b);
  conv_dw(u, 2, u->p1, u->g1b);
  conv_t(u, 2, u->g1b, nullptr, u->g1a);  // dL/dp1
  fc::unet::pool_adjoint(u->g[0], u->g[1], B(u->g1a), B(u->gs0), B(u->s0), B(u->g0a), st);  // dL/ds0
  conv_dw(u, 1, u->a0, u->g0a);
  conv_t(u, 1, u->g0a, &u->a0, u->g0b);
  conv_dw(u, 0, u->x, u->g0b);
}

double *scal(fc_unet *u, int k) { return u->scal.as<double>() + k; }

// z = M(r) on u's stream
void apply(fc_unet *u, const double *r, double *z) {
  cudaStream_t st = u->stream;
  const double *a[1] = {r}, *b[1] = {r};
  fc::unet::dots(u->n, 1, a, b, u->dotpart.as<double>(), scal(u, 2), st);
  fc::unet::input_scales(u->n, scal(u, 2), u->kref, scal(u, 0), st);
  fc::unet::scatter_input(u->g[0], u->eq.as<int64_t>(), r, u->feat.as<float>(), scal(u, 0), B(u->x), st);
  forward(u);
  cudaMemsetAsync(z, 0, sizeof(double) * (size_t)u->n, st);
  fc::unet::gather_output(u->g[0], u->eq.as<int64_t>(), B(u->y), scal(u, 0), z, st);
}

int cuda_fail(fc_status *st, cudaError_t e, const char *where) {
  set_status(st, FC_CUDA_ERROR, -1, 0, 0, std::string(where) + ": " + cudaGetErrorString(e));
  return FC_CUDA_ERROR;
}

}  // namespace

extern "C" {

int fc_unet_create(int32_t nx, int32_t ny, int32_t nz, int64_t n, const int64_t *eq, const float *feat, double kref,
                   uint64_t seed, int32_t device, fc_unet **out, fc_status *status) {
  if (!out || nx < 1 || ny < 1 || nz < 1 || n < 1 || !eq || !feat || !(kref > 0)) {
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
  u->g[0] = Grid{nx + 1, ny + 1, nz + 1};
  u->g[1] = coarser(u->g[0]);
  u->g[2] = coarser(u->g[1]);
  int64_t off = 0, woff = 0;
  size_t part = 8192;
  for (int l = 0; l < LAYERS; ++l) {
    const int64_t nw = (int64_t)27 * LAYER_CIN[l] * LAYER_COUT[l];
    u->w_off[l] = off;
    off += nw;
    u->b_off[l] = off;
    off += LAYER_COUT[l];
    u->wb_off[l] = woff;
    woff += nw;
    part = std::max(part, (size_t)fc::unet::dw_chunks(u->g[LAYER_LEVEL[l]]) * (size_t)nw);
  }
  u->params = off;
  u->wcount = woff;
  const int64_t nodes = u->g[0].voxels();
  std::vector<float> host(off, 0.f);
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> normal(0.f, 1.f);
  for (int l = 0; l < LAYERS - 1; ++l) {  // the last layer starts at zero: M(r) = 0, a loss of one
    const float sd = std::sqrt(2.f / (27.f * (l == 0 ? 4 : LAYER_CIN[l])));
    const int64_t nw = (int64_t)27 * LAYER_CIN[l] * LAYER_COUT[l];
    for (int64_t q = 0; q < nw; ++q) host[u->w_off[l] + q] = sd * normal(rng);
  }
  bool ok = u->p.alloc(sizeof(float) * off) == cudaSuccess && u->grad.alloc(sizeof(float) * off) == cudaSuccess &&
            u->m.alloc(sizeof(float) * off) == cudaSuccess && u->v.alloc(sizeof(float) * off) == cudaSuccess &&
            u->wb.alloc(sizeof(bf16) * woff) == cudaSuccess && u->wt.alloc(sizeof(bf16) * woff) == cudaSuccess &&
            u->eq.alloc(sizeof(int64_t) * 3 * nodes) == cudaSuccess &&
            u->feat.alloc(sizeof(float) * nodes) == cudaSuccess && u->part.alloc(sizeof(float) * part) == cudaSuccess &&
            u->scal.alloc(sizeof(double) * 64) == cudaSuccess &&
            u->dotpart.alloc(sizeof(double) * 8 * 512) == cudaSuccess &&
            u->tz.alloc(sizeof(double) * n) == cudaSuccess && u->td.alloc(sizeof(double) * n) == cudaSuccess;
  const Grid &g0 = u->g[0], &g1 = u->g[1], &g2 = u->g[2];
  ok = ok && alloc_bf16(u->x, g0, CIO) == cudaSuccess && alloc_bf16(u->y, g0, CIO) == cudaSuccess &&
       alloc_bf16(u->dy, g0, CIO) == cudaSuccess;
  for (DeviceBuf *b : {&u->a0, &u->s0, &u->u0, &u->a4, &u->d0, &u->g0a, &u->g0b, &u->gs0})
    ok = ok && alloc_bf16(*b, g0, C) == cudaSuccess;
  for (DeviceBuf *b : {&u->p1, &u->a1, &u->s1, &u->u1, &u->a3, &u->d1, &u->g1a, &u->g1b, &u->gs1})
    ok = ok && alloc_bf16(*b, g1, C) == cudaSuccess;
  for (DeviceBuf *b : {&u->p2, &u->a2, &u->m2, &u->g2a, &u->g2b}) ok = ok && alloc_bf16(*b, g2, C) == cudaSuccess;
  ok = ok && u->tf.alloc(sizeof(float) * (size_t)g0.voxels() * CIO) == cudaSuccess;
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
  apply(u, d_r, d_z);
  return cudaGetLastError() == cudaSuccess ? FC_OK : FC_CUDA_ERROR;
}

int fc_unet_train_step(fc_unet *u, const double *d_r, const double *d_e, const int64_t *d_ptr, const int32_t *d_idx,
                       const double *d_val, float lr, int32_t step, double *d_loss) {
  if (!u || !d_r || !d_e || step < 1 || (d_ptr && (!d_idx || !d_val))) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(u->lock);
  cudaSetDevice(u->device);
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
  fc::unet::scatter_grad(u->g[0], u->eq.as<int64_t>(), d, scal(u, 0), B(u->dy), st);
  backward(u);
  fc::unet::adam(u->params, u->p.as<float>(), u->grad.as<float>(), u->m.as<float>(), u->v.as<float>(), lr, 0.9f,
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
  double *s = sc.as<double>();  // [0] b.b [1] r.r [2] p.r [3] p.q [4] alpha [8..8+ring) z.q_j [16..16+ring) p_j.q_j
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
  while (!converged && it < max_iter) {
    // z = M(r)
    if (net)
      apply(net, r, z);
    else
      copy_kernel<<<blocks(n), 256, 0, st>>>(n, r, z);
    // p = z - sum_j (z.q_j / p_j.q_j) p_j over the stored directions
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
      // the denominators p_j.q_j were kept when each direction was made
      for (size_t j = 0; j < slot.size(); ++j)
        cudaMemcpyAsync(s + 24 + j, s + 16 + slot[j], sizeof(double), cudaMemcpyDeviceToDevice, st);
      fc::unet::fcg_direction(n, (int)slot.size(), z, pj.data(), s + 8, s + 24, p, st);
    } else {
      copy_kernel<<<blocks(n), 256, 0, st>>>(n, z, p);
    }
    fc::launch_spmv(n, d_ptr, d_idx, d_val, p, n, q, n, 1, st);
    {
      const double *a[2] = {p, p}, *b[2] = {r, q};
      fc::unet::dots(n, 2, a, b, part.as<double>(), s + 2, st);
    }
    cudaMemcpyAsync(s + 16 + (it % ring), s + 3, sizeof(double), cudaMemcpyDeviceToDevice, st);
    ratio_kernel<<<1, 1, 0, st>>>(s + 2, s + 4);
    fc::unet::axpy_dev(n, s + 4, 1.0, p, d_x, st);
    fc::unet::axpy_dev(n, s + 4, -1.0, q, r, st);
    {
      const double *a[1] = {r}, *b[1] = {r};
      fc::unet::dots(n, 1, a, b, part.as<double>(), s + 1, st);
    }
    cudaMemcpyAsync(&rr, s + 1, sizeof(double), cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(status, e, "FCG");
    ++it;
    stored = std::min(stored + 1, ring);
    converged = rr <= target;
    if (!(rr == rr)) break;  // NaN: give up on FCG
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
