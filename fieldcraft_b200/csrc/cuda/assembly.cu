// K_ff of a structured hex8 box assembled on the device (include/fieldcraft_fem.h): the element
// matrices (host/hex8.hpp, one thread per element), then every entry as the sum over the elements
// holding both its nodes in element label order (host/assembly.hpp, one thread per row), the
// host builder's operations in its order, so the values are its bits. After the solve: the motion
// of every DOF, the reactions at the held ones, and the stresses (host/stress.hpp).
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/fieldcraft_fem.h"
#include "device_buf.hpp"
#include "host/assembly.hpp"
#include "host/stress.hpp"

struct fc_fem_device {
  fc::assembly::Box box{};
  int64_t n = 0, nnz = 0, elements = 0;
  int device = 0;
  int64_t dofs = 0;  // 3 nodes
  fc::host::DeviceBuf d_ptr, d_idx, d_node, d_eq, d_ke, d_bad;
  fc::host::DeviceBuf d_corner;  // stress recovery: each element's corner values (48 doubles)
};

namespace {

__global__ void element_kernel(fc::assembly::Box box, int64_t elements, const double *__restrict__ young, double nu,
                               double *__restrict__ ke, int *__restrict__ bad) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < elements; e += (int64_t)gridDim.x * blockDim.x) {
    double x[24];
    fc::assembly::element_corners(box, e, x);
    if (!fc::hex8::stiffness(x, young[e], nu, ke + e * 576)) atomicExch(bad, 1);
  }
}

__global__ void entry_kernel(fc::assembly::Box box, int64_t n, const int64_t *__restrict__ ptr,
                             const int32_t *__restrict__ idx, const int64_t *__restrict__ node,
                             const double *__restrict__ ke, double *__restrict__ val) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = node[r / 3];
    const int a = (int)(r % 3);
    for (int64_t q = ptr[r]; q < ptr[r + 1]; ++q) {
      const int32_t col = idx[q];
      val[q] = fc::assembly::entry(box, v, a, node[col / 3], col % 3, ke);
    }
  }
}

// The reactions (zero at free DOFs) and the expanded motion over every DOF, one thread per DOF.
__global__ void reaction_kernel(fc::assembly::Box box, int64_t dofs, const int64_t *__restrict__ eq,
                                const double *__restrict__ q, const double *__restrict__ f,
                                const double *__restrict__ ke, double *__restrict__ r, double *__restrict__ u) {
  for (int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d < dofs; d += (int64_t)gridDim.x * blockDim.x) {
    if (u) u[d] = fc::assembly::expanded(eq, q, d);
    if (r) r[d] = eq[d] >= 0 ? 0.0 : fc::assembly::reaction(box, d / 3, (int)(d % 3), eq, q, f ? f[d] : 0.0, ke);
  }
}

// Stress recovery: per element its Gauss-point and corner stresses (one thread per element),
// then per node the mean over its elements and its von Mises stress (one thread per node).
__global__ void stress_element_kernel(fc::assembly::Box box, int64_t elements, const double *__restrict__ young,
                                      double nu, const double *__restrict__ u, double *__restrict__ points,
                                      double *__restrict__ corner, int *__restrict__ bad) {
  const int64_t px = box.nx + 1, py = box.ny + 1;
  const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < elements; e += (int64_t)gridDim.x * blockDim.x) {
    double x[24], ue[24], pts[48];
    fc::assembly::element_corners(box, e, x);
    const int64_t ex = e % box.nx, ey = (e / box.nx) % box.ny, ez = e / ((int64_t)box.nx * box.ny);
    for (int c = 0; c < 8; ++c) {
      const int64_t v = (ex + off[c][0]) + px * ((ey + off[c][1]) + py * (ez + off[c][2]));
      for (int a = 0; a < 3; ++a) ue[3 * c + a] = u[3 * v + a];
    }
    if (!fc::stress::element_stresses(x, young[e], nu, ue, pts, corner + e * 48)) atomicExch(bad, 1);
    if (points)
      for (int q = 0; q < 48; ++q) points[e * 48 + q] = pts[q];
  }
}

__global__ void stress_node_kernel(fc::assembly::Box box, int64_t nodes, const double *__restrict__ corner,
                                   double *__restrict__ nodal, double *__restrict__ von_mises) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nodes; v += (int64_t)gridDim.x * blockDim.x) {
    double s[6];
    fc::stress::nodal_mean(box, v, corner, s);
    if (nodal)
      for (int k = 0; k < 6; ++k) nodal[v * 6 + k] = s[k];
    if (von_mises) von_mises[v] = fc::stress::von_mises(s);
  }
}

int blocks_for(int64_t count) {
  const int64_t b = (count + 127) / 128;
  return (int)(b < 8192 ? (b > 0 ? b : 1) : 8192);
}

}  // namespace

extern "C" {

int fc_fem_device_create(int nx, int ny, int nz, double lx, double ly, double lz, int64_t n, const int64_t *ptr,
                         const int32_t *idx, const int64_t *eq, int device, fc_fem_device **out) {
  if (!out || nx <= 0 || ny <= 0 || nz <= 0 || n < 0 || n % 3 != 0 || (n > 0 && (!ptr || !idx || !eq)) ||
      !(lx > 0 && ly > 0 && lz > 0))
    return FC_FEM_INVALID;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return FC_FEM_INVALID;
  auto d = new fc_fem_device();
  d->box = {nx, ny, nz, lx, ly, lz};
  d->n = n;
  d->nnz = n > 0 ? ptr[n] : 0;
  d->elements = (int64_t)nx * ny * nz;
  d->device = device;
  const int64_t nodes = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
  d->dofs = 3 * nodes;
  std::vector<int64_t> heq(eq, eq + 3 * nodes);
  std::vector<int64_t> node(n / 3, -1), hptr(ptr, ptr + n + 1);
  std::vector<int32_t> hidx(idx, idx + d->nnz);
  bool ok = true;
  for (int64_t v = 0; v < nodes && ok; ++v) {
    const int64_t e = eq[3 * v];
    if (e < 0) continue;
    if (e % 3 != 0 || e / 3 >= n / 3 || eq[3 * v + 1] != e + 1 || eq[3 * v + 2] != e + 2) ok = false;
    else node[e / 3] = v;
  }
  for (int64_t k = 0; k < n / 3 && ok; ++k) ok = node[k] >= 0;
  for (int64_t q = 0; q < d->nnz && ok; ++q) ok = hidx[q] >= 0 && hidx[q] < n;
  if (!ok) {
    delete d;
    return FC_FEM_INVALID;
  }
  cudaStream_t st = nullptr;
  if (fc::host::upload(d->d_ptr, hptr, st) != cudaSuccess || fc::host::upload(d->d_idx, hidx, st) != cudaSuccess ||
      fc::host::upload(d->d_node, node, st) != cudaSuccess || fc::host::upload(d->d_eq, heq, st) != cudaSuccess ||
      d->d_ke.alloc(sizeof(double) * 576 * (size_t)d->elements) != cudaSuccess ||
      d->d_bad.alloc(sizeof(int)) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
    delete d;
    return FC_FEM_NOMEM;
  }
  *out = d;
  return FC_FEM_OK;
}

int fc_fem_assemble_device(fc_fem_device *d, const double *d_young, double poisson, double *d_val, void *stream) {
  if (!d || !d_young || (d->nnz > 0 && !d_val)) return FC_FEM_INVALID;
  cudaSetDevice(d->device);
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaMemsetAsync(d->d_bad.p, 0, sizeof(int), st);
  element_kernel<<<blocks_for(d->elements), 128, 0, st>>>(d->box, d->elements, d_young, poisson, d->d_ke.as<double>(),
                                                         d->d_bad.as<int>());
  entry_kernel<<<blocks_for(d->n), 128, 0, st>>>(d->box, d->n, d->d_ptr.as<int64_t>(), d->d_idx.as<int32_t>(),
                                                 d->d_node.as<int64_t>(), d->d_ke.as<double>(), d_val);
  int bad = 0;
  if (cudaMemcpyAsync(&bad, d->d_bad.p, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess)
    return FC_FEM_INVALID;
  return bad ? FC_FEM_INVALID : FC_FEM_OK;
}

int fc_fem_reactions_device(fc_fem_device *d, const double *d_q, const double *d_f, double *d_r, double *d_u,
                            void *stream) {
  if (!d || (d->n > 0 && !d_q) || (!d_r && !d_u)) return FC_FEM_INVALID;
  cudaSetDevice(d->device);
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  reaction_kernel<<<blocks_for(d->dofs), 128, 0, st>>>(d->box, d->dofs, d->d_eq.as<int64_t>(), d_q, d_f,
                                                       d->d_ke.as<double>(), d_r, d_u);
  return cudaStreamSynchronize(st) == cudaSuccess && cudaGetLastError() == cudaSuccess ? FC_FEM_OK : FC_FEM_INVALID;
}

int fc_fem_stresses_device(fc_fem_device *d, const double *d_young, double poisson, const double *d_u,
                           double *d_points, double *d_nodal, double *d_von_mises, void *stream) {
  if (!d || !d_young || !d_u) return FC_FEM_INVALID;
  cudaSetDevice(d->device);
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!d->d_corner.p && d->d_corner.alloc(sizeof(double) * 48 * (size_t)d->elements) != cudaSuccess)
    return FC_FEM_NOMEM;
  cudaMemsetAsync(d->d_bad.p, 0, sizeof(int), st);
  stress_element_kernel<<<blocks_for(d->elements), 128, 0, st>>>(d->box, d->elements, d_young, poisson, d_u, d_points,
                                                                  d->d_corner.as<double>(), d->d_bad.as<int>());
  stress_node_kernel<<<blocks_for(d->dofs / 3), 128, 0, st>>>(d->box, d->dofs / 3, d->d_corner.as<double>(), d_nodal,
                                                               d_von_mises);
  int bad = 0;
  if (cudaMemcpyAsync(&bad, d->d_bad.p, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess)
    return FC_FEM_INVALID;
  return bad ? FC_FEM_INVALID : FC_FEM_OK;
}

void fc_fem_device_free(fc_fem_device *d) {
  if (!d) return;
  cudaSetDevice(d->device);
  delete d;
}

}  // extern "C"
