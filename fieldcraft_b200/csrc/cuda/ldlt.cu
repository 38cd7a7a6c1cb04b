// The device LDL^T's pivoted panel step (ldlt_panel.cuh on CUDA threads): one CTA per front of
// a level, each taking its next panel from where the previous one ended. The source of the
// panel is the one the CPU emulation checks against the oracle bit for bit; this file gives it
// the device's block (threads, __syncthreads) and its per-supernode state.
#include <cstdint>

#include "cuda/ldlt_launch.cuh"

namespace fc {
namespace ldlt {

struct DeviceBlock {
  __device__ int tid() const { return threadIdx.x; }
  __device__ int size() const { return blockDim.x; }
  __device__ void sync() { __syncthreads(); }
};

// Per supernode s: pos[s] is where its next panel starts (w when done), twos[s] counts its 2 x 2
// pivots. A singular column lowers *failed to its postorder index (the first failing column in
// postorder is the one reported) and ends the supernode. After the panel the CTA writes the
// update of the later own columns as GEMM tasks (C -= L_panel W^T on the lower tiles, for the
// launch that follows); the slots it does not need stay empty (M = N = K = 0: no work).
__global__ void __launch_bounds__(MAX_THREADS) ldlt_panel_kernel(const PanelTask *__restrict__ tasks,
                                                                 int32_t *__restrict__ pos,
                                                                 int32_t *__restrict__ twos,
                                                                 unsigned long long *__restrict__ failed) {
  __shared__ Shared sh;
  const PanelTask &task = tasks[blockIdx.x];
  const Front &f = task.front;
  const int c0 = pos[task.s];
  int end = f.w;
  bool ok = false;
  if (c0 < f.w) {
    DeviceBlock blk;
    int made = 0;
    end = c0;
    const int singular = panel(blk, sh, f, c0, &end, &made);
    if (singular >= 0) {
      if (threadIdx.x == 0) {
        atomicMin(failed, (unsigned long long)(task.first + singular));
        pos[task.s] = f.w;
      }
      end = f.w;
    } else {
      ok = true;
      panel_w(blk, f, c0, end);
      if (threadIdx.x == 0) twos[task.s] += made;
    }
  }
  // the update tasks (every slot written, so a finished or failed front leaves only empty ones)
  for (int q = threadIdx.x; q < task.nslots; q += blockDim.x) {
    fc::GemmTask g{};
    Tile t;
    if (ok && update_tile(f.m, f.w, end, q, t)) {
      g.C = f.F + t.i0 + (int64_t)t.j0 * f.m;
      g.c_si = 1, g.c_sj = f.m;
      g.A = f.F + t.i0 + (int64_t)c0 * f.m;
      g.a_si = 1, g.a_sk = f.m;
      g.B = f.W + (t.j0 - end);
      g.b_sj = 1, g.b_sk = f.ld_w;
      g.M = t.M, g.N = t.N, g.K = end - c0;
      g.flags = t.lower ? 1 : 0;
    } else {
      g.C = f.F, g.A = f.F, g.B = f.F;
      g.c_si = g.a_si = g.b_sj = 1;
      g.c_sj = g.a_sk = g.b_sk = 1;
    }
    task.slots[q] = g;
  }
  if (!ok) return;
  if (threadIdx.x == 0) pos[task.s] = end;
}

__global__ void __launch_bounds__(MAX_THREADS) ldlt_after_kernel(const AfterTask *__restrict__ tasks) {
  const AfterTask &task = tasks[blockIdx.x];
  DeviceBlock blk;
  if (task.front.m > task.front.w) front_w21(blk, task.front, task.w21, task.front.m - task.front.w);
  split_d(blk, task.front, task.d, task.e);
}

// y <- D^-1 y between the solve's forward and backward passes: n unknowns in postorder, R
// right-hand sides row-major; one thread per unknown (the second column of a 2 x 2 pivot idles).
__global__ void ldlt_d_inverse_kernel(int64_t n, int R, const double *__restrict__ d, const double *__restrict__ e,
                                      const int8_t *__restrict__ pivots, double *__restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    apply_d_inverse(i, R, d, e, pivots, y);
}

// Lower.scale (cholesky.rs:1392-1416): each entry's magnitude to its row's and its column's
// largest, as the bits of non-negative doubles (ordered as integers); a NaN changes nothing, as
// in f64::max. scale_bits starts at zero.
__global__ void ldlt_scale_kernel(int64_t nnz, const int64_t *__restrict__ a_src, const int32_t *__restrict__ a_row,
                                  const int32_t *__restrict__ a_col, const double *__restrict__ val,
                                  unsigned long long *__restrict__ scale_bits) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x) {
    const double v = fabs(val[a_src[q]]);
    if (isnan(v)) continue;
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    atomicMax(scale_bits + a_row[q], b);
    atomicMax(scale_bits + a_col[q], b);
  }
}

// Each supernode's pivots start as its columns in order, every one a 1 x 1 pivot.
__global__ void ldlt_reset_kernel(int64_t n, const int32_t *__restrict__ local, int32_t *__restrict__ order,
                                  int8_t *__restrict__ pivots) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    order[i] = local[i];
    pivots[i] = PIVOT_ONE;
  }
}

__global__ void __launch_bounds__(64) ldlt_inverse_kernel(const InverseTask *__restrict__ tasks) {
  const InverseTask &t = tasks[blockIdx.x];
  DeviceBlock blk;
  unit_lower_inverse(blk, t.L, t.ldl, t.nb, t.X, t.ldx);
}

__global__ void __launch_bounds__(MAX_THREADS) ldlt_permute_kernel(const PermuteTask *__restrict__ tasks) {
  const PermuteTask &t = tasks[blockIdx.x];
  DeviceBlock blk;
  permute_rows_below(blk, t.front, t.from, t.tmp);
}

namespace {
int grid_for(int64_t count, int threads) {
  const int64_t blocks = (count + threads - 1) / threads;
  return (int)(blocks < 4096 ? (blocks > 0 ? blocks : 1) : 4096);
}
}  // namespace

void launch_inverse(const InverseTask *tasks, int count, cudaStream_t st) {
  if (count > 0) ldlt_inverse_kernel<<<count, 64, 0, st>>>(tasks);
}

void launch_permute(const PermuteTask *tasks, int count, cudaStream_t st) {
  if (count > 0) ldlt_permute_kernel<<<count, MAX_THREADS, 0, st>>>(tasks);
}

void launch_panel(const PanelTask *tasks, int count, int32_t *pos, int32_t *twos, unsigned long long *failed,
                  cudaStream_t st) {
  if (count > 0) ldlt_panel_kernel<<<count, MAX_THREADS, 0, st>>>(tasks, pos, twos, failed);
}

void launch_after(const AfterTask *tasks, int count, cudaStream_t st) {
  if (count > 0) ldlt_after_kernel<<<count, MAX_THREADS, 0, st>>>(tasks);
}

void launch_scale(int64_t nnz, const int64_t *a_src, const int32_t *a_row, const int32_t *a_col, const double *val,
                  unsigned long long *scale_bits, cudaStream_t st) {
  if (nnz > 0) ldlt_scale_kernel<<<grid_for(nnz, 256), 256, 0, st>>>(nnz, a_src, a_row, a_col, val, scale_bits);
}

void launch_reset(int64_t n, const int32_t *local, int32_t *order, int8_t *pivots, cudaStream_t st) {
  if (n > 0) ldlt_reset_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, local, order, pivots);
}

void launch_d_inverse(int64_t n, int R, const double *d, const double *e, const int8_t *pivots, double *y,
                      cudaStream_t st) {
  if (n > 0) ldlt_d_inverse_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, R, d, e, pivots, y);
}

}  // namespace ldlt
}  // namespace fc
