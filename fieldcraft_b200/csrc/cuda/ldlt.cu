// The device LDL^T's pivoted panel step (ldlt_panel.cuh on CUDA threads): one CTA per front of
// a level, each taking its next panel from where the previous one ended. The source of the
// panel is the one the CPU emulation checks against the oracle bit for bit; this file gives it
// the device's block (threads, __syncthreads) and its per-supernode state.
#include <cstdint>

#include "cuda/kernels.cuh"
#include "cuda/ldlt_panel.cuh"

namespace fc {
namespace ldlt {

struct DeviceBlock {
  __device__ int tid() const { return threadIdx.x; }
  __device__ int size() const { return blockDim.x; }
  __device__ void sync() { __syncthreads(); }
};

// One front's panel step: the front and its state (Front), where its columns start in the
// analysis' postorder (`first`, for the failing column's name), and the GEMM tasks of the update
// of its later own columns (`slots`, `nslots` of them: update_tiles for the earliest end).
struct PanelTask {
  Front front;
  int64_t first;
  fc::GemmTask *slots;
  int32_t nslots;
  int32_t s;
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

// After a level's panels, per front (one CTA each): W21 = L21 D into w21[s] (leading dimension
// m - w, for the update-matrix GEMM), then D out of the front into d / e at the front's first
// postorder column (split_d), leaving its own block unit lower for the solve.
struct AfterTask {
  Front front;
  double *w21;
  double *d, *e;
};

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

}  // namespace ldlt
}  // namespace fc
