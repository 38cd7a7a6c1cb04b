// The device LDL^T's pivoted panel step (ldlt_panel.cuh on CUDA threads): one CTA per front of
// a level, each taking its next panel from where the previous one ended. The source of the
// panel is the one the CPU emulation checks against the oracle bit for bit; this file gives it
// the device's block (threads, __syncthreads) and its per-supernode state.
#include <cstdint>

#include "cuda/ldlt_panel.cuh"

namespace fc {
namespace ldlt {

struct DeviceBlock {
  __device__ int tid() const { return threadIdx.x; }
  __device__ int size() const { return blockDim.x; }
  __device__ void sync() { __syncthreads(); }
};

// One front's panel step: the front and its state (Front), and where its columns start in the
// analysis' postorder (`first`, for the failing column's name).
struct PanelTask {
  Front front;
  int64_t first;
  int32_t s;
  int32_t pad;
};

// Per supernode s: pos[s] is where its next panel starts (w when done), twos[s] counts its 2 x 2
// pivots. A singular column lowers *failed to its postorder index (the first failing column in
// postorder is the one reported) and ends the supernode.
__global__ void __launch_bounds__(MAX_THREADS) ldlt_panel_kernel(const PanelTask *__restrict__ tasks,
                                                                 int32_t *__restrict__ pos,
                                                                 int32_t *__restrict__ twos,
                                                                 unsigned long long *__restrict__ failed) {
  __shared__ Shared sh;
  const PanelTask &task = tasks[blockIdx.x];
  const Front &f = task.front;
  const int c0 = pos[task.s];
  if (c0 >= f.w) return;
  DeviceBlock blk;
  int end = c0, made = 0;
  const int singular = panel(blk, sh, f, c0, &end, &made);
  if (singular >= 0) {
    if (threadIdx.x == 0) {
      atomicMin(failed, (unsigned long long)(task.first + singular));
      pos[task.s] = f.w;
    }
    return;
  }
  panel_w(blk, f, c0, end);
  if (threadIdx.x == 0) {
    pos[task.s] = end;
    twos[task.s] += made;
  }
}

}  // namespace ldlt
}  // namespace fc
