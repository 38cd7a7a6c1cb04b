// The device LDL^T's tasks and launchers (kernels in ldlt.cu, the panel's source in
// ldlt_panel.cuh).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "cuda/kernels.cuh"
#include "cuda/ldlt_panel.cuh"

namespace fc {
namespace ldlt {

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

// After a level's panels, per front (one CTA each): W21 = L21 D into w21 (leading dimension
// m - w, for the update-matrix GEMM), then D out of the front into d / e (split_d), leaving its
// own block unit lower.
struct AfterTask {
  Front front;
  double *w21;
  double *d, *e;
};

// The solve's 64 x 64 inverse of one unit lower diagonal block: L (leading dimension ldl, nb
// columns) into X (leading dimension ldx) in the inverse arena.
struct InverseTask {
  const double *L;
  double *X;
  int64_t ldl, ldx;
  int32_t nb, pad;
};

// A front's rows below its own columns put in the solve's order (row w + i takes old row
// w + from[i]), through `tmp` (m - w entries).
struct PermuteTask {
  Front front;
  const int32_t *from;
  double *tmp;
};

void launch_inverse(const InverseTask *tasks, int count, cudaStream_t st);
void launch_permute(const PermuteTask *tasks, int count, cudaStream_t st);
void launch_panel(const PanelTask *tasks, int count, int32_t *pos, int32_t *twos, unsigned long long *failed,
                  cudaStream_t st);
void launch_after(const AfterTask *tasks, int count, cudaStream_t st);
void launch_scale(int64_t nnz, const int64_t *a_src, const int32_t *a_row, const int32_t *a_col, const double *val,
                  unsigned long long *scale_bits, cudaStream_t st);
void launch_reset(int64_t n, const int32_t *local, int32_t *order, int8_t *pivots, cudaStream_t st);
void launch_d_inverse(int64_t n, int R, const double *d, const double *e, const int8_t *pivots, double *y,
                      cudaStream_t st);

}  // namespace ldlt
}  // namespace fc
