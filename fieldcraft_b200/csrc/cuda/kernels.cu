// Kernels of the supernodal Cholesky on B200 (sm_100a). FP64 throughout: the dense updates run
// on the FP64 tensor pipe (DMMA, mma.sync m8n8k4 .f64 — Blackwell's tcgen05 has no FP64 kind),
// operands staged through shared memory by cp.async; the rest is SIMT.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstdio>

#include "kernels.cuh"

namespace fc {

namespace {

constexpr double PIVOT_TOLERANCE = 1e-10;  // crates/solver/src/cholesky.rs:48

__device__ __forceinline__ int lower_bound_i32(const int32_t *a, int n, int key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// D = A B + C on one 8x8x4 FP64 tile: a = A[g][tg], b = B[tg][g], c/d = C[g][2 tg + {0, 1}]
// with g = lane / 4, tg = lane % 4.
__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// ---- front assembly ----------------------------------------------------------------------------
// Columns [j0, j1) of supernode s's front: zero them, place A's entries, then add each child's
// update matrix in child order (the front is the multifrontal form of the reference's
// own(rel(i), rel(c)) -= S(i, c), cholesky.rs:636-686, summed child by child).
__global__ void __launch_bounds__(256) assemble_kernel(Tree t, const double *__restrict__ val,
                                                       const AssembleTask *__restrict__ tasks) {
  const AssembleTask task = tasks[blockIdx.x];
  const int s = task.s;
  const int64_t m = t.height[s], w = t.width[s], u = m - w, f = t.first[s];
  double *Ls = t.L + t.loff[s];
  double *Us = t.U + t.uoff[s];
  const int j0 = task.j0, j1 = task.j1;
  const int tid = threadIdx.x;
  for (int j = j0; j < j1; ++j) {
    if (j < w) {
      double *col = Ls + (int64_t)j * m;
      for (int64_t i = tid; i < m; i += blockDim.x) col[i] = 0.0;
    } else {
      double *col = Us + (int64_t)(j - w) * u;
      for (int64_t i = (j - w) + tid; i < u; i += blockDim.x) col[i] = 0.0;
    }
  }
  __syncthreads();
  const int jend = j1 < w ? j1 : (int)w;
  if (j0 < jend) {
    const int64_t e0 = t.a_ptr[f + j0], e1 = t.a_ptr[f + jend];
    for (int64_t e = e0 + tid; e < e1; e += blockDim.x) t.L[t.a_dst[e]] = val[t.a_src[e]];
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
  for (int64_t kp = t.kid_ptr[s]; kp < t.kid_ptr[s + 1]; ++kp) {
    const int c = t.kids[kp];
    const int uc = t.height[c] - t.width[c];
    const int32_t *rel = t.rel + t.rel_off[c];
    const double *Uc = t.U + t.uoff[c];
    const int lo = lower_bound_i32(rel, uc, j0), hi = lower_bound_i32(rel, uc, j1);
    for (int jc = lo + warp; jc < hi; jc += nwarps) {
      const int64_t J = rel[jc];
      const double *src = Uc + (int64_t)jc * uc;
      double *dst = J < w ? Ls + J * m : Us + (J - w) * u - w;
      for (int ic = jc + lane; ic < uc; ic += 32) dst[rel[ic]] += src[ic];
    }
    __syncthreads();
  }
}

// ---- diagonal block: unblocked right-looking Cholesky of a <= 64 x 64 block in shared memory ----
// Pivot test of cholesky.rs:1162-1165: not (d > PIVOT_TOLERANCE |A_jj|) or not finite fails; the
// smallest failing column (postorder) is kept in the status word. A failed pivot makes NaNs and
// nothing else: no index depends on a value.
__global__ void __launch_bounds__(256) potrf_kernel(Tree t, const double *__restrict__ val,
                                                    const PanelTask *__restrict__ tasks, DeviceStatus *status) {
  __shared__ double a[NB * (NB + 1)];
  __shared__ double dpiv;
  const PanelTask task = tasks[blockIdx.x];
  const int s = task.s;
  const int64_t m = t.height[s], f = t.first[s];
  double *Ls = t.L + t.loff[s];
  const int c0 = task.c0, pw = task.c1 - task.c0;
  const int tid = threadIdx.x;
  for (int e = tid; e < pw * pw; e += blockDim.x) {
    const int r = e % pw, c = e / pw;
    if (r >= c) a[c * (NB + 1) + r] = Ls[(c0 + r) + (int64_t)(c0 + c) * m];
  }
  __syncthreads();
  for (int c = 0; c < pw; ++c) {
    if (tid == 0) {
      double d = a[c * (NB + 1) + c];
      const int64_t col = f + c0 + c;
      const int64_t ds = t.diag_src[col];
      const double diag = ds >= 0 ? val[ds] : 0.0;
      if (!(d > PIVOT_TOLERANCE * fabs(diag)) || !isfinite(d))
        atomicMin(&status->failed_column, (unsigned long long)col);
      d = sqrt(d);
      a[c * (NB + 1) + c] = d;
      dpiv = d;
    }
    __syncthreads();
    const double d = dpiv;
    for (int r = c + 1 + tid; r < pw; r += blockDim.x) a[c * (NB + 1) + r] /= d;
    __syncthreads();
    const int rem = pw - c - 1;
    for (int e = tid; e < rem * rem; e += blockDim.x) {
      const int i = c + 1 + e % rem, j = c + 1 + e / rem;
      if (i >= j) a[j * (NB + 1) + i] -= a[c * (NB + 1) + i] * a[c * (NB + 1) + j];
    }
    __syncthreads();
  }
  for (int e = tid; e < pw * pw; e += blockDim.x) {
    const int r = e % pw, c = e / pw;
    if (r >= c) Ls[(c0 + r) + (int64_t)(c0 + c) * m] = a[c * (NB + 1) + r];
  }
}

// ---- rows below a factored diagonal block: X = B L^-T, one row per thread -------------------------
__global__ void __launch_bounds__(TRSM_ROWS) trsm_kernel(Tree t, const PanelTask *__restrict__ tasks) {
  extern __shared__ double smem[];
  double *a = smem;                     // NB x (NB+1)
  double *x = smem + NB * (NB + 1);     // NB x TRSM_ROWS, x[k * TRSM_ROWS + r]
  const PanelTask task = tasks[blockIdx.x];
  const int s = task.s;
  const int64_t m = t.height[s];
  double *Ls = t.L + t.loff[s];
  const int c0 = task.c0, pw = task.c1 - task.c0;
  const int tid = threadIdx.x;
  for (int e = tid; e < pw * pw; e += blockDim.x) {
    const int r = e % pw, c = e / pw;
    if (r >= c) a[c * (NB + 1) + r] = Ls[(c0 + r) + (int64_t)(c0 + c) * m];
  }
  const int64_t row = task.r0 + tid;
  const bool active = row < task.r1;
  if (active)
    for (int k = 0; k < pw; ++k) x[k * TRSM_ROWS + tid] = Ls[row + (int64_t)(c0 + k) * m];
  __syncthreads();
  if (active) {
    for (int c = 0; c < pw; ++c) {
      double acc = x[c * TRSM_ROWS + tid];
      for (int k = 0; k < c; ++k) acc -= x[k * TRSM_ROWS + tid] * a[k * (NB + 1) + c];
      x[c * TRSM_ROWS + tid] = acc / a[c * (NB + 1) + c];
    }
    for (int k = 0; k < pw; ++k) Ls[row + (int64_t)(c0 + k) * m] = x[k * TRSM_ROWS + tid];
  }
}

// ---- tiled C -= A B^T on the FP64 tensor pipe ---------------------------------------------------
// 64 x 64 tile per CTA, 4 warps of 32 x 32 (4 x 4 DMMA tiles), K in chunks of 16 double-buffered
// through shared memory. Shared rows are padded to 68 doubles so the fragment reads of a warp
// (4 k-rows x 8 consecutive doubles) fall in distinct banks.
constexpr int SROW = 68;

__global__ void __launch_bounds__(GEMM_THREADS) gemm_kernel(const GemmTask *__restrict__ tasks) {
  const GemmTask tk = tasks[blockIdx.x];
  __shared__ __align__(16) double As[2][GEMM_KC][SROW];
  __shared__ __align__(16) double Bs[2][GEMM_KC][SROW];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tg = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int M = tk.M, N = tk.N, K = tk.K;
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const bool a_rows = tk.a_si == 1, b_rows = tk.b_sj == 1;
  auto load = [&](int stage, int k0) {
#pragma unroll
    for (int q = 0; q < (GEMM_TM * GEMM_KC) / GEMM_THREADS; ++q) {
      const int e = tid + GEMM_THREADS * q;
      int i, k;
      if (a_rows) {
        i = e & (GEMM_TM - 1);
        k = e / GEMM_TM;
      } else {
        i = e / GEMM_KC;
        k = e & (GEMM_KC - 1);
      }
      const bool ok = i < M && k0 + k < K;
      const double *src = ok ? tk.A + (int64_t)i * tk.a_si + (int64_t)(k0 + k) * tk.a_sk : tk.A;
      cp_async8(&As[stage][k][i], src, ok ? 8 : 0);
      int j;
      if (b_rows) {
        j = e & (GEMM_TN - 1);
        k = e / GEMM_TN;
      } else {
        j = e / GEMM_KC;
        k = e & (GEMM_KC - 1);
      }
      const bool okb = j < N && k0 + k < K;
      const double *srcb = okb ? tk.B + (int64_t)j * tk.b_sj + (int64_t)(k0 + k) * tk.b_sk : tk.B;
      cp_async8(&Bs[stage][k][j], srcb, okb ? 8 : 0);
    }
    cp_async_commit();
  };
  const int nk = (K + GEMM_KC - 1) / GEMM_KC;
  if (nk > 0) load(0, 0);
  for (int kt = 0; kt < nk; ++kt) {
    if (kt + 1 < nk) {
      load((kt + 1) & 1, (kt + 1) * GEMM_KC);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const int st = kt & 1;
#pragma unroll
    for (int kk = 0; kk < GEMM_KC; kk += 4) {
      double av[4], bv[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) av[r] = As[st][kk + tg][wm + r * 8 + g];
#pragma unroll
      for (int c = 0; c < 4; ++c) bv[c] = Bs[st][kk + tg][wn + c * 8 + g];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) dmma(acc[r][c], av[r], bv[c]);
    }
    __syncthreads();
  }
  const bool lower = tk.flags & 1;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int i = wm + r * 8 + g, j = wn + c * 8 + 2 * tg + e;
        if (i < M && j < N && (!lower || i >= j)) {
          double *dst = tk.C + (int64_t)i * tk.c_si + (int64_t)j * tk.c_sj;
          *dst -= acc[r][c][e];
        }
      }
}

// ---- solve -------------------------------------------------------------------------------------
// Rows [i0, i1) of supernode s's solve front: zero its update rows, then add the children's
// update vectors in child order.
__global__ void __launch_bounds__(256) solve_assemble_kernel(Tree t, double *__restrict__ x, double *__restrict__ v,
                                                             const int64_t *__restrict__ voff, int R,
                                                             const RowTask *__restrict__ tasks) {
  const RowTask task = tasks[blockIdx.x];
  const int s = task.s;
  const int64_t m = t.height[s], w = t.width[s], f = t.first[s];
  double *vs = v + voff[s];
  const int tid = threadIdx.x;
  const int64_t z0 = task.i0 > w ? task.i0 : w;
  for (int64_t e = tid; e < (task.i1 - z0) * R; e += blockDim.x) vs[(z0 - w) * R + e] = 0.0;
  __syncthreads();
  for (int64_t kp = t.kid_ptr[s]; kp < t.kid_ptr[s + 1]; ++kp) {
    const int c = t.kids[kp];
    const int uc = t.height[c] - t.width[c];
    const int32_t *rel = t.rel + t.rel_off[c];
    const double *vc = v + voff[c];
    const int lo = lower_bound_i32(rel, uc, task.i0), hi = lower_bound_i32(rel, uc, task.i1);
    for (int64_t e = tid; e < (int64_t)(hi - lo) * R; e += blockDim.x) {
      const int ic = lo + (int)(e / R), j = (int)(e % R);
      const int64_t I = rel[ic];
      double *dst = I < w ? x + (f + I) * R + j : vs + (I - w) * R + j;
      *dst += vc[(int64_t)ic * R + j];
    }
    __syncthreads();
  }
  (void)m;
}

// v_s rows [i0, i1) <- x at the supernode's rows below its columns (final by the backward pass).
__global__ void __launch_bounds__(256) solve_gather_kernel(Tree t, const double *__restrict__ x, double *__restrict__ v,
                                                           const int64_t *__restrict__ voff, int R,
                                                           const RowTask *__restrict__ tasks) {
  const RowTask task = tasks[blockIdx.x];
  const int s = task.s;
  const int64_t w = t.width[s];
  const int32_t *rows = t.rows + t.rows_off[s] + w;
  double *vs = v + voff[s];
  for (int64_t e = threadIdx.x; e < (int64_t)(task.i1 - task.i0) * R; e += blockDim.x) {
    const int64_t i = task.i0 + e / R;
    const int j = (int)(e % R);
    vs[i * R + j] = x[(int64_t)rows[i] * R + j];
  }
}

// Own rows [c0, c1) of supernode s, right-hand sides [j0, j1): forward (L) or backward (L^T)
// substitution with the diagonal block; one right-hand side per thread.
__global__ void __launch_bounds__(64) trsv_kernel(Tree t, double *__restrict__ x, int R, int transpose,
                                                  const SolveTask *__restrict__ tasks) {
  extern __shared__ double smem[];
  double *a = smem;                 // NB x (NB+1)
  double *xs = smem + NB * (NB + 1);  // NB x 64, xs[r * 64 + j]
  const SolveTask task = tasks[blockIdx.x];
  const int s = task.s;
  const int64_t m = t.height[s], f = t.first[s];
  const double *Ls = t.L + t.loff[s];
  const int c0 = task.c0, pw = task.c1 - task.c0, j0 = task.j0, nj = task.j1 - task.j0;
  const int tid = threadIdx.x;
  for (int e = tid; e < pw * pw; e += blockDim.x) {
    const int r = e % pw, c = e / pw;
    if (r >= c) a[c * (NB + 1) + r] = Ls[(c0 + r) + (int64_t)(c0 + c) * m];
  }
  for (int e = tid; e < pw * nj; e += blockDim.x) {
    const int r = e / nj, j = e % nj;
    xs[r * 64 + j] = x[(f + c0 + r) * R + j0 + j];
  }
  __syncthreads();
  if (tid < nj) {
    if (!transpose) {
      for (int r = 0; r < pw; ++r) {
        double acc = xs[r * 64 + tid];
        for (int k = 0; k < r; ++k) acc -= a[k * (NB + 1) + r] * xs[k * 64 + tid];
        xs[r * 64 + tid] = acc / a[r * (NB + 1) + r];
      }
    } else {
      for (int r = pw - 1; r >= 0; --r) {
        double acc = xs[r * 64 + tid];
        for (int k = r + 1; k < pw; ++k) acc -= a[r * (NB + 1) + k] * xs[k * 64 + tid];
        xs[r * 64 + tid] = acc / a[r * (NB + 1) + r];
      }
    }
  }
  __syncthreads();
  for (int e = tid; e < pw * nj; e += blockDim.x) {
    const int r = e / nj, j = e % nj;
    x[(f + c0 + r) * R + j0 + j] = xs[r * 64 + j];
  }
}

__global__ void permute_in_kernel(const int64_t *__restrict__ perm, int64_t n, const double *__restrict__ b,
                                  int64_t ld, double *__restrict__ x, int R) {
  const int64_t total = n * R;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / R;
    const int j = (int)(e % R);
    x[e] = b[perm[i] + j * ld];
  }
}

__global__ void permute_out_kernel(const int64_t *__restrict__ perm, int64_t n, const double *__restrict__ x, int R,
                                   double *__restrict__ b, int64_t ld) {
  const int64_t total = n * R;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / R;
    const int j = (int)(e % R);
    b[perm[i] + j * ld] = x[e];
  }
}

// y = A x: one row per thread, each row summed in column order (crates/solver/src/sparse.rs:42-50).
__global__ void spmv_kernel(int64_t n, const int64_t *__restrict__ ptr, const int32_t *__restrict__ idx,
                            const double *__restrict__ val, const double *__restrict__ x, double *__restrict__ y, int R,
                            int64_t ld) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (r >= n || j >= R) return;
  const double *xj = x + j * ld;
  double acc = -0.0;
  for (int64_t p = ptr[r]; p < ptr[r + 1]; ++p) acc += val[p] * xj[idx[p]];
  y[r + j * ld] = acc;
}

__global__ void pack_kernel(Tree t, const int64_t *__restrict__ toff, double *__restrict__ dst) {
  const int s = blockIdx.x;
  const int64_t m = t.height[s], w = t.width[s];
  const double *Ls = t.L + t.loff[s];
  double *d = dst + toff[s];
  for (int64_t c = 0; c < w; ++c) {
    const int64_t start = c * m - c * (c > 0 ? c - 1 : 0) / 2;
    for (int64_t r = c + threadIdx.x; r < m; r += blockDim.x) d[start + r - c] = Ls[r + c * m];
  }
}

}  // namespace

void launch_assemble(const Tree &t, const double *upper_val, const AssembleTask *tasks, int count, cudaStream_t st) {
  if (count > 0) assemble_kernel<<<count, 256, 0, st>>>(t, upper_val, tasks);
}

void launch_potrf(const Tree &t, const double *upper_val, const PanelTask *tasks, int count, DeviceStatus *status,
                  cudaStream_t st) {
  if (count > 0) potrf_kernel<<<count, 256, 0, st>>>(t, upper_val, tasks, status);
}

void launch_trsm(const Tree &t, const PanelTask *tasks, int count, cudaStream_t st) {
  if (count <= 0) return;
  const size_t smem = sizeof(double) * (NB * (NB + 1) + NB * TRSM_ROWS);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(trsm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    configured = true;
  }
  trsm_kernel<<<count, TRSM_ROWS, smem, st>>>(t, tasks);
}

void launch_gemm(const GemmTask *tasks, int count, cudaStream_t st) {
  if (count > 0) gemm_kernel<<<count, GEMM_THREADS, 0, st>>>(tasks);
}

void launch_solve_assemble(const Tree &t, double *x, double *v, const int64_t *voff, int R, const RowTask *tasks,
                           int count, cudaStream_t st) {
  if (count > 0) solve_assemble_kernel<<<count, 256, 0, st>>>(t, x, v, voff, R, tasks);
}

void launch_solve_gather(const Tree &t, const double *x, double *v, const int64_t *voff, int R, const RowTask *tasks,
                         int count, cudaStream_t st) {
  if (count > 0) solve_gather_kernel<<<count, 256, 0, st>>>(t, x, v, voff, R, tasks);
}

void launch_trsv(const Tree &t, double *x, int R, bool transpose, const SolveTask *tasks, int count, cudaStream_t st) {
  if (count <= 0) return;
  const size_t smem = sizeof(double) * (NB * (NB + 1) + NB * 64);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(trsv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    configured = true;
  }
  trsv_kernel<<<count, 64, smem, st>>>(t, x, R, transpose ? 1 : 0, tasks);
}

void launch_permute_in(const int64_t *perm, int64_t n, const double *b, int64_t ld, double *x, int R, cudaStream_t st) {
  const int64_t total = n * R;
  if (total <= 0) return;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  permute_in_kernel<<<blocks, 256, 0, st>>>(perm, n, b, ld, x, R);
}

void launch_permute_out(const int64_t *perm, int64_t n, const double *x, int R, double *b, int64_t ld,
                        cudaStream_t st) {
  const int64_t total = n * R;
  if (total <= 0) return;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  permute_out_kernel<<<blocks, 256, 0, st>>>(perm, n, x, R, b, ld);
}

void launch_spmv(int64_t n, const int64_t *ptr, const int32_t *idx, const double *val, const double *x, double *y,
                 int R, int64_t ld, cudaStream_t st) {
  if (n <= 0 || R <= 0) return;
  dim3 grid((unsigned)((n + 127) / 128), (unsigned)R);
  spmv_kernel<<<grid, 128, 0, st>>>(n, ptr, idx, val, x, y, R, ld);
}

void launch_pack_trapezoids(const Tree &t, int64_t ns, const int64_t *toff, double *dst, cudaStream_t st) {
  if (ns > 0) pack_kernel<<<(unsigned)ns, 128, 0, st>>>(t, toff, dst);
}

}  // namespace fc
