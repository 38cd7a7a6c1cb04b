// Kernels of the supernodal Cholesky on B200 (sm_100a).
//
// Storage of L and of the update matrices is FP64, or FP32 for the mixed-precision factorisation;
// the diagonal blocks, their inverses, the solve's vectors and every triangular solve stay FP64.
// FP64 updates run on the FP64 tensor pipe (DMMA, mma.sync .f64 — tcgen05 has no FP64 kind); FP32
// updates run as 3xTF32 split products on the tensor pipe with FP32 accumulation. Operands are
// staged through shared memory by cp.async; the rest is SIMT.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstdio>

#include <cooperative_groups.h>

#include "kernels.cuh"
#include "tiles.cuh"

namespace fc {

namespace {

using namespace tiles;

constexpr double PIVOT_TOLERANCE = 1e-10;  // crates/solver/src/cholesky.rs:48

// D = A B + C on one 16x8x8 FP64 tile (sm_90 and later): a = A[g][tg], A[g+8][tg], A[g][tg+4],
// A[g+8][tg+4]; b = B[tg][g], B[tg+4][g]; c/d = C[g][2tg], C[g][2tg+1], C[g+8][2tg], C[g+8][2tg+1].
__device__ __forceinline__ void dmma16(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// The same 16x8x8 shape on TF32 operands with FP32 accumulation (the fragments' positions are
// those of dmma16).
__device__ __forceinline__ void tmma16(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
               : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// x = hi + lo with hi = x rounded to TF32 and lo = (x - hi) rounded to TF32: three products of
// such halves (hi hi + hi lo + lo hi) keep FP32 accuracy (the 3xTF32 split).
__device__ __forceinline__ void tf32_split(float x, uint32_t &hi, uint32_t &lo) {
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(hi) : "f"(x));
  const float rest = x - __uint_as_float(hi);
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(lo) : "f"(rest));
}

// ---- front assembly ----------------------------------------------------------------------------
// One tile of supernode s's front: columns [j0, j1) (at most COLS) by rows [i0, i1) (at
// most ROWS, a thread each), built in shared memory and written once. The tile starts as
//   ASM_L          zero, then A's entries (columns of the L panel, assembled before the panel is
//                  factored; with a scale, the entries of S A S, S = diag(A)^-1/2);
//   ASM_U          the update matrix's tile as its GEMM stored it (-L21 L21^T);
//   ASM_U_PRODUCT  -L21 L21^T formed here (a thin supernode, w <= ASSEMBLE_THIN, whose update
//                  matrix no GEMM writes: each entry is a w-term dot product of two rows of L21);
// then each child's update matrix entries that land in the tile are added, child by child (the
// multifrontal form of the reference's own(rel(i), rel(c)) -= S(i, c), cholesky.rs:636-686).
// ranges[task.ranges + q] = {columns lo, hi, rows lo, hi} of child q's update matrix whose places
// fall in the tile; only its lower triangle (row >= column) is read. No destination is read and
// written through global memory: the child's rows and values stream in coalesced, the scatter is
// to shared memory, and every entry of the tile's lower part is stored once.
template <class T, int COLS, int ROWS>
__global__ void __launch_bounds__(ROWS, ROWS == 256 ? 6 : 8)
    assemble_kernel(Tree t, const double *__restrict__ val, const AssembleTask *__restrict__ tasks,
                    const int4 *__restrict__ ranges) {
  constexpr int THREADS = ROWS, WARPS = THREADS / 32, CPW = COLS / WARPS;  // child columns a warp takes
  static_assert(CPW * WARPS == COLS && CPW >= 1, "tile shape");
  __shared__ T tile[COLS][ROWS];
  __shared__ T lj[ASSEMBLE_THIN][COLS];
  __shared__ int4 s_rg[ASSEMBLE_KIDS];
  __shared__ KidMeta s_km[ASSEMBLE_KIDS];
  const AssembleTask task = tasks[blockIdx.x];
  const int m = task.m, w = task.w, u = m - w, nk = task.nk;
  T *Ls = static_cast<T *>(t.L) + task.loff;
  T *Us = static_cast<T *>(t.U) + task.uoff;
  const int j0 = task.j0, nc = task.j1 - task.j0, i0 = task.i0, nr = task.i1 - task.i0;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // the children's ranges and whereabouts, loaded beside the initial values (the task carries the
  // supernode's own, so no load waits for another before the children's rows)
  if (tid < nk && tid < ASSEMBLE_KIDS) {
    s_rg[tid] = ranges[task.ranges + tid];
    s_km[tid] = t.kid_meta[task.k0 + tid];
  }
  // column jj of the tile, indexed by front row
  auto column = [&](int jj) -> T * {
    const int J = j0 + jj;
    return J < w ? Ls + (int64_t)J * m : Us + (int64_t)(J - w) * u - w;
  };
  // thread tid owns tile row tid for the initial values and the store
  const int ii = tid, r = i0 + tid;
  if (task.mode == ASM_U_PRODUCT) {
    for (int q = tid; q < w * nc; q += THREADS) {
      const int k = q / nc, jj = q - k * nc;
      lj[k][jj] = Ls[(int64_t)k * m + j0 + jj];
    }
    __syncthreads();
    if (ii < nr) {
      // the row's values of L21 four at a time in flight, then their dot products
      T acc[COLS];
#pragma unroll
      for (int jj = 0; jj < COLS; ++jj) acc[jj] = T(0);
      for (int k0 = 0; k0 < w; k0 += 4) {
        T a[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) a[k] = k0 + k < w ? Ls[(int64_t)(k0 + k) * m + r] : T(0);
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (k0 + k < w) {
#pragma unroll
            for (int jj = 0; jj < COLS; ++jj) acc[jj] = fma(a[k], lj[k0 + k][jj], acc[jj]);
          }
      }
#pragma unroll
      for (int jj = 0; jj < COLS; ++jj) tile[jj][ii] = -acc[jj];
    }
  } else if (task.mode == ASM_U) {
    if (ii < nr) {
      T v[COLS];
#pragma unroll
      for (int jj = 0; jj < COLS; ++jj)
        if (jj < nc && r >= j0 + jj) v[jj] = column(jj)[r];
#pragma unroll
      for (int jj = 0; jj < COLS; ++jj)
        if (jj < nc && r >= j0 + jj) tile[jj][ii] = v[jj];
    }
  } else {
#pragma unroll
    for (int jj = 0; jj < COLS; ++jj) tile[jj][ii] = T(0);
    __syncthreads();
    // A's entries of the tile: the block's entries are sorted by row, [e0, e1) are this tile's
    for (int64_t e = task.e0 + tid; e < task.e1; e += THREADS) {
      const int p = (int)(t.a_dst[e] - task.loff), J = p / m, row = p - J * m;
      const double a = t.scale ? val[t.a_src[e]] * t.scale[t.a_row[e]] * t.scale[t.a_col[e]] : val[t.a_src[e]];
      tile[J - j0][row - i0] = T(a);
    }
  }
  __syncthreads();
  // the children: warp q takes the child's columns q, q + WARPS, ... in the tile (a child has at
  // most one column per tile column), its lanes the rows, eight loads a lane a column in flight
  // before the adds
  for (int q = 0; q < nk; ++q) {
    const int4 g = q < ASSEMBLE_KIDS ? s_rg[q] : ranges[task.ranges + q];
    if (g.x < g.y && g.z < g.w) {
      if (g.x + warp < g.y) {
        const KidMeta km = q < ASSEMBLE_KIDS ? s_km[q] : t.kid_meta[task.k0 + q];
        const int32_t *rel = t.rel + km.rel_off;
        int at[CPW][ROWS / 32], jjs[CPW];
        T v[CPW][ROWS / 32];
#pragma unroll
        for (int c = 0; c < CPW; ++c) {
          const int jc = g.x + warp + WARPS * c;
          jjs[c] = -1;
          if (jc < g.y) {
            const T *src = static_cast<const T *>(t.U) + km.uoff + (int64_t)jc * km.uc;
            const int a = g.z > jc ? g.z : jc;
            jjs[c] = rel[jc] - j0;
#pragma unroll
            for (int k = 0; k < ROWS / 32; ++k) {
              const int ic = a + lane + 32 * k;
              at[c][k] = -1;
              if (ic < g.w) {
                at[c][k] = rel[ic];
                v[c][k] = src[ic];
              }
            }
          }
        }
#pragma unroll
        for (int c = 0; c < CPW; ++c)
          if (jjs[c] >= 0) {
#pragma unroll
            for (int k = 0; k < ROWS / 32; ++k)
              if (at[c][k] >= 0) tile[jjs[c]][at[c][k] - i0] += v[c][k];
          }
      }
      __syncthreads();
    }
  }
  if (ii < nr) {
#pragma unroll
    for (int jj = 0; jj < COLS; ++jj)
      if (jj < nc && r >= j0 + jj) column(jj)[r] = tile[jj][ii];
  }
}

// S = diag(A)^-1/2 over the postordered columns (the mixed-precision factorisation's scaling).
__global__ void scale_kernel(int64_t n, const int64_t *__restrict__ diag_src, const double *__restrict__ val,
                             double *__restrict__ scale) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int64_t ds = diag_src[j];
  const double d = ds >= 0 ? fabs(val[ds]) : 0.0;
  scale[j] = d > 0.0 ? 1.0 / sqrt(d) : 1.0;
}

// ---- panel: factor the diagonal block, invert it, solve the rows below --------------------------
// The block (pw <= 64 columns) is factored in FP64 in shared memory by strips of 8 columns; the
// pivot test is the reference's (cholesky.rs:1162-1165): not (d > PIVOT_TOLERANCE |A_jj|) or not
// finite fails, and the smallest failing column (postorder) is kept in the status word. A failed
// pivot makes NaNs and nothing else: no index depends on a value. The inverse comes from 8 x 8
// diagonal blocks and block forward substitution; the rows below are X = B L^-T on the FP64
// tensor pipe. L may be stored in FP32 (widened on load, rounded on store); the diagonal arena
// stays FP64.
constexpr int PANEL_THREADS = 128;
// Shared memory of a panel launch whose widest panel is padded to p8 columns (a multiple of 8).
template <class T>
__host__ __device__ constexpr size_t panel_smem(int p8) {
  return sizeof(double) * (p8 * (65 + TS) + 1024 + 128) + sizeof(T) * p8 * tile_stride<T>();
}

template <class T>
__global__ void __launch_bounds__(PANEL_THREADS) panel_kernel(Tree t, const double *__restrict__ val,
                                                              const PanelTask *__restrict__ tasks,
                                                              DeviceStatus *status, int p8max) {
  extern __shared__ double sm[];
  double *inv = sm;                 // inv[k * TS + i] = Linv(i, k) (p8max rows)
  double *a = inv + p8max * TS;     // factor, column-major, ld 65 (p8max columns)
  double *tt = a + p8max * 65;      // scratch of the inversion's products (<= 1024 doubles)
  T *bt2 = reinterpret_cast<T *>(a);  // after the factor is stored: the second row tile (a and tt)
  double *dg = tt + 1024;           // the matrix's own diagonal entries of the panel's columns
  double *dv = dg + 64;             // the pivots' reciprocals
  T *bt = reinterpret_cast<T *>(dv + 64);  // rows below: bt[k * S + r] = L(r0 + r, c0 + k)
  __shared__ int fail;
  const PanelTask task = tasks[blockIdx.x];
  const int s = task.s;
  const int64_t m = t.height[s], f = t.first[s];
  T *Ls = static_cast<T *>(t.L) + t.loff[s];
  const int c0 = task.c0, pw = task.c1 - task.c0, rows = task.r1 - task.r0;
  const int nb8 = (pw + 7) >> 3, P8 = 8 * nb8, K4 = (pw + 3) & ~3;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) fail = pw;
  // the block's lower triangle (identity past pw, so the padded block inverts to the same leading
  // pw x pw inverse) and the first row tile in flight first, then the matrix's own diagonal
  // entries (two dependent loads each) while those land
  if (rows > 0) load_tile<T>(bt, Ls + task.r0 + (int64_t)c0 * m, 1, m, min(rows, 64), pw, K4);
  if (sizeof(T) == 8) {
    for (int c = warp; c < P8; c += PANEL_THREADS / 32)
      for (int r = lane; r < P8; r += 32) {
        if (r < pw && c < pw && r >= c)
          cp_async8(&a[c * 65 + r], Ls + (c0 + r) + (int64_t)(c0 + c) * m, 8);
        else
          a[c * 65 + r] = (double)(r == c);
      }
  } else {
    // FP32 panels: every load of the thread in flight before the widening stores
    float v[16][2];
#pragma unroll
    for (int ci = 0; ci < 16; ++ci)
#pragma unroll
      for (int ri = 0; ri < 2; ++ri) {
        const int c = warp + 4 * ci, r = lane + 32 * ri;
        v[ci][ri] = r < pw && c < pw && r >= c ? (float)Ls[(c0 + r) + (int64_t)(c0 + c) * m] : (float)(r == c);
      }
#pragma unroll
    for (int ci = 0; ci < 16; ++ci)
#pragma unroll
      for (int ri = 0; ri < 2; ++ri) {
        const int c = warp + 4 * ci, r = lane + 32 * ri;
        if (c < P8 && r < P8) a[c * 65 + r] = (double)v[ci][ri];
      }
  }
  cp_async_commit();
  for (int c = tid; c < pw; c += PANEL_THREADS) {
    const int64_t j = f + c0 + c, ds = t.diag_src[j];
    const double d = ds >= 0 ? val[ds] : 0.0;
    dg[c] = t.scale ? d * t.scale[j] * t.scale[j] : d;
  }
  for (int e = tid; e < P8 * TS; e += PANEL_THREADS) inv[e] = 0.0;
  cp_async_wait<0>();
  __syncthreads();
  // right-looking by strips of 8 columns with look-ahead: warp 0 factors a strip (two rows a
  // lane, pivots and multipliers broadcast by shuffles); then all warps update the next strip's
  // columns, and warp 0 factors that strip while warps 1-3 update the rest of the trailing lower
  // triangle (DMMA, a rank-8 update per 8 x 8 block); padding past pw factors as the identity
  auto factor_strip = [&](int B) {
    const int o = 8 * B;
    const int r0 = o + lane, r1 = o + 32 + lane;
    double s0[8], s1[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      s0[k] = r0 < P8 ? a[(o + k) * 65 + r0] : 0.0;
      s1[k] = r1 < P8 ? a[(o + k) * 65 + r1] : 0.0;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const double acc = __shfl_sync(0xffffffffu, s0[j], j);
      const double rd = rsqrt(acc);
      const double d = acc * rd;
      if (lane == j) {
        s0[j] = d;
        dv[o + j] = rd;
        if (o + j < pw && (!(acc > PIVOT_TOLERANCE * fabs(dg[o + j])) || !isfinite(acc)) && fail == pw) fail = o + j;
      } else if (lane > j) {
        s0[j] *= rd;
      }
      s1[j] *= rd;
#pragma unroll
      for (int k = j + 1; k < 8; ++k) {
        const double lk = __shfl_sync(0xffffffffu, s0[j], k);
        if (lane > j) s0[k] -= s0[j] * lk;
        s1[k] -= s1[j] * lk;
      }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (r0 < P8) a[(o + k) * 65 + r0] = s0[k];
      if (r1 < P8) a[(o + k) * 65 + r1] = s1[k];
    }
  };
  // the rank-8 update by strip B of the 8 x 8 block (I, J) (I >= J > B)
  auto update_tile = [&](int B, int I, int J) {
    const int o = 8 * B, g = lane >> 2, tg = lane & 3;
    double c[2] = {0.0, 0.0};
    dmma(c, a[(o + tg) * 65 + I + g], a[(o + tg) * 65 + J + g]);
    dmma(c, a[(o + 4 + tg) * 65 + I + g], a[(o + 4 + tg) * 65 + J + g]);
    a[(J + 2 * tg) * 65 + I + g] -= c[0];
    a[(J + 2 * tg + 1) * 65 + I + g] -= c[1];
  };
  if (warp == 0) factor_strip(0);
  __syncthreads();
  for (int B = 0; B < nb8; ++B) {
    if (B + 1 < nb8) {
      // the next strip's block column, all warps
      for (int qi = B + 1 + warp; qi < nb8; qi += PANEL_THREADS / 32) update_tile(B, 8 * qi, 8 * (B + 1));
      __syncthreads();
      if (warp == 0) {
        factor_strip(B + 1);
      } else {
        int q = 0;
        for (int qj = B + 2; qj < nb8; ++qj)
          for (int qi = qj; qi < nb8; ++qi, ++q)
            if (q % 3 == warp - 1) update_tile(B, 8 * qi, 8 * qj);
      }
      __syncthreads();
    }
  }
  // inverse: the diagonal 8 x 8 blocks (a column each) ...
  if (tid < P8) {
    const int B = tid >> 3, j = tid & 7, o = 8 * B;
    double y[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (i >= j) {
        double sum = i == j ? 1.0 : 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if (k >= j && k < i) sum -= a[(o + k) * 65 + o + i] * y[k];
        y[i] = sum * dv[o + i];
      } else {
        y[i] = 0.0;
      }
      inv[(o + j) * TS + o + i] = y[i];
    }
  }
  __syncthreads();
  // ... then by doubling (h = 8, 16, 32): neighbouring inverses A^-1, C^-1 of h columns give the
  // inverse of [[A, 0], [B, C]], whose lower-left block is -C^-1 (B A^-1); both products on DMMA,
  // 8 x 8 output tiles round-robin over the warps, T = B A^-1 in the scratch
  for (int h = 8; h < P8; h *= 2) {
    int tile = 0;
    for (int a0 = 0; a0 + h < P8; a0 += 2 * h) {
      const int c0b = a0 + h, hc = min(h, P8 - c0b);
      for (int ti = 0; ti < hc; ti += 8)
        for (int tj = 0; tj < h; tj += 8, ++tile) {
          if ((tile & 3) != warp) continue;
          const int g = lane >> 2, tg = lane & 3;
          double c[2] = {0.0, 0.0};
          for (int k = tj; k < h; k += 4)  // A^-1 (k, j) = 0 for k < j
            dmma(c, a[(a0 + k + tg) * 65 + c0b + ti + g], inv[(a0 + tj + g) * TS + a0 + k + tg]);
          const int base = (a0 / (2 * h)) * h * h;  // the pair's hc x h product, column-major, ld h
          tt[base + (tj + 2 * tg) * h + ti + g] = c[0];
          tt[base + (tj + 2 * tg + 1) * h + ti + g] = c[1];
        }
    }
    __syncthreads();
    tile = 0;
    for (int a0 = 0; a0 + h < P8; a0 += 2 * h) {
      const int c0b = a0 + h, hc = min(h, P8 - c0b);
      const int base = (a0 / (2 * h)) * h * h;
      for (int ti = 0; ti < hc; ti += 8)
        for (int tj = 0; tj < h; tj += 8, ++tile) {
          if ((tile & 3) != warp) continue;
          const int g = lane >> 2, tg = lane & 3;
          double c[2] = {0.0, 0.0};
          for (int k = 0; k <= ti + 4 && k < hc; k += 4)  // C^-1 (i, k) = 0 for k > i
            dmma(c, inv[(c0b + k + tg) * TS + c0b + ti + g], tt[base + (tj + g) * h + k + tg]);
          inv[(a0 + tj + 2 * tg) * TS + c0b + ti + g] = -c[0];
          inv[(a0 + tj + 2 * tg + 1) * TS + c0b + ti + g] = -c[1];
        }
    }
    __syncthreads();
  }
  {
    // this CTA's columns of the factored block and its inverse (the panel's CTAs share the stores)
    double *Dp = t.D + task.doff, *Ip = t.Dinv + task.ioff;
    const int nw = PANEL_THREADS / 32;
    for (int c = task.part * nw + warp; c < pw; c += task.keep * nw)
      for (int r = lane; r < pw; r += 32) {
        Dp[c * pw + r] = r >= c ? a[c * 65 + r] : 0.0;
        Dp[pw * pw + c * pw + r] = inv[c * TS + r];
        Ip[(int64_t)c * task.ild + r] = r >= c ? inv[c * TS + r] : 0.0;
      }
    if (tid == 0 && task.part == 0 && fail < pw)
      atomicMin(&status->failed_column, (unsigned long long)(f + c0 + fail));
  }
  // the rows below, 64 at a time: the first 64 loaded with the block, the next 64 into the factor's
  // and the scratch's space (free once the factor is stored) while the first are solved, any
  // further ones one after another
  if (rows > 64) {
    __syncthreads();  // every thread is done with a and tt
    load_tile<T>(bt2, Ls + task.r0 + 64 + (int64_t)c0 * m, 1, m, min(64, rows - 64), pw, K4);
    cp_async_commit();
  }
  for (int rr = 0; rr < rows; rr += 64) {
    const int nrr = min(64, rows - rr);
    const T *tile = rr == 64 ? bt2 : bt;
    if (rr == 64) {
      cp_async_wait<0>();
      __syncthreads();
    } else if (rr > 64) {
      __syncthreads();  // the previous rows' tile is read
      load_tile<T>(bt, Ls + task.r0 + rr + (int64_t)c0 * m, 1, m, nrr, pw, K4);
      cp_async_commit();
      cp_async_wait<0>();
      __syncthreads();
    }
    double acc[4][4][2];
    zero_acc(acc);
    mma_tiles<T>(tile, inv, K4, acc);
    T *dst = Ls + task.r0 + rr + (int64_t)c0 * m;
    each_acc(acc, [&](int i, int c, double v) {
      if (i < nrr && c < pw) dst[i + (int64_t)c * m] = T(v);
    });
  }
}

// ---- tiled C -= A B^T on the FP64 tensor pipe ---------------------------------------------------
// 64 x 64 tile per CTA, 4 warps of 32 x 32 (2 x 4 DMMA 16x8x8 tiles), K in chunks of 16 through a
// three-stage cp.async pipeline in shared memory (rows padded to 68 doubles so a warp's fragment
// reads of 4 k-rows x 8 consecutive doubles fall in distinct banks). Four CTAs fit an SM. An FP32
// A operand (the solve's L21^T v on an FP32 factor) is staged as FP32 and widened when read.
constexpr int SROW = 68;
constexpr int GEMM_STAGES = 3;
// The solve's short launches with few right-hand sides run with a deeper ring: they have few
// output tiles (often fewer than SMs), and a CTA's K loop is then bound by how many bytes it keeps
// in flight.
constexpr int SOLVE_STAGES = 8;
template <class TA, int STAGES = GEMM_STAGES>
__host__ __device__ constexpr size_t gemm_smem() {
  return STAGES * GEMM_KC * (sizeof(TA) * tile_stride<TA>() + sizeof(double) * SROW);
}

// This thread's elements of a 64 x KC operand tile: a fixed row and k = k0 + 2q when the rows
// are contiguous in memory (si == 1), else a fixed k and row i0 + (128 / KC) q (k contiguous).
template <class T, int KC>
struct TileLoader {
  static constexpr int PER = 64 * KC / GEMM_THREADS;  // elements per thread per stage
  const T *p;
  int64_t dq, dstage;
  int i0, k0, di, dk, lim;
  __device__ __forceinline__ void init(const T *base, int64_t si, int64_t sk, int rows, int tid) {
    if (si == 1) {
      i0 = tid & 63, k0 = tid >> 6, di = 0, dk = 2;
      p = base + i0 + (int64_t)k0 * sk;
      dq = 2 * sk;
      dstage = KC * sk;
    } else {
      i0 = tid / KC, k0 = tid % KC, di = GEMM_THREADS / KC, dk = 0;
      p = base + (int64_t)i0 * si + k0;
      dq = (int64_t)(GEMM_THREADS / KC) * si;
      dstage = KC;
    }
    lim = rows;
  }
  template <int S>
  __device__ __forceinline__ void load(T (*Sm)[S], int kbase, int K, const T *safe) {
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int i = i0 + q * di, k = k0 + q * dk;
      const bool ok = i < lim && kbase + k < K;
      cp_async<sizeof(T)>(&Sm[k][i], ok ? p + q * dq : safe, ok ? (int)sizeof(T) : 0);
    }
    p += dstage;
  }
  // the same tile with row k of the operand at base + rows[k] * sk (unit stride along i, the
  // layout init gives for si == 1): a gather through a row list, the stage's indices loaded first
  template <int S>
  __device__ __forceinline__ void load_rows(T (*Sm)[S], int kbase, int K, const T *base, const int32_t *rows,
                                            int64_t sk, const T *safe) {
    int r[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int k = k0 + q * dk;
      r[q] = kbase + k < K ? rows[kbase + k] : 0;
    }
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int i = i0 + q * di, k = k0 + q * dk;
      const bool ok = i < lim && kbase + k < K;
      cp_async<sizeof(T)>(&Sm[k][i], ok ? base + (int64_t)r[q] * sk + i : safe, ok ? (int)sizeof(T) : 0);
    }
  }
};

// Writes a GEMM task's 64 x 64 tile (acc[r][c][e] of the m16n8k8 fragments of a 32 x 32 warp
// tile) by `flags`: C = +sum (flag 4), -sum (flag 2), or C - sum. For C - sum the old values of a
// half tile are all loaded before any of its stores, so those loads are in flight together.
template <class T, class V>
__device__ __forceinline__ void gemm_store(const GemmTask *tp, int flags, const V (&acc)[2][4][4], int wm, int wn,
                                           int g, int tg) {
  const int M = tp->M, N = tp->N;
  const bool lower = flags & 1, store = flags & 2, partial = flags & 4;
  T *C = static_cast<T *>(tp->C);
  const int64_t c_si = tp->c_si, c_sj = tp->c_sj;
  auto at = [&](int r, int c, int e, T *&dst) {
    const int i = wm + r * 16 + g + 8 * (e >> 1), j = wn + c * 8 + 2 * tg + (e & 1);
    dst = C + (int64_t)i * c_si + (int64_t)j * c_sj;
    return i < M && j < N && (!lower || i >= j);
  };
  if (partial || store) {
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          T *dst;
          if (at(r, c, e, dst)) *dst = T(partial ? acc[r][c][e] : -acc[r][c][e]);
        }
    return;
  }
  // by halves of the warp tile's rows: 16 loads in flight, registers for the accumulator besides
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    T old[4][4];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        T *dst;
        old[c][e] = at(r, c, e, dst) ? *dst : T(0);
      }
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        T *dst;
        if (at(r, c, e, dst)) *dst = T(old[c][e] - acc[r][c][e]);
      }
  }
}

// One chunk of a split sum (GemmTask flag 8): v[e] is this thread's value at position at[e] of
// the 64 x 64 tile. Stores the chunk's partial and, in the CTA that finishes the sum, leaves the
// total in v and returns true (false in every other CTA). Additions run in the order the split
// fixes (chunks in order within a group, groups in order), each thread over its own positions
// with a chunk's loads in flight together.
template <int E>
__device__ __forceinline__ bool split_sum(const GemmTask *tp, double *part, int32_t *counters, double (&v)[E],
                                          const int (&at)[E]) {
  __shared__ int last;
  double *P = part + tp->part_off;
  const int chunks = tp->chunks, groups = split_groups(chunks);
  const int grp = groups ? tp->chunk / SPLIT_GROUP : 0;
  const int q0 = groups ? grp * SPLIT_GROUP : 0, qn = groups ? min(SPLIT_GROUP, chunks - q0) : chunks;
  // adds tiles [t0, t0 + tn) of `src` in order into v
  auto add_tiles = [&](const double *src, int t0, int tn) {
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = 0.0;
    for (int q = t0; q < t0 + tn; ++q) {
      const double *Pq = src + (int64_t)q * 4096;
      double u[E];
#pragma unroll
      for (int e = 0; e < E; ++e) u[e] = __ldcg(Pq + at[e]);
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] += u[e];
    }
  };
  double *mine = P + (int64_t)tp->chunk * 4096;
#pragma unroll
  for (int e = 0; e < E; ++e) mine[at[e]] = v[e];
  __threadfence();
  __syncthreads();
  int32_t *cnt = counters + tp->counter + (groups ? 1 + grp : 0);
  if (threadIdx.x == 0) last = atomicAdd(cnt, 1) == qn - 1;
  __syncthreads();
  if (!last) return false;
  __threadfence();
  add_tiles(P, q0, qn);
  if (threadIdx.x == 0) *cnt = 0;
  if (!groups) return true;
  double *sums = P + (int64_t)chunks * 4096;  // the groups' sums, after the chunks' partials
#pragma unroll
  for (int e = 0; e < E; ++e) sums[(int64_t)grp * 4096 + at[e]] = v[e];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counters + tp->counter, 1) == groups - 1;
  __syncthreads();
  if (!last) return false;
  __threadfence();
  add_tiles(sums, 0, groups);
  if (threadIdx.x == 0) counters[tp->counter] = 0;
  return true;
}

// The tile by the task's flags; for one chunk of a split sum (flag 8, FP64 C): split_sum, then the
// CTA that finishes the sum writes the total.
template <class T, class V>
__device__ __forceinline__ void gemm_epilogue(const GemmTask *tp, const V (&acc)[2][4][4], int wm, int wn, int g,
                                              int tg, double *part = nullptr, int32_t *counters = nullptr) {
  if constexpr (sizeof(T) == sizeof(double)) {
    if (tp->flags & 8) {
      double v[32];
      int at[32];
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int i = wm + r * 16 + g + 8 * (e >> 1), j = wn + c * 8 + 2 * tg + (e & 1);
            v[(r * 4 + c) * 4 + e] = acc[r][c][e];
            at[(r * 4 + c) * 4 + e] = i * 64 + j;
          }
      if (!split_sum(tp, part, counters, v, at)) return;
      double tot[2][4][4];
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
          for (int e = 0; e < 4; ++e) tot[r][c][e] = v[(r * 4 + c) * 4 + e];
      gemm_store<T>(tp, tp->flags & ~8, tot, wm, wn, g, tg);
      return;
    }
  }
  gemm_store<T>(tp, tp->flags, acc, wm, wn, g, tg);
}

// The main loop of a 64 x 64 tile of C -= A B^T over K range [kbeg, kend) of the task: 3-stage
// cp.async ring in `gsm`, DMMA into acc (this thread's fragments).
template <class TA, int STAGES = GEMM_STAGES>
__device__ __forceinline__ void gemm_mainloop(const GemmTask *tp, int kbeg, int kend, double (&acc)[2][4][4],
                                              double *gsm) {
  constexpr int SA = tile_stride<TA>();
  double(*Bs)[GEMM_KC][SROW] = reinterpret_cast<double(*)[GEMM_KC][SROW]>(gsm);
  TA(*As)[GEMM_KC][SA] = reinterpret_cast<TA(*)[GEMM_KC][SA]>(gsm + STAGES * GEMM_KC * SROW);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tg = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int K = kend - kbeg;
  const bool gather = tp->flags & 16;
  const TA *abase = static_cast<const TA *>(tp->A) + (int64_t)kbeg * tp->a_sk;
  const double *bbase = static_cast<const double *>(tp->B) + (gather ? 0 : (int64_t)kbeg * tp->b_sk);
  TileLoader<TA, GEMM_KC> la;
  TileLoader<double, GEMM_KC> lb;
  la.init(abase, tp->a_si, tp->a_sk, tp->M, tid);
  lb.init(bbase, tp->b_sj, tp->b_sk, tp->N, tid);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = acc[i][j][2] = acc[i][j][3] = 0.0;
  const int nk = (K + GEMM_KC - 1) / GEMM_KC;
  const int32_t *brows = gather ? tp->b_rows + kbeg : nullptr;
  const int64_t bsk = tp->b_sk;
  auto load_b = [&](int stage, int kb) {
    if (gather)
      lb.load_rows(Bs[stage], kb, K, bbase, brows, bsk, bbase);
    else
      lb.load(Bs[stage], kb, K, bbase);
  };
  // the first stages' A tiles go out together, before any B tile and before pdl_wait (A is a
  // factor or inverse block, which no kernel of a solve writes; a factorisation's launches are
  // ordinary, pdl_wait returns at once); the first commit group holds them with the first B tile.
  // A's bytes in flight from the start: with few right-hand sides, where A is nearly all of a
  // tile's bytes, the FP64 solve of the 48^3 block took 7.8 ms instead of 9.6
  for (int st = 0; st < STAGES - 1; ++st)
    if (st < nk) la.load(As[st], st * GEMM_KC, K, abase);
  pdl_wait();
  pdl_trigger();
  for (int st = 0; st < STAGES - 1; ++st) {
    if (st < nk) load_b(st, st * GEMM_KC);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const int pf = kt + STAGES - 1;
    if (pf < nk) {
      la.load(As[pf % STAGES], pf * GEMM_KC, K, abase);
      load_b(pf % STAGES, pf * GEMM_KC);
    }
    cp_async_commit();
    const int st = kt % STAGES;
#pragma unroll
    for (int kk = 0; kk < GEMM_KC; kk += 8) {
      double av[2][4], bv[4][2];
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int i = wm + r * 16 + g;
        av[r][0] = (double)As[st][kk + tg][i];
        av[r][1] = (double)As[st][kk + tg][i + 8];
        av[r][2] = (double)As[st][kk + tg + 4][i];
        av[r][3] = (double)As[st][kk + tg + 4][i + 8];
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        bv[c][0] = Bs[st][kk + tg][wn + c * 8 + g];
        bv[c][1] = Bs[st][kk + tg + 4][wn + c * 8 + g];
      }
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) dmma16(acc[r][c], av[r], bv[c]);
    }
  }
  cp_async_wait<0>();
}

template <class TA, int STAGES = GEMM_STAGES>
__global__ void __launch_bounds__(GEMM_THREADS, STAGES == GEMM_STAGES ? 3 : 1)
    gemm_kernel(const GemmTask *__restrict__ tasks, double *part, int32_t *counters) {
  extern __shared__ __align__(16) double gsm[];
  const GemmTask *tp = tasks + blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, tg = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  double acc[2][4][4];
  gemm_mainloop<TA, STAGES>(tp, 0, tp->K, acc, gsm);
  gemm_epilogue<double>(tp, acc, wm, wn, g, tg, part, counters);
}

// ---- the solve's products for a few right-hand sides -------------------------------------------
// With at most 16 right-hand sides a 64 x 64 tile spends most of its DMMA work on zero columns.
// This kernel's tile is 64 x NW (NW = 8 or 16 columns): warp w takes rows [16 w, 16 w + 16) with
// NW / 8 fragments of 8 columns. Its K loop is gemm_kernel's (the same stages, the same m16n8k8
// instruction over the same K order) and a split sum's chunks are added in the same order, so every
// element's bits are the ones gemm_kernel gives: a column's solution does not depend on how many
// right-hand sides were solved together. B rows are NW + 4 doubles apart, so a half-warp's fragment
// reads of 4 k-rows x 4 columns fall in distinct banks.
template <int NW>
__host__ __device__ constexpr int narrow_row() {
  return NW + 4;
}
template <class TA, int NW, int STAGES = GEMM_STAGES>
__host__ __device__ constexpr size_t gemm_narrow_smem() {
  return STAGES * GEMM_KC * (sizeof(TA) * tile_stride<TA>() + sizeof(double) * narrow_row<NW>());
}

template <class TA, int NW, int STAGES = GEMM_STAGES>
__global__ void __launch_bounds__(GEMM_THREADS, STAGES == GEMM_STAGES ? 6 : 2)
    gemm_narrow_kernel(const GemmTask *__restrict__ tasks, double *part, int32_t *counters) {
  constexpr int NF = NW / 8, SA = tile_stride<TA>(), SN = narrow_row<NW>();
  constexpr int BPER = NW * GEMM_KC / GEMM_THREADS;  // B elements per thread per stage
  static_assert(BPER >= 1 && NW * GEMM_KC % GEMM_THREADS == 0, "narrow tile");
  extern __shared__ __align__(16) double gsm[];
  double(*Bs)[GEMM_KC][SN] = reinterpret_cast<double(*)[GEMM_KC][SN]>(gsm);
  TA(*As)[GEMM_KC][SA] = reinterpret_cast<TA(*)[GEMM_KC][SA]>(gsm + STAGES * GEMM_KC * SN);
  const GemmTask *tp = tasks + blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tg = lane & 3;
  const int wm = warp * 16;
  const int K = tp->K, N = tp->N;
  const bool gather = tp->flags & 16;
  const TA *abase = static_cast<const TA *>(tp->A);
  const double *bbase = static_cast<const double *>(tp->B);
  const int64_t bsj = tp->b_sj, bsk = tp->b_sk;
  const int32_t *brows = tp->b_rows;
  TileLoader<TA, GEMM_KC> la;
  la.init(abase, tp->a_si, tp->a_sk, tp->M, tid);
  // B element (k, j) at B + k b_sk + j b_sj (through the row list: B + rows[k] b_sk + j, b_sj = 1);
  // this thread's: j fixed, k = k0 + q * dk (the unit-stride index runs along the warp)
  const bool jfast = bsj == 1;
  const int bj = jfast ? tid % NW : tid / GEMM_KC;
  const int bk0 = jfast ? tid / NW : tid % GEMM_KC;
  const int bdk = jfast ? GEMM_THREADS / NW : 0;
  const int bdj = jfast ? 0 : GEMM_THREADS / GEMM_KC;
  auto load_b = [&](int stage, int kb) {
#pragma unroll
    for (int q = 0; q < BPER; ++q) {
      const int k = bk0 + q * bdk, j = bj + q * bdj;
      const bool ok = j < N && kb + k < K;
      const double *src = bbase;
      if (ok) src = gather ? bbase + (int64_t)brows[kb + k] * bsk + j : bbase + (int64_t)(kb + k) * bsk + j * bsj;
      cp_async<sizeof(double)>(&Bs[stage][k][j], src, ok ? (int)sizeof(double) : 0);
    }
  };
  double acc[NF][4];
#pragma unroll
  for (int c = 0; c < NF; ++c) acc[c][0] = acc[c][1] = acc[c][2] = acc[c][3] = 0.0;
  const int nk = (K + GEMM_KC - 1) / GEMM_KC;
  // as in gemm_mainloop: the first stages' A tiles before pdl_wait, in the first commit group
  for (int st = 0; st < STAGES - 1; ++st)
    if (st < nk) la.load(As[st], st * GEMM_KC, K, abase);
  pdl_wait();
  pdl_trigger();
  for (int st = 0; st < STAGES - 1; ++st) {
    if (st < nk) load_b(st, st * GEMM_KC);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const int pf = kt + STAGES - 1;
    if (pf < nk) {
      la.load(As[pf % STAGES], pf * GEMM_KC, K, abase);
      load_b(pf % STAGES, pf * GEMM_KC);
    }
    cp_async_commit();
    const int st = kt % STAGES;
#pragma unroll
    for (int kk = 0; kk < GEMM_KC; kk += 8) {
      double av[4], bv[NF][2];
      const int i = wm + g;
      av[0] = (double)As[st][kk + tg][i];
      av[1] = (double)As[st][kk + tg][i + 8];
      av[2] = (double)As[st][kk + tg + 4][i];
      av[3] = (double)As[st][kk + tg + 4][i + 8];
#pragma unroll
      for (int c = 0; c < NF; ++c) {
        bv[c][0] = Bs[st][kk + tg][c * 8 + g];
        bv[c][1] = Bs[st][kk + tg + 4][c * 8 + g];
      }
#pragma unroll
      for (int c = 0; c < NF; ++c) dmma16(acc[c], av, bv[c]);
    }
  }
  cp_async_wait<0>();
  // fragment element e of column block c: row wm + g + 8 (e >> 1), column 8 c + 2 tg + (e & 1)
  int flags = tp->flags;
  if (flags & 8) {
    double v[NF * 4];
    int at[NF * 4];
#pragma unroll
    for (int c = 0; c < NF; ++c)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        v[c * 4 + e] = acc[c][e];
        at[c * 4 + e] = (wm + g + 8 * (e >> 1)) * 64 + c * 8 + 2 * tg + (e & 1);
      }
    if (!split_sum(tp, part, counters, v, at)) return;
#pragma unroll
    for (int c = 0; c < NF; ++c)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[c][e] = v[c * 4 + e];
    flags &= ~8;
  }
  const int M = tp->M;
  const bool lower = flags & 1;
  double *C = static_cast<double *>(tp->C);
#pragma unroll
  for (int c = 0; c < NF; ++c)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int i = wm + g + 8 * (e >> 1), j = c * 8 + 2 * tg + (e & 1);
      if (i < M && j < N && (!lower || i >= j)) {
        double *dst = C + (int64_t)i * tp->c_si + (int64_t)j * tp->c_sj;
        *dst = (flags & 4) ? acc[c][e] : (flags & 2) ? -acc[c][e] : *dst - acc[c][e];
      }
    }
}

// ---- the solve's short products, K split over a thread-block cluster -------------------------
// A launch of the solve with few output tiles leaves most SMs idle and each CTA walks a long K
// alone. Here the 8 CTAs of a cluster share one 64 x 64 tile: CTA rank q takes the q-th of 8 equal
// slices of K (multiples of GEMM_KC), keeps its partial tile in its shared memory, and after a
// cluster barrier each CTA adds the 8 partials of 8 of the tile's rows in rank order, reading the
// others' shared memory directly (distributed shared memory), and applies the task's epilogue to
// those rows. A chunk of a longer sum (flag 8) stores its rows' totals as the chunk's partial; the
// last cluster to finish (an atomic count) adds the chunks in order, each CTA its 8 rows. Every
// sum's order depends on K alone, not on the number of right-hand sides.
template <class TA>
__global__ void __cluster_dims__(SOLVE_CLUSTER, 1, 1) __launch_bounds__(GEMM_THREADS, 3)
    gemm_cluster_kernel(const GemmTask *__restrict__ tasks, double *part, int32_t *counters) {
  extern __shared__ __align__(16) double gsm[];
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int q = (int)cluster.block_rank();
  const GemmTask *tp = tasks + blockIdx.x / SOLVE_CLUSTER;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tg = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int K = tp->K;
  const int slice = ((K + SOLVE_CLUSTER - 1) / SOLVE_CLUSTER + GEMM_KC - 1) / GEMM_KC * GEMM_KC;
  const int kb = min(K, q * slice), ke = min(K, kb + slice);
  double acc[2][4][4];
  gemm_mainloop<TA>(tp, kb, ke, acc, gsm);
  __syncthreads();  // the ring is drained: its space takes the partial tile
  double *mine = gsm;  // [i * 64 + j]
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int e = 0; e < 4; ++e)
        mine[(wm + r * 16 + g + 8 * (e >> 1)) * 64 + wn + c * 8 + 2 * tg + (e & 1)] = acc[r][c][e];
  cluster.sync();
  // this CTA's 8 rows: 512 values, 4 a thread, the 8 partials added in rank order
  constexpr int ROWS = 64 / SOLVE_CLUSTER, PER = ROWS * 64 / GEMM_THREADS;
  double tot[PER];
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int e = tid + u * GEMM_THREADS, i = q * ROWS + e / 64, j = e % 64;
    double sum = 0.0;
#pragma unroll
    for (int p = 0; p < SOLVE_CLUSTER; ++p) sum += cluster.map_shared_rank(mine, p)[i * 64 + j];
    tot[u] = sum;
  }
  const int M = tp->M, N = tp->N, flags = tp->flags;
  if (flags & 8) {
    // a chunk of a split sum: its rows' totals are the chunk's partial; the last cluster adds them
    __shared__ int last;
    double *P = part + tp->part_off;
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int e = tid + u * GEMM_THREADS;
      P[(int64_t)tp->chunk * 4096 + q * ROWS * 64 + e] = tot[u];
    }
    __threadfence();
    cluster.sync();  // every CTA's rows are stored (and the peers are done with `mine`)
    if (q == 0 && tid == 0) {
      const int done = atomicAdd(counters + tp->counter, 1) == tp->chunks - 1;
      for (int p = 0; p < SOLVE_CLUSTER; ++p) *cluster.map_shared_rank(&last, p) = done;
    }
    cluster.sync();
    if (!last) return;
    __threadfence();
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int e = tid + u * GEMM_THREADS;
      double sum = 0.0;
      for (int c = 0; c < tp->chunks; ++c) sum += __ldcg(P + (int64_t)c * 4096 + q * ROWS * 64 + e);
      tot[u] = sum;
    }
    cluster.sync();  // every CTA has read the counter's round
    if (q == 0 && tid == 0) counters[tp->counter] = 0;
  } else {
    cluster.sync();  // the peers are done reading this CTA's partial
  }
  const bool lower = flags & 1;
  double *C = static_cast<double *>(tp->C);
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int e = tid + u * GEMM_THREADS, i = q * ROWS + e / 64, j = e % 64;
    if (i < M && j < N && (!lower || i >= j)) {
      double *dst = C + (int64_t)i * tp->c_si + (int64_t)j * tp->c_sj;
      *dst = (flags & 4) ? tot[u] : (flags & 2) ? -tot[u] : *dst - tot[u];
    }
  }
}

// ---- tiled C -= A B^T in FP32 by 3xTF32 on the tensor pipe ---------------------------------------
// The FP32 factorisation's updates: the same 64 x 64 tiles and 32 x 32 warp tiles as gemm_kernel,
// K in chunks of 32 floats; every operand x = hi + lo (TF32 halves) and each product is
// hi*hi + hi*lo + lo*hi, accumulated in FP32.
constexpr int FKC = 32, FS = 72;
constexpr size_t GEMM_F32_SMEM = sizeof(float) * GEMM_STAGES * 2 * FKC * FS;

__global__ void __launch_bounds__(GEMM_THREADS, 4) gemm_tf32x3_kernel(const GemmTask *__restrict__ tasks) {
  extern __shared__ __align__(16) float fsm[];
  float(*As)[FKC][FS] = reinterpret_cast<float(*)[FKC][FS]>(fsm);
  float(*Bs)[FKC][FS] = reinterpret_cast<float(*)[FKC][FS]>(fsm + GEMM_STAGES * FKC * FS);
  const GemmTask *tp = tasks + blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tg = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int K = tp->K;
  const float *abase = static_cast<const float *>(tp->A), *bbase = static_cast<const float *>(tp->B);
  TileLoader<float, FKC> la, lb;
  la.init(abase, tp->a_si, tp->a_sk, tp->M, tid);
  lb.init(bbase, tp->b_sj, tp->b_sk, tp->N, tid);
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = acc[i][j][2] = acc[i][j][3] = 0.f;
  const int nk = (K + FKC - 1) / FKC;
#pragma unroll
  for (int st = 0; st < GEMM_STAGES - 1; ++st) {
    if (st < nk) {
      la.load(As[st], st * FKC, K, abase);
      lb.load(Bs[st], st * FKC, K, bbase);
    }
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<GEMM_STAGES - 2>();
    __syncthreads();
    const int pf = kt + GEMM_STAGES - 1;
    if (pf < nk) {
      la.load(As[pf % GEMM_STAGES], pf * FKC, K, abase);
      lb.load(Bs[pf % GEMM_STAGES], pf * FKC, K, bbase);
    }
    cp_async_commit();
    const int st = kt % GEMM_STAGES;
#pragma unroll
    for (int kk = 0; kk < FKC; kk += 8) {
      uint32_t ah[2][4], al[2][4], bh[4][2], bl[4][2];
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int i = wm + r * 16 + g;
        tf32_split(As[st][kk + tg][i], ah[r][0], al[r][0]);
        tf32_split(As[st][kk + tg][i + 8], ah[r][1], al[r][1]);
        tf32_split(As[st][kk + tg + 4][i], ah[r][2], al[r][2]);
        tf32_split(As[st][kk + tg + 4][i + 8], ah[r][3], al[r][3]);
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        tf32_split(Bs[st][kk + tg][wn + c * 8 + g], bh[c][0], bl[c][0]);
        tf32_split(Bs[st][kk + tg + 4][wn + c * 8 + g], bh[c][1], bl[c][1]);
      }
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          tmma16(acc[r][c], al[r], bh[c]);
          tmma16(acc[r][c], ah[r], bl[c]);
          tmma16(acc[r][c], ah[r], bh[c]);
        }
    }
  }
  cp_async_wait<0>();
  gemm_epilogue<float>(tp, acc, wm, wn, g, tg);
}

// ---- solve -------------------------------------------------------------------------------------
// Rows [i0, i1) of supernode s's solve front: zero its update rows, then add the children's
// update vectors in child order.
__global__ void __launch_bounds__(256) solve_assemble_kernel(Tree t, double *__restrict__ x, double *__restrict__ v,
                                                             const int64_t *__restrict__ voff, int R,
                                                             const RowTask *__restrict__ tasks,
                                                             const int2 *__restrict__ ranges) {
  const RowTask task = tasks[blockIdx.x];
  const int s = task.s;
  const int64_t w = t.width[s], f = t.first[s];
  double *vs = v + voff[s];
  const int tid = threadIdx.x;
  const int64_t z0 = task.i0 > w ? task.i0 : w;
  pdl_wait();
  pdl_trigger();
  for (int64_t e = tid; e < (task.i1 - z0) * R; e += blockDim.x) vs[(z0 - w) * R + e] = 0.0;
  __syncthreads();
  const int64_t k0 = t.kid_ptr[s], k1 = t.kid_ptr[s + 1];
  for (int64_t kp = k0; kp < k1; ++kp) {
    const int c = t.kids[kp];
    const int32_t *rel = t.rel + t.rel_off[c];
    const double *vc = v + voff[c];
    const int2 range = ranges[task.ranges + (kp - k0)];
    const int lo = range.x, hi = range.y;
    for (int64_t e = tid; e < (int64_t)(hi - lo) * R; e += blockDim.x) {
      const int ic = lo + (int)(e / R), j = (int)(e % R);
      const int64_t I = rel[ic];
      double *dst = I < w ? x + (f + I) * R + j : vs + (I - w) * R + j;
      *dst += vc[(int64_t)ic * R + j];
    }
    __syncthreads();
  }
}

// ---- thin supernodes' solve steps ---------------------------------------------------------------
// Forward, one tile (THIN_ROWS rows) of a thin supernode's update vector: the own rows (x plus the
// children's rows that land on them, child by child), y = Dinv x, then the tile = -L(rows, :) y
// plus the children's rows that land in it, stored once. Every tile of the supernode forms y the
// same way (w <= SOLVE_THIN rows), so no tile waits for another. Each phase issues its global
// loads together (the tile's rows of L, the inverse and the own rows are staged in shared memory
// first; a child's rows are read a warp per row, several rows in flight). Values stay FP64; an
// FP32 L is widened. Per entry the operations and their order do not depend on R.
constexpr int THIN_THREADS = 256, THIN_WARPS = THIN_THREADS / 32;

template <class T>
__global__ void __launch_bounds__(THIN_THREADS) thin_fwd_kernel(Tree t, const double *__restrict__ x,
                                                                double *__restrict__ x2, double *__restrict__ v,
                                                                const int64_t *__restrict__ voff, int R, int lg,
                                                                const ThinTask *__restrict__ tasks,
                                                                const int4 *__restrict__ ranges) {
  __shared__ double tile[THIN_ROWS * 64];
  __shared__ double xs[SOLVE_THIN * 64], ys[SOLVE_THIN * 64];
  __shared__ double lt[SOLVE_THIN * THIN_ROWS];  // lt[k * THIN_ROWS + r] = L(i0 + r, k)
  __shared__ double di[SOLVE_THIN * SOLVE_THIN];
  const ThinTask task = tasks[blockIdx.x];
  const int s = task.s, RP = 1 << lg, j0 = task.j0, nj = min(RP, R - j0);
  const int m = t.height[s], w = t.width[s];
  const int64_t f = t.first[s];
  const T *Ls = static_cast<const T *>(t.L) + t.loff[s];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int k0 = (int)t.kid_ptr[s], k1 = (int)t.kid_ptr[s + 1];
  const int i0 = task.i0, nr = task.i1 - task.i0;
#pragma unroll
  for (int q = 0; q < SOLVE_THIN * 64 / THIN_THREADS; ++q) {
    const int e = tid + q * THIN_THREADS, k = e >> 6, j = e & 63;
    if (k < w) lt[k * THIN_ROWS + j] = j < nr ? (double)Ls[(int64_t)k * m + i0 + j] : 0.0;
  }
  if (tid < w * w) di[tid] = t.Dinv[task.dinv + tid];
  pdl_wait();  // L and the inverse above; x and the update vectors below
  pdl_trigger();
#pragma unroll
  for (int q = 0; q < SOLVE_THIN * 64 / THIN_THREADS; ++q) {
    const int e = tid + q * THIN_THREADS, k = e >> 6, j = e & 63;
    if (k < w && j < RP) xs[(k << lg) + j] = j < nj ? x[(f + k) * R + j0 + j] : 0.0;
  }
  __syncthreads();
  for (int kp = k0; kp < k1; ++kp) {
    const int4 g = ranges[task.ranges + (kp - k0)];
    if (g.x == 0) continue;  // the same for the whole block
    const int c = t.kids[kp];
    const int32_t *rel = t.rel + t.rel_off[c];
    const double *vc = v + voff[c];
    // at most w rows: a warp each
    for (int ic = warp; ic < g.x; ic += THIN_WARPS) {
      const int row = rel[ic];
      for (int j = lane; j < nj; j += 32) xs[(row << lg) + j] += vc[(int64_t)ic * R + j0 + j];
    }
    __syncthreads();
  }
  for (int e = tid; e < w << lg; e += THIN_THREADS) {
    const int i = e >> lg, j = e & (RP - 1);
    double acc = 0.0;
    for (int k = 0; k <= i; ++k) acc = fma(di[i + k * w], xs[(k << lg) + j], acc);
    ys[e] = acc;
    if (task.first && j < nj) x2[(f + i) * R + j0 + j] = acc;
  }
  __syncthreads();
  for (int e = tid; e < nr << lg; e += THIN_THREADS) {
    const int r = e >> lg, j = e & (RP - 1);
    double acc = 0.0;
    for (int k = 0; k < w; ++k) acc = fma(lt[k * THIN_ROWS + r], ys[(k << lg) + j], acc);
    tile[e] = -acc;
  }
  __syncthreads();
  for (int kp = k0; kp < k1; ++kp) {
    const int4 g = ranges[task.ranges + (kp - k0)];
    if (g.y >= g.z) continue;  // the same for the whole block
    const int c = t.kids[kp];
    const int32_t *rel = t.rel + t.rel_off[c];
    const double *vc = v + voff[c];
    // a warp per child row (they land on distinct rows), four rows a warp in flight
    for (int b = g.y + warp; b < g.z; b += 4 * THIN_WARPS) {
      int at[4];
      double va[4], vb[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int ic = b + q * THIN_WARPS;
        at[q] = -1;
        if (ic < g.z) {
          at[q] = (rel[ic] - i0) << lg;
          const double *src = vc + (int64_t)ic * R + j0;
          va[q] = lane < nj ? src[lane] : 0.0;
          vb[q] = lane + 32 < nj ? src[lane + 32] : 0.0;
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (at[q] >= 0) {
          if (lane < nj) tile[at[q] + lane] += va[q];
          if (lane + 32 < nj) tile[at[q] + lane + 32] += vb[q];
        }
    }
    __syncthreads();
  }
  double *vs = v + voff[s];
  for (int e = tid; e < nr << lg; e += THIN_THREADS) {
    const int r = e >> lg, j = e & (RP - 1);
    if (j < nj) vs[(int64_t)(i0 + r - w) * R + j0 + j] = tile[e];
  }
}

// Backward, one chunk (THIN_CHUNK rows) of a thin supernode's rows past its columns:
// z_part = L21(rows, :)^T x(rows), the rows' final values read straight from x. The chunk's row
// indices and rows of L21 are staged in shared memory; warp q takes rows q, q + 8, ... (a row's
// right-hand sides across its lanes, four rows in flight), and the warps' sums are added in warp
// order, whatever R is. A supernode of several chunks keeps the partial sums; the last chunk to
// finish (an atomic count, reset by it for the next solve; no CTA waits) adds them in chunk order
// and forms z = x2 - sum and x = Dinv^T z on the supernode's own rows.
template <class T>
__global__ void __launch_bounds__(THIN_THREADS) thin_bwd_kernel(Tree t, double *__restrict__ x,
                                                                const double *__restrict__ x2, int R, int lg,
                                                                const ThinBwdTask *__restrict__ tasks,
                                                                double *__restrict__ part,
                                                                int32_t *__restrict__ counters) {
  __shared__ int32_t ridx[THIN_CHUNK];
  __shared__ double lt[THIN_CHUNK * SOLVE_THIN];  // lt[i * SOLVE_THIN + k] = L21(k0 + i, k)
  __shared__ double red[THIN_WARPS * SOLVE_THIN * 64];
  __shared__ double zs[SOLVE_THIN * 64];
  __shared__ int last;
  const ThinBwdTask task = tasks[blockIdx.x];
  const int s = task.s, RP = 1 << lg, j0 = task.j0, nj = min(RP, R - j0);
  const int m = t.height[s], w = t.width[s];
  const int64_t f = t.first[s];
  const T *Lb = static_cast<const T *>(t.L) + t.loff[s] + w;  // Lb[k m + i] = L21(i, k)
  const int32_t *rows = t.rows + t.rows_off[s] + w;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n = task.k1 - task.k0;
  if (tid < n) ridx[tid] = rows[task.k0 + tid];
#pragma unroll
  for (int q = 0; q < THIN_CHUNK * SOLVE_THIN / THIN_THREADS; ++q) {
    const int e = tid + q * THIN_THREADS, k = e / THIN_CHUNK, i = e - k * THIN_CHUNK;
    if (k < w && i < n) lt[i * SOLVE_THIN + k] = (double)Lb[(int64_t)k * m + task.k0 + i];
  }
  pdl_wait();  // the row list and L above; x, x2, the partial sums and counters below
  pdl_trigger();
  __syncthreads();
  double acc[SOLVE_THIN][2];
#pragma unroll
  for (int k = 0; k < SOLVE_THIN; ++k) acc[k][0] = acc[k][1] = 0.0;
  const bool la = lane < nj, lb = lane + 32 < nj;
  for (int b = warp; b < n; b += 4 * THIN_WARPS) {
    double xa[4], xb[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = b + q * THIN_WARPS;
      xa[q] = xb[q] = 0.0;
      if (i < n) {
        const double *src = x + (int64_t)ridx[i] * R + j0;
        if (la) xa[q] = src[lane];
        if (lb) xb[q] = src[lane + 32];
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = b + q * THIN_WARPS;
      if (i < n) {
#pragma unroll
        for (int k = 0; k < SOLVE_THIN; ++k)
          if (k < w) {
            const double l = lt[i * SOLVE_THIN + k];
            acc[k][0] = fma(l, xa[q], acc[k][0]);
            acc[k][1] = fma(l, xb[q], acc[k][1]);
          }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < SOLVE_THIN; ++k)
    if (k < w) {
      red[(warp * SOLVE_THIN + k) * 64 + lane] = acc[k][0];
      red[(warp * SOLVE_THIN + k) * 64 + lane + 32] = acc[k][1];
    }
  __syncthreads();
  for (int e = tid; e < w * 64; e += THIN_THREADS) {
    const int k = e >> 6, j = e & 63;
    double sum = 0.0;
    for (int q = 0; q < THIN_WARPS; ++q) sum += red[(q * SOLVE_THIN + k) * 64 + j];
    zs[e] = sum;
  }
  if (task.chunks > 1) {
    double *mine = part + task.part + (int64_t)task.chunk * SOLVE_THIN * 64;
    for (int e = tid; e < w * 64; e += THIN_THREADS) mine[e] = zs[e];
    __threadfence();
    __syncthreads();
    if (tid == 0) last = atomicAdd(counters + task.counter, 1) == task.chunks - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const double *all = part + task.part;
    for (int e = tid; e < w * 64; e += THIN_THREADS) {
      double sum = 0.0;
      for (int q = 0; q < task.chunks; ++q) sum += __ldcg(all + (int64_t)q * SOLVE_THIN * 64 + e);
      zs[e] = sum;
    }
    if (tid == 0) counters[task.counter] = 0;
  }
  __syncthreads();
  for (int e = tid; e < w * 64; e += THIN_THREADS) {
    const int k = e >> 6, j = e & 63;
    zs[e] = j < nj ? x2[(f + k) * R + j0 + j] - zs[e] : 0.0;
  }
  __syncthreads();
  const double *Di = t.Dinv + task.dinv;
  for (int e = tid; e < w * 64; e += THIN_THREADS) {
    const int i = e >> 6, j = e & 63;
    if (j >= nj) continue;
    double acc2 = 0.0;
    for (int k = i; k < w; ++k) acc2 = fma(Di[k + i * w], zs[(k << 6) + j], acc2);
    x[(f + i) * R + j0 + j] = acc2;
  }
}

// x[i*R + j] = b[perm[i] + j*ld] (times scale[i] when scaled), and back.
__global__ void permute_in_kernel(const int64_t *__restrict__ perm, int64_t n, const double *__restrict__ b,
                                  int64_t ld, double *__restrict__ x, int R, const double *__restrict__ scale) {
  const int64_t total = n * R;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / R;
    const int j = (int)(e % R);
    const double v = b[perm[i] + j * ld];
    x[e] = scale ? v * scale[i] : v;
  }
}

__global__ void permute_out_kernel(const int64_t *__restrict__ perm, int64_t n, const double *__restrict__ x, int R,
                                   double *__restrict__ b, int64_t ld, const double *__restrict__ scale) {
  const int64_t total = n * R;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / R;
    const int j = (int)(e % R);
    b[perm[i] + j * ld] = scale ? x[e] * scale[i] : x[e];
  }
}

// y = A x with x and y row-major (n x R: a row's right-hand sides contiguous): one warp per row and
// block of 64 right-hand sides, two a lane, the row's entries in order (index and value the same
// for the whole warp, the x row of each entry read as 512 contiguous bytes; four entries in
// flight). Each output is one thread's sum over the row in entry order, whatever R is.
__global__ void __launch_bounds__(256) spmv_rows_kernel(int64_t n, const int64_t *__restrict__ ptr,
                                                        const int32_t *__restrict__ idx,
                                                        const double *__restrict__ val,
                                                        const double *__restrict__ x, double *__restrict__ y, int R) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (row >= n) return;
  const int ja = blockIdx.y * 64 + lane, jb = ja + 32;
  const bool oka = ja < R, okb = jb < R;
  double a0 = 0.0, a1 = 0.0;
  const int64_t e1 = ptr[row + 1];
  int64_t e = ptr[row];
  for (; e + 3 < e1; e += 4) {
    int c[4];
    double v[4], xa[4], xb[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      c[q] = idx[e + q];
      v[q] = val[e + q];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double *xr = x + (int64_t)c[q] * R;
      xa[q] = oka ? xr[ja] : 0.0;
      xb[q] = okb ? xr[jb] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      a0 = fma(v[q], xa[q], a0);
      a1 = fma(v[q], xb[q], a1);
    }
  }
  for (; e < e1; ++e) {
    const double v = val[e];
    const double *xr = x + (int64_t)idx[e] * R;
    if (oka) a0 = fma(v, xr[ja], a0);
    if (okb) a1 = fma(v, xr[jb], a1);
  }
  if (oka) y[row * R + ja] = a0;
  if (okb) y[row * R + jb] = a1;
}

// dst (n x R row-major) <- src (column-major, leading dimension ld), and back: 32 x 32 tiles
// through shared memory, both sides coalesced.
__global__ void __launch_bounds__(256) to_rows_kernel(int64_t n, int R, const double *__restrict__ src, int64_t ld,
                                                      double *__restrict__ dst) {
  __shared__ double tile[32][33];
  const int64_t i0 = (int64_t)blockIdx.x * 32;
  const int j0 = blockIdx.y * 32, tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int k = ty; k < 32; k += 8) {
    const int64_t i = i0 + tx;
    const int j = j0 + k;
    if (i < n && j < R) tile[k][tx] = src[i + (int64_t)j * ld];
  }
  __syncthreads();
  for (int k = ty; k < 32; k += 8) {
    const int64_t i = i0 + k;
    const int j = j0 + tx;
    if (i < n && j < R) dst[i * R + j] = tile[tx][k];
  }
}

__global__ void __launch_bounds__(256) to_cols_kernel(int64_t n, int R, const double *__restrict__ src,
                                                      double *__restrict__ dst, int64_t ld) {
  __shared__ double tile[32][33];
  const int64_t i0 = (int64_t)blockIdx.x * 32;
  const int j0 = blockIdx.y * 32, tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int k = ty; k < 32; k += 8) {
    const int64_t i = i0 + k;
    const int j = j0 + tx;
    if (i < n && j < R) tile[tx][k] = src[i * R + j];
  }
  __syncthreads();
  for (int k = ty; k < 32; k += 8) {
    const int64_t i = i0 + tx;
    const int j = j0 + k;
    if (i < n && j < R) dst[i + (int64_t)j * ld] = tile[k][tx];
  }
}

// y = A x for RB right-hand sides at once: one warp per row, its lanes over the row's entries
// (so a warp reads the row's indices and values once, contiguously, for all RB vectors), then a
// butterfly sum of the lanes. x and y are column-major with leading dimensions ldx and ldy.
template <int RB>
__global__ void __launch_bounds__(256) spmv_kernel(int64_t n, const int64_t *__restrict__ ptr,
                                                   const int32_t *__restrict__ idx, const double *__restrict__ val,
                                                   const double *__restrict__ x, int64_t ldx, double *__restrict__ y,
                                                   int64_t ldy, int R) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int j0 = blockIdx.y * RB;
  if (row >= n) return;
  const int nb = min(RB, R - j0);
  const double *xj = x + j0 * ldx;
  double acc[RB];
#pragma unroll
  for (int j = 0; j < RB; ++j) acc[j] = 0.0;
  for (int64_t p = ptr[row] + lane; p < ptr[row + 1]; p += 32) {
    const double v = val[p];
    const int64_t c = idx[p];
#pragma unroll
    for (int j = 0; j < RB; ++j)
      if (j < nb) acc[j] += v * xj[c + j * ldx];
  }
#pragma unroll
  for (int j = 0; j < RB; ++j) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
    if (lane == j && j < nb) y[row + (j0 + j) * ldy] = acc[j];
  }
}

// The refinement's vector steps on column-major n x R blocks: r = b - Ax (residual, in place of
// Ax) and x += d (update), each block with its own leading dimension.
__global__ void residual_kernel(int64_t n, int R, const double *__restrict__ b, int64_t ldb, double *__restrict__ ax,
                                int64_t ldax) {
  const int64_t total = n * R;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e % n, j = e / n;
    ax[i + j * ldax] = b[i + j * ldb] - ax[i + j * ldax];
  }
}

__global__ void update_kernel(int64_t n, int R, const double *__restrict__ d, int64_t ldd, double *__restrict__ x,
                              int64_t ldx) {
  const int64_t total = n * R;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e % n, j = e / n;
    x[i + j * ldx] += d[i + j * ldd];
  }
}

// Preconditioned CG on column-major n x R blocks, one independent recurrence per column, every
// scalar on the device: out[j] = sum_i a(i, j) b(i, j) (one CTA a column, a fixed tree order).
__global__ void __launch_bounds__(256) coldot_kernel(int64_t n, const double *__restrict__ a, int64_t lda,
                                                     const double *__restrict__ b, int64_t ldb,
                                                     double *__restrict__ out) {
  __shared__ double part[256];
  const double *ca = a + blockIdx.x * lda, *cb = b + blockIdx.x * ldb;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += ca[i] * cb[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) part[threadIdx.x] += part[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = part[0];
}

// alpha_j = rz[j] / pq[j]; x_j += alpha_j p_j; r_j -= alpha_j q_j (columns with done[j] set keep x, r).
__global__ void pcg_step_kernel(int64_t n, int R, const double *__restrict__ rz, const double *__restrict__ pq,
                                const int *__restrict__ done, const double *__restrict__ p, const double *__restrict__ q,
                                double *__restrict__ x, int64_t ldx, double *__restrict__ r) {
  const int64_t total = n * R;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e % n, j = e / n;
    if (done[j]) continue;
    const double alpha = pq[j] != 0.0 ? rz[j] / pq[j] : 0.0;
    x[i + j * ldx] += alpha * p[e];
    r[e] -= alpha * q[e];
  }
}

// p_j = z_j + (rz_new[j] / rz_old[j]) p_j
__global__ void pcg_direction_kernel(int64_t n, int R, const double *__restrict__ rz_new,
                                     const double *__restrict__ rz_old, const double *__restrict__ z,
                                     double *__restrict__ p) {
  const int64_t total = n * R;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = e / n;
    const double beta = rz_old[j] != 0.0 ? rz_new[j] / rz_old[j] : 0.0;
    p[e] = z[e] + beta * p[e];
  }
}

// out[j] = sum_i v(i, j)^2 for each column j (one CTA a column, a fixed tree order).
__global__ void __launch_bounds__(256) sumsq_kernel(int64_t n, int64_t ld, const double *__restrict__ v,
                                                    double *__restrict__ out) {
  __shared__ double part[256];
  const double *col = v + blockIdx.x * ld;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += col[i] * col[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) part[threadIdx.x] += part[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = part[0];
}

// The factor in the reference's packed trapezoids; an FP32 factor of S A S is brought back to A's
// (L(A) = S^-1 L(S A S), row by row).
template <class T>
__global__ void pack_kernel(Tree t, const int64_t *__restrict__ toff, double *__restrict__ dst) {
  const int s = blockIdx.x;
  const int64_t m = t.height[s], w = t.width[s];
  const T *Ls = static_cast<const T *>(t.L) + t.loff[s];
  const int32_t *rows = t.rows + t.rows_off[s];
  double *d = dst + toff[s];
  for (int64_t c = 0; c < w; ++c) {
    const int64_t start = c * m - c * (c > 0 ? c - 1 : 0) / 2;
    const int64_t p = c / NB, c0 = p * NB, c1 = c0 + NB < w ? c0 + NB : w, pw = c1 - c0;
    const double *Dp = t.D + t.doff[s] + 2 * (int64_t)NB * NB * p;
    for (int64_t r = c + threadIdx.x; r < m; r += blockDim.x) {
      const double v = r < c1 ? Dp[(c - c0) * pw + (r - c0)] : (double)Ls[r + c * m];
      d[start + r - c] = t.scale ? v / t.scale[rows[r]] : v;
    }
  }
}

template <class K>
void set_smem(K kernel, size_t bytes) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

void configure_kernels() {
  static bool done = false;
  if (done) return;
  set_smem(panel_kernel<double>, panel_smem<double>(64));
  set_smem(panel_kernel<float>, panel_smem<float>(64));
  set_smem(gemm_kernel<double>, gemm_smem<double>());
  set_smem(gemm_kernel<float>, gemm_smem<float>());
  set_smem(gemm_cluster_kernel<double>, gemm_smem<double>());
  set_smem(gemm_cluster_kernel<float>, gemm_smem<float>());
  set_smem(gemm_narrow_kernel<double, 8, SOLVE_STAGES>, gemm_narrow_smem<double, 8, SOLVE_STAGES>());
  set_smem(gemm_narrow_kernel<float, 8, SOLVE_STAGES>, gemm_narrow_smem<float, 8, SOLVE_STAGES>());
  set_smem(gemm_narrow_kernel<double, 16, SOLVE_STAGES>, gemm_narrow_smem<double, 16, SOLVE_STAGES>());
  set_smem(gemm_narrow_kernel<float, 16, SOLVE_STAGES>, gemm_narrow_smem<float, 16, SOLVE_STAGES>());
  set_smem(gemm_narrow_kernel<double, 8>, gemm_narrow_smem<double, 8>());
  set_smem(gemm_narrow_kernel<float, 8>, gemm_narrow_smem<float, 8>());
  set_smem(gemm_narrow_kernel<double, 16>, gemm_narrow_smem<double, 16>());
  set_smem(gemm_narrow_kernel<float, 16>, gemm_narrow_smem<float, 16>());
  set_smem(gemm_tf32x3_kernel, GEMM_F32_SMEM);
  configure_solve_dag();
  done = true;
}

void launch_scale(int64_t n, const int64_t *diag_src, const double *val, double *scale, cudaStream_t st) {
  if (n > 0) scale_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, diag_src, val, scale);
}

void launch_assemble(const Tree &t, bool fp32, const double *upper_val, const AssembleTask *tasks, const int4 *ranges,
                     int count, cudaStream_t st) {
  if (count <= 0) return;
  configure_kernels();
  if (fp32)
    assemble_kernel<float, ASSEMBLE_COLS_F32, ASSEMBLE_ROWS_F32>
        <<<count, ASSEMBLE_ROWS_F32, 0, st>>>(t, upper_val, tasks, ranges);
  else
    assemble_kernel<double, ASSEMBLE_COLS, ASSEMBLE_ROWS><<<count, ASSEMBLE_ROWS, 0, st>>>(t, upper_val, tasks, ranges);
}

void launch_panel(const Tree &t, bool fp32, const double *upper_val, const PanelTask *tasks, int count,
                  DeviceStatus *status, int p8max, cudaStream_t st) {
  if (count <= 0) return;
  configure_kernels();
  if (fp32)
    panel_kernel<float><<<count, PANEL_THREADS, panel_smem<float>(p8max), st>>>(t, upper_val, tasks, status, p8max);
  else
    panel_kernel<double><<<count, PANEL_THREADS, panel_smem<double>(p8max), st>>>(t, upper_val, tasks, status, p8max);
}

// A launch of `count` CTAs, as a programmatic dependent of the stream's previous kernel when pdl.
template <class... P, class... A>
void launch_ex(void (*kernel)(P...), int count, int threads, size_t smem, cudaStream_t st, bool pdl, A... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)count);
  cfg.blockDim = dim3((unsigned)threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kernel, args...);
}

void launch_gemm_pdl(const GemmTask *tasks, int count, bool fp32_a, cudaStream_t st, double *part, int32_t *counters,
                     bool pdl) {
  if (count <= 0) return;
  configure_kernels();
  if (fp32_a)
    launch_ex(gemm_kernel<float>, count, GEMM_THREADS, gemm_smem<float>(), st, pdl, tasks, part, counters);
  else
    launch_ex(gemm_kernel<double>, count, GEMM_THREADS, gemm_smem<double>(), st, pdl, tasks, part, counters);
}

void launch_gemm(const GemmTask *tasks, int count, GemmKind kind, cudaStream_t st, double *part, int32_t *counters) {
  if (count <= 0) return;
  configure_kernels();
  switch (kind) {
    case GemmKind::F64:
      gemm_kernel<double><<<count, GEMM_THREADS, gemm_smem<double>(), st>>>(tasks, part, counters);
      break;
    case GemmKind::F32A_F64:
      gemm_kernel<float><<<count, GEMM_THREADS, gemm_smem<float>(), st>>>(tasks, part, counters);
      break;
    case GemmKind::F32_TF32X3: gemm_tf32x3_kernel<<<count, GEMM_THREADS, GEMM_F32_SMEM, st>>>(tasks); break;
  }
}

template <int S>
void launch_narrow(const GemmTask *tasks, int count, bool fp32_a, int cols, cudaStream_t st, double *part,
                   int32_t *counters, bool pdl) {
  if (count <= 0) return;
  configure_kernels();
  if (cols <= 8) {
    if (fp32_a)
      launch_ex(gemm_narrow_kernel<float, 8, S>, count, GEMM_THREADS, gemm_narrow_smem<float, 8, S>(), st, pdl, tasks,
                part, counters);
    else
      launch_ex(gemm_narrow_kernel<double, 8, S>, count, GEMM_THREADS, gemm_narrow_smem<double, 8, S>(), st, pdl,
                tasks, part, counters);
  } else {
    if (fp32_a)
      launch_ex(gemm_narrow_kernel<float, 16, S>, count, GEMM_THREADS, gemm_narrow_smem<float, 16, S>(), st, pdl,
                tasks, part, counters);
    else
      launch_ex(gemm_narrow_kernel<double, 16, S>, count, GEMM_THREADS, gemm_narrow_smem<double, 16, S>(), st, pdl,
                tasks, part, counters);
  }
}

void launch_gemm_solve(const GemmTask *tasks, int count, bool fp32_a, int cols, cudaStream_t st, double *part,
                       int32_t *counters, bool pdl) {
  launch_narrow<SOLVE_STAGES>(tasks, count, fp32_a, cols, st, part, counters, pdl);
}

void launch_gemm_narrow(const GemmTask *tasks, int count, bool fp32_a, int cols, cudaStream_t st, double *part,
                        int32_t *counters, bool pdl) {
  launch_narrow<GEMM_STAGES>(tasks, count, fp32_a, cols, st, part, counters, pdl);
}

void launch_gemm_cluster(const GemmTask *tasks, int count, bool fp32_a, cudaStream_t st, double *part,
                         int32_t *counters) {
  if (count <= 0) return;
  configure_kernels();
  const unsigned grid = (unsigned)count * SOLVE_CLUSTER;
  if (fp32_a)
    gemm_cluster_kernel<float><<<grid, GEMM_THREADS, gemm_smem<float>(), st>>>(tasks, part, counters);
  else
    gemm_cluster_kernel<double><<<grid, GEMM_THREADS, gemm_smem<double>(), st>>>(tasks, part, counters);
}

void launch_solve_assemble(const Tree &t, double *x, double *v, const int64_t *voff, int R, const RowTask *tasks,
                           const int2 *ranges, int count, cudaStream_t st, bool pdl) {
  if (count <= 0) return;
  configure_kernels();
  launch_ex(solve_assemble_kernel, count, 256, 0, st, pdl, t, x, v, voff, R, tasks, ranges);
}

void launch_thin_fwd(const Tree &t, bool fp32, const double *x, double *x2, double *v, const int64_t *voff, int R,
                     int lg, const ThinTask *tasks, const int4 *ranges, int count, cudaStream_t st, bool pdl) {
  if (count <= 0) return;
  configure_kernels();
  if (fp32)
    launch_ex(thin_fwd_kernel<float>, count, THIN_THREADS, 0, st, pdl, t, x, x2, v, voff, R, lg, tasks, ranges);
  else
    launch_ex(thin_fwd_kernel<double>, count, THIN_THREADS, 0, st, pdl, t, x, x2, v, voff, R, lg, tasks, ranges);
}

void launch_thin_bwd(const Tree &t, bool fp32, double *x, const double *x2, int R, int lg, const ThinBwdTask *tasks,
                     double *part, int32_t *counters, int count, cudaStream_t st, bool pdl) {
  if (count <= 0) return;
  configure_kernels();
  if (fp32)
    launch_ex(thin_bwd_kernel<float>, count, THIN_THREADS, 0, st, pdl, t, x, x2, R, lg, tasks, part, counters);
  else
    launch_ex(thin_bwd_kernel<double>, count, THIN_THREADS, 0, st, pdl, t, x, x2, R, lg, tasks, part, counters);
}

void launch_permute_in(const int64_t *perm, int64_t n, const double *b, int64_t ld, double *x, int R,
                       const double *scale, cudaStream_t st) {
  const int64_t total = n * R;
  if (total <= 0) return;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  permute_in_kernel<<<blocks, 256, 0, st>>>(perm, n, b, ld, x, R, scale);
}

void launch_permute_out(const int64_t *perm, int64_t n, const double *x, int R, double *b, int64_t ld,
                        const double *scale, cudaStream_t st) {
  const int64_t total = n * R;
  if (total <= 0) return;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  permute_out_kernel<<<blocks, 256, 0, st>>>(perm, n, x, R, b, ld, scale);
}

void launch_spmv(int64_t n, const int64_t *ptr, const int32_t *idx, const double *val, const double *x, int64_t ldx,
                 double *y, int64_t ldy, int R, cudaStream_t st, double *scratch) {
  if (n <= 0 || R <= 0) return;
  if (scratch && R >= SPMV_ROWS_MIN_R) {
    double *xr = scratch, *yr = scratch + n * R;
    const dim3 tgrid((unsigned)((n + 31) / 32), (unsigned)((R + 31) / 32));
    to_rows_kernel<<<tgrid, 256, 0, st>>>(n, R, x, ldx, xr);
    spmv_rows_kernel<<<dim3((unsigned)((n + 7) / 8), (unsigned)((R + 63) / 64)), 256, 0, st>>>(n, ptr, idx, val, xr,
                                                                                              yr, R);
    to_cols_kernel<<<tgrid, 256, 0, st>>>(n, R, yr, y, ldy);
    return;
  }
  constexpr int RB = 8;
  dim3 grid((unsigned)((n + 7) / 8), (unsigned)((R + RB - 1) / RB));
  spmv_kernel<RB><<<grid, 256, 0, st>>>(n, ptr, idx, val, x, ldx, y, ldy, R);
}

void launch_residual(int64_t n, int R, const double *b, int64_t ldb, double *ax, int64_t ldax, cudaStream_t st) {
  const int64_t total = n * R;
  if (total <= 0) return;
  residual_kernel<<<(int)std::min<int64_t>((total + 255) / 256, 148 * 16), 256, 0, st>>>(n, R, b, ldb, ax, ldax);
}

void launch_update(int64_t n, int R, const double *d, int64_t ldd, double *x, int64_t ldx, cudaStream_t st) {
  const int64_t total = n * R;
  if (total <= 0) return;
  update_kernel<<<(int)std::min<int64_t>((total + 255) / 256, 148 * 16), 256, 0, st>>>(n, R, d, ldd, x, ldx);
}

void launch_coldot(int64_t n, int R, const double *a, int64_t lda, const double *b, int64_t ldb, double *out,
                   cudaStream_t st) {
  if (n <= 0 || R <= 0) return;
  coldot_kernel<<<R, 256, 0, st>>>(n, a, lda, b, ldb, out);
}

void launch_pcg_step(int64_t n, int R, const double *rz, const double *pq, const int *done, const double *p,
                     const double *q, double *x, int64_t ldx, double *r, cudaStream_t st) {
  const int64_t total = n * R;
  if (total <= 0) return;
  pcg_step_kernel<<<(int)std::min<int64_t>((total + 255) / 256, 148 * 16), 256, 0, st>>>(n, R, rz, pq, done, p, q, x,
                                                                                         ldx, r);
}

void launch_pcg_direction(int64_t n, int R, const double *rz_new, const double *rz_old, const double *z, double *p,
                          cudaStream_t st) {
  const int64_t total = n * R;
  if (total <= 0) return;
  pcg_direction_kernel<<<(int)std::min<int64_t>((total + 255) / 256, 148 * 16), 256, 0, st>>>(n, R, rz_new, rz_old, z,
                                                                                              p);
}

void launch_sumsq(int64_t n, int R, int64_t ld, const double *v, double *out, cudaStream_t st) {
  if (R > 0) sumsq_kernel<<<R, 256, 0, st>>>(n, ld, v, out);
}

void launch_pack_trapezoids(const Tree &t, bool fp32, int64_t ns, const int64_t *toff, double *dst, cudaStream_t st) {
  if (ns <= 0) return;
  if (fp32)
    pack_kernel<float><<<(unsigned)ns, 128, 0, st>>>(t, toff, dst);
  else
    pack_kernel<double><<<(unsigned)ns, 128, 0, st>>>(t, toff, dst);
}

}  // namespace fc
