// Shared-memory tiles of 64 x 64 (FP64 or FP32) moved by cp.async, and their product on the FP64
// tensor pipe (DMMA). Used by the factorisation's kernels and by the persistent solve.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fc {
namespace tiles {

template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem, const void *gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(gmem), "n"(BYTES), "r"(src_bytes));
}
static __device__ __forceinline__ void cp_async8(void *smem, const void *gmem, int src_bytes) { cp_async<8>(smem, gmem, src_bytes); }
static __device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// D = A B + C on one 8x8x4 FP64 tile: a = A[g][tg], b = B[tg][g], c/d = C[g][2 tg + {0, 1}]
// with g = lane / 4, tg = lane % 4.
static __device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// ---- shared-memory tiles and the DMMA product of two of them --------------------------------------
// A tile holds 64 x 64 elements as [k][i] with a padded row stride: 68 doubles or 72 floats, so a
// warp's fragment reads of 4 k-rows x 8 consecutive elements fall in distinct banks.
template <class T>
__host__ __device__ constexpr int tile_stride() {
  return sizeof(T) == 8 ? 68 : 72;
}
constexpr int TS = 68;

// dst[k * S + i] = src[i * si + k * sk] for i < rows, k < kk, zero for the other i < 64 and
// kk <= k < kpad (rows k >= kpad of the tile are not touched). Issued as cp.async copies, so a
// tile's loads are all in flight at once; the caller commits, waits and synchronises. One warp per
// k (rows contiguous in memory) or one warp per i (k contiguous): every warp reads a contiguous run.
template <class T>
__device__ __forceinline__ void load_tile(T *dst, const T *__restrict__ src, int64_t si, int64_t sk, int rows, int kk,
                                          int kpad) {
  constexpr int S = tile_stride<T>();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (si == 1) {
    for (int k = warp; k < kpad; k += nw)
      for (int i = lane; i < 64; i += 32) {
        const bool ok = i < rows && k < kk;
        cp_async<sizeof(T)>(&dst[k * S + i], ok ? src + i + (int64_t)k * sk : src, ok ? (int)sizeof(T) : 0);
      }
  } else {
    for (int i = warp; i < 64; i += nw)
      for (int k = lane; k < kpad; k += 32) {
        const bool ok = i < rows && k < kk;
        cp_async<sizeof(T)>(&dst[k * S + i], ok ? src + (int64_t)i * si + k * sk : src, ok ? (int)sizeof(T) : 0);
      }
  }
}

// acc(i, j) += sum_{k < K} As[k][i] Bs[k][j] over a 64 x 64 output, 4 warps of 32 x 32, in FP64
// (an FP32 A tile is widened as it is read).
template <class TA>
__device__ __forceinline__ void mma_tiles(const TA *As, const double *Bs, int K, double (&acc)[4][4][2]) {
  constexpr int SA = tile_stride<TA>();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, tg = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  for (int kk = 0; kk < K; kk += 4) {
    double av[4], bv[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) av[r] = (double)As[(kk + tg) * SA + wm + r * 8 + g];
#pragma unroll
    for (int c = 0; c < 4; ++c) bv[c] = Bs[(kk + tg) * TS + wn + c * 8 + g];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) dmma(acc[r][c], av[r], bv[c]);
  }
}

static __device__ __forceinline__ void zero_acc(double (&acc)[4][4][2]) {
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c][0] = acc[r][c][1] = 0.0;
}

// Calls f(i, j, value) for every output of a 64 x 64 accumulator held by this thread.
template <class F>
__device__ __forceinline__ void each_acc(const double (&acc)[4][4][2], F f) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, tg = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int e = 0; e < 2; ++e) f(wm + r * 8 + g, wn + c * 8 + 2 * tg + e, acc[r][c][e]);
}

// *addr(i, j) -= acc(i, j) for i < rows, j < cols: every old value is loaded before any store,
// so the loads are in flight together (a store could alias a later load otherwise).
template <class Addr>
__device__ __forceinline__ void sub_acc(const double (&acc)[4][4][2], int rows, int cols, Addr addr) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, tg = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  double old[4][4][2];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int i = wm + r * 8 + g, j = wn + c * 8 + 2 * tg + e;
        old[r][c][e] = i < rows && j < cols ? *addr(i, j) : 0.0;
      }
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int i = wm + r * 8 + g, j = wn + c * 8 + 2 * tg + e;
        if (i < rows && j < cols) *addr(i, j) = old[r][c][e] - acc[r][c][e];
      }
}

}  // namespace tiles
}  // namespace fc
