// The supernodal triangular solves (forward L y = b, backward L^T x = y) as one persistent,
// dependency-driven launch per direction.
//
// The level-by-level form needs a launch per panel step of every level of the supernodal tree
// (hundreds of launches per direction, each waiting for the slowest task of the step). Here one
// grid of resident CTAs takes tasks from a topologically ordered list with an atomic ticket; each
// task waits on counters raised by the tasks it reads from. Small supernodes (most of the tree,
// little of the work) are one task each, solved start to finish by one CTA; large ones are split
// in 64-row chunks, so that their panel steps spread over many CTAs. Every entry of the solution
// takes the same operations in the same order on every run (no atomics on values): the counters
// order the updates of a chunk exactly as the level-by-level launches do.
//
// Vectors are row-major with R columns (R right-hand sides): x (in postorder) receives the
// right-hand sides, x2 the forward solution; the backward pass leaves the solution in x. The
// update vectors v_s (a supernode's rows past its columns) live in their own slots.
#include <algorithm>

#include "kernels.cuh"
#include "tiles.cuh"

namespace fc {

namespace {

using namespace tiles;

constexpr int DAG_THREADS = 128;
constexpr int DAG_KC = 32;  // K chunk of the products over the rows past the columns

__device__ __forceinline__ int32_t ld_acquire_gpu(const int32_t *p) {
  int32_t v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}

// Warp 0: waits until every dependency of task `id` is met, one lane per dependency. False when
// the list has failed (this wait ran past the limit, or another one did).
__device__ bool dag_wait(const SolveDag &d, const DagTask &tk, int id) {
  const int lane = threadIdx.x & 31;
  bool ok = true;
  for (int e0 = tk.dep0; e0 < tk.dep1; e0 += 32) {
    const int e = e0 + lane;
    if (e < tk.dep1 && ok) {
      const DagDep dep = d.deps[e];
      unsigned long long start = 0;
      while (ld_acquire_gpu(d.counters + dep.counter) < dep.value) {
        if (*(volatile int32_t *)&d.ctl->error) {
          ok = false;
          break;
        }
        const unsigned long long now = global_ns();
        if (start == 0) {
          start = now;
        } else if (now - start > (unsigned long long)d.limit_ns) {
          if (atomicCAS(&d.ctl->error, 0, DAG_TIMEOUT) == 0) d.ctl->task = id;
          ok = false;
          break;
        }
        __nanosleep(64);
      }
    }
    ok = __all_sync(0xffffffffu, ok);
    if (!ok) return false;
  }
  __threadfence();
  return true;
}

// The supernode's numbers a task needs, loaded once per task.
struct Node {
  int64_t m, w, f, loff, rows_off, voff;
};

__device__ __forceinline__ void signal(int32_t *counter, int inc) {
  __threadfence();
  atomicAdd(counter, inc);
}

// Rows [i0, i1) of s's solve front for right-hand sides [j0, j1): zero the update rows, then add
// the children's update vectors in child order (a child's rows land on distinct rows, so four
// elements per thread are in flight at once).
__device__ void front_assemble(const Tree &t, const SolveDag &d, const DagTask &tk, const Node &nd, int i0, int i1) {
  const int R = d.R, j0 = tk.j0, nj = tk.j1 - tk.j0;
  const int64_t w = nd.w, f = nd.f;
  double *vs = d.v + nd.voff;
  const int tid = threadIdx.x;
  const int64_t z0 = i0 > w ? i0 : w;
  for (int e = tid; e < (int)(i1 - z0) * nj; e += blockDim.x) vs[(z0 - w + e / nj) * R + j0 + e % nj] = 0.0;
  __syncthreads();
  const int64_t k0 = t.kid_ptr[tk.s], k1 = t.kid_ptr[tk.s + 1];
  for (int64_t kp = k0; kp < k1; ++kp) {
    const DagChild ch = d.children[tk.child + (kp - k0)];
    const int32_t *rel = t.rel + ch.rel;
    const double *vc = d.v + ch.v;
    const int total = (ch.hi - ch.lo) * nj;
    for (int e0 = tid; e0 < total; e0 += 4 * DAG_THREADS) {
      double *dst[4];
      double add[4], old[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int e = e0 + q * DAG_THREADS;
        dst[q] = nullptr;
        if (e < total) {
          const int ic = ch.lo + e / nj, j = j0 + e % nj;
          const int64_t I = __ldg(rel + ic);
          dst[q] = I < w ? d.x + (f + I) * R + j : vs + (I - w) * R + j;
          add[q] = vc[(int64_t)ic * R + j];
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (dst[q]) old[q] = *dst[q];
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (dst[q]) *dst[q] = old[q] + add[q];
    }
    __syncthreads();
  }
}

// Rows of front chunk c of a supernode with P panels.
__device__ __forceinline__ void chunk_rows(const Node &nd, int P, int c, int &r0, int &r1) {
  if (c < P) {
    r0 = 64 * c;
    r1 = min((int)nd.w, r0 + 64);
  } else {
    r0 = (int)nd.w + 64 * (c - P);
    r1 = min((int)nd.m, r0 + 64);
  }
}

// Panel p of a supernode for right-hand sides [j0, j0 + nj), then its front chunks [cf, cl) one
// after another, each chunk's L tile loaded while the previous one is multiplied.
// Forward: y = Linv x_p (stored in x2), chunk rows (x own rows, v past the columns) -= L(rows, p) y.
// Backward: z = Linv^T x2_p (stored in x), chunk rows (own rows above, x2) -= L(p, rows)^T z.
template <bool BACKWARD, class T>
__device__ void panel_chunks(const Tree &t, const SolveDag &d, const Node &nd, int p, int cf, int cl, int keep,
                             int64_t doff, int j0, int nj, int32_t sig0, int sigstep, int32_t sigmid, double *sm) {
  double *xs = sm;
  double *buf[2] = {sm + 64 * TS, sm + 2 * 64 * TS};
  const int R = d.R;
  const int64_t m = nd.m, w = nd.w, f = nd.f;
  const int P = (int)((w + 63) / 64);
  const T *Ls = static_cast<const T *>(t.L) + nd.loff;
  const int c0 = 64 * p, pw = (int)min(w, (int64_t)c0 + 64) - c0;
  const int K4 = (pw + 3) & ~3;
  double *out = BACKWARD ? d.x : d.x2;
  auto load_chunk = [&](int k) {
    int r0, r1;
    chunk_rows(nd, P, cf + k, r0, r1);
    T *bt = reinterpret_cast<T *>(buf[k & 1]);
    if (BACKWARD)
      load_tile<T>(bt, Ls + c0 + (int64_t)r0 * m, m, 1, r1 - r0, pw, K4);  // bt[k][r] = L(c0 + k, r0 + r)
    else
      load_tile<T>(bt, Ls + r0 + (int64_t)c0 * m, 1, m, r1 - r0, pw, K4);  // bt[k][r] = L(r0 + r, c0 + k)
  };
  const int nc = cl - cf;
  double acc[4][4][2];
  if (keep > 0) {
    // the inverse goes to buf[1], free until chunk 1 is loaded
    const double *Li = t.D + doff + (int64_t)pw * pw;
    if (BACKWARD)
      load_tile<double>(buf[1], Li, pw, 1, pw, pw, K4);  // inv[k][i] = Linv(k, i)
    else
      load_tile<double>(buf[1], Li, 1, pw, pw, pw, K4);  // inv[k][i] = Linv(i, k)
    load_tile<double>(xs, (BACKWARD ? d.x2 : d.x) + (f + c0) * R + j0, 1, R, nj, pw, K4);
    if (nc > 0) load_chunk(0);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    zero_acc(acc);
    mma_tiles<double>(buf[1], xs, K4, acc);
    __syncthreads();
    each_acc(acc, [&](int i, int j, double val) {
      if (i < K4) xs[i * TS + j] = val;
      if (i < pw && j < nj) out[(f + c0 + i) * R + j0 + j] = val;
    });
    __syncthreads();
    if (threadIdx.x == 0 && sigmid >= 0) signal(d.counters + sigmid, 1);
  } else {
    load_tile<double>(xs, out + (f + c0) * R + j0, 1, R, nj, pw, K4);
    if (nc > 0) load_chunk(0);
    cp_async_commit();
  }
  for (int k = 0; k < nc; ++k) {
    if (k + 1 < nc) {
      load_chunk(k + 1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    zero_acc(acc);
    mma_tiles<T>(reinterpret_cast<const T *>(buf[k & 1]), xs, K4, acc);
    int r0, r1;
    chunk_rows(nd, P, cf + k, r0, r1);
    double *dst;
    if (BACKWARD)
      dst = d.x2 + (f + r0) * R + j0;
    else
      dst = r0 < w ? d.x + (f + r0) * R + j0 : d.v + nd.voff + (r0 - w) * R + j0;
    sub_acc(acc, r1 - r0, nj, [&](int i, int j) { return dst + (int64_t)i * R + j; });
    __syncthreads();
    if (threadIdx.x == 0 && sig0 >= 0) signal(d.counters + sig0 + k * sigstep, 1);
  }
}

// Own rows [i0, i1) of a supernode: sum over k in [k0, k1) of L(w + k, row) x(row k of the
// structure, final by then) — the backward update by the rows past the columns, its right-hand
// side gathered straight from x. Subtracted from x2, or stored as a partial tile at `part`.
template <class T>
__device__ void rows_product(const Tree &t, const SolveDag &d, const Node &nd, int i0, int i1, int k0, int k1,
                             int j0, int nj, double *part, double *sm) {
  constexpr int SA = tile_stride<T>();
  const int R = d.R;
  const int64_t m = nd.m, w = nd.w, f = nd.f;
  const int M = i1 - i0, K = k1 - k0;
  const T *A = static_cast<const T *>(t.L) + nd.loff + w + k0 + (int64_t)i0 * m;
  const int32_t *rows = t.rows + nd.rows_off + w + k0;
  double *bs[2] = {sm, sm + DAG_KC * TS};
  T *as[2];
  as[0] = reinterpret_cast<T *>(sm + 2 * DAG_KC * TS);
  as[1] = as[0] + DAG_KC * SA;
  const int nq = (K + DAG_KC - 1) / DAG_KC;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  auto load = [&](int q) {
    const int kc = q * DAG_KC, kk = min(DAG_KC, K - kc);
    load_tile<T>(as[q & 1], A + kc, m, 1, M, kk, DAG_KC);
    // bs[k][j] = x[rows[kc + k]][j0 + j]: one warp per k, a contiguous run of x per row
    for (int k = warp; k < DAG_KC; k += DAG_THREADS / 32) {
      const bool krow = k < kk;
      const double *src = krow ? d.x + (int64_t)rows[kc + k] * R + j0 : d.x;
      for (int j = lane; j < 64; j += 32) {
        const bool ok = krow && j < nj;
        cp_async<8>(&bs[q & 1][k * TS + j], ok ? src + j : d.x, ok ? 8 : 0);
      }
    }
    cp_async_commit();
  };
  double acc[4][4][2];
  zero_acc(acc);
  load(0);
  for (int q = 0; q < nq; ++q) {
    if (q + 1 < nq) {
      load(q + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    mma_tiles<T>(as[q & 1], bs[q & 1], DAG_KC, acc);
    __syncthreads();
  }
  if (part) {
    each_acc(acc, [&](int i, int j, double val) {
      if (i < M && j < nj) part[i * 64 + j] = val;
    });
  } else {
    double *C = d.x2 + (f + i0) * R + j0;
    sub_acc(acc, M, nj, [&](int i, int j) { return C + (int64_t)i * R + j; });
  }
}

// Own rows [i0, i1) -= the partial tiles from `part` on, summed in order.
__device__ void reduce_rows(const SolveDag &d, const Node &nd, const DagTask &tk) {
  const int R = d.R, M = tk.i1 - tk.i0, nj = tk.j1 - tk.j0;
  const double *P = d.part + tk.aux;
  double *C = d.x2 + (nd.f + tk.i0) * R + tk.j0;
  for (int e = threadIdx.x; e < M * 64; e += blockDim.x) {
    const int i = e >> 6, j = e & 63;
    if (j >= nj) continue;
    double sum = 0.0;
    for (int q = 0; q < tk.count; ++q) sum += P[(int64_t)q * 4096 + i * 64 + j];
    C[(int64_t)i * R + j] -= sum;
  }
}

template <bool BACKWARD, class T>
__device__ void run_task(const Tree &t, const SolveDag &d, const DagTask &tk, const Node &nd, double *sm) {
  const int nj = tk.j1 - tk.j0;
  const int P = (int)((nd.w + 63) / 64), C = P + (int)((nd.m - nd.w + 63) / 64);
  if (tk.kind == DAG_PANEL) {
    panel_chunks<BACKWARD, T>(t, d, nd, tk.i0 / 64, tk.r0, tk.r1, tk.keep, tk.aux, tk.j0, nj, tk.sig0, tk.sigstep,
                              tk.sigmid, sm);
  } else if (tk.kind == DAG_NODE) {
    const int64_t doff = t.doff[tk.s];
    if (!BACKWARD) {
      front_assemble(t, d, tk, nd, 0, (int)nd.m);
      for (int p = 0; p < P; ++p) {
        panel_chunks<false, T>(t, d, nd, p, p + 1, C, 1, doff + 2 * (int64_t)NB * NB * p, tk.j0, nj, -1, 0, -1, sm);
        __syncthreads();
      }
    } else {
      const int u = (int)(nd.m - nd.w);
      if (u > 0)
        for (int i = 0; i < P; ++i) {
          rows_product<T>(t, d, nd, 64 * i, (int)min(nd.w, (int64_t)64 * i + 64), 0, u, tk.j0, nj, nullptr, sm);
          __syncthreads();
        }
      for (int p = P - 1; p >= 0; --p) {
        panel_chunks<true, T>(t, d, nd, p, 0, p, 1, doff + 2 * (int64_t)NB * NB * p, tk.j0, nj, -1, 0, -1, sm);
        __syncthreads();
      }
    }
  } else if (!BACKWARD) {
    front_assemble(t, d, tk, nd, tk.i0, tk.i1);
  } else if (tk.kind == DAG_GEMM) {
    rows_product<T>(t, d, nd, tk.i0, tk.i1, tk.r0, tk.r1, tk.j0, nj, tk.aux >= 0 ? d.part + tk.aux : nullptr, sm);
  } else {
    reduce_rows(d, nd, tk);
  }
}

template <bool BACKWARD, class T>
__global__ void __launch_bounds__(DAG_THREADS) solve_dag_kernel(Tree t, SolveDag d) {
  extern __shared__ double sm[];
  __shared__ int32_t s_id, s_ok;
  __shared__ Node s_node;
  for (;;) {
    if (threadIdx.x < 32) {
      unsigned long long t0 = 0;
      int id = 0;
      if (threadIdx.x == 0) {
        if (d.trace) t0 = global_ns();
        id = atomicAdd(&d.ctl->next[BACKWARD ? 1 : 0], 1);
      }
      id = __shfl_sync(0xffffffffu, id, 0);
      bool ok = id < d.count && *(volatile int32_t *)&d.ctl->error == 0;
      if (ok) ok = dag_wait(d, d.tasks[id], id);
      if (threadIdx.x == 0) {
        s_id = id;
        s_ok = ok;
        if (ok) {
          const int s = d.tasks[id].s;
          s_node = Node{t.height[s], t.width[s], t.first[s], t.loff[s], t.rows_off[s], d.voff[s]};
        }
        if (d.trace && id < d.count) {
          d.trace[4 * (int64_t)id] = (long long)t0;
          d.trace[4 * (int64_t)id + 1] = (long long)global_ns();
        }
      }
    }
    __syncthreads();
    const int id = s_id;
    if (id >= d.count) return;
    if (s_ok) {
      const DagTask tk = d.tasks[id];
      const Node nd = s_node;
      run_task<BACKWARD, T>(t, d, tk, nd, sm);
      __syncthreads();
      if (threadIdx.x == 0) {
        for (int k = 0; k < tk.nsig; ++k) signal(d.counters + tk.sig0 + k * tk.sigstep, 1);
        if (tk.sig1 >= 0) signal(d.counters + tk.sig1, tk.inc1);
        if (d.trace) {
          unsigned smid;
          asm volatile("mov.u32 %0, %%smid;\n" : "=r"(smid));
          d.trace[4 * (int64_t)id + 2] = (long long)global_ns();
          d.trace[4 * (int64_t)id + 3] = ((long long)tk.kind << 32) | smid;
        }
      }
    }
    __syncthreads();
  }
}

// Shared memory: the panel's vector tile and two tiles (the inverse or L chunks), or the
// product's two pairs of K-chunk tiles.
template <class T>
constexpr size_t dag_smem() {
  const size_t panel = sizeof(double) * 3 * 64 * TS;
  const size_t product = sizeof(double) * 2 * DAG_KC * TS + sizeof(T) * 2 * DAG_KC * tile_stride<T>();
  return panel > product ? panel : product;
}

}  // namespace

void configure_solve_dag() {
  cudaFuncSetAttribute(solve_dag_kernel<false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dag_smem<double>());
  cudaFuncSetAttribute(solve_dag_kernel<true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dag_smem<double>());
  cudaFuncSetAttribute(solve_dag_kernel<false, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dag_smem<float>());
  cudaFuncSetAttribute(solve_dag_kernel<true, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dag_smem<float>());
}

int solve_dag_blocks_per_sm(bool fp32) {
  int blocks = 0;
  if (fp32)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, solve_dag_kernel<false, float>, DAG_THREADS, dag_smem<float>());
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, solve_dag_kernel<false, double>, DAG_THREADS,
                                                  dag_smem<double>());
  return std::max(blocks, 1);
}

void launch_solve_dag(const Tree &t, bool fp32, bool backward, const SolveDag &d, int grid, cudaStream_t st) {
  if (d.count <= 0) return;
  if (fp32) {
    if (backward)
      solve_dag_kernel<true, float><<<grid, DAG_THREADS, dag_smem<float>(), st>>>(t, d);
    else
      solve_dag_kernel<false, float><<<grid, DAG_THREADS, dag_smem<float>(), st>>>(t, d);
  } else {
    if (backward)
      solve_dag_kernel<true, double><<<grid, DAG_THREADS, dag_smem<double>(), st>>>(t, d);
    else
      solve_dag_kernel<false, double><<<grid, DAG_THREADS, dag_smem<double>(), st>>>(t, d);
  }
}

}  // namespace fc
