// The C ABI of include/fieldcraft_chol.h: handles, the plan of the numeric phase on the device,
// and the launches. The numeric phase is multifrontal over the reference's supernodes: every
// supernode's front (its L panel and its update matrix) is assembled from A and its children's
// update matrices in child order, factored by panels of NB columns (diagonal block, rows below,
// right-looking update of the later columns), and its update matrix U = F22 - L21 L21^T is left
// for its parent. Supernodes are taken level by level of the supernodal tree (a level's
// supernodes are independent); within a level, panel by panel. The factor holds the same L as
// the reference's left-looking order (the same numbers up to rounding).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <map>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/fieldcraft_chol.h"
#include <cuda.h>  // CUtensorMap and its encoder's signature (looked up through the runtime)

#include "cuda/kernels.cuh"
#include "cuda/ldlt_launch.cuh"
#include "device_buf.hpp"
#include "host/ldlt_fold.hpp"
#include "host/symbolic.hpp"

struct fc_symbolic {
  fc::Symbolic s;
};

namespace {

using fc::Failure;
using fc::host::DeviceBuf;
using fc::host::set_status;
using fc::host::upload;

int fail_status(fc_status *st, const Failure &f) {
  set_status(st, f.code, f.column, f.entries, f.limit, f.message);
  return f.code;
}

enum Kind {
  K_ASSEMBLE, K_PANEL, K_RETIRED_2, K_GEMM, K_SOLVE_ASSEMBLE, K_RETIRED_5, K_SOLVE_FWD, K_SOLVE_BWD,
  K_SOLVE_DAG_FWD, K_SOLVE_DAG_BWD,
  K_GEMM_MIXED,  // A in the factor's storage type, B and C FP64
  K_GEMM_F64,    // FP64 throughout (the diagonal blocks' inverses)
  K_GEMM_TC,     // FP32 3xTF32 on tcgen05 (the update matrices of the mixed-precision factor)
  K_SOLVE_THIN_FWD, K_SOLVE_THIN_BWD,  // the thin supernodes' steps of a solve level
  K_PACK_TC,                           // the tcgen05 products' operands packed (K-major hi | lo)
  K_LDLT_PANEL,                        // LDL^T: pivoted panel steps (they write the next GEMM's tasks)
  K_LDLT_AFTER,                        // LDL^T: W21 = L21 D and D out of the fronts
  K_LDLT_INVERSE                       // LDL^T: the 64 x 64 inverses of the unit lower diagonal blocks
};

struct Launch {
  int kind;
  int64_t off;
  int count;
  int level;  // the level of the supernodal tree the launch belongs to (cancellation points)
  int width;  // panel launches: the widest panel, padded (sizes the kernel's shared memory)
  // the factorisation runs on three streams (lanes): lane 0 the chain of panels and what needs
  // them, lane 1 the updates of columns past the next outer block (beside the next panels), lane 2
  // the diagonal blocks' inverses (needed by the solve only); `dep` is a launch on another lane
  // this one waits for (-1: none), `record` marks a launch another waits for
  int lane = 0;
  int dep = -1;
  bool record = false;
};

}  // namespace

struct fc_chol {
  int device = 0, precision = FC_PRECISION_FP64;
  bool fp32 = false;   // L and the update matrices in FP32 (the mixed-precision factorisation)
  size_t esize = 8;    // bytes of an entry of L / U
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int64_t n = 0, ns = 0, entries = 0, nnz = 0, levels = 0;
  double flops = 0;
  std::vector<int64_t> first, perm, loff, uoff, rows_off, toff, doff;
  std::vector<int64_t> ioff;  // where each supernode's diagonal-block inverses start in Dinv
  int64_t i_len = 0, t_len = 0;
  std::vector<int32_t> width, height, rows;
  std::vector<int64_t> kid_ptr;
  std::vector<int32_t> kids;
  std::vector<int64_t> rel_off;  // host copies of the relative maps (for planning)
  std::vector<int32_t> rel;
  std::vector<int32_t> level;
  std::vector<int64_t> a_ptr;    // host copies of the input entries' column starts and their rows
  std::vector<int32_t> a_lrow;   // in the front (sorted within each assembly column block)
  int64_t l_len = 0, u_len = 0;
  // device
  DeviceBuf d_first, d_width, d_height, d_rows_off, d_rows, d_loff, d_uoff, d_kid_ptr, d_kids, d_rel_off, d_rel;
  DeviceBuf d_kid_meta;
  DeviceBuf d_a_ptr, d_a_src, d_a_dst, d_diag_src, d_L, d_U, d_D, d_perm, d_val, d_status, d_toff, d_doff;
  DeviceBuf d_a_row, d_a_col, d_scale;   // mixed precision only
  DeviceBuf d_Dinv, d_T;                 // diagonal-block inverses; the doubling's products
  DeviceBuf d_ir_r, d_ir_d, d_ir_sum;    // iterative refinement workspace
  DeviceBuf d_ir_p, d_ir_q, d_ir_t, d_ir_done;
  DeviceBuf d_ir_sc;                     // the refinement's SpMV: row-major copies of x and y
  bool refine_pcg = true;                // refinement by preconditioned CG (else plain refinement)
  bool tc = true;                        // FP32 updates on tcgen05 (FC_TF32_MMA_SYNC=1: on mma.sync)
  DeviceBuf d_asm, d_ranges, d_panel, d_gemm;
  // the mixed-precision factor's tcgen05 update products: packed operands (reused level after
  // level), their pack and tile tasks, and one TMA tensor map per supernode
  DeviceBuf d_pack, d_pack_t, d_tc_t, d_maps;
  int64_t pack_len = 0;
  // the symmetric indefinite factor (FC_PRECISION_LDLT): the rows' largest |A| (as bits), each
  // column's place in its supernode, the pivot orders and kinds, the panels' progress and 2 x 2
  // counts, the first singular column, per-level scratch, D (diagonal, subdiagonal), the tasks
  bool ldlt = false;
  DeviceBuf d_lscale, d_llocal, d_lorder, d_lpivots, d_lpos, d_ltwos, d_lfailed, d_lscratch, d_ldd, d_lde;
  DeviceBuf d_lpanel, d_lafter, d_linv;
  // the LDL^T solve's structure: the pivot orders folded in after each factorisation (host/
  // ldlt_fold.cpp), its rows, relative maps and permutation on the device, the L21 rows' move;
  // the structure's own rows and maps kept for the next fold; the tree the solve's kernels read
  bool ldlt_folded = false;
  std::vector<int32_t> ldlt_rows0, ldlt_rel0;
  std::vector<int64_t> ldlt_sparent, ldlt_from_off;
  std::vector<int32_t> ldlt_from;
  DeviceBuf d_lsrows, d_lsrel, d_lsperm, d_lfrom, d_ltmp, d_lperm_t;
  fc::Tree stree{};
  fc::Tree tree{};
  std::vector<Launch> program;
  cudaStream_t side = nullptr;            // lane 1 of the factorisation (see Launch), lowest priority
  cudaStream_t hi = nullptr;              // lane 0 of the factorisation, highest priority
  cudaStream_t side2 = nullptr;           // lane 2: the diagonal blocks' inverses, lowest priority
  std::vector<cudaEvent_t> lane_events;   // per launch of the program that another waits for
  cudaEvent_t fork_event = nullptr, join_event = nullptr, hi_join_event = nullptr, join2_event = nullptr;
  int64_t gemm_tasks = 0;
  // solve plan for `solve_R` right-hand sides
  int solve_R = 0;
  DeviceBuf d_x, d_x2, d_v, d_part, d_voff, d_b, d_srow, d_sranges, d_spanel, d_sgemm;
  DeviceBuf d_thin, d_tranges, d_tbwd, d_tpart, d_tcount;  // the thin supernodes' solve tasks
  int solve_lg = 6;
  int64_t solve_tcount = 0;
  std::vector<cudaEvent_t> solve_events;  // the solve's level joins of its two streams
  std::vector<Launch> fwd, bwd;
  // the solve as two dependency-driven persistent launches instead of level by level
  // (FC_OPTION_SOLVE_SCHEDULE, or FC_SOLVE_PERSISTENT=1 in the environment)
  bool dag = false;
  // the solve's launches with few output tiles split K in chunks summed by their last CTA (default)
  // or over thread-block clusters (FC_OPTION_SOLVE_CLUSTER = 1)
  bool solve_cluster = false;
  bool solve_narrow = true;  // the solve's products in 64 x 8 / 64 x 16 tiles for up to 16 right-hand sides
  bool solve_deep = true;    // the solve's short product launches with the deeper cp.async ring
  bool asm_first = true;     // wide update matrices: children added before the panels (lane 1)
  bool solve_pdl = false;    // the level-by-level solve's launches as programmatic dependents
  DeviceBuf d_dtasks, d_ddeps, d_dranges, d_dcount, d_dctl;  // d_dranges: the children's records
  int64_t dag_fwd = 0, dag_bwd = 0, dag_counters = 0;
  int dag_grid = 0;
  long long dag_limit_ns = 4000000000LL;  // a wait longer than this fails the solve (FC_TIMEOUT)
  bool dag_trace = false;                 // per-task times of the persistent solve
  DeviceBuf d_dtrace;
  bool dag_plant = false;                 // test hook: the next plan holds a dependency nothing meets
  int64_t last_factor_launches = 0, last_solve_launches = 0;
  double gemm_flops_factor = 0, gemm_flops_solve = 0;
  double gemm_flops_updates = 0;  // the factor's K_GEMM launches alone (the inverse doubling apart)
  int64_t gemm_big_ordinal = -1, gemm_trail_ordinal = -1;  // the factor's heaviest GEMM launches
  // per-launch event timing (fc_chol_profile)
  bool profiling = false;
  // captured programs, replayed while their inputs stay the same (FC_NO_GRAPHS=1 disables)
  bool graphs = true;
  cudaGraphExec_t factor_graph = nullptr, solve_graph = nullptr;
  const double *factor_graph_val = nullptr;
  cudaStream_t factor_graph_stream = nullptr, solve_graph_stream = nullptr;
  double *solve_graph_b = nullptr;
  int solve_graph_R = 0;
  int64_t solve_graph_ld = 0;
  struct MarkRec {
    int kind, level, count;
    cudaEvent_t a, b;
  };
  std::vector<MarkRec> marks;
  std::vector<cudaEvent_t> event_pool;
  size_t events_used = 0;
  std::mutex lock;
  ~fc_chol() {
    if (factor_graph) cudaGraphExecDestroy(factor_graph);
    if (solve_graph) cudaGraphExecDestroy(solve_graph);
    for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : lane_events)
      if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : solve_events) cudaEventDestroy(e);
    if (fork_event) cudaEventDestroy(fork_event);
    if (hi_join_event) cudaEventDestroy(hi_join_event);
    if (join_event) cudaEventDestroy(join_event);
    if (side) cudaStreamDestroy(side);
    if (hi) cudaStreamDestroy(hi);
    if (side2) cudaStreamDestroy(side2);
    if (join2_event) cudaEventDestroy(join2_event);
  }
};

namespace {

int prop_sms(int device) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
  return v > 0 ? v : 1;
}

int cuda_fail(fc_status *st, cudaError_t e, const char *where) {
  std::string msg = std::string(where) + ": " + cudaGetErrorString(e);
  set_status(st, FC_CUDA_ERROR, -1, 0, 0, msg);
  return FC_CUDA_ERROR;
}

int64_t order_key_work(const fc_chol *h, int64_t s) {
  int64_t m = h->height[s], w = h->width[s], u = m - w;
  return m * w * w + u * u * w;
}

// Supernodes grouped by level (height in the supernodal tree), each level heaviest first.
std::vector<std::vector<int64_t>> levels_of(fc_chol *h) {
  h->level.assign(h->ns, 0);
  int32_t top = 0;
  for (int64_t s = 0; s < h->ns; ++s) {
    int32_t lv = 0;
    for (int64_t q = h->kid_ptr[s]; q < h->kid_ptr[s + 1]; ++q) lv = std::max(lv, h->level[h->kids[q]] + 1);
    h->level[s] = lv;
    top = std::max(top, lv);
  }
  std::vector<std::vector<int64_t>> out(h->ns ? top + 1 : 0);
  for (int64_t s = 0; s < h->ns; ++s) out[h->level[s]].push_back(s);
  for (auto &l : out)
    std::stable_sort(l.begin(), l.end(), [&](int64_t a, int64_t b) { return order_key_work(h, a) > order_key_work(h, b); });
  h->levels = (int64_t)out.size();
  return out;
}

void push(std::vector<Launch> &prog, int kind, int64_t off, int64_t count, int level, int width = 0) {
  if (count > 0) prog.push_back({kind, off, (int)count, level, width});
}

// For front positions [lo, hi) of supernode s: each child's positions (in its update matrix) whose
// place in s's front falls in [lo, hi), appended to `ranges`; returns where they start.
int32_t child_ranges(const fc_chol *h, int64_t s, int lo, int hi, std::vector<int2> &ranges) {
  const int32_t at = (int32_t)ranges.size();
  for (int64_t q = h->kid_ptr[s]; q < h->kid_ptr[s + 1]; ++q) {
    const int64_t c = h->kids[q];
    const int uc = h->height[c] - h->width[c];
    const int32_t *rel = h->rel.data() + h->rel_off[c];
    const int a = (int)(std::lower_bound(rel, rel + uc, lo) - rel);
    const int b = (int)(std::lower_bound(rel, rel + uc, hi) - rel);
    ranges.push_back(make_int2(a, b));
  }
  return at;
}

// The assembly tile's columns: an FP32 front's tiles are twice as wide (the same bytes).
int assemble_cols(const fc_chol *h) { return h->fp32 ? fc::ASSEMBLE_COLS_F32 : fc::ASSEMBLE_COLS; }
int assemble_rows(const fc_chol *h) { return h->fp32 ? fc::ASSEMBLE_ROWS_F32 : fc::ASSEMBLE_ROWS; }

// Assembly tiles of supernode s (see assemble_kernel): ASM_L over the L panel's columns, or the
// update matrix's columns as ASM_U (only tiles some child lands in: the rest keep what the GEMM
// stored), ASM_U_PRODUCT or ASM_U_FIRST (all tiles). A block of assemble_cols(h) columns is cut into row tiles
// of assemble_rows(h) from its first column down; each tile's child ranges come from `at`, per child
// the first row of its update matrix whose place in the front is >= r, for every r in [0, m].
void assemble_tiles(const fc_chol *h, int64_t s, int mode, std::vector<fc::AssembleTask> &out,
                    std::vector<int4> &ranges) {
  const int m = h->height[s], w = h->width[s];
  const int jlo = mode == fc::ASM_L ? 0 : w, jhi = mode == fc::ASM_L ? w : m;
  const int64_t q0 = h->kid_ptr[s], nk = h->kid_ptr[s + 1] - q0;
  std::vector<std::vector<int32_t>> at((size_t)nk);
  for (int64_t q = 0; q < nk; ++q) {
    const int64_t c = h->kids[q0 + q];
    const int uc = h->height[c] - h->width[c];
    const int32_t *rel = h->rel.data() + h->rel_off[c];
    at[q].resize((size_t)m + 1);
    int i = 0;
    for (int r = 0; r <= m; ++r) {
      while (i < uc && rel[i] < r) ++i;
      at[q][r] = i;
    }
  }
  const int64_t f = h->first[s];
  const int cols = assemble_cols(h);
  for (int j0 = jlo; j0 < jhi; j0 += cols) {
    const int j1 = std::min(jhi, j0 + cols);
    for (int i0 = j0; i0 < m; i0 += assemble_rows(h)) {
      const int i1 = std::min(m, i0 + assemble_rows(h));
      const int32_t base = (int32_t)ranges.size();
      bool touched = false;
      for (int64_t q = 0; q < nk; ++q) {
        const int4 g = make_int4(at[q][j0], at[q][j1], at[q][i0], at[q][i1]);
        touched |= g.x < g.y && g.z < g.w && g.w - 1 >= g.x;
        ranges.push_back(g);
      }
      if (mode == fc::ASM_U && !touched) {
        ranges.resize(base);
        continue;
      }
      fc::AssembleTask k{};
      k.s = (int32_t)s, k.j0 = j0, k.j1 = j1, k.i0 = i0, k.i1 = i1, k.mode = mode, k.ranges = base;
      k.nk = (int32_t)nk, k.k0 = (int32_t)q0, k.m = m, k.w = w, k.loff = h->loff[s], k.uoff = h->uoff[s];
      if (mode == fc::ASM_L) {
        const int64_t b0 = h->a_ptr[f + j0], b1 = h->a_ptr[f + j1];
        const int32_t *lr = h->a_lrow.data();
        k.e0 = std::lower_bound(lr + b0, lr + b1, i0) - lr;
        k.e1 = std::lower_bound(lr + b0, lr + b1, i1) - lr;
      }
      out.push_back(k);
    }
  }
}

// The address of entry `off` of the L or U arena (entries of h->esize bytes).
void *arena_at(const DeviceBuf &buf, const fc_chol *h, int64_t off) {
  return static_cast<char *>(buf.p) + (size_t)off * h->esize;
}

// Block b (columns [b SB, b SB + bw)) of supernode s's diagonal-block inverses: its offset in
// Dinv and its width (the leading dimension of its column-major bw x bw storage).
int64_t inv_block(const fc_chol *h, int64_t s, int b, int &bw) {
  const int w = h->width[s];
  bw = std::min(fc::SB, w - b * fc::SB);
  return h->ioff[s] + (int64_t)b * fc::SB * fc::SB;  // every earlier block is full
}

// Useful flops of a GEMM task (a diagonal tile computes its lower triangle only).
double task_flops(const fc::GemmTask &g) {
  double outputs = (double)g.M * g.N;
  if (g.flags & 1) {
    outputs = 0;
    for (int j = 0; j < g.N; ++j) outputs += std::max(0, g.M - j);
  }
  return 2.0 * g.K * outputs;
}


// Offsets in one arena for per-supernode blocks that live from the start of their supernode's
// level to the end of their parent's assembly (the only reader): level by level, the level's
// blocks are taken first-fit from the free space, then its children's blocks are given back.
// Returns the arena's size (entries); offsets are 32-entry aligned.
int64_t arena_offsets(const fc_chol *h, const std::vector<std::vector<int64_t>> &lv, const std::vector<int64_t> &size,
                      std::vector<int64_t> &off) {
  const int64_t ALIGN = 32;
  auto up = [&](int64_t x) { return (x + ALIGN - 1) / ALIGN * ALIGN; };
  std::map<int64_t, int64_t> free_blocks;  // offset -> length
  int64_t top = 0;
  off.assign(h->ns, 0);
  auto take = [&](int64_t len) {
    for (auto it = free_blocks.begin(); it != free_blocks.end(); ++it)
      if (it->second >= len) {
        const int64_t at = it->first, rest = it->second - len;
        free_blocks.erase(it);
        if (rest > 0) free_blocks[at + len] = rest;
        return at;
      }
    const int64_t at = top;
    top += len;
    return at;
  };
  auto give = [&](int64_t at, int64_t len) {
    auto next = free_blocks.lower_bound(at);
    if (next != free_blocks.end() && at + len == next->first) {
      len += next->second;
      free_blocks.erase(next);
    }
    auto prev = free_blocks.lower_bound(at);
    if (prev != free_blocks.begin()) {
      --prev;
      if (prev->first + prev->second == at) {
        prev->second += len;
        return;
      }
    }
    free_blocks[at] = len;
  };
  for (const auto &S : lv) {
    for (int64_t s : S)
      if (size[s] > 0) off[s] = take(up(size[s]));
    for (int64_t s : S)
      for (int64_t q = h->kid_ptr[s]; q < h->kid_ptr[s + 1]; ++q) {
        const int64_t c = h->kids[q];
        if (size[c] > 0) give(off[c], up(size[c]));
      }
  }
  return top;
}

// The factor's program: per level, assemble; per panel, the fused factor/invert/solve of the
// panel, then the update of the later columns; then the update matrices.
// The inverses of the diagonal blocks of the supernodes of one level, by doubling: from the
// panels' 64 x 64 inverses, each step h (64, 128, ... < SB) joins neighbouring inverses A^-1 and
// C^-1 of h columns into the inverse of [[A, 0], [B, C]], whose lower-left block is
// -C^-1 (B A^-1). Step h is two GEMM launches: T = B A^-1 into the scratch T (first), then
// -C^-1 T into Dinv (second); A^-1 and C^-1 are lower triangular, so the K ranges stop at the
// triangle. Returns the scratch doubles the level needs (T may be null to size only).
int64_t inverse_doubling(fc_chol *h, const std::vector<int64_t> &S, double *T, int step_h,
                         std::vector<fc::GemmTask> *first, std::vector<fc::GemmTask> *second) {
  auto Lp = [&](int64_t off) { return arena_at(h->d_L, h, off); };
  double *Dinv = h->d_Dinv.as<double>();
  int64_t toff = 0;
  const int hh = step_h;
  for (int64_t s : S) {
    const int w = h->width[s], m = h->height[s];
    if (w <= hh) continue;
    for (int b = 0; b * fc::SB < w; ++b) {
      int bw;
      const int64_t base = inv_block(h, s, b, bw);
      const int scol = b * fc::SB;
      for (int a0 = 0; a0 + hh < bw; a0 += 2 * hh) {
        const int c0 = a0 + hh, hc = std::min(hh, bw - c0), ha = hh;
        if (first && T) {
          double *Tp = T + toff;
          for (int i = 0; i < hc; i += 64)
            for (int j = 0; j < ha; j += 64) {
              fc::GemmTask g{};  // T(i, j) = sum_k L(c0 + i, a0 + k) Ainv(k, j), k >= j
              g.C = Tp + i + (int64_t)j * hc;
              g.c_si = 1, g.c_sj = hc;
              g.A = Lp(h->loff[s] + (scol + c0 + i) + (int64_t)(scol + a0 + j) * m);
              g.a_si = 1, g.a_sk = m;
              g.B = Dinv + base + (a0 + j) + (int64_t)(a0 + j) * bw;
              g.b_sj = bw, g.b_sk = 1;
              g.M = std::min(64, hc - i), g.N = std::min(64, ha - j), g.K = ha - j;
              g.flags = 4;
              first->push_back(g);
            }
          for (int i = 0; i < hc; i += 64)
            for (int j = 0; j < ha; j += 64) {
              fc::GemmTask g{};  // X(i, j) = -sum_k Cinv(i, k) T(k, j), k <= i
              g.C = Dinv + base + (c0 + i) + (int64_t)(a0 + j) * bw;
              g.c_si = 1, g.c_sj = bw;
              g.A = Dinv + base + (c0 + i) + (int64_t)c0 * bw;
              g.a_si = 1, g.a_sk = bw;
              g.B = Tp + (int64_t)j * hc;
              g.b_sj = hc, g.b_sk = 1;
              g.M = std::min(64, hc - i), g.N = std::min(64, ha - j), g.K = std::min(hc, i + 64);
              g.flags = 2;
              second->push_back(g);
            }
        }
        toff += (int64_t)hc * ha;
      }
    }
  }
  return toff;
}

// A tensor map of a supernode's packed L21 (u rows of 2 wpad FP32 values at pack offset poff).
struct MapSpec {
  int64_t poff, u;
  int wpad;
};

// Panels per outer block of the factorisation of a front's own columns (see plan_factor).
constexpr int OUTER_PANELS = 4;

void plan_factor(fc_chol *h, const std::vector<std::vector<int64_t>> &lv, std::vector<fc::AssembleTask> &asm_t,
                 std::vector<int4> &ranges, std::vector<fc::PanelTask> &panel_t, std::vector<fc::GemmTask> &gemm_t,
                 std::vector<fc::PackTask> &pack_t, std::vector<fc::TcTask> &tc_t, std::vector<MapSpec> &maps) {
  auto Lp = [&](int64_t off) { return arena_at(h->d_L, h, off); };
  auto Up = [&](int64_t off) { return arena_at(h->d_U, h, off); };
  const int NB = fc::NB;
  // a factor GEMM tile: 64 x 64, and 128 x 128 for the update matrices' long products on the
  // tcgen05 path (the first tile of a column block starts on the diagonal, so 'lower' still means
  // local i >= j); the panels' short updates of later columns (K <= 64) stay on 64 x 64 tiles
  const int TM = fc::GEMM_TM;
  const bool tc = h->fp32 && h->tc;
  h->pack_len = 0;
  int pending_join = -1;  // a lane-1 launch the next lane-0 launch after the panel steps waits for
  auto join = [&]() {
    if (pending_join >= 0 && (int)h->program.size() > pending_join + 1) {
      for (size_t q = pending_join + 1; q < h->program.size(); ++q)
        if (h->program[q].lane == 0) {
          h->program[q].dep = pending_join;
          h->program[pending_join].record = true;
          pending_join = -1;
          break;
        }
    }
  };
  // a wide supernode (more than ASSEMBLE_THIN columns) with children gets its update matrix's
  // children contributions first (ASM_U_FIRST, on lane 1 beside its panels) and its update GEMM
  // subtracts -L21 L21^T from them; without children the GEMM stores -L21 L21^T
  auto u_first = [&](int64_t s) {
    return h->asm_first && h->height[s] > h->width[s] && h->width[s] > fc::ASSEMBLE_THIN &&
           h->kid_ptr[s + 1] > h->kid_ptr[s];
  };
  for (size_t l = 0; l < lv.size(); ++l) {
    join();
    const auto &S = lv[l];
    int64_t off = (int64_t)asm_t.size();
    for (int64_t s : S) assemble_tiles(h, s, fc::ASM_L, asm_t, ranges);
    push(h->program, K_ASSEMBLE, off, (int64_t)asm_t.size() - off, (int)l);
    // the wide update matrices' children contributions, on lane 1 once the level's children are
    // complete (after the last lane-0 launch so far), beside the level's panels
    int pre_asm = -1;
    {
      const int64_t uo = (int64_t)asm_t.size();
      for (int64_t s : S)
        if (u_first(s)) assemble_tiles(h, s, fc::ASM_U_FIRST, asm_t, ranges);
      if ((int64_t)asm_t.size() > uo) {
        int prev0 = -1;
        for (int q = (int)h->program.size() - 1; q >= 0 && prev0 < 0; --q)
          if (h->program[q].lane == 0) prev0 = q;
        push(h->program, K_ASSEMBLE, uo, (int64_t)asm_t.size() - uo, (int)l);
        Launch &a = h->program.back();
        a.lane = 1;
        if (prev0 >= 0) {
          a.dep = prev0;
          h->program[prev0].record = true;
        }
        pre_asm = (int)h->program.size() - 1;
      }
    }
    int P = 0;
    for (int64_t s : S) P = std::max(P, (h->width[s] + NB - 1) / NB);
    // Two-level blocking: panels are grouped in outer blocks of OUTER_PANELS. A panel's update of
    // the later columns of its own block (K = one panel) runs on lane 0 right after it; the update
    // of the columns past the block by the whole block (K = its width) runs once, after the
    // block's last panel: the next block's columns on lane 0 (after the previous such update on
    // lane 1, which also wrote them), the rest on lane 1 beside the next block's panels.
    const int OP = OUTER_PANELS;
    int last_rest = -1;   // the level's latest lane-1 launch
    int64_t blk_at = 0;   // the level's packed blocks (the update matrices' packs reuse the space)
    auto tc_tiles = [&](int64_t s, int jlo, int jhi, int32_t map, int kw, int wpad, int row0,
                        std::vector<fc::TcTask> &out) {
      const int m = h->height[s];
      const int64_t lo = h->loff[s];
      for (int jc = jlo; jc < jhi; jc += fc::GEMM_TC_N)
        for (int ic = jc; ic < m; ic += fc::GEMM_TC_M) {
          fc::TcTask g{};
          g.map = map, g.bi = ic - row0, g.bj = jc - row0;
          g.M = std::min(fc::GEMM_TC_M, m - ic), g.N = std::min(fc::GEMM_TC_N, jhi - jc), g.K = kw, g.wpad = wpad;
          g.flags = ic == jc ? 1 : 0;
          g.C = static_cast<float *>(Lp(lo + ic + (int64_t)jc * m));
          g.c_sj = m;
          out.push_back(g);
        }
    };
    auto tiles = [&](int64_t s, int jlo, int jhi, int k0, int k1, std::vector<fc::GemmTask> &out) {
      const int m = h->height[s];
      const int64_t lo = h->loff[s];
      for (int jc = jlo; jc < jhi; jc += fc::GEMM_TN)
        for (int ic = jc; ic < m; ic += TM) {
          fc::GemmTask g{};
          g.C = Lp(lo + ic + (int64_t)jc * m);
          g.A = Lp(lo + ic + (int64_t)k0 * m);
          g.B = Lp(lo + jc + (int64_t)k0 * m);
          g.c_si = 1, g.c_sj = m, g.a_si = 1, g.a_sk = m, g.b_sj = 1, g.b_sk = m;
          g.M = std::min(TM, m - ic);
          g.N = std::min(fc::GEMM_TN, jhi - jc);
          g.K = k1 - k0;
          g.flags = ic == jc ? 1 : 0;
          out.push_back(g);
        }
    };
    for (int p = 0; p < P; ++p) {
      int64_t po = (int64_t)panel_t.size(), go = (int64_t)gemm_t.size();
      std::vector<fc::GemmTask> rest;   // updates of the columns past the next block (lane 1)
      std::vector<fc::PackTask> blk_pack;       // tcgen05 path: the ending blocks' columns packed
      std::vector<fc::TcTask> tc_next, tc_rest;  // and their updates past the block (lanes 0, 1)
      bool outer = false;              // this step's lane-0 launch updates a next block's columns
      int p8max = 8;
      for (int64_t s : S) {
        const int m = h->height[s], w = h->width[s];
        const int c0 = p * NB;
        if (c0 >= w) continue;
        const int c1 = std::min(w, c0 + NB);
        p8max = std::max(p8max, (c1 - c0 + 7) / 8 * 8);
        const int64_t doff = h->doff[s] + 2 * (int64_t)NB * NB * p;
        int bw;
        const int64_t ib = inv_block(h, s, c0 / fc::SB, bw), in = c0 % fc::SB;
        const int64_t ioff = ib + in + in * bw;
        // every CTA of the panel stores its share of the factored block and its inverse (keep:
        // the panel's CTA count, pad: this CTA's place among them)
        if (c1 >= m) panel_t.push_back({(int32_t)s, c0, c1, m, m, 1, doff, ioff, bw, 0});
        const int nrt = (m - c1 + fc::PANEL_ROWS - 1) / fc::PANEL_ROWS;
        for (int r0 = c1, q = 0; r0 < m; r0 += fc::PANEL_ROWS, ++q)
          panel_t.push_back({(int32_t)s, c0, c1, r0, std::min(m, r0 + fc::PANEL_ROWS), nrt, doff, ioff, bw, q});
        const int bs = p / OP * OP * NB, be = std::min(w, bs + OP * NB);  // this panel's block
        if (c1 < be) tiles(s, c1, be, c0, c1, gemm_t);                     // within the block
        if (c1 == be && be < w) {                                         // past the block
          const int nx = std::min(w, be + OP * NB);
          outer = true;
          if (tc) {  // the block's columns packed once, the updates on tcgen05
            const int kw = be - bs, wpad = (kw + fc::TC_KPAD - 1) / fc::TC_KPAD * fc::TC_KPAD, ub = m - be;
            const int32_t map = (int32_t)maps.size();
            maps.push_back({blk_at, ub, wpad});
            for (int r0 = 0; r0 < ub; r0 += fc::TC_PACK_ROWS)
              for (int k0 = 0; k0 < wpad; k0 += fc::TC_PACK_K)
                blk_pack.push_back({(int32_t)s, r0, wpad, kw, blk_at, bs, be, k0, std::min(wpad, k0 + fc::TC_PACK_K)});
            blk_at += ((int64_t)ub * 2 * wpad + 63) / 64 * 64;
            tc_tiles(s, be, nx, map, kw, wpad, be, tc_next);
            if (nx < w) tc_tiles(s, nx, w, map, kw, wpad, be, tc_rest);
          } else {
            tiles(s, be, nx, bs, be, gemm_t);
            if (nx < w) tiles(s, nx, w, bs, be, rest);
          }
        }
      }
      push(h->program, K_PANEL, po, (int64_t)panel_t.size() - po, (int)l, p8max);
      int panel_at = (int)h->program.size() - 1;  // lane 1's updates read what it is after
      if (!blk_pack.empty()) {
        const int64_t bo = (int64_t)pack_t.size();
        pack_t.insert(pack_t.end(), blk_pack.begin(), blk_pack.end());
        push(h->program, K_PACK_TC, bo, (int64_t)blk_pack.size(), (int)l);
        panel_at = (int)h->program.size() - 1;
      }
      const size_t before = h->program.size();
      if (!tc_next.empty()) {
        const int64_t to = (int64_t)tc_t.size();
        tc_t.insert(tc_t.end(), tc_next.begin(), tc_next.end());
        push(h->program, K_GEMM_TC, to, (int64_t)tc_next.size(), (int)l);
      }
      push(h->program, K_GEMM, go, (int64_t)gemm_t.size() - go, (int)l);
      if (h->program.size() > before && outer && last_rest >= 0) {  // the next block after rest(b - 1)
        h->program[before].dep = last_rest;
        h->program[last_rest].record = true;
      }
      if (!rest.empty() || !tc_rest.empty()) {
        if (!rest.empty()) {
          const int64_t ro = (int64_t)gemm_t.size();
          gemm_t.insert(gemm_t.end(), rest.begin(), rest.end());
          push(h->program, K_GEMM, ro, (int64_t)rest.size(), (int)l);
        } else {
          const int64_t to = (int64_t)tc_t.size();
          tc_t.insert(tc_t.end(), tc_rest.begin(), tc_rest.end());
          push(h->program, K_GEMM_TC, to, (int64_t)tc_rest.size(), (int)l);
        }
        Launch &r = h->program.back();
        r.lane = 1;
        r.dep = panel_at;
        h->program[panel_at].record = true;
        last_rest = (int)h->program.size() - 1;
      }
    }
    pending_join = last_rest;
    // the diagonal blocks' inverses serve only the solve: lane 2, after the level's panels, beside
    // everything after them (the doublings of all levels in order on that one stream)
    int panels_done = -1;
    for (int q = (int)h->program.size() - 1; q >= 0 && panels_done < 0; --q)
      if (h->program[q].lane == 0) panels_done = q;
    for (int hh = NB; hh < fc::SB; hh *= 2) {
      std::vector<fc::GemmTask> first, second;
      inverse_doubling(h, S, h->d_T.as<double>(), hh, &first, &second);
      if (first.empty()) break;
      int64_t go = (int64_t)gemm_t.size();
      gemm_t.insert(gemm_t.end(), first.begin(), first.end());
      push(h->program, K_GEMM_MIXED, go, (int64_t)first.size(), (int)l);
      h->program.back().lane = 2;
      if (hh == NB && panels_done >= 0) {
        h->program.back().dep = panels_done;
        h->program[panels_done].record = true;
      }
      go = (int64_t)gemm_t.size();
      gemm_t.insert(gemm_t.end(), second.begin(), second.end());
      push(h->program, K_GEMM_F64, go, (int64_t)second.size(), (int)l);
      h->program.back().lane = 2;
    }
    if (tc) {
      // pack each supernode's L21 (K-major hi | lo), then its 128 x 128 tiles by TMA + tcgen05
      const int64_t po = (int64_t)pack_t.size(), to = (int64_t)tc_t.size();
      int64_t at = 0;
      for (int64_t s : S) {
        const int m = h->height[s], w = h->width[s], u = m - w;
        if (u <= 0 || w <= fc::ASSEMBLE_THIN) continue;  // a thin one's is formed by its assembly
        const int wpad = (w + fc::TC_KPAD - 1) / fc::TC_KPAD * fc::TC_KPAD;
        const int32_t map = (int32_t)maps.size();
        maps.push_back({at, u, wpad});
        for (int r0 = 0; r0 < u; r0 += fc::TC_PACK_ROWS)
          for (int k0 = 0; k0 < wpad; k0 += fc::TC_PACK_K)
            pack_t.push_back({(int32_t)s, r0, wpad, w, at, 0, w, k0, std::min(wpad, k0 + fc::TC_PACK_K)});
        at += ((int64_t)u * 2 * wpad + 63) / 64 * 64;  // 256-byte aligned regions
        const int64_t uo = h->uoff[s];
        for (int bj = 0; bj < u; bj += fc::GEMM_TC_N)
          for (int bi = bj; bi < u; bi += fc::GEMM_TC_M) {
            fc::TcTask g{};
            g.map = map, g.bi = bi, g.bj = bj;
            g.M = std::min(fc::GEMM_TC_M, u - bi), g.N = std::min(fc::GEMM_TC_N, u - bj), g.K = w, g.wpad = wpad;
            g.flags = (bi == bj ? 1 : 0) | (u_first(s) ? 0 : 2);
            g.C = static_cast<float *>(Up(uo + bi + (int64_t)bj * u));
            g.c_sj = u;
            tc_t.push_back(g);
          }
      }
      h->pack_len = std::max(h->pack_len, std::max(at, blk_at));
      push(h->program, K_PACK_TC, po, (int64_t)pack_t.size() - po, (int)l);
      push(h->program, K_GEMM_TC, to, (int64_t)tc_t.size() - to, (int)l);
      if (pre_asm >= 0 && (int64_t)tc_t.size() > to) {  // the products subtract from the children's sum
        h->program.back().dep = pre_asm;
        h->program[pre_asm].record = true;
      }
    } else {
      int64_t go = (int64_t)gemm_t.size();
      for (int64_t s : S) {
        const int m = h->height[s], w = h->width[s], u = m - w;
        if (u <= 0 || w <= fc::ASSEMBLE_THIN) continue;  // a thin one's is formed by its assembly
        const int64_t lo = h->loff[s], uo = h->uoff[s];
        for (int bj = 0; bj < u; bj += fc::GEMM_TN)
          for (int bi = bj; bi < u; bi += fc::GEMM_TM) {
            fc::GemmTask g{};
            g.C = Up(uo + bi + (int64_t)bj * u);
            g.A = Lp(lo + w + bi);
            g.B = Lp(lo + w + bj);
            g.c_si = 1, g.c_sj = u, g.a_si = 1, g.a_sk = m, g.b_sj = 1, g.b_sk = m;
            g.M = std::min(fc::GEMM_TM, u - bi);
            g.N = std::min(fc::GEMM_TN, u - bj);
            g.K = w;
            g.flags = (bi == bj ? 1 : 0) | (u_first(s) ? 0 : 2);
            gemm_t.push_back(g);
          }
      }
      push(h->program, K_GEMM, go, (int64_t)gemm_t.size() - go, (int)l);
      if (pre_asm >= 0 && (int64_t)gemm_t.size() > go) {
        // the products subtract from the children's sum (lane 1); they also read the columns the
        // level's lane-1 updates wrote, which come after the children's sum on that lane
        Launch &g = h->program.back();
        g.dep = pending_join >= 0 ? pending_join : pre_asm;
        h->program[g.dep].record = true;
        pending_join = -1;
      }
    }
    // the children's contributions to the update matrices, on top of -L21 L21^T
    // (a thin supernode's update matrix is formed here whole, -L21 L21^T included)
    off = (int64_t)asm_t.size();
    for (int64_t s : S) {
      const int m = h->height[s], w = h->width[s];
      if (m == w) continue;
      if (w <= fc::ASSEMBLE_THIN)
        assemble_tiles(h, s, fc::ASM_U_PRODUCT, asm_t, ranges);
      else if (h->kid_ptr[s + 1] > h->kid_ptr[s] && !u_first(s))
        assemble_tiles(h, s, fc::ASM_U, asm_t, ranges);
    }
    push(h->program, K_ASSEMBLE, off, (int64_t)asm_t.size() - off, (int)l);
  }
  join();
}

// The factorisation's launch program and task arrays (again after an option changes the kernels'
// tiles), uploaded; the captured factor graph is dropped.
int plan_factor_upload(fc_chol *h, fc_status *st) {
  cudaStream_t stream = h->stream;
  cudaError_t e;
  if (h->factor_graph) {
    cudaGraphExecDestroy(h->factor_graph);
    h->factor_graph = nullptr;
  }
  h->program.clear();
  const std::vector<std::vector<int64_t>> lv = levels_of(h);
  std::vector<fc::AssembleTask> asm_t;
  std::vector<int4> ranges;
  std::vector<fc::PanelTask> panel_t;
  std::vector<fc::GemmTask> gemm_t;
  std::vector<fc::PackTask> pack_t;
  std::vector<fc::TcTask> tc_t;
  std::vector<MapSpec> specs;
  plan_factor(h, lv, asm_t, ranges, panel_t, gemm_t, pack_t, tc_t, specs);
  h->gemm_tasks = (int64_t)(gemm_t.size() + tc_t.size());
  h->gemm_flops_factor = 0;
  for (const auto &g : gemm_t) h->gemm_flops_factor += task_flops(g);
  h->gemm_flops_updates = 0;
  for (const Launch &l : h->program)
    if (l.kind == K_GEMM)
      for (int64_t q = l.off; q < l.off + l.count; ++q) h->gemm_flops_updates += task_flops(gemm_t[q]);
  for (const auto &g : tc_t) {
    double outputs = (double)g.M * g.N;
    if (g.flags & 1) {
      outputs = 0;
      for (int j = 0; j < g.N; ++j) outputs += std::max(0, g.M - j);
    }
    h->gemm_flops_factor += 2.0 * g.K * outputs;
  }
  if (!tc_t.empty()) {
    // the packed operands and their tensor maps (TMA boxes of 128 rows x 16 FP32, 64-byte swizzle)
    if (h->d_pack.alloc(sizeof(float) * (size_t)std::max<int64_t>(h->pack_len, 1)) != cudaSuccess) {
      set_status(st, FC_OUT_OF_MEMORY, -1, h->pack_len, 0, "device memory for the packed operands");
      return FC_OUT_OF_MEMORY;
    }
    using Encode = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      set_status(st, FC_CUDA_ERROR, -1, 0, 0, "cuTensorMapEncodeTiled is not available");
      return FC_CUDA_ERROR;
    }
    const Encode encode = reinterpret_cast<Encode>(fn);
    std::vector<CUtensorMap> maps(specs.size());
    for (size_t i = 0; i < specs.size(); ++i) {
      const MapSpec &m = specs[i];
      const cuuint64_t dims[2] = {(cuuint64_t)2 * m.wpad, (cuuint64_t)m.u};
      const cuuint64_t strides[1] = {(cuuint64_t)2 * m.wpad * sizeof(float)};
      const cuuint32_t box[2] = {(cuuint32_t)fc::TC_KBOX, (cuuint32_t)fc::GEMM_TC_M};
      const cuuint32_t estr[2] = {1, 1};
      const CUresult r = encode(&maps[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, h->d_pack.as<float>() + m.poff, dims,
                                strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) {
        set_status(st, FC_CUDA_ERROR, -1, (int64_t)r, 0, "cuTensorMapEncodeTiled of a packed operand");
        return FC_CUDA_ERROR;
      }
    }
    if ((e = upload(h->d_maps, maps, stream)) != cudaSuccess || (e = upload(h->d_pack_t, pack_t, stream)) != cudaSuccess ||
        (e = upload(h->d_tc_t, tc_t, stream)) != cudaSuccess)
      return cuda_fail(st, e, "upload of the tcgen05 plan");
  }
  {
    // ordinals (among the factor's GEMM launches) of the heaviest launch and of the heaviest one
    // whose tasks all have K <= NB (a panel's update of the later columns)
    int64_t ordinal = 0;
    double big = -1, trail = -1;
    for (const Launch &l : h->program) {
      if (l.kind != K_GEMM) continue;
      double fl = 0;
      int kmax = 0;
      for (int64_t q = l.off; q < l.off + l.count; ++q) {
        fl += task_flops(gemm_t[q]);
        kmax = std::max(kmax, gemm_t[q].K);
      }
      if (fl > big) big = fl, h->gemm_big_ordinal = ordinal;
      if (kmax <= fc::NB && fl > trail) trail = fl, h->gemm_trail_ordinal = ordinal;
      ++ordinal;
    }
  }
  if ((e = upload(h->d_asm, asm_t, stream)) != cudaSuccess || (e = upload(h->d_ranges, ranges, stream)) != cudaSuccess ||
      (e = upload(h->d_panel, panel_t, stream)) != cudaSuccess ||
      (e = upload(h->d_gemm, gemm_t, stream)) != cudaSuccess)
    return cuda_fail(st, e, "upload of the plan");
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_fail(st, e, "plan upload");
  for (cudaEvent_t ev : h->lane_events)
    if (ev) cudaEventDestroy(ev);
  h->lane_events.assign(h->program.size(), nullptr);
  for (size_t q = 0; q < h->program.size(); ++q)
    if (h->program[q].record && (e = cudaEventCreateWithFlags(&h->lane_events[q], cudaEventDisableTiming)) != cudaSuccess)
      return cuda_fail(st, e, "lane events");
  // lane 0 (the panels' chain, on the critical path) at the highest priority, lane 1 (the long
  // updates beside it) at the lowest: a free SM takes the next panel's CTAs before more updates
  int least = 0, greatest = 0;
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  if (!h->side && ((e = cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, least)) != cudaSuccess ||
                   (e = cudaStreamCreateWithPriority(&h->hi, cudaStreamNonBlocking, greatest)) != cudaSuccess ||
                   (e = cudaStreamCreateWithPriority(&h->side2, cudaStreamNonBlocking, least)) != cudaSuccess ||
                   (e = cudaEventCreateWithFlags(&h->join2_event, cudaEventDisableTiming)) != cudaSuccess ||
                   (e = cudaEventCreateWithFlags(&h->fork_event, cudaEventDisableTiming)) != cudaSuccess ||
                   (e = cudaEventCreateWithFlags(&h->join_event, cudaEventDisableTiming)) != cudaSuccess ||
                   (e = cudaEventCreateWithFlags(&h->hi_join_event, cudaEventDisableTiming)) != cudaSuccess))
    return cuda_fail(st, e, "lane stream");
  return FC_OK;
}

// The symmetric indefinite factor's program (FC_PRECISION_LDLT, one stream), per level: the
// fronts' assembly; ceil(w / 64) pivoted panel steps, each followed by the GEMM of the update
// tasks the panel step wrote (slots sized for the earliest panel end, the rest left empty);
// W21 = L21 D and D out of the fronts; the update matrices -L21 W21^T; the children's entries in
// them. The panels' scratch (two columns and W per front) and W21 are reused level after level.
int plan_ldlt_upload(fc_chol *h, fc_status *st) {
  namespace L = fc::ldlt;
  if (h->factor_graph) {
    cudaGraphExecDestroy(h->factor_graph);
    h->factor_graph = nullptr;
  }
  h->program.clear();
  const std::vector<std::vector<int64_t>> lv = levels_of(h);
  auto ldw = [](int w) { return std::max(w - L::PANEL, 1); };
  auto up32 = [](int64_t x) { return (x + 31) / 32 * 32; };
  int64_t most = 0;
  for (const auto &S : lv) {
    int64_t need = 0;
    for (int64_t s : S) {
      const int64_t m = h->height[s], w = h->width[s];
      need += 2 * up32(m) + up32((int64_t)ldw((int)w) * (L::PANEL + 1)) + up32((m - w) * w);
    }
    most = std::max(most, need);
  }
  const int64_t n = h->n;
  cudaStream_t stream = h->stream;
  cudaError_t e = cudaSuccess;
  if (h->d_lscratch.alloc(sizeof(double) * (size_t)std::max<int64_t>(most, 1)) != cudaSuccess ||
      h->d_lscale.alloc(sizeof(double) * (size_t)std::max<int64_t>(n, 1)) != cudaSuccess ||
      h->d_lorder.alloc(sizeof(int32_t) * (size_t)std::max<int64_t>(n, 1)) != cudaSuccess ||
      h->d_lpivots.alloc((size_t)std::max<int64_t>(n, 1)) != cudaSuccess ||
      h->d_lpos.alloc(sizeof(int32_t) * (size_t)std::max<int64_t>(h->ns, 1)) != cudaSuccess ||
      h->d_ltwos.alloc(sizeof(int32_t) * (size_t)std::max<int64_t>(h->ns, 1)) != cudaSuccess ||
      h->d_lfailed.alloc(sizeof(unsigned long long)) != cudaSuccess ||
      h->d_ldd.alloc(sizeof(double) * (size_t)std::max<int64_t>(n, 1)) != cudaSuccess ||
      h->d_lde.alloc(sizeof(double) * (size_t)std::max<int64_t>(n, 1)) != cudaSuccess) {
    set_status(st, FC_OUT_OF_MEMORY, -1, h->entries, 0, "device memory for the LDL^T factor");
    return FC_OUT_OF_MEMORY;
  }
  {
    std::vector<int32_t> local(n);
    for (int64_t s = 0; s < h->ns; ++s)
      for (int64_t j = h->first[s]; j < h->first[s + 1]; ++j) local[j] = (int32_t)(j - h->first[s]);
    if ((e = upload(h->d_llocal, local, stream)) != cudaSuccess) return cuda_fail(st, e, "upload of the LDL^T plan");
  }
  auto Lp = [&](int64_t off) { return static_cast<double *>(arena_at(h->d_L, h, off)); };
  auto Up = [&](int64_t off) { return static_cast<double *>(arena_at(h->d_U, h, off)); };
  double *scratch = h->d_lscratch.as<double>();
  std::vector<fc::AssembleTask> asm_t;
  std::vector<int4> ranges;
  std::vector<fc::GemmTask> gemm_t;
  std::vector<L::PanelTask> pan_t;
  std::vector<int64_t> pan_slot;  // each panel task's first slot in gemm_t (its pointer set at upload)
  std::vector<L::AfterTask> aft_t;
  std::vector<L::InverseTask> inv_t;
  // the structure's rows and relative maps (the solve's are folded from them after each
  // factorisation) and the supernodal tree's parents
  h->ldlt_rows0 = h->rows;
  h->ldlt_rel0 = h->rel;
  h->ldlt_sparent.assign(h->ns, -1);
  for (int64_t s = 0; s < h->ns; ++s)
    for (int64_t q = h->kid_ptr[s]; q < h->kid_ptr[s + 1]; ++q) h->ldlt_sparent[h->kids[q]] = s;
  for (size_t l = 0; l < lv.size(); ++l) {
    const auto &S = lv[l];
    int64_t off = (int64_t)asm_t.size();
    for (int64_t s : S) assemble_tiles(h, s, fc::ASM_L, asm_t, ranges);
    push(h->program, K_ASSEMBLE, off, (int64_t)asm_t.size() - off, (int)l);
    // the level's fronts and their scratch
    std::vector<L::Front> fronts;
    std::vector<double *> w21;
    int64_t at = 0;
    int P = 0;
    for (int64_t s : S) {
      const int m = h->height[s], w = h->width[s];
      const int64_t f = h->first[s];
      L::Front fr{};
      fr.F = Lp(h->loff[s]);
      fr.m = m;
      fr.w = w;
      fr.scale = h->d_lscale.as<double>() + f;
      fr.order = h->d_lorder.as<int32_t>() + f;
      fr.pivots = h->d_lpivots.as<int8_t>() + f;
      fr.a = scratch + at;
      at += up32(m);
      fr.b = scratch + at;
      at += up32(m);
      fr.W = scratch + at;
      fr.ld_w = ldw(w);
      at += up32((int64_t)ldw(w) * (L::PANEL + 1));
      w21.push_back(scratch + at);
      at += up32((int64_t)(m - w) * w);
      fronts.push_back(fr);
      P = std::max(P, (w + L::PANEL - 1) / L::PANEL);
    }
    for (int p = 0; p < P; ++p) {
      const int64_t po = (int64_t)pan_t.size(), go = (int64_t)gemm_t.size();
      for (size_t q = 0; q < S.size(); ++q) {
        const int64_t s = S[q];
        const int m = h->height[s], w = h->width[s];
        if (p * L::PANEL >= w) continue;
        const int earliest = (p + 1) * L::PANEL;
        const int64_t slots = earliest < w ? L::update_tiles(m, w, earliest) : 0;
        L::PanelTask t{};
        t.front = fronts[q];
        t.first = h->first[s];
        t.nslots = (int32_t)slots;
        t.s = (int32_t)s;
        pan_t.push_back(t);
        pan_slot.push_back((int64_t)gemm_t.size());
        for (int64_t k = 0; k < slots; ++k) {
          gemm_t.push_back(fc::GemmTask{});  // empty until the panel step writes it
        }
      }
      push(h->program, K_LDLT_PANEL, po, (int64_t)pan_t.size() - po, (int)l);
      push(h->program, K_GEMM, go, (int64_t)gemm_t.size() - go, (int)l);
    }
    const int64_t ao = (int64_t)aft_t.size();
    for (size_t q = 0; q < S.size(); ++q) {
      const int64_t f = h->first[S[q]];
      aft_t.push_back({fronts[q], w21[q], h->d_ldd.as<double>() + f, h->d_lde.as<double>() + f});
    }
    push(h->program, K_LDLT_AFTER, ao, (int64_t)aft_t.size() - ao, (int)l);
    // the solve's diagonal-block inverses: 64 x 64 ones of the unit lower own blocks, then the
    // doubling to blocks of up to SB columns (as the Cholesky factor's, from its panels' inverses)
    const int64_t io = (int64_t)inv_t.size();
    for (int64_t s : S) {
      const int m = h->height[s], w = h->width[s];
      for (int c0 = 0; c0 < w; c0 += L::PANEL) {
        int bw;
        const int64_t ib = inv_block(h, s, c0 / fc::SB, bw), in = c0 % fc::SB;
        L::InverseTask t{};
        t.L = Lp(h->loff[s] + c0 + (int64_t)c0 * m);
        t.ldl = m;
        t.X = h->d_Dinv.as<double>() + ib + in + in * bw;
        t.ldx = bw;
        t.nb = std::min(L::PANEL, w - c0);
        inv_t.push_back(t);
      }
    }
    push(h->program, K_LDLT_INVERSE, io, (int64_t)inv_t.size() - io, (int)l);
    for (int hh = fc::NB; hh < fc::SB; hh *= 2) {
      std::vector<fc::GemmTask> first_t, second_t;
      inverse_doubling(h, S, h->d_T.as<double>(), hh, &first_t, &second_t);
      if (first_t.empty()) break;
      int64_t d0 = (int64_t)gemm_t.size();
      gemm_t.insert(gemm_t.end(), first_t.begin(), first_t.end());
      push(h->program, K_GEMM_MIXED, d0, (int64_t)first_t.size(), (int)l);
      d0 = (int64_t)gemm_t.size();
      gemm_t.insert(gemm_t.end(), second_t.begin(), second_t.end());
      push(h->program, K_GEMM_F64, d0, (int64_t)second_t.size(), (int)l);
    }
    // the update matrices: U = -L21 W21^T (lower tiles)
    const int64_t go = (int64_t)gemm_t.size();
    for (size_t q = 0; q < S.size(); ++q) {
      const int64_t s = S[q];
      const int m = h->height[s], w = h->width[s], u = m - w;
      const int64_t lo = h->loff[s], uo = h->uoff[s];
      for (int bj = 0; bj < u; bj += fc::GEMM_TN)
        for (int bi = bj; bi < u; bi += fc::GEMM_TM) {
          fc::GemmTask g{};
          g.C = Up(uo + bi + (int64_t)bj * u);
          g.A = Lp(lo + w + bi);
          g.B = w21[q] + bj;
          g.c_si = 1, g.c_sj = u, g.a_si = 1, g.a_sk = m, g.b_sj = 1, g.b_sk = u;
          g.M = std::min(fc::GEMM_TM, u - bi);
          g.N = std::min(fc::GEMM_TN, u - bj);
          g.K = w;
          g.flags = (bi == bj ? 1 : 0) | 2;
          gemm_t.push_back(g);
        }
    }
    push(h->program, K_GEMM, go, (int64_t)gemm_t.size() - go, (int)l);
    // the children's entries on top of the update matrices
    off = (int64_t)asm_t.size();
    for (int64_t s : S)
      if (h->height[s] > h->width[s] && h->kid_ptr[s + 1] > h->kid_ptr[s]) assemble_tiles(h, s, fc::ASM_U, asm_t, ranges);
    push(h->program, K_ASSEMBLE, off, (int64_t)asm_t.size() - off, (int)l);
  }
  h->gemm_tasks = (int64_t)gemm_t.size();
  if ((e = upload(h->d_asm, asm_t, stream)) != cudaSuccess || (e = upload(h->d_ranges, ranges, stream)) != cudaSuccess ||
      (e = upload(h->d_gemm, gemm_t, stream)) != cudaSuccess)
    return cuda_fail(st, e, "upload of the LDL^T plan");
  for (size_t q = 0; q < pan_t.size(); ++q) pan_t[q].slots = h->d_gemm.as<fc::GemmTask>() + pan_slot[q];
  if ((e = upload(h->d_lpanel, pan_t, stream)) != cudaSuccess || (e = upload(h->d_lafter, aft_t, stream)) != cudaSuccess ||
      (e = upload(h->d_linv, inv_t, stream)) != cudaSuccess)
    return cuda_fail(st, e, "upload of the LDL^T plan");
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_fail(st, e, "plan upload");
  for (cudaEvent_t ev : h->lane_events)
    if (ev) cudaEventDestroy(ev);
  h->lane_events.assign(h->program.size(), nullptr);
  return FC_OK;
}

int build(fc_chol *h, const fc::Symbolic &sym, fc_status *st) {
  const int64_t ns = sym.ns, n = sym.n;
  h->n = n;
  h->ns = ns;
  h->entries = sym.entries;
  h->fp32 = h->precision == FC_PRECISION_FP32_IR;
  h->ldlt = h->precision == FC_PRECISION_LDLT;
  h->esize = h->fp32 ? sizeof(float) : sizeof(double);
  h->nnz = (int64_t)sym.upper_idx.size();
  h->first = sym.first;
  h->perm = sym.perm;
  h->rows.assign(sym.rows.begin(), sym.rows.end());
  h->rows_off.assign(sym.rptr.begin(), sym.rptr.end() - (ns ? 1 : 0));
  if (ns == 0) h->rows_off.clear();
  h->width.resize(ns);
  h->height.resize(ns);
  h->loff.resize(ns);
  h->uoff.resize(ns);
  h->toff.resize(ns);
  h->doff.resize(ns);
  h->ioff.resize(ns);
  int64_t lsum = 0, usum = 0, tsum = 0, dsum = 0, isum = 0;
  double flops = 0;
  for (int64_t s = 0; s < ns; ++s) {
    const int64_t m = sym.height(s), w = sym.width(s), u = m - w;
    if (m * w > INT32_MAX) {
      // the assembly addresses a supernode's own panel with 32-bit offsets
      set_status(st, FC_TOO_LARGE, -1, m * w, INT32_MAX, "a supernode's panel holds more than 2^31 - 1 entries");
      return FC_TOO_LARGE;
    }
    h->width[s] = (int32_t)w;
    h->height[s] = (int32_t)m;
    h->loff[s] = lsum;
    h->toff[s] = tsum;
    lsum += m * w;
    usum += u * u;
    tsum += fc::trapezoid(m, w);
    h->doff[s] = dsum;
    h->ioff[s] = isum;
    for (int64_t b = 0; b * fc::SB < w; ++b) {
      const int64_t bw = std::min<int64_t>(fc::SB, w - b * fc::SB);
      isum += bw * bw;
    }
    {
      const int64_t full = w / fc::NB, last = w % fc::NB;
      dsum += 2 * (int64_t)fc::NB * fc::NB * full + 2 * last * last;
    }
    for (int64_t c = 0; c < w; ++c) flops += (double)(m - c) * (double)(m - c);
  }
  h->l_len = lsum;
  h->u_len = usum;
  h->flops = flops;
  // children and relative maps
  h->kid_ptr.assign(ns + 1, 0);
  for (int64_t s = 0; s < ns; ++s)
    if (sym.sparent[s] != fc::NONE) ++h->kid_ptr[sym.sparent[s] + 1];
  for (int64_t s = 0; s < ns; ++s) h->kid_ptr[s + 1] += h->kid_ptr[s];
  h->kids.resize(h->kid_ptr[ns]);
  {
    std::vector<int64_t> at(h->kid_ptr.begin(), h->kid_ptr.end() - 1);
    for (int64_t s = 0; s < ns; ++s)
      if (sym.sparent[s] != fc::NONE) h->kids[at[sym.sparent[s]]++] = (int32_t)s;
  }
  std::vector<int64_t> rel_off(ns, 0);
  std::vector<int32_t> rel;
  for (int64_t c = 0; c < ns; ++c) {
    rel_off[c] = (int64_t)rel.size();
    const int64_t p = sym.sparent[c];
    if (p == fc::NONE) continue;
    const int32_t *cr = sym.rows.data() + sym.rptr[c];
    const int32_t *pr = sym.rows.data() + sym.rptr[p];
    const int64_t pm = sym.height(p);
    int64_t at = 0;
    for (int64_t i = sym.width(c); i < sym.height(c); ++i) {
      while (at < pm && pr[at] < cr[i]) ++at;
      if (at >= pm || pr[at] != cr[i]) {
        Failure f;
        f.code = fc::INTERNAL;
        f.message = "supernodal structure: a child's row outside its parent";
        return fail_status(st, f);
      }
      rel.push_back((int32_t)at);
    }
  }
  // input entries by postordered column, with their place in L
  std::vector<int64_t> snode(n);
  for (int64_t s = 0; s < ns; ++s)
    for (int64_t j = sym.first[s]; j < sym.first[s + 1]; ++j) snode[j] = s;
  std::vector<int64_t> a_ptr(n + 1, 0), a_src(h->nnz), a_dst(h->nnz), diag_src(n, -1);
  for (int64_t e = 0; e < h->nnz; ++e) ++a_ptr[sym.ccol[e] + 1];
  for (int64_t j = 0; j < n; ++j) a_ptr[j + 1] += a_ptr[j];
  {
    std::vector<int64_t> at(a_ptr.begin(), a_ptr.end() - 1);
    for (int64_t e = 0; e < h->nnz; ++e) {
      const int64_t r = sym.crow[e], c = sym.ccol[e];
      const int64_t s = snode[c];
      const int32_t *sr = sym.rows.data() + sym.rptr[s];
      const int64_t m = sym.height(s);
      const int32_t *hit = std::lower_bound(sr, sr + m, (int32_t)r);
      if (hit == sr + m || *hit != r || (hit - sr) < c - sym.first[s]) {
        Failure f;
        f.code = fc::INTERNAL;
        f.message = "supernodal factorization: an entry of A outside the structure";
        return fail_status(st, f);
      }
      const int64_t pos = at[c]++;
      a_src[pos] = e;
      a_dst[pos] = h->loff[s] + (hit - sr) + (c - sym.first[s]) * m;
      if (r == c) diag_src[c] = e;
    }
  }
  // within each block of assemble_cols(h) columns of a supernode, the entries by their row in the
  // front (an assembly tile takes the contiguous run of its rows)
  std::vector<int32_t> a_lrow(h->nnz);
  {
    std::vector<std::pair<int32_t, int64_t>> run;
    std::vector<int64_t> src2, dst2;
    for (int64_t s = 0; s < ns; ++s) {
      const int64_t f = sym.first[s], w = sym.first[s + 1] - f, m = sym.height(s);
      const int64_t cols = assemble_cols(h);
      for (int64_t j0 = 0; j0 < w; j0 += cols) {
        const int64_t b0 = a_ptr[f + j0], b1 = a_ptr[f + std::min(w, j0 + cols)];
        run.clear();
        for (int64_t q = b0; q < b1; ++q) run.emplace_back((int32_t)((a_dst[q] - h->loff[s]) % m), q);
        std::sort(run.begin(), run.end());
        src2.resize(run.size());
        dst2.resize(run.size());
        for (size_t q = 0; q < run.size(); ++q) {
          src2[q] = a_src[run[q].second];
          dst2[q] = a_dst[run[q].second];
          a_lrow[b0 + q] = run[q].first;
        }
        std::copy(src2.begin(), src2.end(), a_src.begin() + b0);
        std::copy(dst2.begin(), dst2.end(), a_dst.begin() + b0);
      }
    }
  }
  h->a_ptr = a_ptr;
  h->a_lrow = std::move(a_lrow);
  h->rel_off = rel_off;
  h->rel = rel;
  auto lv = levels_of(h);
  {
    std::vector<int64_t> usize(ns);
    for (int64_t s = 0; s < ns; ++s) usize[s] = (int64_t)(h->height[s] - h->width[s]) * (h->height[s] - h->width[s]);
    usum = arena_offsets(h, lv, usize, h->uoff);
    h->u_len = usum;
  }
  cudaStream_t stream = h->stream;
  cudaError_t e = cudaSuccess;
#define UP(buf, vec)                                    \
  if ((e = upload(buf, vec, stream)) != cudaSuccess) { \
    return cuda_fail(st, e, "upload " #vec);            \
  }
  UP(h->d_first, h->first);
  UP(h->d_width, h->width);
  UP(h->d_height, h->height);
  UP(h->d_rows_off, h->rows_off);
  UP(h->d_rows, h->rows);
  UP(h->d_loff, h->loff);
  UP(h->d_uoff, h->uoff);
  UP(h->d_kid_ptr, h->kid_ptr);
  UP(h->d_kids, h->kids);
  {
    std::vector<fc::KidMeta> meta(h->kids.size());
    for (size_t q = 0; q < h->kids.size(); ++q) {
      const int64_t c = h->kids[q];
      meta[q] = {h->uoff[c], rel_off[c], h->height[c] - h->width[c], 0};
    }
    UP(h->d_kid_meta, meta);
  }
  UP(h->d_rel_off, rel_off);
  UP(h->d_rel, rel);
  UP(h->d_a_ptr, a_ptr);
  UP(h->d_a_src, a_src);
  UP(h->d_a_dst, a_dst);
  UP(h->d_diag_src, diag_src);
  UP(h->d_perm, h->perm);
  UP(h->d_toff, h->toff);
  UP(h->d_doff, h->doff);
  if (h->fp32 || h->ldlt) {
    std::vector<int32_t> a_row(h->nnz), a_col(h->nnz);
    for (int64_t q = 0; q < h->nnz; ++q) {
      a_row[q] = sym.crow[a_src[q]];
      a_col[q] = sym.ccol[a_src[q]];
    }
    UP(h->d_a_row, a_row);
    UP(h->d_a_col, a_col);
  }
#undef UP
  if (h->d_L.alloc(h->esize * (size_t)std::max<int64_t>(lsum, 1)) != cudaSuccess ||
      h->d_U.alloc(h->esize * (size_t)std::max<int64_t>(usum, 1)) != cudaSuccess ||
      (h->fp32 && h->d_scale.alloc(sizeof(double) * (size_t)std::max<int64_t>(n, 1)) != cudaSuccess) ||
      h->d_D.alloc(sizeof(double) * (size_t)std::max<int64_t>(dsum, 1)) != cudaSuccess ||
      h->d_Dinv.alloc(sizeof(double) * (size_t)std::max<int64_t>(isum, 1)) != cudaSuccess ||
      h->d_val.alloc(sizeof(double) * (size_t)std::max<int64_t>(h->nnz, 1)) != cudaSuccess ||
      h->d_status.alloc(sizeof(fc::DeviceStatus)) != cudaSuccess) {
    Failure f;
    f.code = fc::OUT_OF_MEMORY;
    f.entries = h->entries;
    f.message = "device memory for the factor";
    return fail_status(st, f);
  }
  fc::Tree &t = h->tree;
  t.first = h->d_first.as<int64_t>();
  t.width = h->d_width.as<int32_t>();
  t.height = h->d_height.as<int32_t>();
  t.rows_off = h->d_rows_off.as<int64_t>();
  t.rows = h->d_rows.as<int32_t>();
  t.loff = h->d_loff.as<int64_t>();
  t.uoff = h->d_uoff.as<int64_t>();
  t.kid_ptr = h->d_kid_ptr.as<int64_t>();
  t.kids = h->d_kids.as<int32_t>();
  t.kid_meta = h->d_kid_meta.as<fc::KidMeta>();
  t.rel_off = h->d_rel_off.as<int64_t>();
  t.rel = h->d_rel.as<int32_t>();
  t.a_ptr = h->d_a_ptr.as<int64_t>();
  t.a_src = h->d_a_src.as<int64_t>();
  t.a_dst = h->d_a_dst.as<int64_t>();
  t.diag_src = h->d_diag_src.as<int64_t>();
  t.doff = h->d_doff.as<int64_t>();
  t.a_row = h->d_a_row.as<int32_t>();
  t.a_col = h->d_a_col.as<int32_t>();
  t.scale = h->fp32 ? h->d_scale.as<double>() : nullptr;
  t.L = h->d_L.p;
  t.U = h->d_U.p;
  t.D = h->d_D.as<double>();
  t.Dinv = h->d_Dinv.as<double>();
  h->i_len = isum;
  {
    // the inverses' upper triangles stay zero; the doubling's scratch fits its largest level step
    cudaError_t e = cudaMemsetAsync(h->d_Dinv.p, 0, sizeof(double) * (size_t)std::max<int64_t>(isum, 1), h->stream);
    int64_t most = 0;
    for (const auto &S : lv)
      for (int hh = fc::NB; hh < fc::SB; hh *= 2) most = std::max(most, inverse_doubling(h, S, nullptr, hh, nullptr, nullptr));
    h->t_len = most;
    if (e != cudaSuccess || h->d_T.alloc(sizeof(double) * (size_t)std::max<int64_t>(most, 1)) != cudaSuccess) {
      Failure f;
      f.code = fc::OUT_OF_MEMORY;
      f.entries = h->entries;
      f.message = "device memory for the diagonal-block inverses";
      return fail_status(st, f);
    }
  }
  return h->ldlt ? plan_ldlt_upload(h, st) : plan_factor_upload(h, st);
}

cudaEvent_t next_event(fc_chol *h) {
  if (h->events_used == h->event_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    h->event_pool.push_back(e);
  }
  return h->event_pool[h->events_used++];
}

// Brackets one launch with events when profiling.
struct Mark {
  fc_chol *h;
  int kind, level, count;
  cudaEvent_t a = nullptr;
  Mark(fc_chol *h_, int kind_, int level_ = -1, int count_ = 0) : h(h_), kind(kind_), level(level_), count(count_) {
    if (h->profiling) {
      a = next_event(h);
      cudaEventRecord(a, h->stream);
    }
  }
  ~Mark() {
    if (h->profiling) {
      cudaEvent_t b = next_event(h);
      cudaEventRecord(b, h->stream);
      h->marks.push_back({kind, level, count, a, b});
    }
  }
};

// Runs `enqueue` under stream capture and keeps the instantiated graph in *exec; false if the
// capture or the instantiation failed (the work is then enqueued directly by the caller).
template <class F>
bool capture(fc_chol *h, cudaGraphExec_t *exec, F enqueue) {
  if (*exec) {
    cudaGraphExecDestroy(*exec);
    *exec = nullptr;
  }
  cudaGraph_t graph = nullptr;
  if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  enqueue();
  cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
  if (e != cudaSuccess || !graph) {
    cudaGetLastError();
    return false;
  }
  e = cudaGraphInstantiate(exec, graph, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *exec = nullptr;
    return false;
  }
  return true;
}

int enqueue_factor_direct(fc_chol *h, const double *d_val, const volatile int32_t *cancel);

// Enqueues the factor's program (as a replayed graph when it can). Returns FC_CANCELLED when the
// flag was set between levels.
int enqueue_factor(fc_chol *h, const double *d_val, const volatile int32_t *cancel) {
  h->ldlt_folded = false;
  if (cancel || h->profiling || !h->graphs) return enqueue_factor_direct(h, d_val, cancel);
  if (!h->factor_graph || h->factor_graph_val != d_val || h->factor_graph_stream != h->stream) {
    if (!capture(h, &h->factor_graph, [&] { enqueue_factor_direct(h, d_val, nullptr); })) {
      h->graphs = false;
      return enqueue_factor_direct(h, d_val, nullptr);
    }
    h->factor_graph_val = d_val;
    h->factor_graph_stream = h->stream;
  }
  cudaGraphLaunch(h->factor_graph, h->stream);
  h->last_factor_launches = (int64_t)h->program.size();
  return FC_OK;
}

int enqueue_factor_direct(fc_chol *h, const double *d_val, const volatile int32_t *cancel) {
  const cudaStream_t user = h->stream;
  cudaMemsetAsync(h->d_status.p, 0xff, sizeof(fc::DeviceStatus), user);
  if (h->ldlt) {
    // the rows' largest |A| from the values, every supernode's pivots reset, no panel done
    cudaMemsetAsync(h->d_lscale.p, 0, sizeof(double) * (size_t)std::max<int64_t>(h->n, 1), user);
    cudaMemsetAsync(h->d_lpos.p, 0, sizeof(int32_t) * (size_t)std::max<int64_t>(h->ns, 1), user);
    cudaMemsetAsync(h->d_ltwos.p, 0, sizeof(int32_t) * (size_t)std::max<int64_t>(h->ns, 1), user);
    cudaMemsetAsync(h->d_lfailed.p, 0xff, sizeof(unsigned long long), user);
    fc::ldlt::launch_reset(h->n, h->d_llocal.as<int32_t>(), h->d_lorder.as<int32_t>(), h->d_lpivots.as<int8_t>(), user);
    fc::ldlt::launch_scale(h->nnz, h->d_a_src.as<int64_t>(), h->d_a_row.as<int32_t>(), h->d_a_col.as<int32_t>(), d_val,
                           h->d_lscale.as<unsigned long long>(), user);
  }
  if (h->fp32) fc::launch_scale(h->n, h->d_diag_src.as<int64_t>(), d_val, h->d_scale.as<double>(), user);
  const fc::GemmKind gk = h->fp32 ? fc::GemmKind::F32_TF32X3 : fc::GemmKind::F64;
  const fc::Tree &t = h->tree;
  // both lanes fork from the caller's stream here and join it at the end (lane 0 on the
  // high-priority stream, lane 1 on the low-priority one); profiling keeps one lane
  const bool lanes = h->side && h->hi && h->side2 && !h->profiling;
  const cudaStream_t main = lanes ? h->hi : user;
  if (lanes) {
    cudaEventRecord(h->fork_event, user);
    cudaStreamWaitEvent(h->side, h->fork_event, 0);
    cudaStreamWaitEvent(h->side2, h->fork_event, 0);
    cudaStreamWaitEvent(h->hi, h->fork_event, 0);
  }
  auto join = [&]() {
    if (lanes) {
      cudaEventRecord(h->join_event, h->side);
      cudaStreamWaitEvent(user, h->join_event, 0);
      cudaEventRecord(h->join2_event, h->side2);
      cudaStreamWaitEvent(user, h->join2_event, 0);
      cudaEventRecord(h->hi_join_event, h->hi);
      cudaStreamWaitEvent(user, h->hi_join_event, 0);
    }
  };
  int last_level = -1;
  int64_t launches = 0;
  for (size_t li = 0; li < h->program.size(); ++li) {
    const Launch &l = h->program[li];
    if (cancel && l.level != last_level) {
      if (*cancel != 0) {
        join();
        h->last_factor_launches = launches;
        return FC_CANCELLED;
      }
      last_level = l.level;
    }
    const cudaStream_t st = !lanes || l.lane == 0 ? main : l.lane == 1 ? h->side : h->side2;
    if (lanes && l.dep >= 0) cudaStreamWaitEvent(st, h->lane_events[l.dep], 0);
    Mark mark(h, l.kind, l.level, l.count);
    switch (l.kind) {
      case K_ASSEMBLE:
        fc::launch_assemble(t, h->fp32, d_val, h->d_asm.as<fc::AssembleTask>() + l.off, h->d_ranges.as<int4>(), l.count,
                            st);
        break;
      case K_PANEL:
        fc::launch_panel(t, h->fp32, d_val, h->d_panel.as<fc::PanelTask>() + l.off, l.count,
                         h->d_status.as<fc::DeviceStatus>(), l.width, st);
        break;
      case K_GEMM: fc::launch_gemm(h->d_gemm.as<fc::GemmTask>() + l.off, l.count, gk, st); break;
      case K_PACK_TC: fc::launch_pack_tc(t, h->d_pack_t.as<fc::PackTask>() + l.off, h->d_pack.as<float>(), l.count, st); break;
      case K_GEMM_TC:
        fc::launch_syrk_tc(h->d_tc_t.as<fc::TcTask>() + l.off, h->d_maps.p, l.count, h->d_status.as<fc::DeviceStatus>(),
                           st);
        break;
      case K_GEMM_MIXED:
        fc::launch_gemm(h->d_gemm.as<fc::GemmTask>() + l.off, l.count,
                        h->fp32 ? fc::GemmKind::F32A_F64 : fc::GemmKind::F64, st);
        break;
      case K_GEMM_F64: fc::launch_gemm(h->d_gemm.as<fc::GemmTask>() + l.off, l.count, fc::GemmKind::F64, st); break;
      case K_LDLT_PANEL:
        fc::ldlt::launch_panel(h->d_lpanel.as<fc::ldlt::PanelTask>() + l.off, l.count, h->d_lpos.as<int32_t>(),
                               h->d_ltwos.as<int32_t>(), h->d_lfailed.as<unsigned long long>(), st);
        break;
      case K_LDLT_AFTER: fc::ldlt::launch_after(h->d_lafter.as<fc::ldlt::AfterTask>() + l.off, l.count, st); break;
      case K_LDLT_INVERSE: fc::ldlt::launch_inverse(h->d_linv.as<fc::ldlt::InverseTask>() + l.off, l.count, st); break;
    }
    if (lanes && l.record) cudaEventRecord(h->lane_events[li], st);
    ++launches;
  }
  join();
  h->last_factor_launches = launches;
  return FC_OK;
}

int read_status(fc_chol *h, fc_status *st) {
  fc::DeviceStatus ds{};
  cudaError_t e = cudaMemcpyAsync(&ds, h->d_status.p, sizeof(ds), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_fail(st, e, "factorisation");
  if (ds.timeout != 0xFFFFFFFFu) {
    set_status(st, FC_TIMEOUT, -1, 0, 0, "a bounded wait of the tensor-core GEMM gave up");
    return FC_TIMEOUT;
  }
  if (ds.failed_column != ULLONG_MAX) {
    const int64_t col = (int64_t)ds.failed_column;
    const int64_t orig = col < h->n ? h->perm[col] : col;
    set_status(st, FC_NOT_POSITIVE_DEFINITE, orig, 0, 0, "the pivot is not positive (relative to the diagonal)");
    return FC_NOT_POSITIVE_DEFINITE;
  }
  if (h->ldlt) {
    unsigned long long failed = ULLONG_MAX;
    e = cudaMemcpy(&failed, h->d_lfailed.p, sizeof(failed), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(st, e, "factorisation");
    if (failed != ULLONG_MAX) {
      const int64_t col = (int64_t)failed;
      set_status(st, FC_SINGULAR, col < h->n ? h->perm[col] : col, 0, 0,
                 "no pivot in the column's supernode exceeds the tolerance (singular to working precision)");
      return FC_SINGULAR;
    }
  }
  set_status(st, FC_OK);
  return FC_OK;
}

// The LDL^T factor solves level by level (refined by plain refinement only; not without
// allocation, not persistent): the no-alloc solve is refused for it.
bool ldlt_refused(const fc_chol *h, fc_status *st) {
  if (!h->ldlt) return false;
  set_status(st, FC_INVALID_ARGUMENT, -1, 0, 0, "the LDL^T factor has no solve without allocation");
  return true;
}

// The LDL^T solve's structure, once per factorisation: the pivot orders read back and folded
// into the structure (host/ldlt_fold.cpp), the solve's rows, relative maps and permutation
// uploaded, each front's rows below moved to their new order, and the solve's plan dropped (the
// next solve plans on the folded structure). Its own blocks are unit lower (split_d), so the
// Cholesky solve then runs on them as it is, with D^-1 between its passes.
int ldlt_prepare_solve(fc_chol *h, fc_status *st) {
  if (h->ldlt_folded) return FC_OK;
  const int64_t n = h->n, ns = h->ns;
  std::vector<int32_t> order(n);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess && n > 0)
    e = cudaMemcpy(order.data(), h->d_lorder.p, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(st, e, "the LDL^T factor's pivot orders");
  std::vector<int64_t> rptr(h->rows_off.begin(), h->rows_off.end());
  rptr.push_back((int64_t)h->ldlt_rows0.size());
  if (ns == 0) rptr.assign(1, 0);
  fc::LdltFold fold;
  if (!fc::ldlt_fold(n, ns, h->first.data(), rptr.data(), h->ldlt_rows0.data(), h->perm.data(), h->ldlt_sparent.data(),
                     order.data(), fold)) {
    set_status(st, FC_INTERNAL, -1, 0, 0, "the LDL^T factor's pivot orders are not permutations");
    return FC_INTERNAL;
  }
  std::vector<fc::ldlt::PermuteTask> moves;
  if ((e = upload(h->d_lsrows, fold.rows, h->stream)) != cudaSuccess ||
      (e = upload(h->d_lsrel, fold.rel, h->stream)) != cudaSuccess ||
      (e = upload(h->d_lsperm, fold.perm, h->stream)) != cudaSuccess ||
      (e = upload(h->d_lfrom, fold.from, h->stream)) != cudaSuccess ||
      (e = h->d_ltmp.alloc(sizeof(double) * (size_t)std::max<int64_t>(fold.from_off[ns], 1))) != cudaSuccess)
    return cuda_fail(st, e, "the LDL^T solve's structure");
  for (int64_t s = 0; s < ns; ++s) {
    const int m = h->height[s], w = h->width[s];
    if (m == w) continue;
    fc::ldlt::PermuteTask t{};
    t.front.F = static_cast<double *>(arena_at(h->d_L, h, h->loff[s]));
    t.front.m = m;
    t.front.w = w;
    t.from = h->d_lfrom.as<int32_t>() + fold.from_off[s];
    t.tmp = h->d_ltmp.as<double>() + fold.from_off[s];
    moves.push_back(t);
  }
  if ((e = upload(h->d_lperm_t, moves, h->stream)) != cudaSuccess) return cuda_fail(st, e, "the LDL^T solve's structure");
  fc::ldlt::launch_permute(h->d_lperm_t.as<fc::ldlt::PermuteTask>(), (int)moves.size(), h->stream);
  if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess)
    return cuda_fail(st, e, "the LDL^T solve's structure");
  h->ldlt_from = std::move(fold.from);
  h->ldlt_from_off = std::move(fold.from_off);
  h->rows = std::move(fold.rows);  // what the solve's planner reads
  h->rel = std::move(fold.rel);
  h->stree = h->tree;
  h->stree.rows = h->d_lsrows.as<int32_t>();
  h->stree.rel = h->d_lsrel.as<int32_t>();
  h->solve_R = 0;
  if (h->solve_graph) {
    cudaGraphExecDestroy(h->solve_graph);
    h->solve_graph = nullptr;
  }
  h->ldlt_folded = true;
  return FC_OK;
}

// The solve's program for R right-hand sides (built once per R). Forward, level by level: a thin
// supernode is one launch of tiles (own rows, y = Dinv x, its update vector); a wide one's front
// collects its children's update vectors, then per block of up to SB columns y = Dinv x and the
// rows below -= L y (x accumulates, y lands in x2). Backward, top level first: thin supernodes by
// chunks summing L21^T x; a wide one's own rows -= L21^T x(rows past its columns, read through
// its row list), then per block from the last z = Dinv^T x2 and the own rows above -= L^T z (x2
// accumulates, z lands in x). The task lists hold the update vectors' offsets (liveness-reused,
// like the update matrices) and the tasks over given device vectors x, x2 (n x R each) and v.
struct SolvePlan {
  std::vector<int64_t> voff;
  int64_t vsum = 0;
  int64_t psum = 0;    // doubles of the split GEMMs' partial tiles (the largest launch's)
  int64_t scount = 0;  // their counters (the largest launch's), after the thin ones
  int lg = 6;        // the thin tasks' block of right-hand sides: 1 << lg columns
  int64_t tpart = 0, tcount = 0;  // the thin backward chunks' partial sums and counters (a level's)
  std::vector<fc::ThinTask> thin;
  std::vector<int4> tranges;
  std::vector<fc::ThinBwdTask> tbwd;
  std::vector<fc::RowTask> rows;
  std::vector<int2> ranges;
  std::vector<fc::SolveTask> panels;
  std::vector<fc::GemmTask> gemm;
  std::vector<Launch> fwd, bwd;
};

void solve_offsets(const fc_chol *h, int R, SolvePlan &p) {
  std::vector<std::vector<int64_t>> lv(h->levels);
  for (int64_t s = 0; s < h->ns; ++s) lv[h->level[s]].push_back(s);
  std::vector<int64_t> vsize(h->ns);
  for (int64_t s = 0; s < h->ns; ++s) vsize[s] = (int64_t)(h->height[s] - h->width[s]) * R;
  p.vsum = arena_offsets(h, lv, vsize, p.voff);
  p.lg = 0;
  while ((1 << p.lg) < std::min(R, 64)) ++p.lg;
  const int64_t jb = (R + 63) / 64;
  for (const auto &S : lv) {
    int64_t part = 0, count = 0;
    for (int64_t s : S) {
      const int64_t u = h->height[s] - h->width[s];
      if (h->width[s] > fc::SOLVE_THIN || u <= fc::THIN_CHUNK) continue;
      part += (u + fc::THIN_CHUNK - 1) / fc::THIN_CHUNK * fc::SOLVE_THIN * 64 * jb;
      count += jb;
    }
    p.tpart = std::max(p.tpart, part);
    p.tcount = std::max(p.tcount, count);
  }
}

// In a solve launch with too few output tiles to fill the GPU twice, a GEMM whose K is long is
// split in chunks of SOLVE_KC: the chunks run as separate CTAs and the last one adds their
// partials in order, in groups of SPLIT_GROUP chunks when there are more (GemmTask flag 8: with
// the last chunk alone adding 30 partial tiles, a top supernode's backward product took twice its
// main loop's time). The choice depends on the tiles of one block of 64
// right-hand sides and on K, not on how many right-hand sides are solved together, so a column's
// result does not either. Partials and counters are offsets into buffers given at launch, reused
// launch after launch.
constexpr int SOLVE_KC = 256;
// With clusters a chunk is SOLVE_CLUSTER times longer: each CTA of the cluster walks SOLVE_KC of it.
constexpr int SOLVE_KC_CLUSTER = SOLVE_KC * fc::SOLVE_CLUSTER;

struct SplitPush {
  SolvePlan &p;
  int waves_tiles;  // a launch with fewer output tiles (per block of right-hand sides) is split
  bool cluster;     // split over thread-block clusters (else in chunks of separate CTAs)
  std::vector<std::pair<fc::GemmTask, std::pair<size_t, size_t>>> pending;
  int tiles = 0;
  // g's K range [0, K) may be split; a_es / b_es: bytes of an A / B element; first: g is in the
  // first block of right-hand sides (counts the launch's tiles)
  void add(const fc::GemmTask &g, size_t a_es, size_t b_es, bool first) {
    pending.push_back({g, {a_es, b_es}});
    tiles += first ? 1 : 0;
  }
  // the end of a launch: its tasks go to the plan (split when the launch is short of tiles); its
  // partials and counters are free again after it. Returns whether the launch runs on clusters.
  bool close() {
    const bool split = tiles < waves_tiles;
    const bool on_clusters = split && cluster;
    const int kc = on_clusters ? SOLVE_KC_CLUSTER : SOLVE_KC;
    int64_t at = 0;
    int32_t cnt = 0;
    for (auto &pg : pending) {
      const fc::GemmTask &g = pg.first;
      if (!split || g.K <= kc + kc / 2) {
        p.gemm.push_back(g);
        continue;
      }
      const int chunks = (g.K + kc - 1) / kc;
      for (int q = 0; q < chunks; ++q) {
        fc::GemmTask c = g;
        const int64_t k0 = (int64_t)q * kc;
        c.A = static_cast<const char *>(g.A) + k0 * g.a_sk * (int64_t)pg.second.first;
        if (g.flags & 16)
          c.b_rows = g.b_rows + k0;  // B's rows through the row list
        else
          c.B = static_cast<const char *>(g.B) + k0 * g.b_sk * (int64_t)pg.second.second;
        c.K = (int)std::min<int64_t>(kc, g.K - k0);
        c.flags = g.flags | 8;
        c.part_off = at, c.chunks = chunks, c.chunk = q, c.counter = (int32_t)p.tcount + cnt;
        p.gemm.push_back(c);
      }
      // the chunks' partials, then the groups' sums; a counter for the sum and one a group
      at += (int64_t)(chunks + fc::split_groups(chunks)) * 4096;
      cnt += 1 + fc::split_groups(chunks);
    }
    p.psum = std::max(p.psum, at);
    p.scount = std::max<int64_t>(p.scount, cnt);
    pending.clear();
    tiles = 0;
    return on_clusters;
  }
};

void solve_tasks(const fc_chol *h, int R, double *x, double *x2, double *v, SolvePlan &p) {
  std::vector<std::vector<int64_t>> lv(h->levels);
  for (int64_t s = 0; s < h->ns; ++s) lv[h->level[s]].push_back(s);
  const std::vector<int64_t> &voff = p.voff;
  std::vector<fc::RowTask> &rows = p.rows;
  std::vector<fc::GemmTask> &gemm = p.gemm;
  SplitPush sp{p, 2 * prop_sms(h->device), h->solve_cluster};
  const size_t es = h->esize;
  p.psum = 0, p.scount = 0;
  std::vector<Launch> &fwd = p.fwd, &bwd = p.bwd;
  auto Lp = [&](int64_t off) { return arena_at(h->d_L, h, off); };
  auto thin = [&](int64_t s) { return h->width[s] <= fc::SOLVE_THIN; };
  const int RP = 1 << p.lg, TR = fc::THIN_ROWS;
  // forward
  for (size_t l = 0; l < lv.size(); ++l) {
    const auto &S = lv[l];
    const int64_t to = (int64_t)p.thin.size();
    for (int64_t s : S) {
      if (!thin(s)) continue;
      const int m = h->height[s], w = h->width[s];
      const int64_t q0 = h->kid_ptr[s], q1 = h->kid_ptr[s + 1];
      for (int i0 = w; i0 < m || i0 == w; i0 += TR) {
        const int i1 = std::min(m, i0 + TR);
        const int32_t at = (int32_t)p.tranges.size();
        for (int64_t q = q0; q < q1; ++q) {
          const int64_t c = h->kids[q];
          const int uc = h->height[c] - h->width[c];
          const int32_t *rel = h->rel.data() + h->rel_off[c];
          auto pos = [&](int r) { return (int)(std::lower_bound(rel, rel + uc, r) - rel); };
          p.tranges.push_back(make_int4(pos(w), pos(i0), pos(i1), 0));
        }
        for (int j0 = 0; j0 < R; j0 += RP)
          p.thin.push_back({(int32_t)s, i0, i1, j0, at, i0 == w ? 1 : 0, h->ioff[s]});
        if (i1 >= m) break;
      }
    }
    push(fwd, K_SOLVE_THIN_FWD, to, (int64_t)p.thin.size() - to, (int)l);
    int64_t ro = (int64_t)rows.size();
    for (int64_t s : S) {
      const int m = h->height[s], w = h->width[s];
      const bool kids = h->kid_ptr[s + 1] > h->kid_ptr[s];
      if (thin(s) || (!kids && m == w)) continue;
      for (int i0 = kids ? 0 : w; i0 < m; i0 += 64) {
        const int i1 = std::min(m, i0 + 64);
        rows.push_back({(int32_t)s, i0, i1, child_ranges(h, s, i0, i1, p.ranges)});
      }
    }
    push(fwd, K_SOLVE_ASSEMBLE, ro, (int64_t)rows.size() - ro, (int)l);
    // blocks of SB columns: y = Dinv x (a GEMM with the block's inverse), then the front rows
    // below the block -= L(rows, block) y
    int K = 0;
    for (int64_t s : S)
      if (!thin(s)) K = std::max(K, (h->width[s] + fc::SB - 1) / fc::SB);
    for (int k = 0; k < K; ++k) {
      int64_t go = (int64_t)gemm.size();
      for (int64_t s : S) {
        const int w = h->width[s];
        const int64_t f = h->first[s];
        if (thin(s) || k * fc::SB >= w) continue;
        int bw;
        const int64_t base = inv_block(h, s, k, bw);
        const int c0 = k * fc::SB;
        for (int i0 = 0; i0 < bw; i0 += 64)
          for (int j0 = 0; j0 < R; j0 += 64) {
            fc::GemmTask g{};
            g.C = x2 + (f + c0 + i0) * R + j0;
            g.c_si = R, g.c_sj = 1;
            g.A = h->d_Dinv.as<double>() + base + i0;
            g.a_si = 1, g.a_sk = bw;
            g.B = x + (f + c0) * R + j0;
            g.b_sj = 1, g.b_sk = R;
            g.M = std::min(64, bw - i0), g.N = std::min(64, R - j0), g.K = std::min(bw, i0 + 64);
            g.flags = 4;
            sp.add(g, sizeof(double), sizeof(double), j0 == 0);
          }
      }
      bool cl = sp.close();
      push(fwd, K_SOLVE_FWD, go, (int64_t)gemm.size() - go, (int)l, cl ? 1 : 0);
      go = (int64_t)gemm.size();
      for (int64_t s : S) {
        const int w = h->width[s], m = h->height[s];
        const int64_t f = h->first[s];
        if (thin(s) || k * fc::SB >= w) continue;
        int bw;
        inv_block(h, s, k, bw);
        const int c0 = k * fc::SB, c1 = c0 + bw;
        for (int r0 = c1; r0 < m;) {
          const int r1 = std::min(r0 < w ? w : m, r0 + 64);
          for (int j0 = 0; j0 < R; j0 += 64) {
            fc::GemmTask g{};
            g.C = r0 < w ? x + (f + r0) * R + j0 : v + voff[s] + (int64_t)(r0 - w) * R + j0;
            g.c_si = R, g.c_sj = 1;
            g.A = Lp(h->loff[s] + r0 + (int64_t)c0 * m);
            g.a_si = 1, g.a_sk = m;
            g.B = x2 + (f + c0) * R + j0;
            g.b_sj = 1, g.b_sk = R;
            g.M = r1 - r0, g.N = std::min(64, R - j0), g.K = bw;
            sp.add(g, es, sizeof(double), j0 == 0);
          }
          r0 = r1;
        }
      }
      cl = sp.close();
      push(fwd, K_GEMM, go, (int64_t)gemm.size() - go, (int)l, cl ? 1 : 0);
    }
  }
  // backward
  for (int64_t l = (int64_t)lv.size() - 1; l >= 0; --l) {
    const auto &S = lv[l];
    const int64_t tb = (int64_t)p.tbwd.size();
    int64_t tpat = 0;
    int32_t tcnt = 0;
    for (int64_t s : S) {
      if (!thin(s)) continue;
      const int u = h->height[s] - h->width[s];
      const int chunks = u > fc::THIN_CHUNK ? (u + fc::THIN_CHUNK - 1) / fc::THIN_CHUNK : 1;
      for (int j0 = 0; j0 < R; j0 += RP) {
        for (int q = 0; q < chunks; ++q)
          p.tbwd.push_back({(int32_t)s, q * fc::THIN_CHUNK, std::min(u, (q + 1) * fc::THIN_CHUNK), j0, chunks, q,
                            chunks > 1 ? tcnt : -1, 0, h->ioff[s], chunks > 1 ? tpat : 0});
        if (chunks > 1) {
          tpat += (int64_t)chunks * fc::SOLVE_THIN * 64;
          ++tcnt;
        }
      }
    }
    push(bwd, K_SOLVE_THIN_BWD, tb, (int64_t)p.tbwd.size() - tb, (int)l);
    // own rows -= L21^T x(rows past the columns): the GEMM reads those rows of x through the
    // supernode's row list (final by now: they belong to supernodes of higher levels)
    int64_t go = (int64_t)gemm.size();
    for (int64_t s : S) {
      const int m = h->height[s], w = h->width[s], u = m - w;
      if (u <= 0 || thin(s)) continue;
      const int64_t lo = h->loff[s];
      for (int i0 = 0; i0 < w; i0 += fc::GEMM_TM)
        for (int j0 = 0; j0 < R; j0 += fc::GEMM_TN) {
          fc::GemmTask g{};
          g.C = x2 + (h->first[s] + i0) * (int64_t)R + j0;
          g.c_si = R, g.c_sj = 1;
          g.A = Lp(lo + w + (int64_t)i0 * m);
          g.a_si = m, g.a_sk = 1;
          g.B = x + j0;
          g.b_sj = 1, g.b_sk = R;
          g.b_rows = (h->ldlt ? h->d_lsrows : h->d_rows).as<int32_t>() + h->rows_off[s] + w;
          g.flags = 16;
          g.M = std::min(fc::GEMM_TM, w - i0), g.N = std::min(fc::GEMM_TN, R - j0), g.K = u;
          sp.add(g, es, sizeof(double), j0 == 0);
        }
    }
    bool cl = sp.close();
    push(bwd, K_GEMM, go, (int64_t)gemm.size() - go, (int)l, cl ? 1 : 0);
    // blocks of SB columns from the last: z = Dinv^T x2 (into x), then the own rows above the
    // block -= L(block, rows)^T z
    int K = 0;
    for (int64_t s : S)
      if (!thin(s)) K = std::max(K, (h->width[s] + fc::SB - 1) / fc::SB);
    for (int k = K - 1; k >= 0; --k) {
      int64_t go = (int64_t)gemm.size();
      for (int64_t s : S) {
        const int w = h->width[s];
        const int64_t f = h->first[s];
        if (thin(s) || k * fc::SB >= w) continue;
        int bw;
        const int64_t base = inv_block(h, s, k, bw);
        const int c0 = k * fc::SB;
        for (int i0 = 0; i0 < bw; i0 += 64)
          for (int j0 = 0; j0 < R; j0 += 64) {
            fc::GemmTask g{};
            g.C = x + (f + c0 + i0) * R + j0;
            g.c_si = R, g.c_sj = 1;
            g.A = h->d_Dinv.as<double>() + base + i0 + (int64_t)i0 * bw;
            g.a_si = bw, g.a_sk = 1;
            g.B = x2 + (f + c0 + i0) * R + j0;
            g.b_sj = 1, g.b_sk = R;
            g.M = std::min(64, bw - i0), g.N = std::min(64, R - j0), g.K = bw - i0;
            g.flags = 4;
            sp.add(g, sizeof(double), sizeof(double), j0 == 0);
          }
      }
      cl = sp.close();
      push(bwd, K_SOLVE_BWD, go, (int64_t)gemm.size() - go, (int)l, cl ? 1 : 0);
      go = (int64_t)gemm.size();
      for (int64_t s : S) {
        const int w = h->width[s], m = h->height[s];
        const int64_t f = h->first[s];
        if (thin(s) || k * fc::SB >= w || k == 0) continue;
        int bw;
        inv_block(h, s, k, bw);
        const int c0 = k * fc::SB;
        for (int r0 = 0; r0 < c0; r0 += 64)
          for (int j0 = 0; j0 < R; j0 += 64) {
            fc::GemmTask g{};
            g.C = x2 + (f + r0) * R + j0;
            g.c_si = R, g.c_sj = 1;
            g.A = Lp(h->loff[s] + c0 + (int64_t)r0 * m);
            g.a_si = m, g.a_sk = 1;
            g.B = x + (f + c0) * R + j0;
            g.b_sj = 1, g.b_sk = R;
            g.M = std::min(64, c0 - r0), g.N = std::min(64, R - j0), g.K = bw;
            sp.add(g, es, sizeof(double), j0 == 0);
          }
      }
      cl = sp.close();
      if ((int64_t)gemm.size() > go) push(bwd, K_GEMM, go, (int64_t)gemm.size() - go, (int)l, cl ? 1 : 0);
    }
  }
}


// The solve as two task lists, forward and backward, for the persistent kernel. Supernodes with
// at most NODE_ROWS front rows are one task per direction (and block of 64 right-hand sides);
// larger ones are split in chunks of 64 front rows. Per chunk and block of right-hand sides a
// counter counts the updates the chunk has taken, in the order the level-by-level launches apply
// them: forward, its assembly (if any) then one per earlier panel; backward, its product with the
// rows past the columns (if any) then one per later panel. A task waits for the counts its inputs
// must have reached, so every entry sees the same operations in the same order on every run.
// FIN(s) counts the final update vectors of s (the parent assembles them), DONE(s) the solved
// panels of s (the children's backward products read them). Update vectors and split-product
// partials get space of their own: levels overlap here.
constexpr int NODE_ROWS = 512;
constexpr int ASSEMBLE_GROUP = 4;  // chunks per assembly task of a large supernode
constexpr int PANEL_GROUP = 4;     // chunks per panel task past the first chunk

struct DagPlan {
  std::vector<fc::DagTask> fwd, bwd;
  std::vector<fc::DagDep> deps;
  std::vector<fc::DagChild> children;
  std::vector<int64_t> voff;
  int64_t vsum = 0, psum = 0, counters = 0;
};

void dag_plan(const fc_chol *h, int R, bool plant, DagPlan &p) {
  const int NB = fc::NB;
  const int J = (R + 63) / 64;
  const int64_t ns = h->ns;
  std::vector<std::vector<int64_t>> lv(h->levels);
  for (int64_t s = 0; s < ns; ++s) lv[h->level[s]].push_back(s);
  std::vector<int64_t> parent(ns, -1), cbase(ns + 1, 0);
  for (int64_t s = 0; s < ns; ++s)
    for (int64_t q = h->kid_ptr[s]; q < h->kid_ptr[s + 1]; ++q) parent[h->kids[q]] = s;
  auto panels = [&](int64_t s) { return (h->width[s] + NB - 1) / NB; };
  auto below = [&](int64_t s) { return (h->height[s] - h->width[s] + 63) / 64; };
  auto whole = [&](int64_t s) { return h->height[s] <= NODE_ROWS; };
  p.voff.assign(ns, 0);
  for (int64_t s = 0; s < ns; ++s) {
    p.voff[s] = p.vsum;
    p.vsum += (int64_t)(h->height[s] - h->width[s]) * R;
    cbase[s + 1] = cbase[s] + panels(s) + below(s);
  }
  const int64_t NC = cbase[ns] * J;
  auto F = [&](int64_t s, int c, int jc) { return (int32_t)((cbase[s] + c) * J + jc); };
  auto G = [&](int64_t s, int c, int jc) { return (int32_t)(NC + (cbase[s] + c) * J + jc); };
  auto PC = [&](int64_t s, int c, int jc) { return (int32_t)(2 * NC + (cbase[s] + c) * J + jc); };
  auto Y = [&](int64_t s, int c, int jc) { return (int32_t)(3 * NC + (cbase[s] + c) * J + jc); };
  auto Z = [&](int64_t s, int c, int jc) { return (int32_t)(4 * NC + (cbase[s] + c) * J + jc); };
  auto FIN = [&](int64_t s, int jc) { return (int32_t)(5 * NC + s * J + jc); };
  auto DONE = [&](int64_t s, int jc) { return (int32_t)(5 * NC + (ns + s) * J + jc); };
  p.counters = 5 * NC + 2 * ns * J;
  auto kids = [&](int64_t s) { return h->kid_ptr[s + 1] > h->kid_ptr[s]; };
  auto assembled = [&](int64_t s, int c) { return kids(s) || c >= panels(s); };
  auto chunk = [&](int64_t s, int c, int &i0, int &i1) {
    const int P = panels(s), w = h->width[s], m = h->height[s];
    if (c < P) {
      i0 = c * 64, i1 = std::min(w, i0 + 64);
    } else {
      i0 = w + (c - P) * 64, i1 = std::min(m, i0 + 64);
    }
  };
  auto dep = [&](int32_t counter, int32_t value) {
    if (value > 0) p.deps.push_back({counter, value});
  };
  auto task = [&](int32_t kind, int64_t s, int i0, int i1, int r0, int r1, int jc) {
    fc::DagTask t{};
    t.kind = kind, t.s = (int32_t)s, t.i0 = i0, t.i1 = i1, t.r0 = r0, t.r1 = r1;
    t.j0 = jc * 64, t.j1 = std::min(R, jc * 64 + 64);
    t.dep0 = t.dep1 = (int32_t)p.deps.size();
    t.sig0 = t.sig1 = t.sigmid = -1;
    t.aux = -1;
    return t;
  };
  // the children's rows landing in front rows [i0, i1) of s
  auto children = [&](int64_t s, int i0, int i1) {
    std::vector<int2> r;
    child_ranges(h, s, i0, i1, r);
    const int32_t at = (int32_t)p.children.size();
    for (int64_t q = h->kid_ptr[s]; q < h->kid_ptr[s + 1]; ++q) {
      const int64_t c = h->kids[q];
      const int2 rg = r[q - h->kid_ptr[s]];
      p.children.push_back({h->rel_off[c], p.voff[c], rg.x, rg.y});
    }
    return at;
  };
  auto wait_children = [&](int64_t s, int jc) {
    for (int64_t q = h->kid_ptr[s]; q < h->kid_ptr[s + 1]; ++q) dep(FIN(h->kids[q], jc), below(h->kids[q]));
  };
  auto doff = [&](int64_t s, int pp) { return h->doff[s] + 2 * (int64_t)NB * NB * pp; };
  // forward
  for (size_t l = 0; l < lv.size(); ++l) {
    const auto &S = lv[l];
    for (int64_t s : S) {
      if (!whole(s)) continue;
      const int32_t rec = children(s, 0, h->height[s]);
      for (int jc = 0; jc < J; ++jc) {
        fc::DagTask t = task(fc::DAG_NODE, s, 0, h->height[s], 0, 0, jc);
        t.child = rec;
        wait_children(s, jc);
        t.dep1 = (int32_t)p.deps.size();
        if (below(s) > 0) t.sig1 = FIN(s, jc), t.inc1 = below(s);
        p.fwd.push_back(t);
      }
    }
    for (int64_t s : S) {
      if (whole(s)) continue;
      const int P = panels(s), C = P + below(s);
      for (int c = kids(s) ? 0 : P; c < C; c += ASSEMBLE_GROUP) {
        const int ce = std::min(C, c + ASSEMBLE_GROUP);
        int i0, i1, e0, e1;
        chunk(s, c, i0, e0);
        chunk(s, ce - 1, e1, i1);
        const int32_t rec = children(s, i0, i1);
        for (int jc = 0; jc < J; ++jc) {
          fc::DagTask t = task(fc::DAG_ASSEMBLE, s, i0, i1, c, ce, jc);
          t.child = rec;
          wait_children(s, jc);
          t.dep1 = (int32_t)p.deps.size();
          t.sig0 = F(s, c, jc), t.sigstep = J, t.nsig = ce - c;
          p.fwd.push_back(t);
        }
      }
    }
    int Pmax = 0;
    for (int64_t s : S)
      if (!whole(s)) Pmax = std::max(Pmax, panels(s));
    for (int pp = 0; pp < Pmax; ++pp) {
      for (int64_t s : S) {
        const int P = panels(s), C = P + below(s), m = h->height[s], w = h->width[s];
        if (whole(s) || pp >= P) continue;
        const int c0 = pp * NB, c1 = std::min(w, c0 + NB);
        const int need_p = (assembled(s, pp) ? 1 : 0) + pp;
        for (int jc = 0; jc < J; ++jc) {
          if (c1 >= m) {  // no rows below: the panel's solution only
            fc::DagTask t = task(fc::DAG_PANEL, s, c0, c1, C, C, jc);
            dep(F(s, pp, jc), need_p);
            t.dep1 = (int32_t)p.deps.size();
            t.keep = 1, t.aux = doff(s, pp);
            p.fwd.push_back(t);
            continue;
          }
          // the first chunk below applies the inverse and stores y; the others read y
          for (int c = pp + 1; c < C;) {
            const bool first = c == pp + 1;
            const int ce = first ? c + 1 : std::min(C, c + PANEL_GROUP);
            fc::DagTask t = task(fc::DAG_PANEL, s, c0, c1, c, ce, jc);
            if (first)
              dep(F(s, pp, jc), need_p);
            else
              dep(Y(s, pp, jc), 1);
            for (int q = c; q < ce; ++q) dep(F(s, q, jc), (assembled(s, q) ? 1 : 0) + pp);
            t.dep1 = (int32_t)p.deps.size();
            t.keep = first ? 1 : -1, t.aux = doff(s, pp);
            t.sigmid = first ? Y(s, pp, jc) : -1;
            t.sig0 = F(s, c, jc), t.sigstep = J;
            if (pp == P - 1) t.sig1 = FIN(s, jc), t.inc1 = ce - c;  // final update vectors
            p.fwd.push_back(t);
            c = ce;
          }
        }
      }
    }
  }
  // backward
  for (int64_t l = (int64_t)lv.size() - 1; l >= 0; --l) {
    const auto &S = lv[l];
    auto wait_parent = [&](int64_t s, int jc) {
      if (parent[s] >= 0) dep(DONE(parent[s], jc), panels(parent[s]));
    };
    for (int64_t s : S) {
      if (!whole(s)) continue;
      for (int jc = 0; jc < J; ++jc) {
        fc::DagTask t = task(fc::DAG_NODE, s, 0, h->height[s], 0, 0, jc);
        wait_parent(s, jc);
        t.dep1 = (int32_t)p.deps.size();
        t.sig1 = DONE(s, jc), t.inc1 = panels(s);
        p.bwd.push_back(t);
      }
    }
    std::vector<fc::DagTask> reduce;
    for (int64_t s : S) {
      const int u = h->height[s] - h->width[s], w = h->width[s], P = panels(s);
      if (whole(s) || u <= 0) continue;
      const bool split = u > 2 * fc::SPLIT_K;
      const int chunks = split ? (u + fc::SPLIT_K - 1) / fc::SPLIT_K : 1;
      for (int i = 0; i < P; ++i)
        for (int jc = 0; jc < J; ++jc) {
          const int i0 = 64 * i, i1 = std::min(w, i0 + 64);
          for (int q = 0; q < chunks; ++q) {
            const int k0 = split ? q * fc::SPLIT_K : 0, k1 = split ? std::min(u, k0 + fc::SPLIT_K) : u;
            fc::DagTask t = task(fc::DAG_GEMM, s, i0, i1, k0, k1, jc);
            wait_parent(s, jc);
            t.dep1 = (int32_t)p.deps.size();
            if (split)
              t.aux = p.psum + (int64_t)q * 4096, t.sig1 = PC(s, i, jc);
            else
              t.sig1 = G(s, i, jc);
            t.inc1 = 1;
            p.bwd.push_back(t);
          }
          if (split) {
            fc::DagTask t = task(fc::DAG_REDUCE, s, i0, i1, 0, 0, jc);
            t.count = chunks, t.aux = p.psum;
            t.sig1 = G(s, i, jc), t.inc1 = 1;
            reduce.push_back(t);
            p.psum += (int64_t)chunks * 4096;
          }
        }
    }
    for (fc::DagTask t : reduce) {  // after the level's products
      t.dep0 = (int32_t)p.deps.size();
      dep(PC(t.s, t.i0 / 64, t.j0 / 64), t.count);
      t.dep1 = (int32_t)p.deps.size();
      p.bwd.push_back(t);
    }
    int Pmax = 0;
    for (int64_t s : S)
      if (!whole(s)) Pmax = std::max(Pmax, panels(s));
    for (int pp = Pmax - 1; pp >= 0; --pp) {
      for (int64_t s : S) {
        const int P = panels(s), u = h->height[s] - h->width[s], w = h->width[s];
        if (whole(s) || pp >= P) continue;
        const int c0 = pp * NB, c1 = std::min(w, c0 + NB);
        const int need = (u > 0 ? 1 : 0) + (P - 1 - pp);
        for (int jc = 0; jc < J; ++jc) {
          if (c0 == 0) {
            fc::DagTask t = task(fc::DAG_PANEL, s, c0, c1, 0, 0, jc);
            dep(G(s, pp, jc), need);
            t.dep1 = (int32_t)p.deps.size();
            t.keep = 1, t.aux = doff(s, pp);
            t.sig1 = DONE(s, jc), t.inc1 = 1;
            p.bwd.push_back(t);
            continue;
          }
          // the chunk just above (the next panel to solve) applies the inverse and stores z; the
          // chunks further up read z
          {
            fc::DagTask t = task(fc::DAG_PANEL, s, c0, c1, pp - 1, pp, jc);
            dep(G(s, pp, jc), need);
            dep(G(s, pp - 1, jc), need);
            t.dep1 = (int32_t)p.deps.size();
            t.keep = 1, t.aux = doff(s, pp);
            t.sigmid = Z(s, pp, jc);
            t.sig0 = G(s, pp - 1, jc), t.sigstep = J;
            t.sig1 = DONE(s, jc), t.inc1 = 1;
            p.bwd.push_back(t);
          }
          for (int r = 0; r < pp - 1; r += PANEL_GROUP) {
            const int re = std::min(pp - 1, r + PANEL_GROUP);
            fc::DagTask t = task(fc::DAG_PANEL, s, c0, c1, r, re, jc);
            dep(Z(s, pp, jc), 1);
            for (int q = r; q < re; ++q) dep(G(s, q, jc), need);
            t.dep1 = (int32_t)p.deps.size();
            t.keep = -1, t.aux = doff(s, pp);
            t.sig0 = G(s, r, jc), t.sigstep = J;
            p.bwd.push_back(t);
          }
        }
      }
    }
  }
  if (plant && !p.fwd.empty()) {  // the last forward task also waits for a count nothing reaches
    fc::DagTask &t = p.fwd.back();
    std::vector<fc::DagDep> extra(p.deps.begin() + t.dep0, p.deps.begin() + t.dep1);
    extra.push_back({0, INT32_MAX});
    t.dep0 = (int32_t)p.deps.size();
    p.deps.insert(p.deps.end(), extra.begin(), extra.end());
    t.dep1 = (int32_t)p.deps.size();
  }
}

// Runs the lists in order on the host's counters (one CTA taking every task in turn): every wait
// must be met by earlier tasks, and every counter index must be in range. Each counter is raised
// either by a chain of tasks that each wait for the count before their own, or by tasks whose
// waiter needs all of them, so a count is never reached early with more CTAs.
bool check_dag(const DagPlan &p, std::string &why) {
  std::vector<int32_t> cnt((size_t)p.counters, 0);
  int64_t id = 0;
  for (const auto *list : {&p.fwd, &p.bwd}) {
    for (const fc::DagTask &t : *list) {
      if (t.dep0 < 0 || t.dep1 < t.dep0 || t.dep1 > (int64_t)p.deps.size()) {
        why = "task " + std::to_string(id) + ": dependency range";
        return false;
      }
      for (int32_t e = t.dep0; e < t.dep1; ++e) {
        const fc::DagDep d = p.deps[e];
        if (d.counter < 0 || d.counter >= p.counters || cnt[d.counter] < d.value) {
          why = "task " + std::to_string(id) + " waits for a count no earlier task reaches";
          return false;
        }
      }
      std::vector<std::pair<int64_t, int32_t>> raised;
      const int nsig = t.kind == fc::DAG_PANEL ? t.r1 - t.r0 : t.nsig;
      if (t.sig0 >= 0)
        for (int k = 0; k < nsig; ++k) raised.push_back({(int64_t)t.sig0 + (int64_t)k * t.sigstep, 1});
      if (t.sig1 >= 0) raised.push_back({t.sig1, t.inc1});
      if (t.sigmid >= 0) raised.push_back({t.sigmid, 1});
      for (const auto &r : raised) {
        if (r.first < 0 || r.first >= p.counters) {
          why = "task " + std::to_string(id) + ": counter out of range";
          return false;
        }
        cnt[r.first] += r.second;
      }
      ++id;
    }
  }
  return true;
}

int plan_solve_dag(fc_chol *h, int R, fc_status *st) {
  DagPlan p;
  dag_plan(h, R, h->dag_plant, p);
  std::string why;
  if (!h->dag_plant && !check_dag(p, why)) {
    set_status(st, FC_INTERNAL, -1, 0, 0, "solve plan: " + why);
    return FC_INTERNAL;
  }
  h->dag_plant = false;
  if (p.counters >= INT32_MAX || p.deps.size() >= (size_t)INT32_MAX || p.fwd.size() >= (size_t)INT32_MAX ||
      p.bwd.size() >= (size_t)INT32_MAX) {
    set_status(st, FC_INTERNAL, -1, 0, 0, "solve plan too large");
    return FC_INTERNAL;
  }
  if (h->d_x.alloc(sizeof(double) * (size_t)std::max<int64_t>(h->n * R, 1)) != cudaSuccess ||
      h->d_x2.alloc(sizeof(double) * (size_t)std::max<int64_t>(h->n * R, 1)) != cudaSuccess ||
      h->d_v.alloc(sizeof(double) * (size_t)std::max<int64_t>(p.vsum, 1)) != cudaSuccess ||
      h->d_part.alloc(sizeof(double) * (size_t)std::max<int64_t>(p.psum, 1)) != cudaSuccess ||
      h->d_dcount.alloc(sizeof(int32_t) * (size_t)std::max<int64_t>(p.counters, 1)) != cudaSuccess ||
      h->d_dctl.alloc(sizeof(fc::DagControl)) != cudaSuccess) {
    h->solve_R = 0;
    set_status(st, FC_OUT_OF_MEMORY, -1, h->entries, 0, "device memory for the solve");
    return FC_OUT_OF_MEMORY;
  }
  std::vector<fc::DagTask> all(p.fwd);
  all.insert(all.end(), p.bwd.begin(), p.bwd.end());
  cudaError_t e;
  if ((e = upload(h->d_voff, p.voff, h->stream)) != cudaSuccess || (e = upload(h->d_dtasks, all, h->stream)) != cudaSuccess ||
      (e = upload(h->d_ddeps, p.deps, h->stream)) != cudaSuccess ||
      (e = upload(h->d_dranges, p.children, h->stream)) != cudaSuccess)
    return cuda_fail(st, e, "solve plan");
  if ((e = cudaMemsetAsync(h->d_dctl.p, 0, sizeof(fc::DagControl), h->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(h->stream)) != cudaSuccess)
    return cuda_fail(st, e, "solve plan");
  if (h->dag_trace && h->d_dtrace.alloc(sizeof(long long) * 4 * std::max<size_t>(all.size(), 1)) != cudaSuccess) {
    set_status(st, FC_OUT_OF_MEMORY, -1, h->entries, 0, "device memory for the solve trace");
    return FC_OUT_OF_MEMORY;
  }
  h->dag_fwd = (int64_t)p.fwd.size();
  h->dag_bwd = (int64_t)p.bwd.size();
  h->dag_counters = p.counters;
  h->dag_grid = prop_sms(h->device) * fc::solve_dag_blocks_per_sm(h->fp32);
  h->gemm_flops_solve = 0;
  h->solve_R = R;
  return FC_OK;
}

// The launch record of one direction of the persistent solve.
fc::SolveDag solve_dag(fc_chol *h, bool backward, int R) {
  fc::SolveDag d{};
  d.tasks = h->d_dtasks.as<fc::DagTask>() + (backward ? h->dag_fwd : 0);
  d.count = (int32_t)(backward ? h->dag_bwd : h->dag_fwd);
  d.deps = h->d_ddeps.as<fc::DagDep>();
  d.counters = h->d_dcount.as<int32_t>();
  d.ctl = h->d_dctl.as<fc::DagControl>();
  d.x = h->d_x.as<double>();
  d.x2 = h->d_x2.as<double>();
  d.v = h->d_v.as<double>();
  d.part = h->d_part.as<double>();
  d.voff = h->d_voff.as<int64_t>();
  d.children = h->d_dranges.as<fc::DagChild>();
  d.R = R;
  d.limit_ns = h->dag_limit_ns;
  d.trace = h->dag_trace ? h->d_dtrace.as<long long>() + (backward ? 4 * h->dag_fwd : 0) : nullptr;
  return d;
}

// FC_TIMEOUT when the last persistent solve gave up on a wait (after the stream is idle).
int solve_wait_status(fc_chol *h, fc_status *st) {
  if (!h->dag || !h->d_dctl.p) return FC_OK;
  fc::DagControl c{};
  cudaError_t e = cudaMemcpy(&c, h->d_dctl.p, sizeof(c), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(st, e, "solve status");
  if (c.error) {
    h->solve_R = 0;  // the next solve plans (and captures) afresh
    if (h->solve_graph) {
      cudaGraphExecDestroy(h->solve_graph);
      h->solve_graph = nullptr;
    }
    set_status(st, FC_TIMEOUT, -1, 0, 0, "a wait of the solve ran past its limit (task " + std::to_string(c.task) + ")");
    return FC_TIMEOUT;
  }
  return FC_OK;
}

// The handle's own solve buffers and task arrays for R right-hand sides (built once per R).
std::vector<char> beside(const std::vector<Launch> &prog);

// Events the two-stream solve uses: a fork and a join per level with a thin launch beside wide ones.
size_t solve_events_needed(const fc_chol *h) {
  size_t n = 0;
  for (const auto *prog : {&h->fwd, &h->bwd})
    for (char c : beside(*prog)) n += c ? 2 : 0;
  return n;
}

int plan_solve(fc_chol *h, int R, fc_status *st) {
  if (h->solve_R == R) return FC_OK;
  if (h->solve_graph) {
    cudaGraphExecDestroy(h->solve_graph);
    h->solve_graph = nullptr;
  }
  if (h->dag) return plan_solve_dag(h, R, st);
  SolvePlan p;
  solve_offsets(h, R, p);
  cudaError_t e;
  if (h->d_x.alloc(sizeof(double) * (size_t)std::max<int64_t>(h->n * R, 1)) != cudaSuccess ||
      h->d_x2.alloc(sizeof(double) * (size_t)std::max<int64_t>(h->n * R, 1)) != cudaSuccess ||
      h->d_v.alloc(sizeof(double) * (size_t)std::max<int64_t>(p.vsum, 1)) != cudaSuccess) {
    h->solve_R = 0;
    set_status(st, FC_OUT_OF_MEMORY, -1, h->entries, 0, "device memory for the solve");
    return FC_OUT_OF_MEMORY;
  }
  if ((e = upload(h->d_voff, p.voff, h->stream)) != cudaSuccess) return cuda_fail(st, e, "solve plan");
  solve_tasks(h, R, h->d_x.as<double>(), h->d_x2.as<double>(), h->d_v.as<double>(), p);
  if (h->d_part.alloc(sizeof(double) * (size_t)std::max<int64_t>(p.psum, 1)) != cudaSuccess ||
      h->d_tpart.alloc(sizeof(double) * (size_t)std::max<int64_t>(p.tpart, 1)) != cudaSuccess ||
      h->d_tcount.alloc(sizeof(int32_t) * (size_t)std::max<int64_t>(p.tcount + p.scount, 1)) != cudaSuccess) {
    h->solve_R = 0;
    set_status(st, FC_OUT_OF_MEMORY, -1, h->entries, 0, "device memory for the solve");
    return FC_OUT_OF_MEMORY;
  }
  h->fwd = std::move(p.fwd);
  h->bwd = std::move(p.bwd);
  h->gemm_flops_solve = 0;
  for (const auto &g : p.gemm) h->gemm_flops_solve += task_flops(g);
  if ((e = upload(h->d_srow, p.rows, h->stream)) != cudaSuccess || (e = upload(h->d_sranges, p.ranges, h->stream)) != cudaSuccess ||
      (e = upload(h->d_spanel, p.panels, h->stream)) != cudaSuccess ||
      (e = upload(h->d_sgemm, p.gemm, h->stream)) != cudaSuccess || (e = upload(h->d_thin, p.thin, h->stream)) != cudaSuccess ||
      (e = upload(h->d_tranges, p.tranges, h->stream)) != cudaSuccess ||
      (e = upload(h->d_tbwd, p.tbwd, h->stream)) != cudaSuccess)
    return cuda_fail(st, e, "solve plan");
  if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_fail(st, e, "solve plan");
  h->solve_lg = p.lg;
  h->solve_tcount = p.tcount + p.scount;
  while (h->solve_events.size() < solve_events_needed(h)) {
    cudaEvent_t ev;
    if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return cuda_fail(st, e, "solve events");
    h->solve_events.push_back(ev);
  }
  h->solve_R = R;
  return FC_OK;
}

// The device buffers a solve program runs on.
struct SolveBuffers {
  double *x, *x2, *v;
  const int64_t *voff;
  const fc::RowTask *rows;
  const int2 *ranges;
  const fc::SolveTask *panels;
  const fc::GemmTask *gemm;
  double *part;
  const fc::ThinTask *thin;
  const int4 *tranges;
  const fc::ThinBwdTask *tbwd;
  double *tpart;
  int32_t *tcount;
  int lg;
};

SolveBuffers own_buffers(fc_chol *h) {
  return {h->d_x.as<double>(),         h->d_x2.as<double>(),           h->d_v.as<double>(),
          h->d_voff.as<int64_t>(),       h->d_srow.as<fc::RowTask>(),    h->d_sranges.as<int2>(),
          h->d_spanel.as<fc::SolveTask>(), h->d_sgemm.as<fc::GemmTask>(), h->d_part.as<double>(),
          h->d_thin.as<fc::ThinTask>(),  h->d_tranges.as<int4>(),        h->d_tbwd.as<fc::ThinBwdTask>(),
          h->d_tpart.as<double>(),       h->d_tcount.as<int32_t>(),      h->solve_lg};
}

// Whether each launch of a solve program is the thin launch of a level that also has wide ones
// (then it can run beside them).
std::vector<char> beside(const std::vector<Launch> &prog) {
  std::vector<char> out(prog.size(), 0);
  for (size_t a = 0; a < prog.size();) {
    size_t b = a;
    bool thin = false, wide = false;
    for (; b < prog.size() && prog[b].level == prog[a].level; ++b) {
      const bool t = prog[b].kind == K_SOLVE_THIN_FWD || prog[b].kind == K_SOLVE_THIN_BWD;
      thin |= t;
      wide |= !t;
    }
    if (thin && wide)
      for (size_t q = a; q < b; ++q)
        out[q] = prog[q].kind == K_SOLVE_THIN_FWD || prog[q].kind == K_SOLVE_THIN_BWD;
    a = b;
  }
  return out;
}

// With `events` (two per level that has both a thin and a wide launch, from *ev on), such a
// level's thin launch runs on the side stream beside its wide launches: the side stream forks
// from the main one at the level's start and joins it at the level's end (the next level reads
// what both wrote). Other levels stay on the main stream.
void run_solve_program(fc_chol *h, const std::vector<Launch> &prog, const SolveBuffers &b, int R, int64_t &launches,
                       const std::vector<cudaEvent_t> *events = nullptr, size_t *ev = nullptr) {
  const cudaStream_t main = h->stream;
  const fc::Tree &t = h->ldlt ? h->stree : h->tree;
  const bool narrow = h->solve_narrow && R <= 16;  // every task's N is R then
  // with few right-hand sides, a launch of fewer CTAs than two per SM: each CTA walks its K with
  // the deeper ring (with 64-column tiles the ring's shared memory would leave one CTA an SM,
  // and the measured solve was slower)
  const int short_launch = h->solve_deep && narrow ? 2 * prop_sms(h->device) : 0;
  const bool lanes = events && ev && h->side;
  const std::vector<char> side = lanes ? beside(prog) : std::vector<char>(prog.size(), 0);
  // (option) every launch of the program as a programmatic dependent of its stream's previous
  // kernel: its CTAs are scheduled while that kernel finishes and load their task, L and inverse
  // tiles before waiting for it (the program's first kernel follows the ordinary permutation
  // launch, which starts only after everything before the solve is done)
  const bool pdl = h->solve_pdl;
  bool forked = false;
  int level = INT_MIN;
  for (size_t q = 0; q < prog.size(); ++q) {
    const Launch &l = prog[q];
    if (l.level != level) {
      if (forked) {  // the previous level's join
        cudaEventRecord((*events)[*ev], h->side);
        cudaStreamWaitEvent(main, (*events)[(*ev)++], 0);
        forked = false;
      }
      level = l.level;
    }
    if (side[q] && !forked) {
      cudaEventRecord((*events)[*ev], main);
      cudaStreamWaitEvent(h->side, (*events)[(*ev)++], 0);
      forked = true;
    }
    const cudaStream_t st = side[q] ? h->side : main;
    Mark mark(h, l.kind + 16, l.level, l.count);
    switch (l.kind) {
      case K_SOLVE_ASSEMBLE:
        fc::launch_solve_assemble(t, b.x, b.v, b.voff, R, b.rows + l.off, b.ranges, l.count, st, pdl);
        break;
      case K_SOLVE_FWD:  // the diagonal blocks' inverses applied (FP64 throughout)
      case K_SOLVE_BWD:
        if (l.width == 1)
          fc::launch_gemm_cluster(b.gemm + l.off, l.count, false, st, b.part, b.tcount);
        else if (l.count < short_launch)
          fc::launch_gemm_solve(b.gemm + l.off, l.count, false, R, st, b.part, b.tcount, pdl);
        else if (narrow)
          fc::launch_gemm_narrow(b.gemm + l.off, l.count, false, R, st, b.part, b.tcount, pdl);
        else
          fc::launch_gemm_pdl(b.gemm + l.off, l.count, false, st, b.part, b.tcount, pdl);
        break;
      case K_GEMM:
        if (l.width == 1)
          fc::launch_gemm_cluster(b.gemm + l.off, l.count, h->fp32, st, b.part, b.tcount);
        else if (l.count < short_launch)
          fc::launch_gemm_solve(b.gemm + l.off, l.count, h->fp32, R, st, b.part, b.tcount, pdl);
        else if (narrow)
          fc::launch_gemm_narrow(b.gemm + l.off, l.count, h->fp32, R, st, b.part, b.tcount, pdl);
        else
          fc::launch_gemm_pdl(b.gemm + l.off, l.count, h->fp32, st, b.part, b.tcount, pdl);
        break;
      case K_SOLVE_THIN_FWD:
        fc::launch_thin_fwd(t, h->fp32, b.x, b.x2, b.v, b.voff, R, b.lg, b.thin + l.off, b.tranges, l.count, st, pdl);
        break;
      case K_SOLVE_THIN_BWD:
        fc::launch_thin_bwd(t, h->fp32, b.x, b.x2, R, b.lg, b.tbwd + l.off, b.tpart, b.tcount, l.count, st, pdl);
        break;
    }
    ++launches;
  }
  if (forked) {
    cudaEventRecord((*events)[*ev], h->side);
    cudaStreamWaitEvent(main, (*events)[(*ev)++], 0);
  }
}

void enqueue_solve_direct(fc_chol *h, double *d_b, int R, int64_t ld);

// Solves for the R right-hand sides in device memory at d_b (column-major, leading dimension ld),
// as a replayed graph when it can.
int enqueue_solve(fc_chol *h, double *d_b, int R, int64_t ld, fc_status *st) {
  if (h->ldlt) {
    const int rc = ldlt_prepare_solve(h, st);
    if (rc != FC_OK) return rc;
  }
  const int before = h->solve_R;
  int rc = plan_solve(h, R, st);
  if (rc != FC_OK) return rc;
  if (h->profiling || !h->graphs) {
    enqueue_solve_direct(h, d_b, R, ld);
    return FC_OK;
  }
  if (!h->solve_graph || before != R || h->solve_graph_b != d_b || h->solve_graph_R != R || h->solve_graph_ld != ld ||
      h->solve_graph_stream != h->stream) {
    if (!capture(h, &h->solve_graph, [&] { enqueue_solve_direct(h, d_b, R, ld); })) {
      h->graphs = false;
      enqueue_solve_direct(h, d_b, R, ld);
      return FC_OK;
    }
    h->solve_graph_b = d_b;
    h->solve_graph_R = R;
    h->solve_graph_ld = ld;
    h->solve_graph_stream = h->stream;
  }
  cudaGraphLaunch(h->solve_graph, h->stream);
  h->last_solve_launches = h->dag ? 4 : (int64_t)(h->fwd.size() + h->bwd.size() + 2);
  return FC_OK;
}

void enqueue_solve_direct(fc_chol *h, double *d_b, int R, int64_t ld) {
  int64_t launches = 0;
  if (h->dag && !h->ldlt) {
    cudaMemsetAsync(h->d_dcount.p, 0, sizeof(int32_t) * (size_t)h->dag_counters, h->stream);
    cudaMemsetAsync(h->d_dctl.p, 0, sizeof(fc::DagControl), h->stream);
    fc::launch_permute_in(h->d_perm.as<int64_t>(), h->n, d_b, ld, h->d_x.as<double>(), R, h->tree.scale, h->stream);
    {
      Mark mark(h, K_SOLVE_DAG_FWD + 16, -1, (int)h->dag_fwd);
      fc::launch_solve_dag(h->tree, h->fp32, false, solve_dag(h, false, R), h->dag_grid, h->stream);
    }
    {
      Mark mark(h, K_SOLVE_DAG_BWD + 16, -1, (int)h->dag_bwd);
      fc::launch_solve_dag(h->tree, h->fp32, true, solve_dag(h, true, R), h->dag_grid, h->stream);
    }
    fc::launch_permute_out(h->d_perm.as<int64_t>(), h->n, h->d_x.as<double>(), R, d_b, ld, h->tree.scale, h->stream);
    h->last_solve_launches = 4;
    return;
  }
  const SolveBuffers b = own_buffers(h);
  // the thin backward chunks' counters start at zero (their last chunk also leaves them so)
  cudaMemsetAsync(h->d_tcount.p, 0, sizeof(int32_t) * (size_t)std::max<int64_t>(h->solve_tcount, 1), h->stream);
  // the LDL^T factor's solve permutes through its folded order and applies D^-1 between the passes
  const int64_t *perm = h->ldlt ? h->d_lsperm.as<int64_t>() : h->d_perm.as<int64_t>();
  fc::launch_permute_in(perm, h->n, d_b, ld, h->d_x.as<double>(), R, h->tree.scale, h->stream);
  // the thin launches beside the wide ones (not while profiling: then every launch is timed alone)
  const bool lanes = h->side && !h->profiling && h->solve_events.size() >= solve_events_needed(h);
  size_t ev = 0;
  run_solve_program(h, h->fwd, b, R, launches, lanes ? &h->solve_events : nullptr, &ev);
  if (h->ldlt) {
    fc::ldlt::launch_d_inverse(h->n, R, h->d_ldd.as<double>(), h->d_lde.as<double>(), h->d_lpivots.as<int8_t>(), b.x2,
                               h->stream);
    ++launches;
  }
  run_solve_program(h, h->bwd, b, R, launches, lanes ? &h->solve_events : nullptr, &ev);
  fc::launch_permute_out(perm, h->n, h->d_x.as<double>(), R, d_b, ld, h->tree.scale, h->stream);
  h->last_solve_launches = launches + 2;
}

}  // namespace

// Scratch of fc_chol_solve_device_noalloc: the solve's vectors and task lists for callers that
// cannot allocate device memory. A file-scope device array, so loading the library reserves it
// on every device the process uses, until exit. Host code may not use its name as an address;
// the address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char fc_noalloc_scratch[FC_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex noalloc_setup_lock;
constexpr int NOALLOC_DEVICES = 64;
unsigned char *noalloc_base[NOALLOC_DEVICES] = {};

// The scratch's device address on the current device (set up on the first call there).
cudaError_t noalloc_scratch(int device, unsigned char **base) {
  if (device < 0 || device >= NOALLOC_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(noalloc_setup_lock);
  if (!noalloc_base[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, fc_noalloc_scratch);
    if (e != cudaSuccess) return e;
    noalloc_base[device] = static_cast<unsigned char *>(p);
  }
  *base = noalloc_base[device];
  return cudaSuccess;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" {

const char *fc_version(void) { return "fieldcraft-b200 0.1.0 (sm_100a)"; }

// Not part of the public ABI: the LDL^T solve's structure folding (host/ldlt_fold.cpp) on a
// caller's arrays, for tests. Outputs: perm_out[n], rows_out[rptr[ns]], from_out (the rows-below
// count), rel_out (the same count less the roots'). Returns 0, or -1 on inconsistent input.
int fc_test_ldlt_fold(int64_t n, int64_t ns, const int64_t *first, const int64_t *rptr, const int32_t *rows,
                      const int64_t *perm, const int64_t *sparent, const int32_t *order, int64_t *perm_out,
                      int32_t *rows_out, int32_t *from_out, int32_t *rel_out) {
  fc::LdltFold f;
  if (!fc::ldlt_fold(n, ns, first, rptr, rows, perm, sparent, order, f)) return -1;
  std::copy(f.perm.begin(), f.perm.end(), perm_out);
  std::copy(f.rows.begin(), f.rows.end(), rows_out);
  std::copy(f.from.begin(), f.from.end(), from_out);
  std::copy(f.rel.begin(), f.rel.end(), rel_out);
  return 0;
}

int fc_symbolic_analyse(int64_t n, const int64_t *ptr, const int32_t *idx, uint64_t max_entries, fc_symbolic **out,
                        fc_status *status) {
  if (!out || n < 0 || (n > 0 && (!ptr || !idx))) {
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "null or negative argument");
    return FC_INVALID_ARGUMENT;
  }
  *out = nullptr;
  std::vector<int64_t> zero_ptr(1, 0);
  fc::UpperPattern a{n, n > 0 ? ptr : zero_ptr.data(), idx};
  try {
    auto s = new fc_symbolic();
    Failure f;
    if (!fc::analyse(a, max_entries, s->s, f)) {
      delete s;
      return fail_status(status, f);
    }
    *out = s;
  } catch (const std::bad_alloc &) {
    set_status(status, FC_OUT_OF_MEMORY, -1, 0, 0, "host memory for the analysis");
    return FC_OUT_OF_MEMORY;
  }
  set_status(status, FC_OK);
  return FC_OK;
}

int fc_chol_batch_analyse(int32_t count, const int64_t *n, const int64_t *const *ptr, const int32_t *const *idx,
                          uint64_t max_entries, fc_symbolic **out, int64_t *offsets, fc_status *status) {
  if (!out || count < 0 || (count > 0 && (!n || !ptr || !idx || !offsets))) {
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "null or negative argument");
    return FC_INVALID_ARGUMENT;
  }
  *out = nullptr;
  try {
    // diag(A_0, A_1, ...) by columns: each system's columns shifted by its first unknown
    std::vector<int64_t> bptr(1, 0);
    std::vector<int32_t> bidx;
    int64_t at = 0;
    for (int32_t b = 0; b < count; ++b) {
      if (n[b] < 0 || (n[b] > 0 && (!ptr[b] || !idx[b]))) {
        set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "system " + std::to_string(b) + ": bad pattern");
        return FC_INVALID_ARGUMENT;
      }
      offsets[b] = at;
      if (at + n[b] > INT32_MAX) {
        set_status(status, FC_TOO_LARGE, -1, 0, 0, "the batch has more than 2^31 unknowns");
        return FC_TOO_LARGE;
      }
      for (int64_t k = 0; k < n[b]; ++k) {
        for (int64_t q = ptr[b][k]; q < ptr[b][k + 1]; ++q) bidx.push_back((int32_t)(idx[b][q] + at));
        bptr.push_back((int64_t)bidx.size());
      }
      at += n[b];
    }
    if (count > 0) offsets[count] = at;
    return fc_symbolic_analyse(at, bptr.data(), bidx.data(), max_entries, out, status);
  } catch (const std::bad_alloc &) {
    set_status(status, FC_OUT_OF_MEMORY, -1, 0, 0, "host memory for the batch's analysis");
    return FC_OUT_OF_MEMORY;
  }
}

int fc_chol_batch_locate(int32_t count, const int64_t *offsets, int64_t column, int32_t *system, int64_t *local) {
  if (count < 1 || !offsets || !system || !local || column < 0 || column >= offsets[count]) return FC_INVALID_ARGUMENT;
  const int64_t *hit = std::upper_bound(offsets, offsets + count + 1, column) - 1;
  *system = (int32_t)(hit - offsets);
  *local = column - *hit;
  return FC_OK;
}

void fc_symbolic_free(fc_symbolic *sym) { delete sym; }

int fc_symbolic_get(const fc_symbolic *sym, fc_symbolic_arrays *o) {
  if (!sym || !o) return FC_INVALID_ARGUMENT;
  const fc::Symbolic &s = sym->s;
  o->n = s.n;
  o->ns = s.ns;
  o->entries = s.entries;
  o->nnz = (int64_t)s.upper_idx.size();
  o->rows_len = (int64_t)s.rows.size();
  o->lower_len = (int64_t)s.lidx.size();
  o->updates_len = (int64_t)s.uk.size();
  o->tasks_len = (int64_t)s.task_lo.size();
  o->top_len = (int64_t)s.top.size();
  o->perm = s.perm.data();
  o->first = s.first.data();
  o->rptr = s.rptr.data();
  o->rows = s.rows.data();
  o->upper_ptr = s.upper_ptr.data();
  o->upper_idx = s.upper_idx.data();
  o->lptr = s.lptr.data();
  o->lidx = s.lidx.data();
  o->slot = s.slot.data();
  o->crow = s.crow.data();
  o->ccol = s.ccol.data();
  o->uptr = s.uptr.data();
  o->uk = s.uk.data();
  o->up1 = s.up1.data();
  o->up2 = s.up2.data();
  o->task_lo = s.task_lo.data();
  o->task_hi = s.task_hi.data();
  o->top = s.top.data();
  return FC_OK;
}

int fc_symbolic_import(const fc_symbolic_arrays *in, fc_symbolic **out, fc_status *status) {
  bool args = in && out && in->n >= 0 && in->ns >= 0 && in->nnz >= 0 && in->rows_len >= 0 && in->lower_len >= 0 &&
              in->updates_len >= 0 && in->tasks_len >= 0 && in->top_len >= 0;
  if (args) {
    // every array with a positive length has an address
    auto has = [](const void *p, int64_t len) { return len == 0 || p != nullptr; };
    args = has(in->perm, in->n) && in->first && in->rptr && has(in->rows, in->rows_len) && in->upper_ptr &&
           has(in->upper_idx, in->nnz) && in->lptr && has(in->lidx, in->lower_len) && has(in->slot, in->nnz) &&
           has(in->crow, in->nnz) && has(in->ccol, in->nnz) && in->uptr && has(in->uk, in->updates_len) &&
           has(in->up1, in->updates_len) && has(in->up2, in->updates_len) && has(in->task_lo, in->tasks_len) &&
           has(in->task_hi, in->tasks_len) && has(in->top, in->top_len);
  }
  if (!args) {
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "null or negative argument");
    return FC_INVALID_ARGUMENT;
  }
  *out = nullptr;
  try {
    auto h = new fc_symbolic();
    fc::Symbolic &s = h->s;
    auto cp64 = [](std::vector<int64_t> &v, const int64_t *p, int64_t len) { v.assign(p, p + len); };
    auto cp32 = [](std::vector<int32_t> &v, const int32_t *p, int64_t len) { v.assign(p, p + len); };
    s.n = in->n;
    s.ns = in->ns;
    s.entries = in->entries;
    cp64(s.perm, in->perm, in->n);
    cp64(s.first, in->first, in->ns + 1);
    cp64(s.rptr, in->rptr, in->ns + 1);
    cp32(s.rows, in->rows, in->rows_len);
    cp64(s.upper_ptr, in->upper_ptr, in->n + 1);
    cp32(s.upper_idx, in->upper_idx, in->nnz);
    cp64(s.lptr, in->lptr, in->n + 1);
    cp32(s.lidx, in->lidx, in->lower_len);
    cp64(s.slot, in->slot, in->nnz);
    cp32(s.crow, in->crow, in->nnz);
    cp32(s.ccol, in->ccol, in->nnz);
    cp64(s.uptr, in->uptr, in->ns + 1);
    cp64(s.uk, in->uk, in->updates_len);
    cp64(s.up1, in->up1, in->updates_len);
    cp64(s.up2, in->up2, in->updates_len);
    cp64(s.task_lo, in->task_lo, in->tasks_len);
    cp64(s.task_hi, in->task_hi, in->tasks_len);
    cp64(s.top, in->top, in->top_len);
    // Everything the device plan indexes with is checked here, so that no inconsistent array
    // reaches an index on the host or the device. The supernodal tree follows from the
    // structures: a supernode's parent holds its first row past its own columns.
    const char *why = nullptr;
    if (s.first.front() != 0 || s.first.back() != s.n || s.rptr.front() != 0 ||
        s.rptr.back() != (int64_t)s.rows.size())
      why = "supernodal structure: first/rptr do not span the columns and rows";
    std::vector<int64_t> snode(s.n, 0);
    for (int64_t t = 0; !why && t < s.ns; ++t) {
      if (s.first[t + 1] <= s.first[t] || s.rptr[t + 1] - s.rptr[t] < s.first[t + 1] - s.first[t])
        why = "supernodal structure: a supernode narrower than zero or taller than its rows";
      for (int64_t j = s.first[t]; !why && j < s.first[t + 1]; ++j) snode[j] = t;
    }
    s.sparent.assign(s.ns, fc::NONE);
    for (int64_t t = 0; !why && t < s.ns; ++t) {
      const int64_t w = s.width(t), m = s.height(t);
      const int32_t *r = s.rows.data() + s.rptr[t];
      for (int64_t i = 0; !why && i < m; ++i) {
        if (i < w ? r[i] != s.first[t] + i : (r[i] <= r[i - 1] || r[i] >= s.n))
          why = "supernodal structure: a supernode's rows are not its columns followed by increasing rows below";
      }
      if (!why && m > w) {
        s.sparent[t] = snode[r[w]];
        if (s.sparent[t] <= t) why = "supernodal structure: a parent before its child";
      }
    }
    if (!why) {
      std::vector<char> seen(s.n, 0);
      for (int64_t k = 0; !why && k < s.n; ++k) {
        const int64_t c = s.perm[k];
        if (c < 0 || c >= s.n || seen[c]) why = "perm is not a permutation";
        else seen[c] = 1;
      }
    }
    if (!why && (s.upper_ptr.front() != 0 || s.upper_ptr.back() != in->nnz))
      why = "upper_ptr does not span the entries";
    for (int64_t j = 0; !why && j < s.n; ++j)
      if (s.upper_ptr[j + 1] < s.upper_ptr[j]) why = "upper_ptr decreases";
    for (int64_t e = 0; !why && e < in->nnz; ++e) {
      const int64_t r = s.crow[e], c = s.ccol[e], i = s.upper_idx[e];
      if (r < 0 || r >= s.n || c < 0 || c > r || i < 0 || i >= s.n)
        why = "an entry's coordinates outside the lower triangle";
    }
    if (why) {
      delete h;
      set_status(status, FC_INTERNAL, -1, 0, 0, why);
      return FC_INTERNAL;
    }
    *out = h;
  } catch (const std::bad_alloc &) {
    set_status(status, FC_OUT_OF_MEMORY, -1, 0, 0, "host memory");
    return FC_OUT_OF_MEMORY;
  }
  set_status(status, FC_OK);
  return FC_OK;
}

int fc_chol_create(const fc_symbolic *sym, int precision, int device, fc_chol **out, fc_status *status) {
  if (!sym || !out ||
      (precision != FC_PRECISION_FP64 && precision != FC_PRECISION_FP32_IR && precision != FC_PRECISION_LDLT)) {
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "null argument or unknown precision");
    return FC_INVALID_ARGUMENT;
  }
  *out = nullptr;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(status, e, "cudaSetDevice");
  fc_chol *h = nullptr;
  try {
    h = new fc_chol();
  } catch (const std::bad_alloc &) {
    set_status(status, FC_OUT_OF_MEMORY, -1, 0, 0, "host memory");
    return FC_OUT_OF_MEMORY;
  }
  h->device = device;
  h->precision = precision;
  {
    const char *env = std::getenv("FC_NO_GRAPHS");
    h->graphs = !(env && env[0] == '1');
    const char *mma_sync = std::getenv("FC_TF32_MMA_SYNC");
    h->tc = !(mma_sync && mma_sync[0] == '1');
    const char *persistent = std::getenv("FC_SOLVE_PERSISTENT");
    h->dag = persistent && persistent[0] == '1' && precision != FC_PRECISION_LDLT;
  }
  fc::configure_kernels();
  if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    delete h;
    return cuda_fail(status, e, "cudaStreamCreate");
  }
  h->own_stream = true;
  int rc;
  try {
    rc = build(h, sym->s, status);
  } catch (const std::bad_alloc &) {
    rc = FC_OUT_OF_MEMORY;
    set_status(status, rc, -1, sym->s.entries, 0, "host memory for the plan");
  }
  if (rc != FC_OK) {
    fc_chol_destroy(h);
    return rc;
  }
  *out = h;
  set_status(status, FC_OK);
  return FC_OK;
}

void fc_chol_destroy(fc_chol *h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  cudaStream_t own = h->own_stream ? h->stream : nullptr;
  h->stream = nullptr;
  delete h;  // frees the device buffers
  if (own) cudaStreamDestroy(own);
}

int fc_chol_set_stream(fc_chol *h, void *stream) {
  if (!h) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  if (stream) {
    if (h->own_stream) cudaStreamDestroy(h->stream);
    h->stream = (cudaStream_t)stream;
    h->own_stream = false;
  } else if (!h->own_stream) {
    cudaStream_t own = nullptr;
    if (cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking) != cudaSuccess) return FC_CUDA_ERROR;
    h->stream = own;
    h->own_stream = true;
  }
  return FC_OK;
}

int fc_chol_factor(fc_chol *h, const double *upper_val, int64_t nnz, const volatile int32_t *cancel, fc_status *status) {
  if (!h || (nnz > 0 && !upper_val)) {
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "null handle or values");
    return FC_INVALID_ARGUMENT;
  }
  if (nnz != h->nnz) {
    set_status(status, FC_INTERNAL, -1, 0, 0, "supernodal factorization: the matrix's pattern differs from the analysed one");
    return FC_INTERNAL;
  }
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  cudaError_t e = cudaSuccess;
  if (nnz > 0) e = cudaMemcpyAsync(h->d_val.p, upper_val, sizeof(double) * nnz, cudaMemcpyHostToDevice, h->stream);
  if (e != cudaSuccess) return cuda_fail(status, e, "values upload");
  int rc = enqueue_factor(h, h->d_val.as<double>(), cancel);
  if (rc == FC_CANCELLED) {
    cudaStreamSynchronize(h->stream);
    set_status(status, FC_CANCELLED, -1, 0, 0, "cancelled");
    return FC_CANCELLED;
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(status, e, "factor launch");
  return read_status(h, status);
}

int fc_chol_factor_device_async(fc_chol *h, const double *d_upper_val, int64_t nnz) {
  if (!h || nnz != h->nnz || (nnz > 0 && !d_upper_val)) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  const int rc = enqueue_factor(h, d_upper_val, nullptr);
  if (rc != FC_OK) return rc;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FC_OK : FC_CUDA_ERROR;
}

int fc_chol_check(fc_chol *h, fc_status *status) {
  if (!h) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  const int rc = read_status(h, status);
  if (rc != FC_OK) return rc;
  return solve_wait_status(h, status);
}

int fc_chol_option(fc_chol *h, int32_t option, int64_t value) {
  if (!h) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  auto replan = [&] {
    h->solve_R = 0;
    if (h->solve_graph) {
      cudaGraphExecDestroy(h->solve_graph);
      h->solve_graph = nullptr;
    }
  };
  switch (option) {
    case FC_OPTION_SOLVE_SCHEDULE:
      if ((value != 0 && value != 1) || (value == 1 && h->ldlt)) return FC_INVALID_ARGUMENT;
      h->dag = value == 1;
      replan();
      return FC_OK;
    case FC_OPTION_WAIT_LIMIT_NS:
      if (value <= 0) return FC_INVALID_ARGUMENT;
      h->dag_limit_ns = value;
      replan();
      return FC_OK;
    case FC_OPTION_PLANT_UNMET_WAIT:
      h->dag_plant = value != 0;
      replan();
      return FC_OK;
    case FC_OPTION_TRACE:
      h->dag_trace = value != 0;
      replan();
      return FC_OK;
    case FC_OPTION_REFINEMENT:
      if (value != 0 && value != 1) return FC_INVALID_ARGUMENT;
      h->refine_pcg = value == 0;
      return FC_OK;
    case FC_OPTION_SOLVE_CLUSTER:
      if (value != 0 && value != 1) return FC_INVALID_ARGUMENT;
      h->solve_cluster = value == 1;
      replan();
      return FC_OK;
    case FC_OPTION_SOLVE_NARROW:
      if (value != 0 && value != 1) return FC_INVALID_ARGUMENT;
      h->solve_narrow = value == 1;
      replan();
      return FC_OK;
    case FC_OPTION_SOLVE_DEEP:
      if (value != 0 && value != 1) return FC_INVALID_ARGUMENT;
      h->solve_deep = value == 1;
      replan();
      return FC_OK;
    case FC_OPTION_SOLVE_PDL:
      if (value != 0 && value != 1) return FC_INVALID_ARGUMENT;
      h->solve_pdl = value == 1;
      replan();
      return FC_OK;
    case FC_OPTION_CHILDREN_FIRST: {
      if (value != 0 && value != 1) return FC_INVALID_ARGUMENT;
      if (h->asm_first == (value == 1)) return FC_OK;
      h->asm_first = value == 1;
      fc_status ignore{};
      return h->ldlt ? FC_OK : plan_factor_upload(h, &ignore);
    }
    case FC_OPTION_FP32_UPDATES: {
      if (value != 0 && value != 1) return FC_INVALID_ARGUMENT;
      if (h->tc == (value == 0)) return FC_OK;
      h->tc = value == 0;
      fc_status ignore{};
      return h->fp32 ? plan_factor_upload(h, &ignore) : FC_OK;
    }
  }
  return FC_INVALID_ARGUMENT;
}

int64_t fc_chol_trace_read(fc_chol *h, int64_t *out, int64_t cap) {
  if (!h || cap < 0 || (cap > 0 && !out)) return -FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  if (!h->dag_trace || !h->dag || h->solve_R == 0) return 0;
  const int64_t tasks = h->dag_fwd + h->dag_bwd;
  const int64_t words = std::min(cap, 4 * tasks);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
      (words > 0 && cudaMemcpy(out, h->d_dtrace.p, sizeof(int64_t) * words, cudaMemcpyDeviceToHost) != cudaSuccess))
    return -FC_CUDA_ERROR;
  return tasks;
}

int fc_chol_factor_device(fc_chol *h, const double *d_upper_val, int64_t nnz, fc_status *status) {
  int rc = fc_chol_factor_device_async(h, d_upper_val, nnz);
  if (rc != FC_OK) {
    set_status(status, rc, -1, 0, 0, rc == FC_CUDA_ERROR ? cudaGetErrorString(cudaGetLastError()) : "bad argument");
    return rc;
  }
  return fc_chol_check(h, status);
}

int64_t fc_chol_entries(const fc_chol *h) { return h ? h->entries : -1; }

int fc_chol_solve_device_async(fc_chol *h, double *d_b, int32_t nrhs, int64_t ld) {
  if (!h || nrhs < 0 || (nrhs > 0 && (!d_b || ld < h->n))) return FC_INVALID_ARGUMENT;
  if (nrhs == 0 || h->n == 0) return FC_OK;
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  int rc = enqueue_solve(h, d_b, nrhs, ld, nullptr);
  if (rc != FC_OK) return rc;
  return cudaGetLastError() == cudaSuccess ? FC_OK : FC_CUDA_ERROR;
}

int fc_chol_solve_device(fc_chol *h, double *d_b, int32_t nrhs, int64_t ld, fc_status *status) {
  if (!h || nrhs < 0 || (nrhs > 0 && (!d_b || ld < h->n))) {
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "right-hand side length");
    return FC_INVALID_ARGUMENT;
  }
  if (nrhs == 0 || h->n == 0) {
    set_status(status, FC_OK);
    return FC_OK;
  }
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  int rc = enqueue_solve(h, d_b, nrhs, ld, status);
  if (rc != FC_OK) return rc;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(status, e, "solve");
  if ((rc = solve_wait_status(h, status)) != FC_OK) return rc;
  set_status(status, FC_OK);
  return FC_OK;
}

int fc_chol_solve_device_noalloc(fc_chol *h, double *d_b, int32_t nrhs, int64_t ld, fc_status *status) {
  if (!h || nrhs < 0 || (nrhs > 0 && (!d_b || ld < h->n))) {
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "right-hand side length");
    return FC_INVALID_ARGUMENT;
  }
  if (ldlt_refused(h, status)) return FC_INVALID_ARGUMENT;
  if (nrhs == 0 || h->n == 0) {
    set_status(status, FC_OK);
    return FC_OK;
  }
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  unsigned char *base = nullptr;
  cudaError_t e = noalloc_scratch(h->device, &base);
  if (e != cudaSuccess) return cuda_fail(status, e, "cudaGetSymbolAddress of the solve scratch");
  const int R = nrhs;
  // Layout in the scratch: x | x2 | v | voff | row tasks | child ranges | panel tasks | GEMM tasks
  // | split partial tiles | thin forward tasks | their child ranges | thin backward tasks | their
  // partial sums | the counters (thin, then split).
  SolvePlan p;
  solve_offsets(h, R, p);
  const size_t vec = align256(sizeof(double) * (size_t)h->n * R);
  const size_t at_x = 0, at_x2 = vec, at_v = 2 * vec;
  const size_t at_voff = at_v + align256(sizeof(double) * (size_t)p.vsum);
  auto too_large = [&](size_t need) {
    char msg[160];
    std::snprintf(msg, sizeof(msg), "the solve needs %zu bytes of scratch; the no-allocation limit is %zu",
                  need, (size_t)FC_NOALLOC_SCRATCH_BYTES);
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, msg);
    return FC_INVALID_ARGUMENT;
  };
  if (at_voff > FC_NOALLOC_SCRATCH_BYTES) return too_large(at_voff);
  solve_tasks(h, R, reinterpret_cast<double *>(base + at_x), reinterpret_cast<double *>(base + at_x2),
              reinterpret_cast<double *>(base + at_v), p);
  const size_t at_rows = at_voff + align256(sizeof(int64_t) * p.voff.size());
  const size_t at_ranges = at_rows + align256(sizeof(fc::RowTask) * p.rows.size());
  const size_t at_panels = at_ranges + align256(sizeof(int2) * p.ranges.size());
  const size_t at_gemm = at_panels + align256(sizeof(fc::SolveTask) * p.panels.size());
  const size_t at_part = at_gemm + align256(sizeof(fc::GemmTask) * p.gemm.size());
  const size_t at_thin = at_part + align256(sizeof(double) * (size_t)p.psum);
  const size_t at_tranges = at_thin + align256(sizeof(fc::ThinTask) * p.thin.size());
  const size_t at_tbwd = at_tranges + align256(sizeof(int4) * p.tranges.size());
  const size_t at_tpart = at_tbwd + align256(sizeof(fc::ThinBwdTask) * p.tbwd.size());
  const size_t at_tcount = at_tpart + align256(sizeof(double) * (size_t)p.tpart);
  const size_t counters = (size_t)std::max<int64_t>(p.tcount + p.scount, 1);
  const size_t need = at_tcount + sizeof(int32_t) * counters;
  if (need > FC_NOALLOC_SCRATCH_BYTES) return too_large(need);
  // Every region is written before it is read in this call: the task lists and offsets here, x by
  // the permutation, x2 by the forward panels, each update vector's rows zeroed by its assembly
  // (or stored whole by a thin forward tile), each partial tile stored by its chunk before the
  // last chunk of its sum reads it, the counters zeroed here.
  auto put = [&](size_t at, const void *src, size_t bytes) {
    if (bytes && e == cudaSuccess) e = cudaMemcpyAsync(base + at, src, bytes, cudaMemcpyHostToDevice, h->stream);
  };
  put(at_voff, p.voff.data(), sizeof(int64_t) * p.voff.size());
  put(at_rows, p.rows.data(), sizeof(fc::RowTask) * p.rows.size());
  put(at_ranges, p.ranges.data(), sizeof(int2) * p.ranges.size());
  put(at_panels, p.panels.data(), sizeof(fc::SolveTask) * p.panels.size());
  put(at_gemm, p.gemm.data(), sizeof(fc::GemmTask) * p.gemm.size());
  put(at_thin, p.thin.data(), sizeof(fc::ThinTask) * p.thin.size());
  put(at_tranges, p.tranges.data(), sizeof(int4) * p.tranges.size());
  put(at_tbwd, p.tbwd.data(), sizeof(fc::ThinBwdTask) * p.tbwd.size());
  if (e == cudaSuccess) e = cudaMemsetAsync(base + at_tcount, 0, sizeof(int32_t) * counters, h->stream);
  if (e != cudaSuccess) return cuda_fail(status, e, "copy of the solve plan into the scratch");
  const SolveBuffers b{reinterpret_cast<double *>(base + at_x), reinterpret_cast<double *>(base + at_x2),
                       reinterpret_cast<double *>(base + at_v), reinterpret_cast<const int64_t *>(base + at_voff),
                       reinterpret_cast<const fc::RowTask *>(base + at_rows),
                       reinterpret_cast<const int2 *>(base + at_ranges),
                       reinterpret_cast<const fc::SolveTask *>(base + at_panels),
                       reinterpret_cast<const fc::GemmTask *>(base + at_gemm),
                       reinterpret_cast<double *>(base + at_part),
                       reinterpret_cast<const fc::ThinTask *>(base + at_thin),
                       reinterpret_cast<const int4 *>(base + at_tranges),
                       reinterpret_cast<const fc::ThinBwdTask *>(base + at_tbwd),
                       reinterpret_cast<double *>(base + at_tpart),
                       reinterpret_cast<int32_t *>(base + at_tcount),
                       p.lg};
  int64_t launches = 0;
  fc::launch_permute_in(h->d_perm.as<int64_t>(), h->n, d_b, ld, b.x, R, h->tree.scale, h->stream);
  run_solve_program(h, p.fwd, b, R, launches);
  run_solve_program(h, p.bwd, b, R, launches);
  fc::launch_permute_out(h->d_perm.as<int64_t>(), h->n, b.x, R, d_b, ld, h->tree.scale, h->stream);
  h->last_solve_launches = launches + 2;
  e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(status, e, "solve");
  set_status(status, FC_OK);
  return FC_OK;
}

int fc_chol_refine_solve_device(fc_chol *h, const int64_t *d_ptr, const int32_t *d_idx, const double *d_val,
                                const double *d_b, double *d_x, int32_t nrhs, int64_t ld, double tol, int32_t max_iter,
                                double *relres, int32_t *iterations, fc_status *status) {
  if (iterations) *iterations = 0;
  if (!h || nrhs < 0 || max_iter < 1 || (nrhs > 0 && (!d_b || !d_x || ld < h->n || !d_ptr || !d_idx || !d_val))) {
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "right-hand side length");
    return FC_INVALID_ARGUMENT;
  }
  if (h->ldlt && h->refine_pcg) {  // conjugate gradients needs a positive definite preconditioner
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0,
               "the LDL^T factor refines by plain refinement only (FC_OPTION_REFINEMENT = 1)");
    return FC_INVALID_ARGUMENT;
  }
  if (nrhs == 0 || h->n == 0) {
    set_status(status, FC_OK);
    return FC_OK;
  }
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  const int R = nrhs;
  const int64_t n = h->n;
  const size_t block = sizeof(double) * (size_t)n * R;
  const bool pcg = h->refine_pcg;
  auto need = [&](DeviceBuf &b, size_t bytes) { return b.bytes >= bytes || b.alloc(bytes) == cudaSuccess; };
  if (!need(h->d_ir_r, block) || !need(h->d_ir_d, block) || !need(h->d_ir_sum, 6 * sizeof(double) * R) ||
      !need(h->d_ir_sc, 2 * block) ||
      (pcg && (!need(h->d_ir_p, block) || !need(h->d_ir_q, block) || !need(h->d_ir_t, block) ||
               !need(h->d_ir_done, sizeof(int) * R)))) {
    set_status(status, FC_OUT_OF_MEMORY, -1, h->entries, 0, "device memory for the refinement");
    return FC_OUT_OF_MEMORY;
  }
  cudaStream_t st = h->stream;
  double *r = h->d_ir_r.as<double>(), *z = h->d_ir_d.as<double>(), *sums = h->d_ir_sum.as<double>();
  // sums: [0, R) residual norms^2, [R, 2R) ||b||^2, [2R, 3R) r.z, [3R, 4R) r.z new, [4R, 5R) p.q
  std::vector<double> host(2 * R), rel(R, 0.0);
  std::vector<int> done(R, 0);
  cudaError_t e = cudaSuccess;
  // x = 0, r = b
  for (int j = 0; j < R && e == cudaSuccess; ++j) {
    e = cudaMemsetAsync(d_x + (int64_t)j * ld, 0, sizeof(double) * n, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(r + (int64_t)j * n, d_b + (int64_t)j * ld, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
  }
  if (e != cudaSuccess) return cuda_fail(status, e, "refinement set-up");
  fc::launch_sumsq(n, R, n, r, sums + R, st);
  e = cudaMemcpyAsync(host.data() + R, sums + R, sizeof(double) * R, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(status, e, "refinement set-up");
  // the true residual's relative norms of the current x (into rel); true when every column is done
  auto check = [&](double *t) -> int {
    fc::launch_spmv(n, d_ptr, d_idx, d_val, d_x, ld, t, n, R, st, h->d_ir_sc.as<double>());
    fc::launch_residual(n, R, d_b, ld, t, n, st);
    fc::launch_sumsq(n, R, n, t, sums, st);
    cudaError_t e2 = cudaMemcpyAsync(host.data(), sums, 2 * sizeof(double) * R, cudaMemcpyDeviceToHost, st);
    if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(st);
    if (e2 == cudaSuccess) e2 = cudaGetLastError();
    if (e2 != cudaSuccess) return cuda_fail(status, e2, "refinement");
    int rc2 = solve_wait_status(h, status);
    if (rc2 != FC_OK) return rc2;
    bool all = true;
    for (int j = 0; j < R; ++j) {
      const double bb = host[R + j];
      rel[j] = bb > 0.0 ? std::sqrt(host[j] / bb) : std::sqrt(host[j]);
      done[j] = rel[j] <= tol;  // NaN never converges
      all = all && done[j];
    }
    return all ? -1 : FC_OK;
  };
  int it = 0, rc = FC_OK;
  bool converged = false;
  if (!pcg) {
    // plain refinement: x += M (b - A x)
    while (it < max_iter) {
      e = cudaMemcpyAsync(z, r, block, cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) return cuda_fail(status, e, "refinement");
      if ((rc = enqueue_solve(h, z, R, n, status)) != FC_OK) return rc;
      ++it;
      fc::launch_update(n, R, z, n, d_x, ld, st);
      rc = check(r);
      if (rc == -1) {
        converged = true;
        break;
      }
      if (rc != FC_OK) return rc;
    }
  } else {
    // conjugate gradients preconditioned by this factor (an FP32 factor makes M ~ A^-1 to a few
    // digits), one recurrence per right-hand side; convergence is judged on b - A x itself
    double *p = h->d_ir_p.as<double>(), *q = h->d_ir_q.as<double>(), *t = h->d_ir_t.as<double>();
    double *rz = sums + 2 * R, *rz_new = sums + 3 * R, *pq = sums + 4 * R;
    int *d_done = h->d_ir_done.as<int>();
    e = cudaMemcpyAsync(z, r, block, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(status, e, "refinement");
    if ((rc = enqueue_solve(h, z, R, n, status)) != FC_OK) return rc;
    ++it;
    cudaMemcpyAsync(p, z, block, cudaMemcpyDeviceToDevice, st);
    fc::launch_coldot(n, R, r, n, z, n, rz, st);
    cudaMemsetAsync(d_done, 0, sizeof(int) * R, st);
    // the recurrence's residual r (one norm per column, read each iteration) says when to look
    // at the true residual; only the true residual decides convergence and which columns stop
    auto recurrence_small = [&]() -> int {
      fc::launch_sumsq(n, R, n, r, sums, st);
      cudaError_t e2 = cudaMemcpyAsync(host.data(), sums, sizeof(double) * R, cudaMemcpyDeviceToHost, st);
      if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(st);
      if (e2 == cudaSuccess) e2 = cudaGetLastError();
      if (e2 != cudaSuccess) return cuda_fail(status, e2, "refinement");
      int rc2 = solve_wait_status(h, status);
      if (rc2 != FC_OK) return rc2;
      for (int j = 0; j < R; ++j) {
        const double bb = host[R + j];  // ||b||^2 of column j, read by the last true check
        const double rr = bb > 0.0 ? std::sqrt(host[j] / bb) : std::sqrt(host[j]);
        if (!done[j] && !(rr <= tol)) return FC_OK;
      }
      return -1;
    };
    for (;;) {
      fc::launch_spmv(n, d_ptr, d_idx, d_val, p, n, q, n, R, st, h->d_ir_sc.as<double>());
      fc::launch_coldot(n, R, p, n, q, n, pq, st);
      fc::launch_pcg_step(n, R, rz, pq, d_done, p, q, d_x, ld, r, st);
      rc = recurrence_small();
      if (rc == -1) rc = check(t);
      if (rc == -1) {
        converged = true;
        break;
      }
      if (rc != FC_OK) return rc;
      if (it >= max_iter) break;
      e = cudaMemcpyAsync(d_done, done.data(), sizeof(int) * R, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(z, r, block, cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) return cuda_fail(status, e, "refinement");
      if ((rc = enqueue_solve(h, z, R, n, status)) != FC_OK) return rc;
      ++it;
      fc::launch_coldot(n, R, r, n, z, n, rz_new, st);
      fc::launch_pcg_direction(n, R, rz_new, rz, z, p, st);
      std::swap(rz, rz_new);
    }
  }
  if (relres)
    for (int j = 0; j < R; ++j) relres[j] = rel[j];
  if (iterations) *iterations = it;
  if (!converged) {
    set_status(status, FC_TIMEOUT, -1, 0, 0, "the refinement did not reach the tolerance");
    return FC_TIMEOUT;
  }
  set_status(status, FC_OK);
  return FC_OK;
}

int fc_chol_solve(fc_chol *h, double *b, int32_t nrhs, int64_t ld, fc_status *status) {
  if (!h || nrhs < 0 || (nrhs > 0 && (!b || ld < h->n))) {
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "right-hand side length");
    return FC_INVALID_ARGUMENT;
  }
  if (nrhs == 0 || h->n == 0) {
    set_status(status, FC_OK);
    return FC_OK;
  }
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  const size_t bytes = sizeof(double) * (size_t)h->n * nrhs;
  if (h->d_b.bytes < bytes && h->d_b.alloc(bytes) != cudaSuccess) {
    set_status(status, FC_OUT_OF_MEMORY, -1, h->entries, 0, "device memory for the right-hand sides");
    return FC_OUT_OF_MEMORY;
  }
  cudaError_t e = cudaMemcpy2DAsync(h->d_b.p, sizeof(double) * h->n, b, sizeof(double) * ld, sizeof(double) * h->n, nrhs,
                                    cudaMemcpyHostToDevice, h->stream);
  if (e != cudaSuccess) return cuda_fail(status, e, "right-hand side upload");
  int rc = enqueue_solve(h, h->d_b.as<double>(), nrhs, h->n, status);
  if (rc != FC_OK) return rc;
  e = cudaMemcpy2DAsync(b, sizeof(double) * ld, h->d_b.p, sizeof(double) * h->n, sizeof(double) * h->n, nrhs,
                        cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(status, e, "solve");
  if ((rc = solve_wait_status(h, status)) != FC_OK) return rc;
  set_status(status, FC_OK);
  return FC_OK;
}

int fc_chol_ldlt_pivots(fc_chol *h, int8_t *pivots, int32_t *order, fc_status *status) {
  if (!h || !h->ldlt || (h->n > 0 && (!pivots || !order))) {
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "not an LDL^T factor, or a null argument");
    return FC_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  if (h->n == 0) {
    set_status(status, FC_OK);
    return FC_OK;
  }
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaMemcpy(pivots, h->d_lpivots.p, (size_t)h->n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(order, h->d_lorder.p, sizeof(int32_t) * (size_t)h->n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(status, e, "pivots");
  set_status(status, FC_OK);
  return FC_OK;
}

int fc_chol_values(fc_chol *h, double *dst, fc_status *status) {
  if (!h || (h->entries > 0 && !dst)) {
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "null argument");
    return FC_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  if (h->entries == 0) {
    set_status(status, FC_OK);
    return FC_OK;
  }
  if (h->ldlt) {
    // L as the fronts hold it (own blocks unit lower), D put back on their diagonals and at the
    // 2 x 2 pivots' first subdiagonal entries: the reference's Block::values
    std::vector<double> rect((size_t)std::max<int64_t>(h->l_len, 1)), d(h->n), sub(h->n);
    std::vector<int8_t> piv(h->n);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) e = cudaMemcpy(rect.data(), h->d_L.p, sizeof(double) * (size_t)h->l_len, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(d.data(), h->d_ldd.p, sizeof(double) * (size_t)h->n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(sub.data(), h->d_lde.p, sizeof(double) * (size_t)h->n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(piv.data(), h->d_lpivots.p, (size_t)h->n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(status, e, "values");
    // after a solve the rows below are in the solve's order: row w + i holds row w + from[i]
    int64_t at = 0;
    for (int64_t s = 0; s < h->ns; ++s) {
      const int64_t m = h->height[s], w = h->width[s], f = h->first[s];
      const double *F = rect.data() + h->loff[s];
      std::vector<int64_t> to(m - w);  // the structure's row w + j is at row w + to[j]
      for (int64_t i = 0; i < m - w; ++i) to[i] = i;
      if (h->ldlt_folded)
        for (int64_t i = 0; i < m - w; ++i) to[h->ldlt_from[h->ldlt_from_off[s] + i]] = i;
      for (int64_t c = 0; c < w; ++c) {
        for (int64_t r = c; r < m; ++r) dst[at + r - c] = F[(r >= w ? w + to[r - w] : r) + c * m];
        dst[at] = d[f + c];
        if (piv[f + c] == fc::ldlt::PIVOT_FIRST && c + 1 < m) dst[at + 1] = sub[f + c];
        at += m - c;
      }
    }
    set_status(status, FC_OK);
    return FC_OK;
  }
  DeviceBuf tmp;
  if (tmp.alloc(sizeof(double) * (size_t)h->entries) != cudaSuccess) {
    set_status(status, FC_OUT_OF_MEMORY, -1, h->entries, 0, "device memory for the copy");
    return FC_OUT_OF_MEMORY;
  }
  fc::launch_pack_trapezoids(h->tree, h->fp32, h->ns, h->d_toff.as<int64_t>(), tmp.as<double>(), h->stream);
  cudaError_t e = cudaMemcpyAsync(dst, tmp.p, sizeof(double) * h->entries, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_fail(status, e, "values");
  set_status(status, FC_OK);
  return FC_OK;
}

int fc_chol_inertia(fc_chol *h, int64_t *positive, int64_t *negative, int64_t *two_by_two, fc_status *status) {
  if (!h || !positive || !negative || !two_by_two) {
    set_status(status, FC_INVALID_ARGUMENT, -1, 0, 0, "null argument");
    return FC_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> g(h->lock);
  if (!h->ldlt) {  // a Cholesky factor's matrix is positive definite (ldlt.rs:500-506)
    *positive = h->n, *negative = 0, *two_by_two = 0;
    set_status(status, FC_OK);
    return FC_OK;
  }
  cudaSetDevice(h->device);
  std::vector<double> d(h->n), sub(h->n);
  std::vector<int8_t> piv(h->n);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess && h->n > 0) e = cudaMemcpy(d.data(), h->d_ldd.p, sizeof(double) * (size_t)h->n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && h->n > 0) e = cudaMemcpy(sub.data(), h->d_lde.p, sizeof(double) * (size_t)h->n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && h->n > 0) e = cudaMemcpy(piv.data(), h->d_lpivots.p, (size_t)h->n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(status, e, "inertia");
  // Sylvester's law on D (ldlt.rs:415-447): a 1 x 1 pivot by its sign; a 2 x 2 one has one of
  // each sign when its determinant is negative, else both of the sign of its trace
  int64_t pos = 0, neg = 0, twos = 0;
  for (int64_t c = 0; c < h->n;) {
    if (piv[c] == fc::ldlt::PIVOT_FIRST && c + 1 < h->n) {
      const double d11 = d[c], d21 = sub[c], d22 = d[c + 1];
      const double det = d11 * d22 - d21 * d21;
      if (det < 0.0)
        pos += 1, neg += 1;
      else if (d11 + d22 > 0.0)
        pos += 2;
      else
        neg += 2;
      twos += 1;
      c += 2;
    } else {
      if (d[c] > 0.0)
        pos += 1;
      else
        neg += 1;
      c += 1;
    }
  }
  *positive = pos, *negative = neg, *two_by_two = twos;
  set_status(status, FC_OK);
  return FC_OK;
}

int64_t fc_chol_stat(const fc_chol *h, int what) {
  if (!h) return -1;
  switch (what) {
    case 0: return h->levels;
    case 1: return (int64_t)h->program.size();
    case 2: return h->l_len * 8;
    case 3: return h->u_len * 8;
    case 4: return h->ns;
    case 5: return (int64_t)h->flops;
    case 6: return h->gemm_tasks;
    case 7: return h->last_factor_launches;
    case 8: return h->last_solve_launches;
    case 9: return (int64_t)h->gemm_flops_factor;
    case 10: return (int64_t)h->gemm_flops_solve;
    case 11: return h->gemm_big_ordinal;
    case 12: return h->gemm_trail_ordinal;
    case 13: return h->dag ? h->dag_fwd : 0;
    case 14: return h->dag ? h->dag_bwd : 0;
    case 15: return (int64_t)h->gemm_flops_updates;
  }
  return -1;
}

int fc_chol_profile(fc_chol *h, int enable) {
  if (!h) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  h->profiling = enable != 0;
  h->marks.clear();
  h->events_used = 0;
  return FC_OK;
}

int fc_chol_profile_read(fc_chol *h, double *ms, int64_t *launches, int32_t kinds) {
  if (!h || !ms || !launches || kinds <= 0) return FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return FC_CUDA_ERROR;
  for (int k = 0; k < kinds; ++k) {
    ms[k] = 0;
    launches[k] = 0;
  }
  for (auto &m : h->marks) {
    if (m.kind < 0 || m.kind >= kinds) continue;
    float t = 0;
    if (cudaEventElapsedTime(&t, m.a, m.b) == cudaSuccess) ms[m.kind] += t;
    launches[m.kind] += 1;
  }
  h->marks.clear();
  h->events_used = 0;
  return FC_OK;
}

int64_t fc_chol_profile_launches(fc_chol *h, int32_t *kind, int32_t *level, int32_t *tasks, float *ms, int64_t cap) {
  if (!h || cap < 0 || (cap > 0 && (!kind || !level || !tasks || !ms))) return -FC_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(h->lock);
  cudaSetDevice(h->device);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return -FC_CUDA_ERROR;
  const int64_t count = (int64_t)h->marks.size();
  for (int64_t i = 0; i < std::min(count, cap); ++i) {
    const auto &m = h->marks[i];
    kind[i] = m.kind;
    level[i] = m.level;
    tasks[i] = m.count;
    ms[i] = 0;
    cudaEventElapsedTime(&ms[i], m.a, m.b);
  }
  return count;
}

int fc_csr_spmv_device(int64_t n, const int64_t *d_ptr, const int32_t *d_idx, const double *d_val, const double *d_x,
                       double *d_y, int32_t nrhs, int64_t ld, void *stream) {
  if (n < 0 || nrhs < 0 || (n > 0 && (!d_ptr || !d_idx || !d_val || !d_x || !d_y || ld < n))) return FC_INVALID_ARGUMENT;
  const cudaStream_t st = (cudaStream_t)stream;
  // several right-hand sides: through row-major copies in stream-ordered scratch (freed in order)
  double *scratch = nullptr;
  if (n > 0 && nrhs >= fc::SPMV_ROWS_MIN_R &&
      cudaMallocAsync(reinterpret_cast<void **>(&scratch), sizeof(double) * 2 * (size_t)n * nrhs, st) != cudaSuccess) {
    cudaGetLastError();
    scratch = nullptr;
  }
  fc::launch_spmv(n, d_ptr, d_idx, d_val, d_x, ld, d_y, ld, nrhs, st, scratch);
  if (scratch) cudaFreeAsync(scratch, st);
  return cudaGetLastError() == cudaSuccess ? FC_OK : FC_CUDA_ERROR;
}

}  // extern "C"
