// Device kernels of the supernodal Cholesky and their task records. The host plans the whole
// numeric phase as a fixed list of launches over task arrays (level by level of the supernodal
// tree, panel by panel inside a level); each CTA of a launch takes one task.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fc {

// Panel width of the dense partial factorisation of a front, and the tile of the dense kernels.
constexpr int NB = 64;
constexpr int GEMM_TM = 64, GEMM_TN = 64, GEMM_KC = 16;
constexpr int GEMM_THREADS = 128;
constexpr int PANEL_ROWS = 128;  // rows of a panel solved by one CTA (64 at a time)
// A front is assembled by tiles of ASSEMBLE_COLS columns by ASSEMBLE_ROWS rows, one CTA each
// (a thread per row, a warp per child column); a supernode at most ASSEMBLE_THIN columns wide has
// its update matrix formed by the assembly itself instead of by a GEMM.
constexpr int ASSEMBLE_COLS = 8, ASSEMBLE_ROWS = 256, ASSEMBLE_THIN = 16;
// An FP32 front (mixed precision) is assembled by tiles of 16 columns by 128 rows (a thread a row,
// each warp four child columns): the bytes of a 256-row FP64 tile over half its rows, and eight
// CTAs an SM.
constexpr int ASSEMBLE_COLS_F32 = 16, ASSEMBLE_ROWS_F32 = 128;
constexpr int ASSEMBLE_KIDS = 8;  // children whose ranges a tile keeps in shared memory (the rest: global)
constexpr int SPLIT_K = 512;  // K chunk of the persistent solve's split products
// Chunks of a split sum added by one CTA (GemmTask flag 8): a sum of more chunks is added in
// groups of this many, then the groups' sums, each by the last CTA to finish its part.
constexpr int SPLIT_GROUP = 8;
// Counters and partial tiles (of 4096 doubles) that a split sum of `chunks` chunks takes.
__host__ __device__ constexpr int split_groups(int chunks) {
  return chunks > SPLIT_GROUP ? (chunks + SPLIT_GROUP - 1) / SPLIT_GROUP : 0;
}
// The solve applies the inverse of a supernode's diagonal block SB columns at a time: the inverses
// of its diagonal blocks of up to SB columns are formed during the factorisation (from the 64 x 64
// inverses of the panels, by doubling), so a solve step is a GEMM over SB columns, not a chain of
// SB / 64 dependent panel steps.
constexpr int SB = 2048;
// The solve's short products split K over a cluster of this many CTAs (gemm_cluster_kernel).
constexpr int SOLVE_CLUSTER = 8;

// Programmatic dependent launch. The solve's kernels may be launched so that a kernel's CTAs are
// scheduled while the kernel before it in the stream is still running. A CTA reads before
// pdl_wait() only data that no kernel of the solve writes (task lists, row lists, L, the diagonal
// blocks' inverses) and reads or writes the solve's vectors, partial sums and counters only after
// it; pdl_wait() returns once every grid the kernel depends on has completed with its writes
// visible (at once in a kernel launched the ordinary way). Every CTA passes pdl_wait() before it
// exits, so a kernel completes only after its predecessors have. Right after its wait a CTA lets
// the next kernel be scheduled (pdl_trigger): at most one kernel's CTAs wait at a time, not a
// chain of them holding the SMs.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// A child as its parent's assembly reads it: its update matrix (offset, height) and relative map.
struct KidMeta {
  int64_t uoff, rel_off;
  int32_t uc, pad;
};

// Where each supernode lives on the device. A front of supernode s has m = rows(s) rows and
// w = width(s) columns of L; its update matrix U_s is the (m-w) x (m-w) Schur complement.
struct Tree {
  const int64_t *first;     // [ns+1] first column (postorder)
  const int32_t *width;     // [ns]
  const int32_t *height;    // [ns]  m
  const int64_t *rows_off;  // [ns]
  const int32_t *rows;      // row structures (postorder indices)
  const int64_t *loff;      // [ns] L panel: m x w, column-major, ld m
  const int64_t *uoff;      // [ns] U: (m-w) x (m-w), column-major, ld m-w (lower half used)
  const int64_t *kid_ptr;   // [ns+1]
  const int32_t *kids;      // children in increasing order
  const KidMeta *kid_meta;  // per entry of kids
  const int64_t *rel_off;   // [ns] where a child's relative map starts (its rows past its columns)
  const int32_t *rel;       // positions of a child's rows in its parent's structure
  const int64_t *a_ptr;     // [n+1] input entries by postordered column
  const int64_t *a_src;     // upper-entry index of each
  const int64_t *a_dst;     // its place in the L arena
  const int64_t *diag_src;  // [n] upper-entry index of A(j, j), -1 if absent
  const int64_t *doff;      // [ns] diagonal arena: panel p of s keeps its factored block and its
                            // inverse (pw x pw each, column-major) at doff[s] + 2 NB NB p
  const int32_t *a_row;     // mixed precision: each input entry's postordered row and column
  const int32_t *a_col;
  const double *scale;      // mixed precision: S = diag(A)^-1/2 (postorder); null in FP64
  void *L;                  // L panels and update matrices: double, or float in mixed precision
  void *U;
  double *D;
  double *Dinv;             // inverses of the diagonal blocks of up to SB columns (column-major,
                            // lower triangular, zero above)
};

// Front tile columns [j0, j1) x rows [i0, i1) of supernode s; ranges[q] (from `ranges`) is child
// q's {columns lo, hi, rows lo, hi} of its update matrix that land in the tile; [e0, e1) are the
// input entries of an ASM_L tile.
// ASM_U_FIRST: an update matrix's tile from zero with the children's contributions, written
// before its supernode's panels; the update GEMM then subtracts -L21 L21^T from it.
enum AssembleMode : int32_t { ASM_L = 0, ASM_U = 1, ASM_U_PRODUCT = 2, ASM_U_FIRST = 3 };
struct AssembleTask {
  int32_t s, j0, j1, i0, i1, mode, ranges, nk;  // nk: the supernode's children
  int64_t e0, e1;
  int64_t loff, uoff;    // the supernode's L and update-matrix offsets
  int32_t m, w, k0, pad;  // its height and width; its first child's place in the kid lists
};
// Panel [c0, c1) of supernode s: factor its diagonal block, invert it, and solve the rows
// [r0, r1) below it (r0 >= c1; an empty range for a task that only keeps the block). Every task of
// the panel factors the block itself (no CTA waits on another) and writes its share of the factored
// block and its inverse (to the diagonal arena at `doff` and to Dinv at `ioff`); part 0 reports the
// pivots.
struct PanelTask {
  int32_t s, c0, c1, r0, r1;
  int32_t keep;  // the panel's CTA count: each stores columns part, part + keep, ... (times 4 warps)
  int64_t doff;  // of the factored block and its inverse
  int64_t ioff;  // where the block's inverse goes in Dinv (leading dimension ild)
  int32_t ild, part;
};
// C(i, j) -= sum_k A(i, k) B(j, k) for i < M, j < N, k < K, strided operands. Flags: 1 touches
// i >= j only (a diagonal tile of a symmetric matrix); 2 stores C = -sum instead of subtracting;
// 4 stores C = +sum. Flag 16 (FP64 B, unit j stride): B's row k is at B + b_rows[k] * b_sk (a
// gather through a row list). Flag 8 (FP64 C only): this task is chunk `chunk` of `chunks` of one split
// sum over K; each chunk stores its 64 x 64 partial at part + part_off + chunk * 4096 (`part`
// given at launch). With at most SPLIT_GROUP chunks the last chunk to finish (counters[counter],
// reset by it) adds the partials in chunk order and applies the total to C by the other flags.
// With more, the chunks form groups of SPLIT_GROUP (the last group shorter): the last chunk of a
// group to finish (counters[counter + 1 + group]) adds the group's partials in chunk order and
// stores the group's sum after the partials (part_off + (chunks + group) * 4096); the last group
// to finish (counters[counter]) adds the group sums in group order and applies the total. The
// order of every addition is fixed by the split, whichever CTA finishes last. No chunk waits.
struct GemmTask {
  void *C;
  const void *A;
  const void *B;
  int64_t c_si, c_sj, a_si, a_sk, b_sj, b_sk;
  int32_t M, N, K, flags;
  int64_t part_off;
  int32_t chunks, chunk, counter, pad;
  const int32_t *b_rows;
};
// Solve, panel [c0, c1) of supernode s, right-hand sides [j0, j1): apply the inverse of the
// diagonal block (forward: L^-1, backward: L^-T), then update the front rows [r0, r1) (forward:
// below the panel; backward: the own rows above it). `keep`: this task stores the panel's result.
struct SolveTask {
  int32_t s, c0, c1, r0, r1, j0, j1, keep;
  int64_t doff;
};
// Solve front rows [i0, i1) of supernode s; ranges[q] (from `ranges`) is child q's rows of its
// update vector whose places fall in [i0, i1).
struct RowTask {
  int32_t s, i0, i1, ranges;
};

// A supernode at most SOLVE_THIN columns wide takes each direction of the solve in one launch:
// forward, ThinTask tiles of its update vector (rows [i0, i1) of the front, right-hand sides from
// j0), each forming y = Dinv x of the supernode's own rows itself (`first` also stores it); per
// child the int4 at ranges[q] is {own rows' end, tile rows lo, hi, 0} in its update vector.
// Backward, ThinBwdTask chunks of the rows past the columns: each sums L21^T x over its rows, and
// the last chunk to finish (a counter) adds the chunks' sums in order and applies Dinv^T.
constexpr int SOLVE_THIN = 8;
constexpr int THIN_ROWS = 64;      // update-vector rows of a forward tile (by up to 64 right-hand sides)
constexpr int THIN_CHUNK = 128;    // rows past the columns per backward task
struct ThinTask {
  int32_t s, i0, i1, j0, ranges, first;
  int64_t dinv;  // the supernode's diagonal-block inverse in Dinv (w x w, column-major)
};
struct ThinBwdTask {
  int32_t s, k0, k1, j0, chunks, chunk, counter, pad;
  int64_t dinv, part;  // part: the chunks' partial sums (chunks x SOLVE_THIN x 64 doubles)
};

// ---- the solve as one dependency-driven launch per direction ----------------------------------
// Every CTA of a persistent grid takes the next task of a topologically ordered list (an atomic
// ticket), waits until the task's dependencies are met (counters raised by the tasks it depends
// on), does it, and raises the task's own counters. A task only waits on tasks taken before it, so
// the list completes with any number of resident CTAs. Waits are bounded: past `limit_ns` the
// waiting CTA records FC_TIMEOUT in the control block and every CTA drains the list without work.
//
// A supernode's front rows fall in chunks of at most 64 rows: chunk c < P is own columns
// [64c, 64c + 64) (P panels of 64), chunk P + b is rows past the columns [w + 64b, w + 64b + 64).
constexpr int32_t DAG_TIMEOUT = 7;  // the FC_TIMEOUT status code
enum DagKind : int32_t {
  DAG_ASSEMBLE = 0,  // forward: rows [i0, i1) (chunks [r0, r1)): zero the update rows, add the children
  DAG_PANEL = 1,     // panel columns [i0, i1), front chunks [r0, r1) updated, one after another
  DAG_NODE = 2,      // a whole small supernode: forward, assembly and every panel; backward, the
                     // product with the rows past the columns and every panel
  DAG_GEMM = 3,      // backward: own rows [i0, i1) -= L(w + k, rows)^T x(row k) for k in [r0, r1)
  DAG_REDUCE = 4,    // backward: own rows [i0, i1) -= the `count` partial tiles from aux on, in order
};
// Panel tasks: keep = 1 applies the inverse of the diagonal block and stores the panel's result
// (y in x2 forward, z in x backward), raising `sigmid` once it is stored; keep = -1 reads it from
// there. A panel task raises counter sig0 + k sigstep after its k-th chunk; other tasks raise
// sig0 + k sigstep for k < nsig at the end. Every task adds inc1 to sig1 at the end.
struct DagTask {
  int32_t kind, s, i0, i1, r0, r1, j0, j1;
  int32_t keep, child, count;  // child: first record of the children's ranges (assembly)
  int32_t dep0, dep1;          // [dep0, dep1) in the dependency list
  int32_t sig0, sigstep, nsig, sig1, inc1, sigmid;
  int32_t pad;
  int64_t aux;  // panel: the diagonal block's offset in the diagonal arena; gemm, reduce: partial
                // tile offset (-1: subtract in place)
};
struct DagDep {
  int32_t counter, value;  // wait until counters[counter] >= value
};
// One child's rows [lo, hi) (of its rows past its columns) that land in an assembly task's rows.
struct DagChild {
  int64_t rel;  // offset of the child's relative map
  int64_t v;    // offset of the child's update vectors
  int32_t lo, hi;
};
struct DagControl {
  int32_t next[2];  // tickets of the forward and the backward lists
  int32_t error;    // 0, or the FC_* code of the first failed wait
  int32_t task;     // the task whose wait failed
};
struct SolveDag {
  const DagTask *tasks;
  int32_t count;
  const DagDep *deps;
  const DagChild *children;
  int32_t *counters;
  DagControl *ctl;
  double *x, *x2, *v, *part;
  const int64_t *voff;
  int32_t R;
  long long limit_ns;
  long long *trace;  // null, or per task: taken, ready and done times (ns), kind << 32 | SM
};
// Sets the persistent kernels' shared-memory limits (called by configure_kernels).
void configure_solve_dag();
// CTAs per SM of the solve's persistent kernel (for sizing its grid).
int solve_dag_blocks_per_sm(bool fp32);
void launch_solve_dag(const Tree &t, bool fp32, bool backward, const SolveDag &d, int grid, cudaStream_t st);

// Device status word of a factorisation: the smallest failing pivot column (postorder).
struct DeviceStatus {
  unsigned long long failed_column;  // ULLONG_MAX when none
  unsigned int timeout;              // 0xFFFFFFFF when none; set when a bounded device wait gave up
  unsigned int pad;
};

// Sets the kernels' shared-memory limits (once per process; before any stream capture).
void configure_kernels();

// The operand types of a GEMM launch: FP64 throughout (DMMA); an FP32 A with FP64 B and C (DMMA,
// the solve on an FP32 factor); FP32 throughout by 3xTF32 (the FP32 factorisation).
enum class GemmKind { F64, F32A_F64, F32_TF32X3 };
// The mixed-precision factor's long products on the tcgen05 tensor cores: the update matrices
// (U = -L21 L21^T) and a front's updates past an outer block (C -= L(rows, block) L(cols, block)^T).
// The operand block of L (columns [c0, c0 + kw), front rows from row0 down) is first packed as a
// K-major FP32 array P: row i = [hi(L(row0 + i, c0..c0 + wpad)) | lo(...)], wpad = kw rounded up
// to TC_KPAD, at P + poff, by PackTask row blocks of TC_PACK_ROWS. A TcTask is one tile
// C(bi.., bj..) of up to GEMM_TC_M x GEMM_TC_N (bi, bj: rows of P; flags as GemmTask: 1 lower
// triangle only, 2 store -product, else subtract), its operands read by TMA through tensor map
// `map` of the block's P (an array of 128-byte CUtensorMap objects in device memory); a wait that
// gives up sets status->timeout.
constexpr int GEMM_TC_M = 128, GEMM_TC_N = 128, TC_KPAD = 32, TC_PACK_ROWS = 64;
constexpr int TC_KBOX = 16;  // K values of a TMA box (64 bytes: 64-byte swizzle)
struct PackTask {
  int32_t s, r0, wpad, kw;  // rows [r0, r0 + TC_PACK_ROWS) of the packed block, kw columns
  int64_t poff;
  int32_t c0, row0;  // the block: columns [c0, c0 + kw) of L from front row row0 down
  int32_t k0, k1;    // this task's packed columns [k0, k1) (multiples of TC_KPAD; k1 <= wpad)
};
// A pack task's columns: a wide block is packed by several tasks side by side, not column chunk
// after column chunk in one CTA.
constexpr int TC_PACK_K = 64;
struct TcTask {
  int32_t map, bi, bj, M, N, K, wpad, flags;
  float *C;
  int64_t c_sj;  // C(i, j) at C[i + j c_sj]
};
void launch_pack_tc(const Tree &t, const PackTask *tasks, float *P, int count, cudaStream_t st);
void launch_syrk_tc(const TcTask *tasks, const void *maps, int count, DeviceStatus *status, cudaStream_t st);

// S = diag(A)^-1/2 for the mixed-precision factorisation.
void launch_scale(int64_t n, const int64_t *diag_src, const double *val, double *scale, cudaStream_t st);
void launch_assemble(const Tree &t, bool fp32, const double *upper_val, const AssembleTask *tasks,
                     const int4 *ranges, int count, cudaStream_t st);
// p8max: the widest panel of the launch, rounded up to a multiple of 8 (sizes shared memory).
void launch_panel(const Tree &t, bool fp32, const double *upper_val, const PanelTask *tasks, int count,
                  DeviceStatus *status, int p8max, cudaStream_t st);
// part and counters: the partial sums and counters of split tasks (flag 8), null when there are none.
void launch_gemm(const GemmTask *tasks, int count, GemmKind kind, cudaStream_t st, double *part = nullptr,
                 int32_t *counters = nullptr);
// pdl: launch as a programmatic dependent of the kernel before it in the stream (the solve's
// launches; the kernels keep the rules of pdl_wait).
void launch_gemm_pdl(const GemmTask *tasks, int count, bool fp32_a, cudaStream_t st, double *part, int32_t *counters,
                     bool pdl);
// The solve's products with at most 16 right-hand sides (every task's N <= cols): 64 x 8 or 64 x 16
// tiles, each element's bits those of launch_gemm's F64 / F32A_F64 kernels.
void launch_gemm_narrow(const GemmTask *tasks, int count, bool fp32_a, int cols, cudaStream_t st, double *part,
                        int32_t *counters, bool pdl = false);
// The solve's products with at most 16 right-hand sides (every task's N <= cols <= 16) in 64 x 8 /
// 64 x 16 tiles with a deeper cp.async ring: the same bits as launch_gemm_narrow.
void launch_gemm_solve(const GemmTask *tasks, int count, bool fp32_a, int cols, cudaStream_t st, double *part,
                       int32_t *counters, bool pdl = false);
// The same tasks (FP64 B and C; A FP64 or FP32) with K split over clusters of SOLVE_CLUSTER CTAs.
void launch_gemm_cluster(const GemmTask *tasks, int count, bool fp32_a, cudaStream_t st, double *part,
                         int32_t *counters);
// Solve kernels: x and v are row-major with R columns (R right-hand sides), x in postorder.
void launch_solve_assemble(const Tree &t, double *x, double *v, const int64_t *voff, int R,
                           const RowTask *tasks, const int2 *ranges, int count, cudaStream_t st, bool pdl = false);
// The thin supernodes' steps of a level; lg = log2 of the right-hand-side block (a power of two
// <= 64 covering R, or 64).
void launch_thin_fwd(const Tree &t, bool fp32, const double *x, double *x2, double *v, const int64_t *voff, int R,
                     int lg, const ThinTask *tasks, const int4 *ranges, int count, cudaStream_t st, bool pdl = false);
void launch_thin_bwd(const Tree &t, bool fp32, double *x, const double *x2, int R, int lg, const ThinBwdTask *tasks,
                     double *part, int32_t *counters, int count, cudaStream_t st, bool pdl = false);
// x_post[i*R + j] = b[perm[i] + j*ld] (times scale[i] if given) and back.
void launch_permute_in(const int64_t *perm, int64_t n, const double *b, int64_t ld, double *x, int R,
                       const double *scale, cudaStream_t st);
void launch_permute_out(const int64_t *perm, int64_t n, const double *x, int R, double *b, int64_t ld,
                        const double *scale, cudaStream_t st);
// Iterative refinement on column-major n x R blocks, each with its own leading dimension:
// ax <- b - ax, x <- x + d, out[j] <- sum of squares of column j.
void launch_residual(int64_t n, int R, const double *b, int64_t ldb, double *ax, int64_t ldax, cudaStream_t st);
void launch_update(int64_t n, int R, const double *d, int64_t ldd, double *x, int64_t ldx, cudaStream_t st);
void launch_sumsq(int64_t n, int R, int64_t ld, const double *v, double *out, cudaStream_t st);
// Preconditioned CG per column (scalars on the device): out[j] = a_j . b_j;
// x_j += (rz_j / pq_j) p_j and r_j -= (rz_j / pq_j) q_j unless done[j]; p_j = z_j + (rzn_j / rzo_j) p_j.
// p, q, r, z are n x R with leading dimension n.
void launch_coldot(int64_t n, int R, const double *a, int64_t lda, const double *b, int64_t ldb, double *out,
                   cudaStream_t st);
void launch_pcg_step(int64_t n, int R, const double *rz, const double *pq, const int *done, const double *p,
                     const double *q, double *x, int64_t ldx, double *r, cudaStream_t st);
void launch_pcg_direction(int64_t n, int R, const double *rz_new, const double *rz_old, const double *z, double *p,
                          cudaStream_t st);
// y = A x for column-major x, y (leading dimensions ldx, ldy). With `scratch` (2 n R doubles) and
// R >= SPMV_ROWS_MIN_R, x is transposed to row-major there, multiplied with every row's right-hand
// sides contiguous, and the result transposed back (the column-major gather reads one sector per
// entry and right-hand side).
constexpr int SPMV_ROWS_MIN_R = 4;
void launch_spmv(int64_t n, const int64_t *ptr, const int32_t *idx, const double *val, const double *x, int64_t ldx,
                 double *y, int64_t ldy, int R, cudaStream_t st, double *scratch = nullptr);
// Copies the L panels out into the reference's packed trapezoids (dst offsets per supernode).
void launch_pack_trapezoids(const Tree &t, bool fp32, int64_t ns, const int64_t *toff, double *dst,
                            cudaStream_t st);

}  // namespace fc
