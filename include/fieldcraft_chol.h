/* fieldcraft_chol.h — C ABI of the B200 numeric phase of FieldCraft's supernodal Cholesky.
 *
 * The reference's API for this path is Rust (crates/solver/src/cholesky.rs):
 *   UpperColumns (:102-107), Factor::new(a, max_entries) (:1545), Factor::entries (:1557),
 *   Factor::solve (:1562), Factor::solve_many (:1568), FactorError (:346-361),
 *   and the crate-private Symbolic (:1195-1207) whose arrays a Rust caller hands over.
 * Every entry point below names the reference item it replaces. Plain pointers and sizes only;
 * no C++ exceptions cross this boundary; every call returns an FC_* code and fills *status
 * (when status is not NULL) with the code and, for a numeric failure, the column.
 *
 * Index types: row pointers int64, row/column indices int32, values double (FP64).
 * Host buffers are caller-owned; device memory is owned by the handle; one CUDA stream per
 * handle (settable). Distinct handles may be used from distinct threads.
 */
#ifndef FIELDCRAFT_CHOL_H
#define FIELDCRAFT_CHOL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Codes: FactorError one to one (cholesky.rs:346-361), then the boundary's own. */
#define FC_OK 0
#define FC_NOT_POSITIVE_DEFINITE 1 /* FactorError::NotPositiveDefinite { column } */
#define FC_SINGULAR 2              /* FactorError::Singular { column } (LDLT; unused by Cholesky) */
#define FC_TOO_LARGE 3             /* FactorError::TooLarge { entries, limit } */
#define FC_OUT_OF_MEMORY 4         /* FactorError::OutOfMemory { entries } */
#define FC_INTERNAL 5              /* FactorError::Internal(String) */
#define FC_CANCELLED 6             /* FactorError::Cancelled */
#define FC_TIMEOUT 7               /* a bounded device wait gave up */
#define FC_INVALID_ARGUMENT 8      /* solver::Error::Internal("right-hand side length") and bad pointers */
#define FC_CUDA_ERROR 9            /* the CUDA runtime refused a call (no device, launch failure) */

/* Precision of the numeric phase. */
#define FC_PRECISION_FP64 0
#define FC_PRECISION_FP32_IR 1 /* FP32 factor of S A S, every diagonal block in FP64; FP64 refinement */
/* FP64 symmetric indefinite P A P^T = L D L^T (LdltFactor, crates/solver/src/ldlt.rs): bounded
 * Bunch-Kaufman pivots inside supernodes, on the same analysis; values (fc_chol_values, the
 * reference's Block::values), inertia (fc_chol_inertia) and solves through fc_chol_solve and
 * fc_chol_solve_device (the first solve after a factorisation folds the pivot orders into the
 * solve's structure, which waits for the stream), and fc_chol_refine_solve_device by plain
 * refinement (FC_OPTION_REFINEMENT = 1; conjugate gradients needs a definite preconditioner);
 * no-alloc and persistent solves return FC_INVALID_ARGUMENT. A column with no pivot is
 * FC_SINGULAR (FactorError::Singular). */
#define FC_PRECISION_LDLT 2

typedef struct fc_status {
  int32_t code;
  int32_t reserved;
  int64_t column;  /* original column of a NotPositiveDefinite / Singular pivot, else -1 */
  int64_t entries; /* TooLarge / OutOfMemory: entries of the factor */
  int64_t limit;   /* TooLarge: the cap */
  char message[224];
} fc_status;

typedef struct fc_symbolic fc_symbolic;
typedef struct fc_chol fc_chol;

/* ---- symbolic analysis (replaces Symbolic::new, cholesky.rs:1212-1378) --------------------------
 * The upper triangle of a symmetric matrix by columns (UpperColumns, cholesky.rs:102-107): column
 * k holds rows i <= k, sorted; ptr[n+1], idx[ptr[n]]. Refused with FC_TOO_LARGE before any
 * numeric memory when the factor would hold more than max_entries entries (cholesky.rs:1217). */
int fc_symbolic_analyse(int64_t n, const int64_t *ptr, const int32_t *idx, uint64_t max_entries,
                        fc_symbolic **out, fc_status *status);
void fc_symbolic_free(fc_symbolic *sym);

/* Batches (no reference counterpart; the reference factors one system at a time): `count`
 * independent systems, system b's upper triangle by columns in n[b], ptr[b], idx[b], analysed as
 * the one block-diagonal matrix diag(A_0, A_1, ...). Its elimination forest is the union of the
 * systems' trees, so no supernode spans two systems, and one handle made from the result
 * (fc_chol_create) factors and solves every system in the same launches: values and right-hand
 * sides end to end, system b's unknowns from offsets[b] (offsets[count + 1] is filled; the last is
 * the total). FC_TOO_LARGE when the whole batch's factor would pass max_entries. */
int fc_chol_batch_analyse(int32_t count, const int64_t *n, const int64_t *const *ptr, const int32_t *const *idx,
                          uint64_t max_entries, fc_symbolic **out, int64_t *offsets, fc_status *status);
/* A column of the batch (a failing pivot's, FC_NOT_POSITIVE_DEFINITE) as its system and that
 * system's own column. */
int fc_chol_batch_locate(int32_t count, const int64_t *offsets, int64_t column, int32_t *system, int64_t *local);

/* The arrays of the reference's Symbolic, for a caller that ran its own analysis (the Rust
 * side) or wants to check this one. Field meanings follow cholesky.rs:385-415, 728-737,
 * 1195-1207; the update lists are by target supernode in CSR form. */
typedef struct fc_symbolic_arrays {
  int64_t n, ns, entries, nnz, rows_len, lower_len, updates_len, tasks_len, top_len;
  const int64_t *perm;     /* [n]      perm[k]: original column of factor column k */
  const int64_t *first;    /* [ns+1]   Structure.first */
  const int64_t *rptr;     /* [ns+1]   Structure.rptr */
  const int32_t *rows;     /* [rows_len] Structure.rows */
  const int64_t *upper_ptr;/* [n+1]    Pattern.upper_ptr */
  const int32_t *upper_idx;/* [nnz]    Pattern.upper_idx */
  const int64_t *lptr;     /* [n+1]    Pattern.ptr */
  const int32_t *lidx;     /* [lower_len] Pattern.idx */
  const int64_t *slot;     /* [nnz]    Pattern.slot */
  const int32_t *crow;     /* [nnz]    Pattern.coords .0 */
  const int32_t *ccol;     /* [nnz]    Pattern.coords .1 */
  const int64_t *uptr;     /* [ns+1]   updates by target */
  const int64_t *uk, *up1, *up2; /* [updates_len] Update { k, p1, p2 } */
  const int64_t *task_lo, *task_hi; /* [tasks_len] Symbolic.tasks */
  const int64_t *top;      /* [top_len] Symbolic.top */
} fc_symbolic_arrays;

/* Views of the analysis' arrays (valid while sym lives). */
int fc_symbolic_get(const fc_symbolic *sym, fc_symbolic_arrays *out);
/* An analysis from a caller's arrays (copied). FC_INVALID_ARGUMENT for a negative length or a
 * missing array; FC_INTERNAL (with the reason in the message) unless first/rptr span the columns
 * and rows, each supernode's rows are its own columns followed by increasing rows below, perm is
 * a permutation, upper_ptr spans the nnz entries, and every (crow, ccol) lies in the lower
 * triangle. The update lists, tasks and top are copied for fc_symbolic_get only. */
int fc_symbolic_import(const fc_symbolic_arrays *in, fc_symbolic **out, fc_status *status);

/* ---- numeric factorisation on a B200 (replaces Factor::from_symbolic, cholesky.rs:1549-1554) ----
 * fc_chol_create uploads the structure and plans the level schedule on `device`; no values yet.
 * It copies what it needs: sym may be freed afterwards. FC_TOO_LARGE (entries = the panel's size,
 * limit = 2^31 - 1) when one supernode's panel m x w holds more entries than 32-bit offsets
 * address; FC_OUT_OF_MEMORY when the device arenas do not fit. */
int fc_chol_create(const fc_symbolic *sym, int precision, int device, fc_chol **out, fc_status *status);
void fc_chol_destroy(fc_chol *h);
/* Runs on this CUDA stream (cudaStream_t); NULL for the handle's own stream. */
int fc_chol_set_stream(fc_chol *h, void *stream);

/* Symbolic::numeric + Symbolic::factor (cholesky.rs:1392-1416, 1443-1529) from host values:
 * upper_val[nnz] in the order of the analysed UpperColumns. cancel, when not NULL, is read
 * between levels of the supernodal tree (the reference reads its progress between
 * supernodes, :1476-1484): non-zero stops with FC_CANCELLED. Errors: FC_NOT_POSITIVE_DEFINITE
 * with the original column of the first failing pivot in postorder (:1506-1528). */
int fc_chol_factor(fc_chol *h, const double *upper_val, int64_t nnz, const volatile int32_t *cancel,
                   fc_status *status);
/* The same from values already in device memory; synchronises the stream before returning. */
int fc_chol_factor_device(fc_chol *h, const double *d_upper_val, int64_t nnz, fc_status *status);
/* Enqueues the factorisation without waiting; fc_chol_check reads its status afterwards. */
int fc_chol_factor_device_async(fc_chol *h, const double *d_upper_val, int64_t nnz);
int fc_chol_check(fc_chol *h, fc_status *status);

/* Factor::entries (cholesky.rs:1557): entries of L (the reference's count, trapezoids). */
int64_t fc_chol_entries(const fc_chol *h);
/* Factor::solve / solve_many (cholesky.rs:1562-1570): solves A x = b in place for nrhs
 * right-hand sides stored column-major in b (column j at b + j*ld, ld >= n). */
int fc_chol_solve(fc_chol *h, double *b, int32_t nrhs, int64_t ld, fc_status *status);
/* The same on device memory; synchronises before returning. */
int fc_chol_solve_device(fc_chol *h, double *d_b, int32_t nrhs, int64_t ld, fc_status *status);
int fc_chol_solve_device_async(fc_chol *h, double *d_b, int32_t nrhs, int64_t ld);
/* A solve that allocates no device memory. It has no counterpart in the reference: it exists for
 * callers that cannot call cudaMalloc, such as a host application whose own allocator owns all of
 * the device's memory under a fixed budget, where an extra allocation could fail or fragment
 * that pool. It solves like fc_chol_solve_device (d_b column-major, leading dimension ld, in
 * place), but takes its working memory (the solve vectors and task lists) from one file-scope
 * device array of FC_NOALLOC_SCRATCH_BYTES that the library reserves on every device it is
 * loaded on, until the process exits. Calls that need more than that are refused with
 * FC_INVALID_ARGUMENT and a message giving the size needed. The first call on each device looks
 * the array's address up (cudaGetSymbolAddress); make that first call before any stream capture.
 * The address is kept for the life of the process: a caller that resets the device
 * (cudaDeviceReset) or tears down and recreates its context must not call this entry point
 * again in that process.
 * All calls share the one array and each leaves its contents behind: calls whose work overlaps on
 * the GPU (several handles or threads on one device at once) race on it. Synchronises before
 * returning. */
#define FC_NOALLOC_SCRATCH_BYTES (32u << 20)
int fc_chol_solve_device_noalloc(fc_chol *h, double *d_b, int32_t nrhs, int64_t ld, fc_status *status);
/* The factor's values in the reference's layout: supernode by supernode, each its lower
 * trapezoid by columns (column c holds rows c..m, cholesky.rs:418-425, 1534-1542). dst has
 * fc_chol_entries(h) doubles. */
int fc_chol_values(fc_chol *h, double *dst, fc_status *status);
/* The LDL^T factor's pivots (ldlt.rs:399-447, Pivot): per column in postorder its kind (0 a 1 x 1
 * pivot, 1 / 2 the first / second column of a 2 x 2) and the supernode-local column at that pivot
 * position. n entries each; FC_INVALID_ARGUMENT for a Cholesky factor. */
int fc_chol_ldlt_pivots(fc_chol *h, int8_t *pivots, int32_t *order, fc_status *status);
/* LdltFactor::inertia and two_by_two (ldlt.rs:399-447): the counts of positive and negative
 * eigenvalues of A (Sylvester's law on D) and of 2 x 2 pivots; a Cholesky factor's are (n, 0, 0). */
int fc_chol_inertia(fc_chol *h, int64_t *positive, int64_t *negative, int64_t *two_by_two, fc_status *status);

/* Solve A x = b to a relative residual in FP64 around the handle's factor (the mixed-precision
 * mode's FP32 factor of S A S, or the FP64 factor) as the preconditioner M: by default conjugate
 * gradients preconditioned by M, one recurrence per right-hand side, from x = 0 (the first step is
 * x = M b); FC_OPTION_REFINEMENT = 1 selects plain refinement x += M (b - A x). Convergence is
 * judged on the true residual b - A x (FP64 SpMV on A by rows: d_ptr[n+1], d_idx, d_val, both
 * triangles, the matrix the factor was made from) until ||r_j|| <= tol ||b_j|| for every
 * right-hand side j or max_iter solves. No counterpart in the reference (its only refinement,
 * Symmetric::solve_refined, crates/solver/src/ldlt.rs:529-566, is in working precision).
 * b and x are column-major n x nrhs with leading dimension ld, in device memory. relres (host,
 * nrhs entries, may be NULL) receives the final relative residuals, *iterations the solves done.
 * FC_TIMEOUT when max_iter solves did not reach tol (x holds the last iterate). */
int fc_chol_refine_solve_device(fc_chol *h, const int64_t *d_ptr, const int32_t *d_idx, const double *d_val,
                                const double *d_b, double *d_x, int32_t nrhs, int64_t ld, double tol,
                                int32_t max_iter, double *relres, int32_t *iterations, fc_status *status);

/* Plan statistics: 0 levels, 1 launches of the factor, 2 bytes of L on device, 3 bytes of the
 * update matrices, 4 supernodes, 5 factor flops (sum of column counts squared), 6 GEMM tasks,
 * 7 kernels launched by the last factorisation, 8 kernels launched by the last solve, 9 flops of
 * the factor's GEMM tasks, 10 flops of the last solve plan's GEMM tasks, 11 the ordinal among the
 * factor's GEMM launches of the one with the most flops, 12 the same among the launches whose
 * tasks all have K <= 64 (the panels' updates of later columns), 13 and 14 the tasks of the
 * persistent solve's forward and backward lists, 15 flops of the factor's update GEMM launches
 * alone (9 without the diagonal blocks' inverse doubling). */
int64_t fc_chol_stat(const fc_chol *h, int what);

/* Execution options of a handle (no reference counterpart). Each takes effect from the next solve.
 *   FC_OPTION_SOLVE_SCHEDULE   0: the solve runs level by level, one launch per panel step
 *                              (default); 1: as two persistent dependency-driven launches.
 *   FC_OPTION_WAIT_LIMIT_NS    a wait of the persistent solve longer than this many nanoseconds
 *                              fails the solve with FC_TIMEOUT (default 4e9).
 *   FC_OPTION_PLANT_UNMET_WAIT (tests) value != 0: the next solve plan holds one dependency that no
 *                              task meets, so that solve ends with FC_TIMEOUT after the limit.
 *   FC_OPTION_TRACE            value != 0: the persistent solve records per task when it was taken,
 *                              when its inputs were ready and when it was done (fc_chol_trace_read).
 *   FC_OPTION_REFINEMENT       fc_chol_refine_solve_device's iteration: 0 conjugate gradients
 *                              preconditioned by the factor (default), 1 plain refinement
 *                              x += M (b - A x).
 *   FC_OPTION_FP32_UPDATES     the mixed-precision factor's update-matrix products: 0 on tcgen05
 *                              in 128 x 128 tiles (default), 1 on mma.sync in 64 x 64 tiles
 *                              (re-plans the factorisation; takes effect from the next one).
 *   FC_OPTION_SOLVE_CLUSTER    the level-by-level solve's products in launches with few output
 *                              tiles: 0 K split in chunks of separate CTAs, the last adding the
 *                              partials (default); 1 each tile's K split over a cluster of 8 CTAs
 *                              that add their partials through distributed shared memory.
 *   FC_OPTION_SOLVE_NARROW     with at most 16 right-hand sides, the level-by-level solve's
 *                              products in 64 x 8 or 64 x 16 tiles: 1 (default) on, 0 in the
 *                              64 x 64 tiles of more right-hand sides. The results are the same
 *                              bit for bit (the same products in the same order).
 *   FC_OPTION_SOLVE_DEEP       1 (default): with at most 16 right-hand sides, the level-by-level
 *                              solve's product launches of fewer CTAs than two per SM run with an
 *                              8-stage copy ring (more bytes in flight a CTA); 0: the factor's
 *                              3-stage ring. The same bits.
 *   FC_OPTION_CHILDREN_FIRST   1 (default): a supernode wider than 16 columns with children gets
 *                              its update matrix's children contributions summed first, beside
 *                              its panels, and its update product subtracts -L21 L21^T from them;
 *                              0: the product stores -L21 L21^T and the children are added after
 *                              it (re-plans the factorisation; the factor agrees to rounding).
 *   FC_OPTION_SOLVE_PDL        1: the level-by-level solve's kernels are launched as programmatic
 *                              dependents (each starts while the one before it in its stream
 *                              finishes, loading its tasks and factor tiles before it waits for
 *                              that kernel); 0 (default): ordinary launches. The same bits. */
#define FC_OPTION_SOLVE_SCHEDULE 1
#define FC_OPTION_WAIT_LIMIT_NS 2
#define FC_OPTION_PLANT_UNMET_WAIT 3
#define FC_OPTION_TRACE 4
#define FC_OPTION_REFINEMENT 5
#define FC_OPTION_FP32_UPDATES 6
#define FC_OPTION_SOLVE_CLUSTER 7
#define FC_OPTION_SOLVE_NARROW 8
#define FC_OPTION_SOLVE_DEEP 9
#define FC_OPTION_CHILDREN_FIRST 10
#define FC_OPTION_SOLVE_PDL 11
int fc_chol_option(fc_chol *h, int32_t option, int64_t value);
/* The last traced persistent solve: 4 words per task, forward tasks then backward (fc_chol_stat 13
 * and 14 count them): taken, ready and done times in nanoseconds (%globaltimer), and kind << 32 |
 * SM index (kinds 0 assembly, 1 panel, 2 gather, 3 product, 4 reduction). Copies at most cap words;
 * returns the number of tasks (0 when not tracing; negative: -FC_INVALID_ARGUMENT, -FC_CUDA_ERROR). */
int64_t fc_chol_trace_read(fc_chol *h, int64_t *out, int64_t cap);

/* Per-launch timing with CUDA events on the handle's stream (no reference counterpart: the
 * measurement hook of the benchmark). enable != 0 starts recording; fc_chol_profile_read waits for
 * the stream and returns, per launch kind, the summed milliseconds and the launch count (arrays of
 * `kinds` entries), then clears them. Kinds: 0 front assembly, 1 panel (factor,
 * invert and solve below a diagonal block), 3 GEMM of the factor, 10 and 11 the two GEMMs of a
 * doubling step of the diagonal-block inverses, 12 the tcgen05 GEMM of the mixed-precision factor
 * and 15 the packing of its operands; 16 the LDL^T factor's pivoted panel steps, 17 its W21 and D
 * split, 18 its unit lower block inverses;
 * 19 GEMM, 20 front assembly, 22 forward inverse, 23
 * backward inverse of the solve (level by level), 24 forward, 25 backward persistent launch of the
 * solve, 29 forward, 30 backward step of the thin supernodes (32 covers all). */
int fc_chol_profile(fc_chol *h, int enable);
int fc_chol_profile_read(fc_chol *h, double *ms, int64_t *launches, int32_t kinds);
/* The recorded launches one by one, oldest first, without clearing them: kind (as above), level
 * of the supernodal tree, number of tasks (CTAs) and milliseconds. Fills at most cap entries and
 * returns how many are recorded (negative: -FC_INVALID_ARGUMENT or -FC_CUDA_ERROR). */
int64_t fc_chol_profile_launches(fc_chol *h, int32_t *kind, int32_t *level, int32_t *tasks, float *ms, int64_t cap);

/* ---- compressed-row products (Csr::mul, crates/solver/src/sparse.rs:42-50) ---------------------
 * y = A x on the device for nrhs vectors, x and y column-major with leading dimension ld. With 4
 * or more vectors the product goes through row-major copies in scratch of 16 n nrhs bytes taken
 * from the stream-ordered allocator on `stream` and released on it (cudaMallocAsync /
 * cudaFreeAsync); if that allocation fails the column-major kernel runs instead. */
int fc_csr_spmv_device(int64_t n, const int64_t *d_ptr, const int32_t *d_idx, const double *d_val,
                       const double *d_x, double *d_y, int32_t nrhs, int64_t ld, void *stream);

/* Version string of the library. */
const char *fc_version(void);

#ifdef __cplusplus
}
#endif
#endif
