// The pivoted panel of the symmetric indefinite LDL^T (crates/solver/src/ldlt.rs:250-335) on one
// front, written once for a thread block: the device kernel runs it with CUDA threads; the tests
// run the same source with host threads and a barrier, against the oracle, bit for bit.
//
// The front holds a supernode's own columns: m rows x w columns, column-major with leading
// dimension m, entries (r, c) with r >= c meaningful. Columns before the panel are final (L below
// the pivots, D on them); the panel's and later columns hold the front after the earlier panels'
// updates. The panel chooses its pivots among all of the supernode's remaining own columns by
// the bounded Bunch-Kaufman (rook) search, interchanging the front's own rows and columns
// symmetrically, and stores 1 x 1 and 2 x 2 pivots; a 2 x 2 pivot may end it one column late.
// Every product and sum is rounded on its own (no fused multiply-add), in the reference's order,
// so a front's pivots and values are the reference's exactly.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define FC_LDLT_FN __device__ __forceinline__
#define FC_LDLT_HD __host__ __device__ __forceinline__  // arithmetic the host plan shares
#else
#include <cmath>
#define FC_LDLT_FN inline
#define FC_LDLT_HD inline
#endif

namespace fc {
namespace ldlt {

constexpr double ALPHA = 0.6403882032022076;  // (1 + sqrt 17) / 8, ldlt.rs:77
constexpr int ROOK_STEPS = 64;                // ldlt.rs:81
constexpr int PANEL = 64;                     // cholesky.rs:54
constexpr double PIVOT_TOLERANCE = 1e-10;     // cholesky.rs:48
constexpr int MAX_THREADS = 256;
constexpr int8_t PIVOT_ONE = 0, PIVOT_FIRST = 1, PIVOT_SECOND = 2;

#if defined(__CUDACC__)
FC_LDLT_FN double mul(double a, double b) { return __dmul_rn(a, b); }
FC_LDLT_FN double add(double a, double b) { return __dadd_rn(a, b); }
FC_LDLT_FN double sub(double a, double b) { return __dsub_rn(a, b); }
FC_LDLT_FN double magnitude(double x) { return fabs(x); }
FC_LDLT_FN bool finite(double x) { return isfinite(x); }
FC_LDLT_FN bool not_a_number(double x) { return isnan(x); }
#else
FC_LDLT_FN double mul(double a, double b) { return a * b; }
FC_LDLT_FN double add(double a, double b) { return a + b; }
FC_LDLT_FN double sub(double a, double b) { return a - b; }
FC_LDLT_FN double magnitude(double x) { return std::fabs(x); }
FC_LDLT_FN bool finite(double x) { return std::isfinite(x); }
FC_LDLT_FN bool not_a_number(double x) { return std::isnan(x); }
#endif

// One front and its per-column state.
struct Front {
  double *F;            // m x w, column-major, leading dimension m
  int64_t m;
  int w;
  const double *scale;  // [w] the largest |A| of each own column (in the structure's order)
  int32_t *order;       // [w] order[c]: the own column (structure's order) at pivot position c
  int8_t *pivots;       // [w] PIVOT_ONE / PIVOT_FIRST / PIVOT_SECOND
  double *a, *b;        // [m] each: the searched column and a candidate (scratch)
  double *W;            // rows [c1, w) of L D over the panel's columns, ld_w x (c1 - c0)
  int64_t ld_w;         // >= w - c0 - PANEL
};

// Block-shared scratch.
struct Shared {
  double row[PANEL + 1];  // a row of L D over the panel's factored columns
  double best_v[MAX_THREADS];
  int best_i[MAX_THREADS];
  int nan[MAX_THREADS];
};

FC_LDLT_FN double &at(const Front &f, int64_t r, int64_t c) { return f.F[r + c * f.m]; }

template <class T>
FC_LDLT_FN void exchange(T &x, T &y) {
  const T t = x;
  x = y;
  y = t;
}

// row[0..len) <- row D for the columns k0.. (times_d, cholesky.rs:458-481); one thread.
FC_LDLT_FN void times_d(double *row, int len, const Front &f, int k0) {
  int k = 0;
  while (k < len) {
    if (f.pivots[k0 + k] == PIVOT_FIRST) {
      const double x = row[k], y = k + 1 < len ? row[k + 1] : 0.0;
      const double d11 = at(f, k0 + k, k0 + k), d21 = at(f, k0 + k + 1, k0 + k), d22 = at(f, k0 + k + 1, k0 + k + 1);
      row[k] = add(mul(x, d11), mul(y, d21));
      if (k + 1 < len) row[k + 1] = add(mul(x, d21), mul(y, d22));
      k += 2;
    } else {
      row[k] = mul(row[k], at(f, k0 + k, k0 + k));
      k += 1;
    }
  }
}

// Column c (local, >= k) of the part still to factor, rows [k, m), into out: the front's entries
// less the products with the panel's factored columns [c0, k) (Block::current, ldlt.rs:173-192).
template <class Block>
FC_LDLT_FN void current(Block &blk, Shared &sh, const Front &f, int c0, int k, int c, double *out) {
  if (blk.tid() == 0) {
    for (int q = c0; q < k; ++q) sh.row[q - c0] = at(f, c, q);
    times_d(sh.row, k - c0, f, c0);
  }
  blk.sync();
  for (int64_t r = k + blk.tid(); r < f.m; r += blk.size()) {
    double v = r >= c ? at(f, r, c) : at(f, c, r);
    for (int q = c0; q < k; ++q) v = sub(v, mul(at(f, r, q), sh.row[q - c0]));
    out[r] = v;
  }
  blk.sync();
}

// The largest magnitude of v over [lo, hi) except `skip`, with the lowest such index (largest,
// ldlt.rs:145-163). Returns false when an entry is not a number (the reference's NaN, which its
// callers treat as a singular column). Every thread gets the same answer.
template <class Block>
FC_LDLT_FN bool largest(Block &blk, Shared &sh, const double *v, int lo, int hi, int skip, int &index, double &value) {
  double bv = 0.0;
  int bi = lo, bn = 0;
  for (int i = lo + blk.tid(); i < hi; i += blk.size()) {
    if (i == skip) continue;
    const double x = magnitude(v[i]);
    if (not_a_number(x)) {
      bn = 1;
    } else if (x > bv) {
      bv = x;
      bi = i;
    }
  }
  sh.best_v[blk.tid()] = bv;
  sh.best_i[blk.tid()] = bi;
  sh.nan[blk.tid()] = bn;
  blk.sync();
  double v0 = 0.0;
  int i0 = lo, n0 = 0;
  for (int t = 0; t < blk.size(); ++t) {
    n0 |= sh.nan[t];
    const double x = sh.best_v[t];
    if (x > v0 || (x == v0 && x > 0.0 && sh.best_i[t] < i0)) {
      v0 = x;
      i0 = sh.best_i[t];
    }
  }
  blk.sync();
  index = i0;
  value = v0;
  return n0 == 0;
}

// Symmetric interchange of local columns p and q (both at pivot positions >= k) in the front,
// the order and the scratch columns (interchange and Block::swap, ldlt.rs:128-143, 194-204).
// Every thread has read what the pivot decision needs (the scratch columns' entries) before
// any thread moves them: the first barrier.
template <class Block>
FC_LDLT_FN void interchange(Block &blk, const Front &f, int p, int q, double *a, double *b) {
  if (p == q) return;
  if (p > q) exchange(p, q);
  blk.sync();
  const int t = blk.tid(), T = blk.size();
  for (int c = t; c < p; c += T) exchange(at(f, p, c), at(f, q, c));
  for (int c = p + 1 + t; c < q; c += T) exchange(at(f, c, p), at(f, q, c));
  for (int64_t r = q + 1 + t; r < f.m; r += T) exchange(at(f, r, p), at(f, r, q));
  if (t == 0) {
    exchange(at(f, p, p), at(f, q, q));
    exchange(f.order[p], f.order[q]);
    exchange(a[p], a[q]);
    exchange(b[p], b[q]);
  }
  blk.sync();
}

// A 1 x 1 pivot at k from the current column (Block::one, ldlt.rs:206-221).
template <class Block>
FC_LDLT_FN void one(Block &blk, const Front &f, int k, const double *col) {
  const double d = col[k];
  for (int64_t r = k + 1 + blk.tid(); r < f.m; r += blk.size()) at(f, r, k) = col[r] / d;
  if (blk.tid() == 0) {
    at(f, k, k) = d;
    f.pivots[k] = PIVOT_ONE;
  }
  blk.sync();
}

// A 2 x 2 pivot at k, k + 1 from the current columns a (k) and b (k + 1) (Block::two,
// ldlt.rs:223-248).
template <class Block>
FC_LDLT_FN void two(Block &blk, const Front &f, int k, const double *a, const double *b) {
  const double d11 = a[k], d21 = a[k + 1], d22 = b[k + 1];
  const double det = sub(mul(d11, d22), mul(d21, d21));
  for (int64_t r = k + 2 + blk.tid(); r < f.m; r += blk.size()) {
    const double x = a[r], y = b[r];
    at(f, r, k) = sub(mul(x, d22), mul(y, d21)) / det;
    at(f, r, k + 1) = sub(mul(y, d11), mul(x, d21)) / det;
  }
  if (blk.tid() == 0) {
    at(f, k, k) = d11;
    at(f, k + 1, k) = d21;
    at(f, k + 1, k + 1) = d22;
    f.pivots[k] = PIVOT_FIRST;
    f.pivots[k + 1] = PIVOT_SECOND;
  }
  blk.sync();
}

// The panel from column c0 (Block::panel, ldlt.rs:250-335). Returns -1, or the own column (the
// structure's order) found singular; *end receives where the panel ended and *twos the 2 x 2
// pivots it made. Every thread returns the same.
template <class Block>
FC_LDLT_FN int panel(Block &blk, Shared &sh, const Front &f, int c0, int *end_out, int *twos) {
  const int w = f.w;
  const int end = c0 + PANEL < w ? c0 + PANEL : w;
  double *a = f.a, *b = f.b;
  int k = c0;
  *twos = 0;
  while (k < end) {
    current(blk, sh, f, c0, k, k, a);
    const double akk = magnitude(a[k]);
    int r0;
    double omega_k;
    const bool numbers = largest(blk, sh, a, k + 1, w, -1, r0, omega_k);
    if (!finite(akk) || !numbers || !finite(omega_k)) return f.order[k];
    bool pair = false;
    int p = k, pi = k, pr = k;
    if (!(akk >= ALPHA * omega_k)) {
      // the rook search: `a` holds column i, `b` the candidate r
      int i = k, r = r0, step = 0;
      double omega_i = omega_k;
      for (;;) {
        current(blk, sh, f, c0, k, r, b);
        int s;
        double omega_r;
        const bool fine = largest(blk, sh, b, k, w, r, s, omega_r);
        const double arr = magnitude(b[r]);
        if (!finite(arr) || !fine || !finite(omega_r)) return f.order[k];
        step += 1;
        if (arr >= ALPHA * omega_r) {
          exchange(a, b);
          p = r;
          break;
        }
        if (omega_r <= omega_i || step >= ROOK_STEPS) {
          pair = true;
          pi = i;
          pr = r;
          break;
        }
        exchange(a, b);
        i = r;
        omega_i = omega_r;
        r = s;
      }
    }
    if (!pair) {
      interchange(blk, f, k, p, a, b);
      if (!(magnitude(a[k]) > PIVOT_TOLERANCE * f.scale[f.order[k]])) return f.order[k];
      one(blk, f, k, a);
      k += 1;
    } else {
      // i to k, then r to k + 1 (r was at k if i took its place)
      interchange(blk, f, k, pi, a, b);
      interchange(blk, f, k + 1, pr == k ? pi : pr, a, b);
      const double offdiagonal = magnitude(a[k + 1]);
      const double s0 = f.scale[f.order[k]], s1 = f.scale[f.order[k + 1]];
      const double size = s0 < s1 ? s1 : s0;
      if (!(offdiagonal > PIVOT_TOLERANCE * size)) return f.order[k];
      two(blk, f, k, a, b);
      *twos += 1;
      k += 2;
    }
  }
  *end_out = k;
  return -1;
}

// W = L D for the rows [c1, w) over the panel's columns [c0, c1): the coefficients of the update
// of the later own columns by the panel (products' Y, cholesky.rs:531-548).
template <class Block>
FC_LDLT_FN void panel_w(Block &blk, const Front &f, int c0, int c1) {
  const int kw = c1 - c0;
  for (int64_t r = c1 + blk.tid(); r < f.w; r += blk.size()) {
    double *wr = f.W + (r - c1);
    int k = 0;
    while (k < kw) {
      const int c = c0 + k;
      if (f.pivots[c] == PIVOT_FIRST) {
        const double x = at(f, r, c), y = at(f, r, c + 1);
        const double d11 = at(f, c, c), d21 = at(f, c + 1, c), d22 = at(f, c + 1, c + 1);
        wr[k * f.ld_w] = add(mul(x, d11), mul(y, d21));
        wr[(k + 1) * f.ld_w] = add(mul(x, d21), mul(y, d22));
        k += 2;
      } else {
        wr[k * f.ld_w] = mul(at(f, r, c), at(f, c, c));
        k += 1;
      }
    }
  }
  blk.sync();
}

// W21 = L21 D: the rows [w, m) of the front times its block diagonal, ld_out x w, for the update
// matrix U = -L21 W21^T the parent assembles (products' Y for a descendant, cholesky.rs:531-548,
// with times_d's operations).
template <class Block>
FC_LDLT_FN void front_w21(Block &blk, const Front &f, double *out, int64_t ld_out) {
  for (int64_t r = f.w + blk.tid(); r < f.m; r += blk.size()) {
    double *o = out + (r - f.w);
    int k = 0;
    while (k < f.w) {
      if (f.pivots[k] == PIVOT_FIRST) {
        const double x = at(f, r, k), y = at(f, r, k + 1);
        const double d11 = at(f, k, k), d21 = at(f, k + 1, k), d22 = at(f, k + 1, k + 1);
        o[k * ld_out] = add(mul(x, d11), mul(y, d21));
        o[(k + 1) * ld_out] = add(mul(x, d21), mul(y, d22));
        k += 2;
      } else {
        o[k * ld_out] = mul(at(f, r, k), at(f, k, k));
        k += 1;
      }
    }
  }
  blk.sync();
}

// D out of a factored front: d[c] receives D's diagonal and e[c] its subdiagonal (the 2 x 2
// pivots' d21 at their first column, else 0); the front's own block becomes unit lower (ones on
// the diagonal, zeros where a 2 x 2 pivot's d21 was), the form the triangular solve reads.
template <class Block>
FC_LDLT_FN void split_d(Block &blk, const Front &f, double *d, double *e) {
  for (int c = blk.tid(); c < f.w; c += blk.size()) {
    d[c] = at(f, c, c);
    e[c] = f.pivots[c] == PIVOT_FIRST ? at(f, c + 1, c) : 0.0;
  }
  blk.sync();
  for (int c = blk.tid(); c < f.w; c += blk.size()) {
    at(f, c, c) = 1.0;
    if (f.pivots[c] == PIVOT_FIRST) at(f, c + 1, c) = 0.0;
  }
  blk.sync();
}

// y <- D^-1 y for the unknowns [0, n) of R right-hand sides (row-major, y[i * R + j]), D given by
// its diagonal d, subdiagonal e and the pivot kinds (the solve's block step, cholesky.rs:946-974).
// One thread per pivot group: a 1 x 1 pivot or the first column of a 2 x 2 one.
FC_LDLT_FN void apply_d_inverse(int64_t i, int R, const double *d, const double *e, const int8_t *pivots, double *y) {
  if (pivots[i] == PIVOT_SECOND) return;
  if (pivots[i] == PIVOT_FIRST) {
    const double d11 = d[i], d21 = e[i], d22 = d[i + 1];
    const double det = sub(mul(d11, d22), mul(d21, d21));
    for (int j = 0; j < R; ++j) {
      const double p = y[i * R + j], q = y[(i + 1) * R + j];
      y[i * R + j] = sub(mul(d22, p), mul(d21, q)) / det;
      y[(i + 1) * R + j] = sub(mul(d11, q), mul(d21, p)) / det;
    }
  } else {
    for (int j = 0; j < R; ++j) y[i * R + j] = y[i * R + j] / d[i];
  }
}

// X = L^-1 for an nb x nb unit lower block of a front (nb <= 64; L's diagonal is not read),
// column-major with leading dimension ldx: column j by forward substitution, x_i = -sum over
// k in [j, i) of L(i, k) x_k, summed in k order from zero. One thread per column; the strictly
// upper part of X is left as it is (zero in the solve's inverse arena).
template <class Block>
FC_LDLT_FN void unit_lower_inverse(Block &blk, const double *Lb, int64_t ldl, int nb, double *X, int64_t ldx) {
  for (int j = blk.tid(); j < nb; j += blk.size()) {
    double *x = X + (int64_t)j * ldx;
    x[j] = 1.0;
    for (int i = j + 1; i < nb; ++i) {
      double s = 0.0;
      for (int k = j; k < i; ++k) s = add(s, mul(Lb[i + (int64_t)k * ldl], x[k]));
      x[i] = -s;
    }
  }
  blk.sync();
}

// Rows [w, m) of every own column of a front put in a new order: row w + i takes the old row
// w + from[i] (from: a permutation of [0, m - w)). One column at a time through `tmp` (m - w
// entries), threads over its rows.
template <class Block>
FC_LDLT_FN void permute_rows_below(Block &blk, const Front &f, const int32_t *from, double *tmp) {
  const int64_t u = f.m - f.w;
  for (int c = 0; c < f.w; ++c) {
    double *col = f.F + f.w + (int64_t)c * f.m;
    for (int64_t i = blk.tid(); i < u; i += blk.size()) tmp[i] = col[from[i]];
    blk.sync();
    for (int64_t i = blk.tid(); i < u; i += blk.size()) col[i] = tmp[i];
    blk.sync();
  }
}

// The update of the later own columns by a panel that ended at c1, as tiles of at most 64 x 64:
// the front's rows [c1, m) of its columns [c1, w), lower part only; column blocks of 64 from c1,
// in each the row blocks from the diagonal down. Tile `slot` of that list, or false past its end.
struct Tile {
  int64_t i0;   // first row
  int j0;       // first column
  int M, N;     // rows, columns
  bool lower;   // a diagonal tile: only rows >= columns
};
constexpr int TILE_ROWS = 64;

FC_LDLT_HD bool update_tile(int64_t m, int w, int c1, int64_t slot, Tile &t) {
  for (int j0 = c1; j0 < w; j0 += TILE_ROWS) {
    const int64_t rows = (m - j0 + TILE_ROWS - 1) / TILE_ROWS;
    if (slot < rows) {
      t.i0 = j0 + slot * TILE_ROWS;
      t.j0 = j0;
      t.M = (int)(m - t.i0 < TILE_ROWS ? m - t.i0 : TILE_ROWS);
      t.N = w - j0 < TILE_ROWS ? w - j0 : TILE_ROWS;
      t.lower = slot == 0;
      return true;
    }
    slot -= rows;
  }
  return false;
}

// The tiles of that update: at most this many for a panel that ends at c1 or later (the count
// falls as c1 grows), so a plan sized for the earliest end holds every case.
FC_LDLT_HD int64_t update_tiles(int64_t m, int w, int c1) {
  int64_t count = 0;
  for (int j0 = c1; j0 < w; j0 += TILE_ROWS) count += (m - j0 + TILE_ROWS - 1) / TILE_ROWS;
  return count;
}

}  // namespace ldlt
}  // namespace fc
