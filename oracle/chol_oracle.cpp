// ORACLE — test infrastructure, not product code. A CPU restatement of the reference's
// supernodal Cholesky (crates/solver/src/cholesky.rs, FieldCraft 0.8.1), of its symmetric
// indefinite LDL^T on the same structure (crates/solver/src/ldlt.rs: bounded Bunch-Kaufman pivots
// inside supernodes) and of its sparse product (crates/solver/src/sparse.rs:42-50), used only by
// the tests, by the smoke check and by the benchmark's CPU-baseline leg as the checker and the
// timed CPU reference. Nothing in the product links or calls it.
//
// It follows the reference's operation order entry by entry: sums over a supernode's columns
// in column order from zero, updates subtracted in supernode order, panels of PANEL columns,
// tiles of TILE rows, no fused multiply-add (built with -ffp-contract=off, no -ffast-math), so
// each entry of the factor is the one the reference computes. The reference is Rust with
// crates.io dependencies that are not present here, so it cannot be built; the restatement is
// pinned by every known answer the reference's own tests hold, among them the FNV-1a
// fingerprints the reference froze of the bits of its Cholesky solution and of four LDL^T
// factors and solutions, which this code reproduces bit for bit (tests/test_oracle_pins.py,
// tests/test_oracle_ldlt.py, which cite each).
//
// Threads: subtree tasks run concurrently and large dense kernels split their row tiles, as in
// cholesky.rs:1443-1529 and :625-629; neither changes any entry's operations.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

namespace {

constexpr int64_t NONE = -1;
constexpr double PIVOT_TOLERANCE = 1e-10;  // cholesky.rs:48
constexpr int64_t TILE = 64;               // cholesky.rs:51
constexpr int64_t PANEL = 64;              // cholesky.rs:54
constexpr int64_t MR = 8;                  // cholesky.rs:57 (scalar.rs PACKED_ROWS)
constexpr int64_t NR = 4;                  // cholesky.rs:61
constexpr int64_t BLOCK = 3;               // cholesky.rs:221
constexpr uint64_t PARALLEL_WORK = 1ull << 21;  // cholesky.rs:67
constexpr uint64_t SUBTREE_SHARE = 256;         // cholesky.rs:97
constexpr int GROUP = 6;                        // cholesky.rs:870

enum Code : int32_t {
  OK = 0, NOT_POSITIVE_DEFINITE = 1, SINGULAR = 2, TOO_LARGE = 3, OUT_OF_MEMORY = 4, INTERNAL = 5, CANCELLED = 6
};

// The pivots of an LDL^T factor's block diagonal D per column (cholesky.rs:447-457): a 1 x 1
// pivot, or the first or second column of a 2 x 2 one.
enum PivotKind : int8_t { PIVOT_ONE = 0, PIVOT_FIRST = 1, PIVOT_SECOND = 2 };
constexpr double ALPHA = 0.6403882032022076;  // ldlt.rs:77: (1 + sqrt 17) / 8
constexpr int ROOK_STEPS = 64;                // ldlt.rs:81

struct Error {
  Code code;
  int64_t column;
};

uint64_t sat_add(uint64_t a, uint64_t b) { return a + b < a ? UINT64_MAX : a + b; }
uint64_t sat_mul(uint64_t a, uint64_t b) { return (a && b && a > UINT64_MAX / b) ? UINT64_MAX : a * b; }

// ---- a small pool: parallel_for over an index range; nested calls run serially --------------
thread_local bool in_pool = false;
int g_threads = 1;

void parallel_for(int64_t count, const std::function<void(int64_t)> &fn) {
  if (count <= 0) return;
  if (g_threads <= 1 || in_pool || count == 1) {
    for (int64_t i = 0; i < count; ++i) fn(i);
    return;
  }
  std::atomic<int64_t> next{0};
  auto work = [&]() {
    in_pool = true;
    for (;;) {
      int64_t i = next.fetch_add(1);
      if (i >= count) break;
      fn(i);
    }
    in_pool = false;
  };
  const int nt = (int)std::min<int64_t>(g_threads, count);
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(work);
  work();
  for (auto &t : pool) t.join();
}

// ---- symbolic (cholesky.rs:150-342, 728-813, 1195-1378) --------------------------------------

struct Upper {
  int64_t n;
  const int64_t *ptr;
  const int32_t *idx;
};

void etree(const Upper &a, std::vector<int64_t> &parent) {
  parent.assign(a.n, NONE);
  std::vector<int64_t> ancestor(a.n, NONE);
  for (int64_t k = 0; k < a.n; ++k)
    for (int64_t p = a.ptr[k]; p < a.ptr[k + 1]; ++p) {
      int64_t i = a.idx[p];
      while (i != NONE && i < k) {
        int64_t next = ancestor[i];
        ancestor[i] = k;
        if (next == NONE) parent[i] = k;
        i = next;
      }
    }
}

int64_t ereach(const Upper &a, int64_t k, const std::vector<int64_t> &parent, std::vector<int64_t> &stack,
               std::vector<int64_t> &mark, std::vector<int64_t> &path) {
  int64_t top = a.n;
  mark[k] = k;
  for (int64_t p = a.ptr[k]; p < a.ptr[k + 1]; ++p) {
    int64_t i = a.idx[p];
    if (i > k) continue;
    path.clear();
    while (i != NONE && mark[i] != k) {
      path.push_back(i);
      mark[i] = k;
      i = parent[i];
    }
    while (!path.empty()) {
      stack[--top] = path.back();
      path.pop_back();
    }
  }
  return top;
}

void symbolic_by_columns(const Upper &a, std::vector<int64_t> &parent, std::vector<int64_t> &counts) {
  etree(a, parent);
  counts.assign(a.n, 1);
  std::vector<int64_t> stack(a.n, 0), mark(a.n, NONE), path;
  for (int64_t k = 0; k < a.n; ++k) {
    int64_t top = ereach(a, k, parent, stack, mark, path);
    for (int64_t t = top; t < a.n; ++t) counts[stack[t]] += 1;
  }
}

bool uniform_blocks(const Upper &a, std::vector<int64_t> &bptr, std::vector<int32_t> &bidx) {
  if (a.n == 0 || a.n % BLOCK != 0) return false;
  bptr.assign(1, 0);
  bidx.clear();
  for (int64_t q = 0; q < a.n / BLOCK; ++q) {
    int64_t s = a.ptr[BLOCK * q], e = a.ptr[BLOCK * q + 1];
    if (e == s) return false;
    if (a.idx[e - 1] != BLOCK * q) return false;
    int64_t above = e - 1 - s;
    if (above % BLOCK) return false;
    for (int64_t b = 0; b < above; b += BLOCK) {
      int64_t f = a.idx[s + b];
      if (f % BLOCK) return false;
      for (int64_t i = 0; i < BLOCK; ++i)
        if (a.idx[s + b + i] != f + i) return false;
      bidx.push_back((int32_t)(f / BLOCK));
    }
    bidx.push_back((int32_t)q);
    for (int64_t c = 1; c < BLOCK; ++c) {
      int64_t cs = a.ptr[BLOCK * q + c], ce = a.ptr[BLOCK * q + c + 1];
      if (ce - cs < above) return false;
      for (int64_t t = 0; t < above; ++t)
        if (a.idx[cs + t] != a.idx[s + t]) return false;
      if (ce - cs - above != c + 1) return false;
      for (int64_t i = 0; i < c + 1; ++i)
        if (a.idx[cs + above + i] != BLOCK * q + i) return false;
    }
    bptr.push_back((int64_t)bidx.size());
  }
  return true;
}

void symbolic(const Upper &a, std::vector<int64_t> &parent, std::vector<int64_t> &counts, bool &blocks) {
  std::vector<int64_t> bptr;
  std::vector<int32_t> bidx;
  blocks = uniform_blocks(a, bptr, bidx);
  if (!blocks) {
    symbolic_by_columns(a, parent, counts);
    return;
  }
  Upper b{a.n / BLOCK, bptr.data(), bidx.data()};
  std::vector<int64_t> bp, bc;
  symbolic_by_columns(b, bp, bc);
  parent.clear();
  counts.clear();
  for (int64_t q = 0; q < b.n; ++q)
    for (int64_t c = 0; c < BLOCK; ++c) {
      parent.push_back(c + 1 < BLOCK ? BLOCK * q + c + 1 : (bp[q] == NONE ? NONE : BLOCK * bp[q]));
      counts.push_back(BLOCK * bc[q] - c);
    }
}

std::vector<int64_t> postorder(const std::vector<int64_t> &parent) {
  int64_t n = (int64_t)parent.size();
  std::vector<int64_t> head(n, NONE), next(n, NONE);
  for (int64_t j = n - 1; j >= 0; --j) {
    int64_t p = parent[j];
    if (p == NONE || p >= n) continue;
    next[j] = head[p];
    head[p] = j;
  }
  std::vector<int64_t> post, stack;
  for (int64_t root = 0; root < n; ++root) {
    if (parent[root] != NONE) continue;
    stack.push_back(root);
    while (!stack.empty()) {
      int64_t top = stack.back();
      int64_t child = head[top];
      if (child == NONE) {
        post.push_back(top);
        stack.pop_back();
      } else {
        head[top] = next[child];
        stack.push_back(child);
      }
    }
  }
  return post;
}

struct Pattern {
  std::vector<int64_t> ptr;
  std::vector<int32_t> idx;
  std::vector<int64_t> slot;
  std::vector<int32_t> crow, ccol;
};

void pattern_new(const Upper &a, const std::vector<int64_t> &inverse, Pattern &pt) {
  int64_t n = a.n;
  pt.ptr.assign(n + 1, 0);
  for (int64_t k = 0; k < n; ++k)
    for (int64_t p = a.ptr[k]; p < a.ptr[k + 1]; ++p) pt.ptr[std::min(inverse[a.idx[p]], inverse[k]) + 1] += 1;
  for (int64_t j = 0; j < n; ++j) pt.ptr[j + 1] += pt.ptr[j];
  std::vector<std::pair<int64_t, int64_t>> entries(pt.ptr[n]);
  std::vector<int64_t> next(pt.ptr.begin(), pt.ptr.begin() + n);
  int64_t nnz = a.ptr[n];
  pt.crow.resize(nnz);
  pt.ccol.resize(nnz);
  for (int64_t k = 0; k < n; ++k) {
    int64_t first = a.ptr[k];
    for (int64_t t = 0; first + t < a.ptr[k + 1]; ++t) {
      int64_t i = a.idx[first + t];
      int64_t r = std::max(inverse[i], inverse[k]), c = std::min(inverse[i], inverse[k]);
      pt.crow[first + t] = (int32_t)r;
      pt.ccol[first + t] = (int32_t)c;
      entries[next[c]++] = {r, first + t};
    }
  }
  for (int64_t j = 0; j < n; ++j)
    std::stable_sort(entries.begin() + pt.ptr[j], entries.begin() + pt.ptr[j + 1],
                     [](auto &x, auto &y) { return x.first < y.first; });
  pt.slot.assign(nnz, 0);
  pt.idx.resize(entries.size());
  for (size_t pos = 0; pos < entries.size(); ++pos) {
    pt.slot[entries[pos].second] = (int64_t)pos;
    pt.idx[pos] = (int32_t)entries[pos].first;
  }
}

struct Update {
  int64_t k, p1, p2;
};

}  // namespace

struct or_sym {
  int64_t n = 0, ns = 0, entries = 0;
  bool blocks = false;
  std::vector<int64_t> perm, first, rptr, sparent;
  std::vector<int32_t> rows;
  Pattern pattern;
  std::vector<int64_t> upper_ptr;
  std::vector<int32_t> upper_idx;
  std::vector<std::vector<Update>> updates;
  std::vector<int64_t> task_lo, task_hi, top;
  int64_t cols_start(int64_t s) const { return first[s]; }
  int64_t width(int64_t s) const { return first[s + 1] - first[s]; }
  const int32_t *rows_of(int64_t s) const { return rows.data() + rptr[s]; }
  int64_t height(int64_t s) const { return rptr[s + 1] - rptr[s]; }
};

struct or_factor {
  const or_sym *sym = nullptr;
  std::vector<std::vector<double>> values;
};

struct LdltBlock;
struct or_ldlt;

namespace {

// Symbolic::new (cholesky.rs:1212-1378).
int analyse(const Upper &a, uint64_t max_entries, or_sym &s, int64_t *info) {
  int64_t n = a.n;
  std::vector<int64_t> parent0, counts0;
  symbolic(a, parent0, counts0, s.blocks);
  uint64_t total = 0;
  for (auto c : counts0) total = sat_add(total, (uint64_t)c);
  if (total > max_entries) {
    info[0] = (int64_t)std::min<uint64_t>(total, INT64_MAX);
    info[1] = (int64_t)std::min<uint64_t>(max_entries, INT64_MAX);
    return TOO_LARGE;
  }
  s.n = n;
  s.entries = (int64_t)total;
  s.perm = postorder(parent0);
  if ((int64_t)s.perm.size() != n) return INTERNAL;
  std::vector<int64_t> inverse(n, 0);
  for (int64_t k = 0; k < n; ++k) inverse[s.perm[k]] = k;
  std::vector<int64_t> parent(n), counts(n);
  for (int64_t k = 0; k < n; ++k) {
    int64_t j = s.perm[k];
    parent[k] = parent0[j] == NONE ? NONE : inverse[parent0[j]];
    counts[k] = counts0[j];
  }
  pattern_new(a, inverse, s.pattern);
  s.upper_ptr.assign(a.ptr, a.ptr + n + 1);
  s.upper_idx.assign(a.idx, a.idx + a.ptr[n]);
  std::vector<int64_t> children(n, 0);
  for (int64_t p : parent)
    if (p != NONE) children[p] += 1;
  s.first.assign(1, 0);
  for (int64_t j = 1; j < n; ++j) {
    bool joins = parent[j - 1] == j && children[j] == 1 && counts[j - 1] == counts[j] + 1;
    if (!joins) s.first.push_back(j);
  }
  if (n > 0) s.first.push_back(n);
  s.ns = (int64_t)s.first.size() - 1;
  std::vector<int64_t> snode(n, 0);
  for (int64_t t = 0; t < s.ns; ++t)
    for (int64_t j = s.first[t]; j < s.first[t + 1]; ++j) snode[j] = t;
  s.sparent.resize(s.ns);
  for (int64_t t = 0; t < s.ns; ++t) {
    int64_t last = s.first[t + 1] - 1;
    s.sparent[t] = parent[last] == NONE ? NONE : snode[parent[last]];
  }
  std::vector<std::vector<int64_t>> kids(s.ns);
  for (int64_t t = 0; t < s.ns; ++t)
    if (s.sparent[t] != NONE) kids[s.sparent[t]].push_back(t);
  s.rptr.assign(1, 0);
  std::vector<int64_t> mark(n, NONE);
  std::vector<int32_t> set;
  for (int64_t t = 0; t < s.ns; ++t) {
    int64_t f = s.first[t], l = s.first[t + 1];
    set.clear();
    auto add = [&](int64_t r) {
      if (mark[r] != t) {
        mark[r] = t;
        set.push_back((int32_t)r);
      }
    };
    for (int64_t j = f; j < l; ++j) {
      add(j);
      for (int64_t p = s.pattern.ptr[j]; p < s.pattern.ptr[j + 1]; ++p) add(s.pattern.idx[p]);
    }
    for (int64_t c : kids[t]) {
      int64_t cw = s.first[c + 1] - s.first[c];
      for (int64_t p = s.rptr[c] + cw; p < s.rptr[c + 1]; ++p) add(s.rows[p]);
    }
    std::sort(set.begin(), set.end());
    if ((int64_t)set.size() != counts[f] || set.empty() || set[0] != f) return INTERNAL;
    s.rows.insert(s.rows.end(), set.begin(), set.end());
    s.rptr.push_back((int64_t)s.rows.size());
  }
  s.updates.assign(s.ns, {});
  for (int64_t k = 0; k < s.ns; ++k) {
    const int32_t *kr = s.rows_of(k);
    int64_t m = s.height(k), p = s.width(k);
    while (p < m) {
      int64_t target = snode[kr[p]];
      int64_t end = s.first[target + 1];
      int64_t q = p;
      while (q < m && kr[q] < end) ++q;
      s.updates[target].push_back({k, p, q});
      p = q;
    }
  }
  std::vector<uint64_t> subtree(s.ns);
  std::vector<int64_t> start(s.ns);
  for (int64_t t = 0; t < s.ns; ++t) {
    uint64_t m = s.height(t), w = s.width(t), work = 0;
    for (uint64_t c = 0; c < w; ++c) work = sat_add(work, sat_mul(m - c, m - c));
    subtree[t] = work;
    start[t] = t;
  }
  for (int64_t t = 0; t < s.ns; ++t) {
    int64_t p = s.sparent[t];
    if (p != NONE) {
      subtree[p] = sat_add(subtree[p], subtree[t]);
      start[p] = std::min(start[p], start[t]);
    }
  }
  uint64_t all = 0;
  for (int64_t t = 0; t < s.ns; ++t)
    if (s.sparent[t] == NONE) all = sat_add(all, subtree[t]);
  uint64_t share = std::max(all / SUBTREE_SHARE, PARALLEL_WORK);
  int64_t t = 0;
  while (t < s.ns) {
    int64_t root = NONE, r = t;
    while (r != NONE && start[r] == t && subtree[r] <= share) {
      root = r;
      r = s.sparent[r];
    }
    if (root == NONE) {
      s.top.push_back(t);
      ++t;
    } else {
      s.task_lo.push_back(t);
      s.task_hi.push_back(root + 1);
      t = root + 1;
    }
  }
  return OK;
}

// ---- numeric (cholesky.rs:418-720, 1040-1188, 1392-1529) -------------------------------------

inline int64_t offset(int64_t m, int64_t c) { return c * m - c * (c > 0 ? c - 1 : 0) / 2; }

// Entries of an m-row, w-column lower trapezoid (cholesky.rs:418-420).
int64_t trapezoid_size(int64_t m, int64_t w) {
  int64_t s = 0;
  for (int64_t c = 0; c < w; ++c) s += m > c ? m - c : 0;
  return s;
}

struct PanelRef {
  int64_t m;
  const double *data;
  int64_t size;
  double at(int64_t r, int64_t c) const { return data[offset(m, c) + r - c]; }
  // Rows r..r+len of column c; nullptr when outside the trapezoid.
  const double *column(int64_t c, int64_t r, int64_t len) const {
    int64_t start = offset(m, c) + r - c;
    if (r < c || start < 0 || start + len > size) return nullptr;
    return data + start;
  }
};

// times_d (cholesky.rs:458-481): row <- row D, with D the block diagonal the trapezoid holds
// for its columns k0.. and `pivots` their pivots from k0.
void times_d(double *row, int64_t len, const PanelRef &l, int64_t k0, const int8_t *pivots) {
  int64_t k = 0;
  while (k < len) {
    if (pivots[k] == PIVOT_FIRST) {
      const double a = row[k], b = k + 1 < len ? row[k + 1] : 0.0;
      const double d11 = l.at(k0 + k, k0 + k), d21 = l.at(k0 + k + 1, k0 + k), d22 = l.at(k0 + k + 1, k0 + k + 1);
      row[k] = a * d11 + b * d21;
      if (k + 1 < len) row[k + 1] = a * d21 + b * d22;
      k += 2;
    } else {
      row[k] *= l.at(k0 + k, k0 + k);
      k += 1;
    }
  }
}

// products (cholesky.rs:531-630) with the reference's packing and micro-tiles (MR x NR, two
// columns a pass); tiles[t][c * TILE + i]. Y is L, or L D when `pivots` (of the columns k0..)
// are given. Returns false on a tile outside the panel.
bool products_tiled(const PanelRef &l, int64_t k0, int64_t kw, int64_t p, int64_t mu, int64_t wu,
                    std::vector<std::vector<double>> &tiles, const int8_t *pivots = nullptr) {
  std::vector<double> yt(wu * kw, 0.0);
  for (int64_t k = 0; k < kw; ++k) {
    const double *col = l.column(k0 + k, p, wu);
    if (!col) return false;
    for (int64_t c = 0; c < wu; ++c) yt[c * kw + k] = col[c];
  }
  if (pivots && kw > 0)
    for (int64_t c = 0; c < wu; ++c) times_d(&yt[c * kw], kw, l, k0, pivots);
  int64_t nb = (wu + NR - 1) / NR;
  std::vector<double> yp(nb * kw * NR, 0.0);
  for (int64_t c = 0; c < wu; ++c)
    for (int64_t k = 0; k < kw; ++k) yp[((c / NR) * kw + k) * NR + c % NR] = yt[c * kw + k];
  int64_t ntiles = (mu + TILE - 1) / TILE;
  tiles.assign(ntiles, {});
  std::atomic<bool> bad{false};
  auto tile = [&](int64_t t) {
    int64_t i0 = t * TILE, h = std::min(TILE, mu - i0), cols = std::min(wu, i0 + h);
    std::vector<double> out(cols * TILE, 0.0);
    std::vector<double> xp((TILE / MR) * kw * MR, 0.0);
    for (int64_t k = 0; k < kw; ++k) {
      const double *column = l.column(k0 + k, p + i0, h);
      if (!column) {
        bad = true;
        return;
      }
      for (int64_t r = 0; r * MR < h; ++r) {
        int64_t len = std::min(MR, h - r * MR);
        for (int64_t i = 0; i < len; ++i) xp[(r * kw + k) * MR + i] = column[r * MR + i];
      }
    }
    for (int64_t b = 0; b < (cols + NR - 1) / NR; ++b)
      for (int64_t r = 0; r < TILE / MR; ++r)
        for (int64_t pair = 0; pair < NR / 2; ++pair) {
          double first[MR], second[MR];
          for (int64_t i = 0; i < MR; ++i) first[i] = second[i] = 0.0;
          for (int64_t k = 0; k < kw; ++k) {
            const double *x = &xp[(r * kw + k) * MR];
            const double y0 = yp[(b * kw + k) * NR + 2 * pair], y1 = yp[(b * kw + k) * NR + 2 * pair + 1];
            for (int64_t i = 0; i < MR; ++i) first[i] += x[i] * y0;
            for (int64_t i = 0; i < MR; ++i) second[i] += x[i] * y1;
          }
          for (int j = 0; j < 2; ++j) {
            int64_t c = b * NR + 2 * pair + j;
            if (c < cols) std::memcpy(&out[c * TILE + r * MR], j ? second : first, sizeof(double) * MR);
          }
        }
    tiles[t] = std::move(out);
  };
  if (sat_mul(sat_mul(mu, wu), kw) >= PARALLEL_WORK)
    parallel_for(ntiles, tile);
  else
    for (int64_t t = 0; t < ntiles; ++t) tile(t);
  return !bad;
}

// The column-at-a-time products (the reference test's products_by_columns, cholesky.rs:1581-1623).
bool products_by_columns(const PanelRef &l, int64_t k0, int64_t kw, int64_t p, int64_t mu, int64_t wu,
                         std::vector<std::vector<double>> &tiles) {
  std::vector<double> yt(wu * kw, 0.0);
  for (int64_t k = 0; k < kw; ++k) {
    const double *col = l.column(k0 + k, p, wu);
    if (!col) return false;
    for (int64_t c = 0; c < wu; ++c) yt[c * kw + k] = col[c];
  }
  int64_t ntiles = (mu + TILE - 1) / TILE;
  tiles.assign(ntiles, {});
  for (int64_t t = 0; t < ntiles; ++t) {
    int64_t i0 = t * TILE, h = std::min(TILE, mu - i0), cols = std::min(wu, i0 + h);
    std::vector<double> x(kw * TILE, 0.0);
    for (int64_t k = 0; k < kw; ++k) {
      const double *column = l.column(k0 + k, p + i0, h);
      if (!column) return false;
      std::memcpy(&x[k * TILE], column, sizeof(double) * h);
    }
    std::vector<double> out(cols * TILE, 0.0);
    for (int64_t c = 0; c < cols; ++c) {
      double acc[TILE];
      for (int64_t i = 0; i < TILE; ++i) acc[i] = 0.0;
      for (int64_t k = 0; k < kw; ++k) {
        double b = yt[c * kw + k];
        for (int64_t i = 0; i < TILE; ++i) acc[i] += x[k * TILE + i] * b;
      }
      std::memcpy(&out[c * TILE], acc, sizeof(acc));
    }
    tiles[t] = std::move(out);
  }
  return true;
}

// subtract (cholesky.rs:636-686): own(rel(i), rel(c)) -= S(i, c), i >= c. False on a broken
// structure (a column of the update not in own after the one before it).
template <class Rel>
bool subtract(double *own, int64_t own_size, int64_t m, const std::vector<std::vector<double>> &tiles, int64_t mu,
              int64_t wu, Rel rel) {
  int64_t at = 0;
  std::vector<std::pair<int64_t, double *>> columns;
  for (int64_t c = 0; c < std::min(wu, mu); ++c) {
    int64_t cc = rel(c);
    int64_t start = offset(m, cc);
    if (!(cc < m) || start < at || start + (m - cc) > own_size) return false;
    columns.push_back({c, own + start});
    at = start + m - cc;
  }
  auto column = [&](int64_t idx) {
    int64_t c = columns[idx].first;
    double *target = columns[idx].second;
    int64_t cc = rel(c);
    for (int64_t t = c / TILE; t < (int64_t)tiles.size(); ++t) {
      int64_t i0 = t * TILE, h = std::min(TILE, mu - i0);
      for (int64_t i = std::max(i0, c); i < i0 + h; ++i) target[rel(i) - cc] -= tiles[t][c * TILE + i - i0];
    }
  };
  if (sat_mul(mu, wu) >= (1u << 16))
    parallel_for((int64_t)columns.size(), column);
  else
    for (int64_t i = 0; i < (int64_t)columns.size(); ++i) column(i);
  return true;
}

// solve_below (cholesky.rs:691-720).
void solve_below(const PanelRef &l, int64_t c0, int64_t c1, std::vector<std::vector<double>> &out) {
  int64_t m = l.m, pw = c1 - c0;
  int64_t ntiles = (m - c1 + TILE - 1) / TILE;
  out.assign(ntiles, {});
  auto tile = [&](int64_t t) {
    int64_t i0 = c1 + t * TILE, h = std::min(TILE, m - i0);
    std::vector<double> buf(pw * TILE, 0.0);
    for (int64_t c = 0; c < pw; ++c) std::memcpy(&buf[c * TILE], l.column(c0 + c, i0, h), sizeof(double) * h);
    for (int64_t c = 0; c < pw; ++c) {
      double *target = &buf[c * TILE];
      for (int64_t k = 0; k < c; ++k) {
        const double *src = &buf[k * TILE];
        double lck = l.at(c0 + c, c0 + k);
        for (int64_t i = 0; i < TILE; ++i) target[i] -= src[i] * lck;
      }
      double d = l.at(c0 + c, c0 + c);
      for (int64_t i = 0; i < TILE; ++i) target[i] /= d;
    }
    out[t] = std::move(buf);
  };
  if (sat_mul(sat_mul(m - c1, pw), pw) >= PARALLEL_WORK)
    parallel_for(ntiles, tile);
  else
    for (int64_t t = 0; t < ntiles; ++t) tile(t);
}

struct Lower {
  std::vector<double> val, diag, scale;
};

// Context::assemble (cholesky.rs:1044-1125): supernode j's columns of A, then minus the
// product L_K Y_K^T of every descendant K that reaches it, in supernode order (Y = L, or L D when
// `pivots_of(k)` is not null). `values_of(k)` is descendant k's trapezoid.
template <class ValuesOf, class PivotsOf>
Error assemble(const or_sym &s, const Lower &a, int64_t j, double *own, int64_t own_size, ValuesOf values_of,
               PivotsOf pivots_of) {
  const int32_t *rows = s.rows_of(j);
  int64_t m = s.height(j), w = s.width(j), f = s.first[j];
  if (own_size != trapezoid_size(m, w)) return {INTERNAL, -1};
  std::fill(own, own + own_size, 0.0);
  for (int64_t c = 0; c < w; ++c)
    for (int64_t p = s.pattern.ptr[f + c]; p < s.pattern.ptr[f + c + 1]; ++p) {
      int32_t r = s.pattern.idx[p];
      const int32_t *hit = std::lower_bound(rows, rows + m, r);
      if (hit == rows + m || *hit != r) return {INTERNAL, -1};
      int64_t at = hit - rows;
      if (at < c) return {INTERNAL, -1};
      own[offset(m, c) + at - c] = a.val[p];
    }
  std::vector<std::vector<double>> tiles;
  std::vector<int64_t> relative;
  for (const Update &u : s.updates[j]) {
    const int32_t *kr = s.rows_of(u.k);
    int64_t km = s.height(u.k), kw = s.width(u.k);
    int64_t mu = km - u.p1, wu = u.p2 - u.p1;
    relative.clear();
    int64_t at = 0;
    for (int64_t i = u.p1; i < km; ++i) {
      while (at < m && rows[at] < kr[i]) ++at;
      if (at >= m || rows[at] != kr[i]) return {INTERNAL, -1};
      relative.push_back(at);
    }
    const std::vector<double> &vk = values_of(u.k);
    PanelRef lk{km, vk.data(), (int64_t)vk.size()};
    if (!products_tiled(lk, 0, kw, u.p1, mu, wu, tiles, pivots_of(u.k))) return {INTERNAL, -1};
    if (!subtract(own, own_size, m, tiles, mu, wu, [&](int64_t i) { return relative[i]; })) return {INTERNAL, -1};
  }
  return {OK, -1};
}

// Context::supernode (cholesky.rs:1131-1188): assemble, then panels.
Error supernode(const or_sym &s, const Lower &a, int64_t j, std::vector<std::vector<double>> &values) {
  int64_t m = s.height(j), w = s.width(j), f = s.first[j];
  std::vector<double> &ownv = values[j];
  double *own = ownv.data();
  int64_t own_size = (int64_t)ownv.size();
  Error assembled = assemble(
      s, a, j, own, own_size, [&](int64_t k) -> const std::vector<double> & { return values[k]; },
      [](int64_t) -> const int8_t * { return nullptr; });
  if (assembled.code != OK) return assembled;
  std::vector<std::vector<double>> tiles;
  for (int64_t c0 = 0; c0 < w; c0 += PANEL) {
    int64_t c1 = std::min(c0 + PANEL, w), pw = c1 - c0;
    if (c0 > 0) {
      PanelRef lp{m, own, own_size};
      if (!products_tiled(lp, 0, c0, c0, m - c0, pw, tiles)) return {INTERNAL, -1};
      if (!subtract(own, own_size, m, tiles, m - c0, pw, [&](int64_t i) { return c0 + i; })) return {INTERNAL, -1};
    }
    for (int64_t c = c0; c < c1; ++c) {
      int64_t dst = offset(m, c);
      for (int64_t k = c0; k < c; ++k) {
        int64_t src = offset(m, k) + c - k;
        double lck = own[src];
        for (int64_t r = 0; r < c1 - c; ++r) own[dst + r] -= own[src + r] * lck;
      }
      double d = own[dst];
      double diag = a.diag[f + c];
      if (!(d > PIVOT_TOLERANCE * std::fabs(diag)) || !std::isfinite(d)) return {NOT_POSITIVE_DEFINITE, f + c};
      d = std::sqrt(d);
      own[dst] = d;
      for (int64_t r = dst + 1; r < dst + c1 - c; ++r) own[r] /= d;
    }
    if (c1 < m) {
      PanelRef lp{m, own, own_size};
      solve_below(lp, c0, c1, tiles);
      for (int64_t t = 0; t < (int64_t)tiles.size(); ++t) {
        int64_t i0 = c1 + t * TILE, h = std::min(TILE, m - i0);
        for (int64_t c = 0; c < pw; ++c) {
          int64_t start = offset(m, c0 + c) + i0 - (c0 + c);
          std::memcpy(own + start, &tiles[t][c * TILE], sizeof(double) * h);
        }
      }
    }
  }
  return {OK, -1};
}

// Symbolic::factor (cholesky.rs:1443-1529): subtree tasks concurrently, each in order, then
// the supernodes above them in order; the earliest failing column in postorder is reported,
// named by its original column.
template <class Supernode>
Error factor(const or_sym &s, const volatile int32_t *cancel, Supernode supernode) {
  int64_t ntasks = (int64_t)s.task_lo.size();
  std::vector<Error> failed(ntasks, Error{OK, -1});
  std::mutex broken_lock;
  Error broken{OK, -1};
  auto cancelled = [&]() { return cancel && *cancel != 0; };
  parallel_for(ntasks, [&](int64_t t) {
    for (int64_t j = s.task_lo[t]; j < s.task_hi[t]; ++j) {
      if (cancelled()) {
        std::lock_guard<std::mutex> g(broken_lock);
        if (broken.code == OK) broken = {CANCELLED, -1};
        break;
      }
      Error e = supernode(j);
      if (e.code == NOT_POSITIVE_DEFINITE || e.code == SINGULAR) {
        failed[t] = e;
        break;
      }
      if (e.code != OK) {
        std::lock_guard<std::mutex> g(broken_lock);
        if (broken.code == OK) broken = e;
        break;
      }
    }
  });
  if (broken.code != OK) return broken;
  Error earliest{OK, -1};
  for (auto &e : failed)
    if (e.code != OK && (earliest.code == OK || e.column < earliest.column)) earliest = e;
  auto named = [&](Error e) {
    if (e.code == NOT_POSITIVE_DEFINITE || e.code == SINGULAR) e.column = s.perm[e.column];
    return e;
  };
  for (int64_t j : s.top) {
    if (cancelled()) return {CANCELLED, -1};
    if (earliest.code != OK && s.first[j] > earliest.column) break;
    Error e = supernode(j);
    if (e.code != OK) return named(e);
  }
  if (earliest.code != OK) return named(earliest);
  return {OK, -1};
}

// solve_group for Cholesky (cholesky.rs:904-1037), `kk` right-hand sides interleaved.
void solve_group(const or_factor &fac, double *x, int kk) {
  const or_sym &s = *fac.sym;
  for (int64_t k = 0; k < s.ns; ++k) {
    const int32_t *rows = s.rows_of(k);
    int64_t m = s.height(k), f = s.first[k], w = s.width(k);
    const double *t = fac.values[k].data();
    double *own = x + f * kk;
    for (int64_t q = 0; q < w; ++q) {
      double yq[GROUP];
      double d = t[offset(m, q)];
      for (int j = 0; j < kk; ++j) {
        yq[j] = own[q * kk + j] / d;
        own[q * kk + j] = yq[j];
      }
      const double *col = t + offset(m, q);  // rows q..m of column q
      for (int64_t r = q + 1; r < w; ++r) {
        double l = col[r - q];
        for (int j = 0; j < kk; ++j) own[r * kk + j] -= l * yq[j];
      }
      for (int64_t r = w; r < m; ++r) {
        double l = col[r - q];
        double *v = x + (int64_t)rows[r] * kk;
        for (int j = 0; j < kk; ++j) v[j] -= l * yq[j];
      }
    }
  }
  for (int64_t k = s.ns - 1; k >= 0; --k) {
    const int32_t *rows = s.rows_of(k);
    int64_t m = s.height(k), f = s.first[k], w = s.width(k);
    const double *t = fac.values[k].data();
    double *own = x + f * kk;
    for (int64_t q = w - 1; q >= 0; --q) {
      double sum[GROUP];
      for (int j = 0; j < kk; ++j) sum[j] = own[q * kk + j];
      const double *col = t + offset(m, q);
      for (int64_t r = q + 1; r < w; ++r) {
        double l = col[r - q];
        for (int j = 0; j < kk; ++j) sum[j] -= l * own[r * kk + j];
      }
      for (int64_t r = w; r < m; ++r) {
        double l = col[r - q];
        const double *v = x + (int64_t)rows[r] * kk;
        for (int j = 0; j < kk; ++j) sum[j] -= l * v[j];
      }
      double d = t[offset(m, q)];
      for (int j = 0; j < kk; ++j) own[q * kk + j] = sum[j] / d;
    }
  }
}

// ---- symmetric indefinite LDL^T (ldlt.rs) --------------------------------------------------
// The same supernodes, tasks and products as the Cholesky factor; inside a supernode, pivots
// chosen by the bounded Bunch-Kaufman (rook) search among the supernode's own columns.

// One supernode of an LDL^T factor (ldlt.rs:88-98): L below the pivots and D on them in the lower
// trapezoid by columns in pivot order; order[c] is the own column (symbolic order) at pivot c.
}  // namespace

struct LdltBlock {
  std::vector<double> values;
  std::vector<int8_t> pivots;
  std::vector<int64_t> order;
  int64_t two_by_two = 0;
};

struct or_ldlt {
  const or_sym *sym = nullptr;
  std::vector<LdltBlock> blocks;
};

namespace {

// interchange (ldlt.rs:128-143): symmetric interchange of local columns p < q of an m-row lower
// trapezoid: the rows of the columns before p, the diagonals, the strip between them and the
// rows below q.
void interchange(std::vector<double> &v, int64_t m, int64_t p, int64_t q) {
  auto at = [m](int64_t r, int64_t c) { return offset(m, c) + r - c; };
  for (int64_t c = 0; c < p; ++c) std::swap(v[at(p, c)], v[at(q, c)]);
  std::swap(v[at(p, p)], v[at(q, q)]);
  for (int64_t c = p + 1; c < q; ++c) std::swap(v[at(c, p)], v[at(q, c)]);
  for (int64_t r = q + 1; r < m; ++r) std::swap(v[at(r, p)], v[at(r, q)]);
}

// largest (ldlt.rs:145-163): the largest magnitude of v over [lo, hi) except `skip`, with the
// lowest such index; NaN at the first entry that is not a number.
std::pair<int64_t, double> largest(const std::vector<double> &v, int64_t lo, int64_t hi, int64_t skip) {
  std::pair<int64_t, double> best{lo, 0.0};
  for (int64_t i = lo; i < hi; ++i) {
    if (i == skip) continue;
    const double x = i < (int64_t)v.size() ? std::fabs(v[i]) : 0.0;
    if (std::isnan(x)) return {i, x};
    if (x > best.second) best = {i, x};
  }
  return best;
}

struct LdltScratch {
  std::vector<double> a, b, w;  // the searched column, a candidate, a row of L D (ldlt.rs:165-172)
};

// Block::current (ldlt.rs:173-192): column c (local, >= k) of the part still to factor, rows
// k..m, into out: the trapezoid's entries less the products with the panel's factored columns
// c0..k, whose L D row is formed from L and D.
void ldlt_current(const LdltBlock &b, int64_t m, int64_t c0, int64_t k, int64_t c, std::vector<double> &out,
                  std::vector<double> &w) {
  const PanelRef t{m, b.values.data(), (int64_t)b.values.size()};
  for (int64_t r = k; r < m; ++r) out[r] = r >= c ? t.at(r, c) : t.at(c, r);
  w.clear();
  for (int64_t q = c0; q < k; ++q) w.push_back(t.at(c, q));
  if (!w.empty()) times_d(w.data(), (int64_t)w.size(), t, c0, b.pivots.data() + c0);
  for (int64_t q = c0; q < k; ++q) {
    const double wq = w[q - c0];
    const double *l = t.column(q, k, m - k);
    for (int64_t r = 0; r < m - k; ++r) out[k + r] -= l[r] * wq;
  }
}

// Block::swap (ldlt.rs:194-204): local columns p and q (pivot positions >= k) in the trapezoid,
// the order and the current columns.
void ldlt_swap(LdltBlock &b, int64_t m, int64_t p, int64_t q, LdltScratch &sc) {
  if (p == q) return;
  if (p > q) std::swap(p, q);
  interchange(b.values, m, p, q);
  std::swap(b.order[p], b.order[q]);
  std::swap(sc.a[p], sc.a[q]);
  std::swap(sc.b[p], sc.b[q]);
}

// Block::one (ldlt.rs:206-221): a 1 x 1 pivot at k from the current column.
void ldlt_one(LdltBlock &b, int64_t m, int64_t k, const std::vector<double> &col) {
  const double d = col[k];
  const int64_t start = offset(m, k);
  b.values[start] = d;
  for (int64_t r = k + 1; r < m; ++r) b.values[start + r - k] = col[r] / d;
  b.pivots[k] = PIVOT_ONE;
}

// Block::two (ldlt.rs:223-248): a 2 x 2 pivot at k, k + 1 from the current columns a (k) and
// b (k + 1).
void ldlt_two(LdltBlock &blk, int64_t m, int64_t k, const std::vector<double> &a, const std::vector<double> &b) {
  const double d11 = a[k], d21 = a[k + 1], d22 = b[k + 1];
  const double det = d11 * d22 - d21 * d21;
  const int64_t s0 = offset(m, k), s1 = offset(m, k + 1);
  blk.values[s0] = d11;
  blk.values[s0 + 1] = d21;
  blk.values[s1] = d22;
  for (int64_t r = k + 2; r < m; ++r) {
    const double x = a[r], y = b[r];
    blk.values[s0 + r - k] = (x * d22 - y * d21) / det;
    blk.values[s1 + r - k - 1] = (y * d11 - x * d21) / det;
  }
  blk.pivots[k] = PIVOT_FIRST;
  blk.pivots[k + 1] = PIVOT_SECOND;
  blk.two_by_two += 1;
}

// Block::panel (ldlt.rs:250-335): the panel from column c0 of a supernode with m rows and w
// columns whose first column is f (postorder), pivots chosen among the columns c0..w by the rook
// search, each column brought up to date with the panel's columns before it. `end` receives
// where the panel ended (one column past c0 + PANEL after a closing 2 x 2 pivot).
Error ldlt_panel(LdltBlock &blk, int64_t m, int64_t w, int64_t c0, int64_t f, const Lower &lower, LdltScratch &sc,
                 int64_t &end_out) {
  const int64_t end = std::min(c0 + PANEL, w);
  auto scale = [&](int64_t at) { return lower.scale[f + blk.order[at]]; };
  auto singular = [&](int64_t at) { return Error{SINGULAR, f + blk.order[at]}; };
  int64_t k = c0;
  while (k < end) {
    ldlt_current(blk, m, c0, k, k, sc.a, sc.w);
    const double akk = std::fabs(sc.a[k]);
    const auto first = largest(sc.a, k + 1, w, NONE);
    const int64_t r0 = first.first;
    const double omega_k = first.second;
    if (!std::isfinite(akk) || !std::isfinite(omega_k)) return singular(k);
    bool two = false;
    int64_t p = k, pi = k, pr = k;
    if (akk >= ALPHA * omega_k) {
      p = k;
    } else {
      // the rook search: `a` holds column i, `b` the candidate r
      int64_t i = k, r = r0;
      double omega_i = omega_k;
      int step = 0;
      for (;;) {
        ldlt_current(blk, m, c0, k, r, sc.b, sc.w);
        const auto next = largest(sc.b, k, w, r);
        const double omega_r = next.second, arr = std::fabs(sc.b[r]);
        if (!std::isfinite(arr) || !std::isfinite(omega_r)) return singular(k);
        step += 1;
        if (arr >= ALPHA * omega_r) {
          std::swap(sc.a, sc.b);
          p = r;
          break;
        }
        if (omega_r <= omega_i || step >= ROOK_STEPS) {
          two = true;
          pi = i;
          pr = r;
          break;
        }
        std::swap(sc.a, sc.b);
        i = r;
        omega_i = omega_r;
        r = next.first;
      }
    }
    if (!two) {
      ldlt_swap(blk, m, k, p, sc);
      if (!(std::fabs(sc.a[k]) > PIVOT_TOLERANCE * scale(k))) return singular(k);
      ldlt_one(blk, m, k, sc.a);
      k += 1;
    } else {
      // i to k, then r to k + 1 (r was at k if i took its place)
      ldlt_swap(blk, m, k, pi, sc);
      ldlt_swap(blk, m, k + 1, pr == k ? pi : pr, sc);
      const double offdiagonal = std::fabs(sc.a[k + 1]);
      const double size = std::max(scale(k), scale(k + 1));
      if (!(offdiagonal > PIVOT_TOLERANCE * size)) return singular(k);
      ldlt_two(blk, m, k, sc.a, sc.b);
      k += 2;
    }
  }
  end_out = k;
  return {OK, -1};
}

// supernode (ldlt.rs:337-363): assemble with the descendants' L D, then panels; after each
// panel the rest of the supernode minus the panel's L D L^T by the tiled products.
Error ldlt_supernode(const or_sym &s, const Lower &a, int64_t j, std::vector<LdltBlock> &blocks) {
  const int64_t m = s.height(j), w = s.width(j), f = s.first[j];
  LdltBlock &own = blocks[j];
  Error assembled = assemble(
      s, a, j, own.values.data(), (int64_t)own.values.size(),
      [&](int64_t k) -> const std::vector<double> & { return blocks[k].values; },
      [&](int64_t k) -> const int8_t * { return blocks[k].pivots.data(); });
  if (assembled.code != OK) return assembled;
  own.pivots.assign(w, PIVOT_ONE);
  own.order.resize(w);
  for (int64_t c = 0; c < w; ++c) own.order[c] = c;
  own.two_by_two = 0;
  LdltScratch sc;
  sc.a.assign(m, 0.0);
  sc.b.assign(m, 0.0);
  std::vector<std::vector<double>> tiles;
  int64_t c0 = 0;
  while (c0 < w) {
    int64_t c1 = c0;
    Error e = ldlt_panel(own, m, w, c0, f, a, sc, c1);
    if (e.code != OK) return e;
    if (c1 < w) {
      const PanelRef l{m, own.values.data(), (int64_t)own.values.size()};
      if (!products_tiled(l, c0, c1 - c0, c1, m - c1, w - c1, tiles, own.pivots.data() + c0)) return {INTERNAL, -1};
      if (!subtract(own.values.data(), (int64_t)own.values.size(), m, tiles, m - c1, w - c1,
                    [&](int64_t i) { return c1 + i; }))
        return {INTERNAL, -1};
    }
    c0 = c1;
  }
  return {OK, -1};
}

// solve_group with LDL^T's unit L, block diagonal D and pivot order (cholesky.rs:904-1037), `kk`
// right-hand sides interleaved: L z = P b and D^-1 by supernodes, each supernode's own unknowns
// left in pivot order for the backward pass; then L^T x = z in reverse, each supernode
// scattering its unknowns back from pivot order.
void ldlt_solve_group(const or_sym &s, const std::vector<LdltBlock> &blocks, double *x, int kk) {
  std::vector<double> y;
  for (int64_t k = 0; k < s.ns; ++k) {
    const int32_t *rows = s.rows_of(k);
    const int64_t m = s.height(k), f = s.first[k], w = s.width(k);
    const LdltBlock &blk = blocks[k];
    const PanelRef t{m, blk.values.data(), (int64_t)blk.values.size()};
    double *own = x + f * kk;
    y.assign(w * kk, 0.0);
    for (int64_t c = 0; c < w; ++c)
      for (int j = 0; j < kk; ++j) y[c * kk + j] = own[blk.order[c] * kk + j];
    for (int64_t q = 0; q < w; ++q) {
      const int64_t end = q + (blk.pivots[q] == PIVOT_FIRST ? 2 : 1);
      double yq[GROUP];
      for (int j = 0; j < kk; ++j) yq[j] = y[q * kk + j];
      for (int64_t r = end; r < w; ++r) {
        const double l = t.at(r, q);
        for (int j = 0; j < kk; ++j) y[r * kk + j] -= l * yq[j];
      }
      for (int64_t r = w; r < m; ++r) {
        const double l = t.at(r, q);
        double *v = x + (int64_t)rows[r] * kk;
        for (int j = 0; j < kk; ++j) v[j] -= l * yq[j];
      }
    }
    int64_t c = 0;
    while (c < w) {
      if (blk.pivots[c] == PIVOT_FIRST) {
        const double d11 = t.at(c, c), d21 = t.at(c + 1, c), d22 = t.at(c + 1, c + 1);
        const double det = d11 * d22 - d21 * d21;
        for (int j = 0; j < kk; ++j) {
          const double p = y[c * kk + j], q = y[(c + 1) * kk + j];
          y[c * kk + j] = (d22 * p - d21 * q) / det;
          y[(c + 1) * kk + j] = (d11 * q - d21 * p) / det;
        }
        c += 2;
      } else {
        const double d = t.at(c, c);
        for (int j = 0; j < kk; ++j) y[c * kk + j] /= d;
        c += 1;
      }
    }
    std::memcpy(own, y.data(), sizeof(double) * w * kk);
  }
  for (int64_t k = s.ns - 1; k >= 0; --k) {
    const int32_t *rows = s.rows_of(k);
    const int64_t m = s.height(k), f = s.first[k], w = s.width(k);
    const LdltBlock &blk = blocks[k];
    const PanelRef t{m, blk.values.data(), (int64_t)blk.values.size()};
    double *own = x + f * kk;
    y.assign(own, own + w * kk);
    for (int64_t c = w - 1; c >= 0; --c) {
      // reverse pivot groups, ascending columns within each 2 x 2 group
      int64_t q = c, end = c + 1;
      if (blk.pivots[c] == PIVOT_SECOND && c > 0) {
        q = c - 1;
        end = c + 1;
      } else if (blk.pivots[c] == PIVOT_FIRST) {
        q = c + 1;
        end = c + 2;
      }
      double sum[GROUP];
      for (int j = 0; j < kk; ++j) sum[j] = y[q * kk + j];
      for (int64_t r = end; r < w; ++r) {
        const double l = t.at(r, q);
        for (int j = 0; j < kk; ++j) sum[j] -= l * y[r * kk + j];
      }
      for (int64_t r = w; r < m; ++r) {
        const double l = t.at(r, q);
        const double *v = x + (int64_t)rows[r] * kk;
        for (int j = 0; j < kk; ++j) sum[j] -= l * v[j];
      }
      for (int j = 0; j < kk; ++j) y[q * kk + j] = sum[j];
    }
    for (int64_t pos = 0; pos < w; ++pos)
      for (int j = 0; j < kk; ++j) own[blk.order[pos] * kk + j] = y[pos * kk + j];
  }
}

}  // namespace

extern "C" {

// Info codes for or_sym_info / or_sym_export.
enum {
  OR_N = 0, OR_NS = 1, OR_ENTRIES = 2, OR_ROWS = 3, OR_LOWER = 4, OR_UPDATES = 5, OR_TASKS = 6, OR_TOP = 7,
  OR_BLOCKS = 8, OR_NNZ = 9
};
enum {
  OR_X_PERM = 0, OR_X_FIRST = 1, OR_X_RPTR = 2, OR_X_ROWS = 3, OR_X_SPARENT = 4, OR_X_LPTR = 5, OR_X_LIDX = 6,
  OR_X_SLOT = 7, OR_X_CROW = 8, OR_X_CCOL = 9, OR_X_UPTR = 10, OR_X_UK = 11, OR_X_UP1 = 12, OR_X_UP2 = 13,
  OR_X_TASK_LO = 14, OR_X_TASK_HI = 15, OR_X_TOP = 16
};

void or_set_threads(int threads) {
  if (threads <= 0) {
    unsigned h = std::thread::hardware_concurrency();
    threads = h ? (int)h : 1;
  }
  g_threads = threads;
}

int or_get_threads(void) { return g_threads; }

// UpperColumns::from_symmetric (cholesky.rs:112-145): rows of a full symmetric CSR, entries with
// column <= row, as the upper triangle by columns. out_ptr[n+1]; out_idx/out_val sized by the
// count this returns when they are null.
int64_t or_upper_from_symmetric(int64_t n, const int64_t *ptr, const int32_t *idx, const double *val, int64_t *out_ptr,
                                int32_t *out_idx, double *out_val) {
  int64_t total = 0;
  if (out_ptr) out_ptr[0] = 0;
  for (int64_t k = 0; k < n; ++k) {
    for (int64_t p = ptr[k]; p < ptr[k + 1]; ++p)
      if (idx[p] <= k) {
        if (out_idx) out_idx[total] = idx[p];
        if (out_val) out_val[total] = val[p];
        ++total;
      }
    if (out_ptr) out_ptr[k + 1] = total;
  }
  return total;
}

int or_analyse(int64_t n, const int64_t *ptr, const int32_t *idx, uint64_t max_entries, or_sym **out, int64_t *info) {
  *out = nullptr;
  try {
    auto s = new or_sym();
    int code = analyse(Upper{n, ptr, idx}, max_entries, *s, info);
    if (code != OK) {
      delete s;
      return code;
    }
    *out = s;
    return OK;
  } catch (const std::bad_alloc &) {
    return OUT_OF_MEMORY;
  }
}

void or_sym_free(or_sym *s) { delete s; }

int64_t or_sym_info(const or_sym *s, int what) {
  switch (what) {
    case OR_N: return s->n;
    case OR_NS: return s->ns;
    case OR_ENTRIES: return s->entries;
    case OR_ROWS: return (int64_t)s->rows.size();
    case OR_LOWER: return (int64_t)s->pattern.idx.size();
    case OR_UPDATES: {
      int64_t t = 0;
      for (auto &l : s->updates) t += (int64_t)l.size();
      return t;
    }
    case OR_TASKS: return (int64_t)s->task_lo.size();
    case OR_TOP: return (int64_t)s->top.size();
    case OR_BLOCKS: return s->blocks ? 1 : 0;
    case OR_NNZ: return (int64_t)s->upper_idx.size();
  }
  return -1;
}

// Copies one array out as int64 values.
int or_sym_export(const or_sym *s, int what, int64_t *dst) {
  auto put64 = [&](const std::vector<int64_t> &v) { std::copy(v.begin(), v.end(), dst); };
  auto put32 = [&](const std::vector<int32_t> &v) {
    for (size_t i = 0; i < v.size(); ++i) dst[i] = v[i];
  };
  switch (what) {
    case OR_X_PERM: put64(s->perm); break;
    case OR_X_FIRST: put64(s->first); break;
    case OR_X_RPTR: put64(s->rptr); break;
    case OR_X_ROWS: put32(s->rows); break;
    case OR_X_SPARENT: put64(s->sparent); break;
    case OR_X_LPTR: put64(s->pattern.ptr); break;
    case OR_X_LIDX: put32(s->pattern.idx); break;
    case OR_X_SLOT: put64(s->pattern.slot); break;
    case OR_X_CROW: put32(s->pattern.crow); break;
    case OR_X_CCOL: put32(s->pattern.ccol); break;
    case OR_X_UPTR: {
      int64_t t = 0;
      dst[0] = 0;
      for (int64_t j = 0; j < s->ns; ++j) dst[j + 1] = (t += (int64_t)s->updates[j].size());
      break;
    }
    case OR_X_UK:
    case OR_X_UP1:
    case OR_X_UP2: {
      int64_t t = 0;
      for (auto &l : s->updates)
        for (auto &u : l) dst[t++] = what == OR_X_UK ? u.k : (what == OR_X_UP1 ? u.p1 : u.p2);
      break;
    }
    case OR_X_TASK_LO: put64(s->task_lo); break;
    case OR_X_TASK_HI: put64(s->task_hi); break;
    case OR_X_TOP: put64(s->top); break;
    default: return -1;
  }
  return 0;
}

// Pattern::new with a caller's inverse permutation (cholesky.rs:738-803): lptr[n+1], lidx,
// slot, crow, ccol (sized by the input's entries).
int or_pattern(int64_t n, const int64_t *ptr, const int32_t *idx, const int64_t *inverse, int64_t *lptr, int32_t *lidx,
               int64_t *slot, int32_t *crow, int32_t *ccol) {
  Pattern pt;
  std::vector<int64_t> inv(inverse, inverse + n);
  pattern_new(Upper{n, ptr, idx}, inv, pt);
  std::copy(pt.ptr.begin(), pt.ptr.end(), lptr);
  std::copy(pt.idx.begin(), pt.idx.end(), lidx);
  std::copy(pt.slot.begin(), pt.slot.end(), slot);
  std::copy(pt.crow.begin(), pt.crow.end(), crow);
  std::copy(pt.ccol.begin(), pt.ccol.end(), ccol);
  return 0;
}

// symbolic (blocks when possible) and symbolic_by_columns: parent[n], counts[n].
int or_tree_counts(int64_t n, const int64_t *ptr, const int32_t *idx, int by_columns, int64_t *parent, int64_t *counts) {
  std::vector<int64_t> p, c;
  bool blocks = false;
  if (by_columns)
    symbolic_by_columns(Upper{n, ptr, idx}, p, c);
  else
    symbolic(Upper{n, ptr, idx}, p, c, blocks);
  std::copy(p.begin(), p.end(), parent);
  std::copy(c.begin(), c.end(), counts);
  return blocks ? 1 : 0;
}

int or_postorder(int64_t n, const int64_t *parent, int64_t *post) {
  std::vector<int64_t> p(parent, parent + n);
  auto q = postorder(p);
  std::copy(q.begin(), q.end(), post);
  return (int)q.size() == n ? 0 : -1;
}

// Symbolic::numeric (cholesky.rs:1392-1416): the values in postorder, the diagonal and the
// largest magnitude of each row (= column) of the symmetric matrix.
static Lower lower_of(const or_sym *s, const double *upper_val) {
  Lower a;
  const Pattern &p = s->pattern;
  a.val.assign(p.idx.size(), 0.0);
  a.diag.assign(s->n, 0.0);
  a.scale.assign(s->n, 0.0);
  for (size_t e = 0; e < p.slot.size(); ++e) {
    double v = upper_val[e];
    a.val[p.slot[e]] = v;
    int64_t r = p.crow[e], c = p.ccol[e];
    if (r == c) a.diag[c] = v;
    a.scale[r] = std::max(a.scale[r], std::fabs(v));
    a.scale[c] = std::max(a.scale[c], std::fabs(v));
  }
  return a;
}

// Symbolic::numeric + allocate + factor. column_out receives the failing original column.
int or_factor_new(const or_sym *s, const double *upper_val, const int32_t *cancel, or_factor **out, int64_t *column_out) {
  *out = nullptr;
  *column_out = -1;
  try {
    Lower a = lower_of(s, upper_val);
    auto f = new or_factor();
    f->sym = s;
    f->values.resize(s->ns);
    for (int64_t j = 0; j < s->ns; ++j) f->values[j].assign(trapezoid_size(s->height(j), s->width(j)), 0.0);
    Error e = factor(*s, cancel, [&](int64_t j) { return supernode(*s, a, j, f->values); });
    if (e.code != OK) {
      *column_out = e.column;
      delete f;
      return e.code;
    }
    *out = f;
    return OK;
  } catch (const std::bad_alloc &) {
    return OUT_OF_MEMORY;
  }
}

void or_factor_free(or_factor *f) { delete f; }

// The factor's values, supernode by supernode, each its packed lower trapezoid.
int64_t or_factor_values(const or_factor *f, double *dst) {
  int64_t at = 0;
  for (auto &v : f->values) {
    if (dst) std::memcpy(dst + at, v.data(), sizeof(double) * v.size());
    at += (int64_t)v.size();
  }
  return at;
}

// Factor::solve_many: b column-major n x nrhs (ld = n), in place, by groups of GROUP.
int or_solve(const or_factor *f, double *b, int64_t nrhs) {
  const int64_t n = f->sym->n;
  const auto &perm = f->sym->perm;
  std::vector<double> x(n * GROUP);
  for (int64_t g0 = 0; g0 < nrhs; g0 += GROUP) {
    int kk = (int)std::min<int64_t>(GROUP, nrhs - g0);
    for (int64_t i = 0; i < n; ++i)
      for (int j = 0; j < kk; ++j) x[i * kk + j] = b[(g0 + j) * n + perm[i]];
    solve_group(*f, x.data(), kk);
    for (int64_t i = 0; i < n; ++i)
      for (int j = 0; j < kk; ++j) b[(g0 + j) * n + perm[i]] = x[i * kk + j];
  }
  return 0;
}

// Csr::mul (sparse.rs:42-50): y = A x, each row summed in column order.
void or_spmv(int64_t n, const int64_t *ptr, const int32_t *idx, const double *val, const double *x, double *y) {
  parallel_for((n + 4095) / 4096, [&](int64_t b) {
    for (int64_t r = b * 4096; r < std::min(n, (b + 1) * 4096); ++r) {
      double acc = -0.0;
      for (int64_t p = ptr[r]; p < ptr[r + 1]; ++p) acc += val[p] * x[idx[p]];
      y[r] = acc;
    }
  });
}

// products through the packed micro-tiles (tiled != 0) or column by column, tiles written one
// after another (each cols*TILE entries); returns the entries written, -1 on a tile past the panel.
int64_t or_products(int64_t m, const double *data, int64_t size, int64_t k0, int64_t kw, int64_t p, int64_t mu,
                    int64_t wu, int tiled, double *out) {
  PanelRef l{m, data, size};
  std::vector<std::vector<double>> tiles;
  bool ok = tiled ? products_tiled(l, k0, kw, p, mu, wu, tiles) : products_by_columns(l, k0, kw, p, mu, wu, tiles);
  if (!ok) return -1;
  int64_t at = 0;
  for (auto &t : tiles) {
    if (out) std::memcpy(out + at, t.data(), sizeof(double) * t.size());
    at += (int64_t)t.size();
  }
  return at;
}

// subtract with rel(i) = rel[i]; tiles as or_products lays them out. 0, or -1 on a broken structure.
int or_subtract(double *own, int64_t own_size, int64_t m, const double *tiles_flat, int64_t mu, int64_t wu,
                const int64_t *rel) {
  std::vector<std::vector<double>> tiles;
  int64_t at = 0;
  for (int64_t t = 0; t * TILE < mu; ++t) {
    int64_t h = std::min(TILE, mu - t * TILE), cols = std::min(wu, t * TILE + h);
    tiles.emplace_back(tiles_flat + at, tiles_flat + at + cols * TILE);
    at += cols * TILE;
  }
  return subtract(own, own_size, m, tiles, mu, wu, [&](int64_t i) { return rel[i]; }) ? 0 : -1;
}

// LdltFactor::from_symbolic (ldlt.rs:378-392): numeric + allocate + factor with pivoting.
// column_out receives the failing original column (SINGULAR).
int or_ldlt_new(const or_sym *s, const double *upper_val, const int32_t *cancel, or_ldlt **out, int64_t *column_out) {
  *out = nullptr;
  *column_out = -1;
  try {
    Lower a = lower_of(s, upper_val);
    auto f = new or_ldlt();
    f->sym = s;
    f->blocks.resize(s->ns);
    for (int64_t j = 0; j < s->ns; ++j) f->blocks[j].values.assign(trapezoid_size(s->height(j), s->width(j)), 0.0);
    Error e = factor(*s, cancel, [&](int64_t j) { return ldlt_supernode(*s, a, j, f->blocks); });
    if (e.code != OK) {
      *column_out = e.column;
      delete f;
      return e.code;
    }
    *out = f;
    return OK;
  } catch (const std::bad_alloc &) {
    return OUT_OF_MEMORY;
  }
}

void or_ldlt_free(or_ldlt *f) { delete f; }

// The factor's values (L below the pivots, D on them), supernode by supernode.
int64_t or_ldlt_values(const or_ldlt *f, double *dst) {
  int64_t at = 0;
  for (auto &b : f->blocks) {
    if (dst) std::memcpy(dst + at, b.values.data(), sizeof(double) * b.values.size());
    at += (int64_t)b.values.size();
  }
  return at;
}

// Every supernode's pivots (0 one, 1 first, 2 second of a 2 x 2) and local order, end to end in
// postorder (n entries each).
void or_ldlt_pivots(const or_ldlt *f, int64_t *pivots, int64_t *order) {
  int64_t at = 0;
  for (auto &b : f->blocks) {
    for (size_t c = 0; c < b.pivots.size(); ++c) {
      pivots[at + (int64_t)c] = b.pivots[c];
      order[at + (int64_t)c] = b.order[c];
    }
    at += (int64_t)b.pivots.size();
  }
}

// 0: the 2 x 2 pivots; 1, 2: the positive and negative eigenvalue counts (Sylvester's law on D,
// ldlt.rs:415-447).
int64_t or_ldlt_info(const or_ldlt *f, int what) {
  int64_t two = 0, positive = 0, negative = 0;
  const or_sym &s = *f->sym;
  for (int64_t k = 0; k < s.ns; ++k) {
    const LdltBlock &b = f->blocks[k];
    two += b.two_by_two;
    const PanelRef t{s.height(k), b.values.data(), (int64_t)b.values.size()};
    int64_t c = 0;
    while (c < (int64_t)b.pivots.size()) {
      if (b.pivots[c] == PIVOT_FIRST) {
        const double d11 = t.at(c, c), d21 = t.at(c + 1, c), d22 = t.at(c + 1, c + 1);
        const double det = d11 * d22 - d21 * d21;
        if (det < 0.0) {
          positive += 1;
          negative += 1;
        } else if (d11 + d22 > 0.0) {
          positive += 2;
        } else {
          negative += 2;
        }
        c += 2;
      } else {
        if (t.at(c, c) > 0.0)
          positive += 1;
        else
          negative += 1;
        c += 1;
      }
    }
  }
  return what == 0 ? two : what == 1 ? positive : negative;
}

// LdltFactor::solve_many (ldlt.rs:404-413): b column-major n x nrhs (ld = n), in place, by
// groups of GROUP.
int or_ldlt_solve(const or_ldlt *f, double *b, int64_t nrhs) {
  const or_sym &s = *f->sym;
  const int64_t n = s.n;
  std::vector<double> x(n * GROUP);
  for (int64_t g0 = 0; g0 < nrhs; g0 += GROUP) {
    int kk = (int)std::min<int64_t>(GROUP, nrhs - g0);
    for (int64_t i = 0; i < n; ++i)
      for (int j = 0; j < kk; ++j) x[i * kk + j] = b[(g0 + j) * n + s.perm[i]];
    ldlt_solve_group(s, f->blocks, x.data(), kk);
    for (int64_t i = 0; i < n; ++i)
      for (int j = 0; j < kk; ++j) b[(g0 + j) * n + s.perm[i]] = x[i * kk + j];
  }
  return 0;
}

}  // extern "C"
