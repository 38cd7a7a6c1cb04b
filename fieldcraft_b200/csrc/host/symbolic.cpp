// Symbolic analysis of the supernodal Cholesky (see symbolic.hpp for what it restates).
#include "symbolic.hpp"

#include <algorithm>
#include <new>

namespace fc {

namespace {

// Unknowns of a block that share one structure (cholesky.rs:221).
constexpr int64_t BLOCK = 3;
// Dense work from which the reference runs a kernel's tiles in parallel (cholesky.rs:67), and
// the share of the total work a subtree task takes (cholesky.rs:97).
constexpr uint64_t PARALLEL_WORK = 1ull << 21;
constexpr uint64_t SUBTREE_SHARE = 256;

uint64_t sat_add(uint64_t a, uint64_t b) { return a + b < a ? UINT64_MAX : a + b; }
uint64_t sat_mul(uint64_t a, uint64_t b) {
  if (a == 0 || b == 0) return 0;
  return a > UINT64_MAX / b ? UINT64_MAX : a * b;
}

struct Cols {
  int64_t n;
  const int64_t *ptr;
  const int32_t *idx;
};

void etree_counts(const Cols &a, std::vector<int64_t> &parent, std::vector<int64_t> &counts) {
  const int64_t n = a.n;
  parent.assign(n, NONE);
  std::vector<int64_t> ancestor(n, NONE);
  for (int64_t k = 0; k < n; ++k)
    for (int64_t p = a.ptr[k]; p < a.ptr[k + 1]; ++p) {
      int64_t i = a.idx[p];
      // Walk to the root of i's current subtree, compressing the path to k (cholesky.rs:157-180).
      while (i != NONE && i < k) {
        int64_t next = ancestor[i];
        ancestor[i] = k;
        if (next == NONE) parent[i] = k;
        i = next;
      }
    }
  counts.assign(n, 1);
  std::vector<int64_t> mark(n, NONE);
  // Row k of L is the reach of column k's entries in the tree (cholesky.rs:185-213); each column
  // it reaches gains one entry.
  for (int64_t k = 0; k < n; ++k) {
    mark[k] = k;
    for (int64_t p = a.ptr[k]; p < a.ptr[k + 1]; ++p) {
      int64_t i = a.idx[p];
      if (i > k) continue;
      while (i != NONE && mark[i] != k) {
        ++counts[i];
        mark[i] = k;
        i = parent[i];
      }
    }
  }
}

// The blocks' matrix when every block of three unknowns has one structure (cholesky.rs:230-262).
bool uniform_blocks(const UpperPattern &a, std::vector<int64_t> &bptr, std::vector<int32_t> &bidx) {
  if (a.n == 0 || a.n % BLOCK != 0) return false;
  const int64_t nb = a.n / BLOCK;
  bptr.assign(1, 0);
  bptr.reserve(nb + 1);
  bidx.clear();
  for (int64_t q = 0; q < nb; ++q) {
    const int64_t c0 = BLOCK * q;
    const int64_t s0 = a.ptr[c0], e0 = a.ptr[c0 + 1];
    if (e0 == s0 || a.idx[e0 - 1] != c0) return false;
    const int64_t above = e0 - 1 - s0;
    if (above % BLOCK != 0) return false;
    for (int64_t t = 0; t < above; t += BLOCK) {
      const int64_t f = a.idx[s0 + t];
      if (f % BLOCK != 0) return false;
      for (int64_t i = 1; i < BLOCK; ++i)
        if (a.idx[s0 + t + i] != f + i) return false;
      bidx.push_back((int32_t)(f / BLOCK));
    }
    bidx.push_back((int32_t)q);
    for (int64_t c = 1; c < BLOCK; ++c) {
      const int64_t s = a.ptr[c0 + c], e = a.ptr[c0 + c + 1];
      if (e - s != above + c + 1) return false;
      for (int64_t t = 0; t < above; ++t)
        if (a.idx[s + t] != a.idx[s0 + t]) return false;
      for (int64_t i = 0; i <= c; ++i)
        if (a.idx[s + above + i] != c0 + i) return false;
    }
    bptr.push_back((int64_t)bidx.size());
  }
  return true;
}

}  // namespace

void tree_and_counts_by_columns(const UpperPattern &a, std::vector<int64_t> &parent, std::vector<int64_t> &counts) {
  etree_counts(Cols{a.n, a.ptr, a.idx}, parent, counts);
}

void tree_and_counts(const UpperPattern &a, std::vector<int64_t> &parent, std::vector<int64_t> &counts,
                     bool *by_blocks) {
  std::vector<int64_t> bptr;
  std::vector<int32_t> bidx;
  const bool blocks = uniform_blocks(a, bptr, bidx);
  if (by_blocks) *by_blocks = blocks;
  if (!blocks) {
    tree_and_counts_by_columns(a, parent, counts);
    return;
  }
  std::vector<int64_t> bparent, bcounts;
  etree_counts(Cols{a.n / BLOCK, bptr.data(), bidx.data()}, bparent, bcounts);
  parent.resize(a.n);
  counts.resize(a.n);
  // Within a block every unknown's parent is the next one; the last one's is the first unknown
  // of the block's parent; unknown c has BLOCK * count - c entries (cholesky.rs:264-287).
  for (int64_t q = 0; q < a.n / BLOCK; ++q)
    for (int64_t c = 0; c < BLOCK; ++c) {
      parent[BLOCK * q + c] = c + 1 < BLOCK ? BLOCK * q + c + 1 : (bparent[q] == NONE ? NONE : BLOCK * bparent[q]);
      counts[BLOCK * q + c] = BLOCK * bcounts[q] - c;
    }
}

std::vector<int64_t> postorder(const std::vector<int64_t> &parent) {
  const int64_t n = (int64_t)parent.size();
  std::vector<int64_t> head(n, NONE), next(n, NONE);
  for (int64_t j = n - 1; j >= 0; --j) {
    const int64_t p = parent[j];
    if (p < 0 || p >= n) continue;
    next[j] = head[p];
    head[p] = j;
  }
  std::vector<int64_t> post;
  post.reserve(n);
  std::vector<int64_t> stack;
  for (int64_t root = 0; root < n; ++root) {
    if (parent[root] != NONE) continue;
    stack.push_back(root);
    while (!stack.empty()) {
      const int64_t top = stack.back();
      const int64_t child = head[top];
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

bool analyse(const UpperPattern &a, uint64_t max_entries, Symbolic &out, Failure &fail) {
  try {
    const int64_t n = a.n;
    auto internal = [&](const char *what) {
      fail.code = INTERNAL;
      fail.message = std::string("supernodal structure: ") + what;
      return false;
    };
    std::vector<int64_t> parent0, counts0;
    tree_and_counts(a, parent0, counts0);
    uint64_t total = 0;
    for (int64_t c : counts0) total = sat_add(total, (uint64_t)c);
    if (total > max_entries) {
      fail.code = TOO_LARGE;
      fail.entries = (int64_t)std::min<uint64_t>(total, INT64_MAX);
      fail.limit = (int64_t)std::min<uint64_t>(max_entries, INT64_MAX);
      return false;
    }
    Symbolic &s = out;
    s = Symbolic();
    s.n = n;
    s.entries = (int64_t)total;
    s.perm = postorder(parent0);
    if ((int64_t)s.perm.size() != n) return internal("postorder");
    std::vector<int64_t> inverse(n);
    for (int64_t k = 0; k < n; ++k) inverse[s.perm[k]] = k;
    std::vector<int64_t> parent(n), counts(n);
    for (int64_t k = 0; k < n; ++k) {
      const int64_t p = parent0[s.perm[k]];
      parent[k] = p == NONE ? NONE : inverse[p];
      counts[k] = counts0[s.perm[k]];
    }
    // Pattern::new: the lower triangle in postorder with the position of each upper entry.
    const int64_t nnz = a.ptr[n];
    s.upper_ptr.assign(a.ptr, a.ptr + n + 1);
    s.upper_idx.assign(a.idx, a.idx + nnz);
    s.lptr.assign(n + 1, 0);
    for (int64_t k = 0; k < n; ++k)
      for (int64_t p = a.ptr[k]; p < a.ptr[k + 1]; ++p)
        s.lptr[std::min(inverse[a.idx[p]], inverse[k]) + 1] += 1;
    for (int64_t j = 0; j < n; ++j) s.lptr[j + 1] += s.lptr[j];
    std::vector<std::pair<int64_t, int64_t>> entries(s.lptr[n]);
    std::vector<int64_t> next(s.lptr.begin(), s.lptr.end() - 1);
    s.crow.resize(nnz);
    s.ccol.resize(nnz);
    for (int64_t k = 0; k < n; ++k)
      for (int64_t p = a.ptr[k]; p < a.ptr[k + 1]; ++p) {
        const int64_t ni = inverse[a.idx[p]], nk = inverse[k];
        const int64_t r = std::max(ni, nk), c = std::min(ni, nk);
        s.crow[p] = (int32_t)r;
        s.ccol[p] = (int32_t)c;
        entries[next[c]++] = {r, p};
      }
    for (int64_t j = 0; j < n; ++j)
      std::stable_sort(entries.begin() + s.lptr[j], entries.begin() + s.lptr[j + 1],
                       [](const auto &x, const auto &y) { return x.first < y.first; });
    s.slot.resize(nnz);
    s.lidx.resize(entries.size());
    for (size_t pos = 0; pos < entries.size(); ++pos) {
      s.slot[entries[pos].second] = (int64_t)pos;
      s.lidx[pos] = (int32_t)entries[pos].first;
    }
    entries.clear();
    entries.shrink_to_fit();
    // Fundamental supernodes (cholesky.rs:1236-1253).
    std::vector<int64_t> children(n, 0);
    for (int64_t p : parent)
      if (p != NONE) ++children[p];
    s.first.assign(1, 0);
    for (int64_t j = 1; j < n; ++j) {
      const bool joins = parent[j - 1] == j && children[j] == 1 && counts[j - 1] == counts[j] + 1;
      if (!joins) s.first.push_back(j);
    }
    if (n > 0) s.first.push_back(n);
    const int64_t ns = (int64_t)s.first.size() - 1 > 0 ? (int64_t)s.first.size() - 1 : 0;
    s.ns = ns;
    if (n == 0) s.first.assign(1, 0);
    std::vector<int64_t> snode(n);
    for (int64_t t = 0; t < ns; ++t)
      for (int64_t j = s.first[t]; j < s.first[t + 1]; ++j) snode[j] = t;
    s.sparent.assign(ns, NONE);
    for (int64_t t = 0; t < ns; ++t) {
      const int64_t last = s.first[t + 1] - 1;
      s.sparent[t] = parent[last] == NONE ? NONE : snode[parent[last]];
    }
    std::vector<int64_t> kptr(ns + 1, 0), kids;
    for (int64_t t = 0; t < ns; ++t)
      if (s.sparent[t] != NONE) ++kptr[s.sparent[t] + 1];
    for (int64_t t = 0; t < ns; ++t) kptr[t + 1] += kptr[t];
    kids.resize(kptr[ns]);
    {
      std::vector<int64_t> at(kptr.begin(), kptr.end() - 1);
      for (int64_t t = 0; t < ns; ++t)
        if (s.sparent[t] != NONE) kids[at[s.sparent[t]]++] = t;
    }
    // Row structures: own columns, rows of A below them, children's rows past their columns.
    s.rptr.assign(1, 0);
    std::vector<int64_t> mark(n, NONE);
    std::vector<int32_t> set;
    for (int64_t t = 0; t < ns; ++t) {
      const int64_t f = s.first[t], l = s.first[t + 1];
      set.clear();
      auto add = [&](int64_t r) {
        if (mark[r] != t) {
          mark[r] = t;
          set.push_back((int32_t)r);
        }
      };
      for (int64_t j = f; j < l; ++j) {
        add(j);
        for (int64_t p = s.lptr[j]; p < s.lptr[j + 1]; ++p) add(s.lidx[p]);
      }
      for (int64_t q = kptr[t]; q < kptr[t + 1]; ++q) {
        const int64_t c = kids[q];
        const int64_t cw = s.first[c + 1] - s.first[c];
        for (int64_t p = s.rptr[c] + cw; p < s.rptr[c + 1]; ++p) add(s.rows[p]);
      }
      std::sort(set.begin(), set.end());
      if ((int64_t)set.size() != counts[f] || set.empty() || set[0] != f)
        return internal("a supernode's rows differ from its column count");
      s.rows.insert(s.rows.end(), set.begin(), set.end());
      s.rptr.push_back((int64_t)s.rows.size());
    }
    // Updates each supernode receives from its descendants, in increasing order (cholesky.rs:1314-1330).
    std::vector<int64_t> ucount(ns + 1, 0);
    std::vector<int64_t> tk, t1, t2, tt;
    for (int64_t k = 0; k < ns; ++k) {
      const int32_t *kr = s.rows.data() + s.rptr[k];
      const int64_t m = s.rptr[k + 1] - s.rptr[k];
      int64_t p = s.first[k + 1] - s.first[k];
      while (p < m) {
        const int64_t target = snode[kr[p]];
        const int64_t end = s.first[target + 1];
        int64_t q = p;
        while (q < m && kr[q] < end) ++q;
        tk.push_back(k);
        t1.push_back(p);
        t2.push_back(q);
        tt.push_back(target);
        ++ucount[target + 1];
        p = q;
      }
    }
    for (int64_t t = 0; t < ns; ++t) ucount[t + 1] += ucount[t];
    s.uptr = ucount;
    s.uk.resize(tk.size());
    s.up1.resize(tk.size());
    s.up2.resize(tk.size());
    {
      std::vector<int64_t> at(ucount.begin(), ucount.end() - 1);
      for (size_t e = 0; e < tk.size(); ++e) {
        const int64_t pos = at[tt[e]]++;
        s.uk[pos] = tk[e];
        s.up1[pos] = t1[e];
        s.up2[pos] = t2[e];
      }
    }
    // Subtree tasks of at most a share of the work each, and the supernodes above them.
    std::vector<uint64_t> subtree(ns);
    std::vector<int64_t> start(ns);
    for (int64_t t = 0; t < ns; ++t) {
      const uint64_t m = (uint64_t)s.height(t), w = (uint64_t)s.width(t);
      uint64_t work = 0;
      for (uint64_t c = 0; c < w; ++c) work = sat_add(work, sat_mul(m - c, m - c));
      subtree[t] = work;
      start[t] = t;
    }
    for (int64_t t = 0; t < ns; ++t) {
      const int64_t p = s.sparent[t];
      if (p != NONE) {
        subtree[p] = sat_add(subtree[p], subtree[t]);
        start[p] = std::min(start[p], start[t]);
      }
    }
    uint64_t all = 0;
    for (int64_t t = 0; t < ns; ++t)
      if (s.sparent[t] == NONE) all = sat_add(all, subtree[t]);
    const uint64_t share = std::max(all / SUBTREE_SHARE, PARALLEL_WORK);
    int64_t t = 0;
    while (t < ns) {
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
    return true;
  } catch (const std::bad_alloc &) {
    fail.code = OUT_OF_MEMORY;
    fail.entries = 0;
    return false;
  }
}

}  // namespace fc
