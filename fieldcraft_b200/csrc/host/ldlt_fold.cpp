// The LDL^T factor's pivot orders folded into the solve's structure. A supernode's own columns
// sit at their pivot positions (pos[f + order[c]] = f + c), so its own block is unit lower in the
// order the factor stored it; every row index elsewhere moves through pos. A supernode's rows below
// are then sorted again (rows of one ancestor's columns change order among themselves only), and
// `from` records how, so that the factor's L21 rows can be moved the same way; the relative maps
// (a child's rows below in its parent's rows) follow from the new rows. The solve then runs as the
// Cholesky solve on unit lower blocks, with D^-1 between its passes (ldlt.rs's solve order:
// cholesky.rs:904-1037 with pivots and order).
#include "ldlt_fold.hpp"

#include <algorithm>
#include <numeric>

namespace fc {

bool ldlt_fold(int64_t n, int64_t ns, const int64_t *first, const int64_t *rptr, const int32_t *rows,
               const int64_t *perm, const int64_t *sparent, const int32_t *order, LdltFold &out) {
  std::vector<int64_t> pos(n, -1);
  for (int64_t s = 0; s < ns; ++s) {
    const int64_t f = first[s], w = first[s + 1] - f;
    for (int64_t c = 0; c < w; ++c) {
      const int64_t o = order[f + c];
      if (o < 0 || o >= w || pos[f + o] >= 0) return false;
      pos[f + o] = f + c;
    }
  }
  out.perm.assign(n, 0);
  for (int64_t i = 0; i < n; ++i) out.perm[pos[i]] = perm[i];
  const int64_t total = ns ? rptr[ns] : 0;
  out.rows.assign(rows, rows + total);
  out.from_off.assign(ns + 1, 0);
  for (int64_t s = 0; s < ns; ++s)
    out.from_off[s + 1] = out.from_off[s] + (rptr[s + 1] - rptr[s]) - (first[s + 1] - first[s]);
  out.from.assign(out.from_off[ns], 0);
  std::vector<std::pair<int32_t, int32_t>> below;
  for (int64_t s = 0; s < ns; ++s) {
    const int64_t f = first[s], w = first[s + 1] - f, m = rptr[s + 1] - rptr[s];
    int32_t *r = out.rows.data() + rptr[s];
    for (int64_t c = 0; c < w; ++c) r[c] = (int32_t)(f + c);
    below.clear();
    for (int64_t i = w; i < m; ++i) below.emplace_back((int32_t)pos[rows[rptr[s] + i]], (int32_t)(i - w));
    std::sort(below.begin(), below.end());
    for (size_t i = 0; i < below.size(); ++i) {
      r[w + (int64_t)i] = below[i].first;
      out.from[out.from_off[s] + (int64_t)i] = below[i].second;
    }
  }
  out.rel_off.assign(ns, 0);
  out.rel.clear();
  for (int64_t c = 0; c < ns; ++c) {
    out.rel_off[c] = (int64_t)out.rel.size();
    const int64_t p = sparent[c];
    if (p < 0) continue;
    const int32_t *cr = out.rows.data() + rptr[c], *pr = out.rows.data() + rptr[p];
    const int64_t cw = first[c + 1] - first[c], cm = rptr[c + 1] - rptr[c], pm = rptr[p + 1] - rptr[p];
    int64_t at = 0;
    for (int64_t i = cw; i < cm; ++i) {
      while (at < pm && pr[at] < cr[i]) ++at;
      if (at >= pm || pr[at] != cr[i]) return false;
      out.rel.push_back((int32_t)at);
    }
  }
  return true;
}

}  // namespace fc
