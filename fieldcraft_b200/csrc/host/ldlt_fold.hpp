// The triangular solve's structure for an LDL^T factor: the factor's pivot orders folded into the
// supernodal structure, so that the Cholesky solve runs on it unchanged (see ldlt_fold.cpp).
#pragma once

#include <cstdint>
#include <vector>

namespace fc {

struct LdltFold {
  std::vector<int64_t> perm;      // [n] the original column at each new place
  std::vector<int32_t> rows;      // like the structure's rows, in new places, each supernode's sorted
  std::vector<int32_t> from;      // per supernode, its rows below: new row i was old row from[i]
  std::vector<int64_t> from_off;  // [ns + 1] where each supernode's `from` starts
  std::vector<int32_t> rel;       // per supernode with a parent: each row below, its place in the parent's rows
  std::vector<int64_t> rel_off;   // [ns]
};

// first[ns + 1], rptr[ns + 1], rows (the structure: own columns first, then the rows below,
// sorted), perm[n] (the analysis' postorder), sparent[ns] (-1 at roots), order[n] (per supernode
// its own column at each pivot position, as the factor left it). False when order is not a
// permutation within each supernode or a row below is not in its parent.
bool ldlt_fold(int64_t n, int64_t ns, const int64_t *first, const int64_t *rptr, const int32_t *rows,
               const int64_t *perm, const int64_t *sparent, const int32_t *order, LdltFold &out);

}  // namespace fc
