// Host-side symbolic analysis of the supernodal Cholesky: the elimination tree and column
// counts (by 3-unknown blocks when the matrix has them), the postorder, the lower pattern in
// postorder with the gather map of the input's entries, the fundamental supernodes, their row
// structures, the per-target update lists and the subtree tasks. It restates
// crates/solver/src/cholesky.rs:150-342 and 1195-1416 so that the structure (and therefore the
// fill and the supernode partition) is the reference's bit for bit.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace fc {

constexpr int64_t NONE = -1;

// Error codes shared with the C ABI (fieldcraft_chol.h FC_* values).
enum Code : int32_t {
  OK = 0,
  NOT_POSITIVE_DEFINITE = 1,
  SINGULAR = 2,
  TOO_LARGE = 3,
  OUT_OF_MEMORY = 4,
  INTERNAL = 5,
  CANCELLED = 6,
  TIMEOUT = 7,
  INVALID_ARGUMENT = 8,
  CUDA_ERROR = 9,
};

struct Failure {
  Code code = OK;
  int64_t column = -1, entries = 0, limit = 0;
  std::string message;
};

// The upper triangle of a symmetric matrix by columns (cholesky.rs:102-107): column k holds the
// rows i <= k, sorted. Only the pattern is needed for the analysis.
struct UpperPattern {
  int64_t n = 0;
  const int64_t *ptr = nullptr;  // n + 1
  const int32_t *idx = nullptr;  // ptr[n]
};

struct Symbolic {
  int64_t n = 0, ns = 0, entries = 0;
  std::vector<int64_t> perm;     // perm[k]: original column of factor column k
  std::vector<int64_t> first;    // ns + 1: first column of each supernode, n at the end
  std::vector<int64_t> rptr;     // ns + 1
  std::vector<int32_t> rows;     // row structure of each supernode, own columns first, sorted
  std::vector<int64_t> sparent;  // supernodal tree, NONE at roots
  // The lower triangle in postorder (Pattern, cholesky.rs:728-803).
  std::vector<int64_t> lptr;     // n + 1
  std::vector<int32_t> lidx;
  std::vector<int64_t> slot;     // per upper entry: its position in lidx
  std::vector<int32_t> crow, ccol;  // per upper entry: (row, column) in postorder, row >= column
  std::vector<int64_t> upper_ptr;
  std::vector<int32_t> upper_idx;
  // Updates each supernode receives (cholesky.rs:385-389, 1314-1330), by target, in order.
  std::vector<int64_t> uptr;     // ns + 1
  std::vector<int64_t> uk, up1, up2;
  // Subtree tasks (ranges of supernodes) and the supernodes above them (cholesky.rs:1332-1375).
  std::vector<int64_t> task_lo, task_hi, top;

  int64_t width(int64_t s) const { return first[s + 1] - first[s]; }
  int64_t height(int64_t s) const { return rptr[s + 1] - rptr[s]; }
};

// Entries of an m-row, w-column lower trapezoid, and where its column c starts (cholesky.rs:418-425).
inline int64_t trapezoid(int64_t m, int64_t w) {
  int64_t s = 0;
  for (int64_t c = 0; c < w; ++c) s += m > c ? m - c : 0;
  return s;
}
inline int64_t trapezoid_offset(int64_t m, int64_t c) { return c * m - c * (c > 0 ? c - 1 : 0) / 2; }

// The postorder of a forest given by parents, children ascending (cholesky.rs:309-342).
std::vector<int64_t> postorder(const std::vector<int64_t> &parent);
// Elimination tree and column counts, by blocks of three when possible (cholesky.rs:230-287).
void tree_and_counts(const UpperPattern &a, std::vector<int64_t> &parent, std::vector<int64_t> &counts,
                     bool *by_blocks = nullptr);
// The same, column by column for any matrix (cholesky.rs:290-305).
void tree_and_counts_by_columns(const UpperPattern &a, std::vector<int64_t> &parent,
                                std::vector<int64_t> &counts);
// Symbolic::new (cholesky.rs:1212-1378). Returns false with `fail` set on TooLarge/Internal/OOM.
bool analyse(const UpperPattern &a, uint64_t max_entries, Symbolic &out, Failure &fail);

}  // namespace fc
