// Structured hex8 models for the Cholesky path: mesh, node graph, fill-reducing order, free-DOF
// numbering, element stiffness and assembly of K_ff. Declared in include/fieldcraft_fem.h, whose
// head names the reference files each part restates.
#include "fieldcraft_fem.h"
#include "assembly.hpp"
#include "hex8.hpp"
#include "stress.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <new>
#include <thread>
#include <vector>

namespace {

constexpr int64_t NONE = -1;
// Parts this small are ordered as they come (crates/solver/src/ordering.rs:25).
constexpr size_t LEAF = 16;
// Pseudo-peripheral searches per part (ordering.rs:114).
constexpr int PERIPHERAL_SEARCHES = 8;

struct Graph {
  int64_t n;
  const int64_t *ptr;
  const int32_t *idx;
  const int32_t *begin(int64_t v) const { return idx + ptr[v]; }
  const int32_t *end(int64_t v) const { return idx + ptr[v + 1]; }
};

// Nested dissection by coordinate bisection (ordering.rs:28-98): split at the median of the
// longest axis (ties by node index), the smaller boundary is the separator, parts then separator.
std::vector<int64_t> nested_dissection(const Graph &g, const double *xyz) {
  const int64_t n = g.n;
  std::vector<int64_t> order;
  order.reserve(n);
  std::vector<uint8_t> side(n, 0);
  struct Task { bool emit; std::vector<int64_t> nodes; };
  std::vector<Task> stack;
  {
    std::vector<int64_t> all(n);
    for (int64_t v = 0; v < n; ++v) all[v] = v;
    stack.push_back({false, std::move(all)});
  }
  while (!stack.empty()) {
    Task task = std::move(stack.back());
    stack.pop_back();
    if (task.emit) {
      order.insert(order.end(), task.nodes.begin(), task.nodes.end());
      continue;
    }
    std::vector<int64_t> &part = task.nodes;
    if (part.size() <= LEAF) {
      order.insert(order.end(), part.begin(), part.end());
      continue;
    }
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t v : part)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], xyz[3 * v + k]);
        hi[k] = std::max(hi[k], xyz[3 * v + k]);
      }
    int axis = 0;
    for (int k = 0; k < 3; ++k)
      if (hi[k] - lo[k] > hi[axis] - lo[axis]) axis = k;
    // total order on doubles (no NaN expected in coordinates), ties by index
    std::sort(part.begin(), part.end(), [&](int64_t a, int64_t b) {
      double ka = xyz[3 * a + axis], kb = xyz[3 * b + axis];
      if (ka < kb) return true;
      if (kb < ka) return false;
      return a < b;
    });
    const size_t half = part.size() / 2;
    for (size_t i = 0; i < part.size(); ++i) side[part[i]] = i < half ? 1 : 2;
    auto touches = [&](int64_t v, uint8_t other) {
      for (const int32_t *w = g.begin(v); w != g.end(v); ++w)
        if (side[*w] == other) return true;
      return false;
    };
    std::vector<int64_t> lb, rb;
    for (size_t i = 0; i < half; ++i)
      if (touches(part[i], 2)) lb.push_back(part[i]);
    for (size_t i = half; i < part.size(); ++i)
      if (touches(part[i], 1)) rb.push_back(part[i]);
    std::vector<int64_t> sep = lb.size() <= rb.size() ? std::move(lb) : std::move(rb);
    for (int64_t v : part) side[v] = 0;
    for (int64_t v : sep) side[v] = 3;
    std::vector<int64_t> a, b;
    for (size_t i = 0; i < half; ++i)
      if (side[part[i]] != 3) a.push_back(part[i]);
    for (size_t i = half; i < part.size(); ++i)
      if (side[part[i]] != 3) b.push_back(part[i]);
    for (int64_t v : sep) side[v] = 0;
    stack.push_back({true, std::move(sep)});
    stack.push_back({false, std::move(b)});
    stack.push_back({false, std::move(a)});
  }
  return order;
}

// Breadth-first level structure of the nodes owned by `token` from `root` (ordering.rs:118-141).
std::vector<std::vector<int64_t>> level_structure(const Graph &g, int64_t root, int64_t token,
                                                  const std::vector<int64_t> &owner,
                                                  std::vector<int64_t> &level) {
  std::vector<std::vector<int64_t>> out;
  out.push_back({root});
  level[root] = 0;
  for (;;) {
    const int64_t depth = (int64_t)out.size();
    std::vector<int64_t> next;
    for (int64_t v : out.back())
      for (const int32_t *w = g.begin(v); w != g.end(v); ++w)
        if (owner[*w] == token && level[*w] == NONE) {
          level[*w] = depth;
          next.push_back(*w);
        }
    if (next.empty()) return out;
    out.push_back(std::move(next));
  }
}

void clear_levels(std::vector<int64_t> &level, const std::vector<std::vector<int64_t>> &s) {
  for (const auto &l : s)
    for (int64_t v : l) level[v] = NONE;
}

// Nested dissection on the graph alone: separators from the middle level of a level structure
// rooted at a pseudo-peripheral node (ordering.rs:157-253).
std::vector<int64_t> graph_dissection(const Graph &g) {
  const int64_t n = g.n;
  std::vector<int64_t> order;
  order.reserve(n);
  std::vector<int64_t> owner(n, 0), level(n, NONE);
  int64_t token = 0;
  struct Task { bool emit; std::vector<int64_t> nodes; };
  std::vector<Task> stack;
  {
    std::vector<int64_t> all(n);
    for (int64_t v = 0; v < n; ++v) all[v] = v;
    stack.push_back({false, std::move(all)});
  }
  while (!stack.empty()) {
    Task task = std::move(stack.back());
    stack.pop_back();
    if (task.emit) {
      order.insert(order.end(), task.nodes.begin(), task.nodes.end());
      continue;
    }
    std::vector<int64_t> &part = task.nodes;
    if (part.empty()) continue;
    const int64_t first = part[0];
    if (part.size() <= LEAF) {
      order.insert(order.end(), part.begin(), part.end());
      continue;
    }
    ++token;
    for (int64_t v : part) owner[v] = token;
    auto degree = [&](int64_t v) {
      int64_t d = 0;
      for (const int32_t *w = g.begin(v); w != g.end(v); ++w) d += owner[*w] == token;
      return d;
    };
    auto structure = level_structure(g, first, token, owner, level);
    for (int it = 0; it < PERIPHERAL_SEARCHES; ++it) {
      const auto &last = structure.back();
      if (last.empty()) break;
      int64_t cand = last[0], cd = degree(last[0]);
      for (int64_t v : last) {
        int64_t d = degree(v);
        if (d < cd || (d == cd && v < cand)) { cand = v; cd = d; }
      }
      clear_levels(level, structure);
      auto deeper = level_structure(g, cand, token, owner, level);
      if (deeper.size() <= structure.size()) {
        clear_levels(level, deeper);
        for (size_t dpt = 0; dpt < structure.size(); ++dpt)
          for (int64_t v : structure[dpt]) level[v] = (int64_t)dpt;
        break;
      }
      structure = std::move(deeper);
    }
    size_t reached = 0;
    for (const auto &l : structure) reached += l.size();
    if (reached < part.size()) {
      std::vector<int64_t> rest;
      for (int64_t v : part)
        if (level[v] == NONE) rest.push_back(v);
      clear_levels(level, structure);
      std::vector<int64_t> comp;
      for (const auto &l : structure) comp.insert(comp.end(), l.begin(), l.end());
      std::sort(comp.begin(), comp.end());
      stack.push_back({false, std::move(rest)});
      stack.push_back({false, std::move(comp)});
      continue;
    }
    if (structure.size() < 3) {
      clear_levels(level, structure);
      order.insert(order.end(), part.begin(), part.end());
      continue;
    }
    size_t count = 0, middle = 1;
    for (size_t i = 1; i < structure.size(); ++i) {
      count += structure[i].size();
      if (2 * count >= part.size()) {
        middle = std::min(i, structure.size() - 2);
        break;
      }
    }
    auto touches_next = [&](int64_t v) {
      for (const int32_t *w = g.begin(v); w != g.end(v); ++w)
        if (owner[*w] == token && level[*w] == (int64_t)middle + 1) return true;
      return false;
    };
    std::vector<int64_t> sep, before, after;
    for (size_t i = 0; i < middle; ++i) before.insert(before.end(), structure[i].begin(), structure[i].end());
    for (int64_t v : structure[middle]) (touches_next(v) ? sep : before).push_back(v);
    for (size_t i = middle + 1; i < structure.size(); ++i)
      after.insert(after.end(), structure[i].begin(), structure[i].end());
    clear_levels(level, structure);
    std::sort(before.begin(), before.end());
    std::sort(sep.begin(), sep.end());
    std::sort(after.begin(), after.end());
    stack.push_back({true, std::move(sep)});
    stack.push_back({false, std::move(after)});
    stack.push_back({false, std::move(before)});
  }
  return order;
}

// Entries of the Cholesky factor of the node graph in `order` (ordering.rs:257-281): column
// counts from the elimination tree and the row subtrees (crates/solver/src/cholesky.rs:157-213,
// 290-305), one unknown per node.
int64_t fill_of(const Graph &g, const int64_t *order) {
  const int64_t n = g.n;
  std::vector<int64_t> position(n, NONE);
  for (int64_t k = 0; k < n; ++k) {
    if (order[k] < 0 || order[k] >= n || position[order[k]] != NONE) return -1;
    position[order[k]] = k;
  }
  // Upper columns: column k holds the positions r <= k of node order[k]'s neighbours.
  std::vector<int64_t> ptr(n + 1, 0);
  std::vector<int64_t> idx;
  idx.reserve(g.ptr[n] / 2 + n);
  std::vector<int64_t> rows;
  for (int64_t k = 0; k < n; ++k) {
    rows.clear();
    const int64_t v = order[k];
    for (const int32_t *w = g.begin(v); w != g.end(v); ++w)
      if (position[*w] < k) rows.push_back(position[*w]);
    rows.push_back(k);
    std::sort(rows.begin(), rows.end());
    rows.erase(std::unique(rows.begin(), rows.end()), rows.end());
    idx.insert(idx.end(), rows.begin(), rows.end());
    ptr[k + 1] = (int64_t)idx.size();
  }
  std::vector<int64_t> parent(n, NONE), ancestor(n, NONE);
  for (int64_t k = 0; k < n; ++k)
    for (int64_t p = ptr[k]; p < ptr[k + 1]; ++p) {
      int64_t i = idx[p];
      while (i != NONE && i < k) {
        int64_t next = ancestor[i];
        ancestor[i] = k;
        if (next == NONE) parent[i] = k;
        i = next;
      }
    }
  std::vector<int64_t> mark(n, NONE);
  int64_t total = n;
  for (int64_t k = 0; k < n; ++k) {
    mark[k] = k;
    for (int64_t p = ptr[k]; p < ptr[k + 1]; ++p) {
      int64_t i = idx[p];
      if (i > k) continue;
      while (i != NONE && mark[i] != k) {
        ++total;
        mark[i] = k;
        i = parent[i];
      }
    }
  }
  return total;
}

std::vector<int64_t> fill_reducing(const Graph &g, const double *xyz) {
  std::vector<int64_t> planes = nested_dissection(g, xyz);
  if ((size_t)g.n <= LEAF) return planes;
  std::vector<int64_t> graph = graph_dissection(g);
  return fill_of(g, graph.data()) < fill_of(g, planes.data()) ? graph : planes;
}

// ---- hex8 element ----------------------------------------------------------------------------

// The element's stiffness (host/hex8.hpp, shared with the device assembly).
bool hex8_stiffness(const double *xyz, double young, double nu, double *k) {
  return fc::hex8::stiffness(xyz, young, nu, k);
}

int hardware_threads(int threads) {
  if (threads > 0) return threads;
  unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

}  // namespace

struct fc_problem {
  int64_t nodes = 0, n = 0;
  std::vector<int64_t> order, eq, ptr;
  std::vector<int32_t> idx;
  std::vector<double> val;
};

extern "C" {

// Not part of the public ABI: K_ff of a box assembled entry by entry on the host with the device
// assembly's code (host/assembly.hpp), for tests; val[ptr[n]] in the pattern's order. eq as
// fc_fem_equations gives it. Returns FC_FEM_OK, or FC_FEM_INVALID for an invalid element.
int fc_test_fem_assemble_host(int nx, int ny, int nz, double lx, double ly, double lz, int64_t n, const int64_t *ptr,
                              const int32_t *idx, const int64_t *eq, const double *young, double poisson,
                              double *val) {
  const fc::assembly::Box box{nx, ny, nz, lx, ly, lz};
  const int64_t elements = (int64_t)nx * ny * nz, nodes = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
  std::vector<double> ke((size_t)elements * 576);
  for (int64_t e = 0; e < elements; ++e) {
    double x[24];
    fc::assembly::element_corners(box, e, x);
    if (!fc::hex8::stiffness(x, young[e], poisson, ke.data() + e * 576)) return FC_FEM_INVALID;
  }
  std::vector<int64_t> node(n / 3);
  for (int64_t v = 0; v < nodes; ++v)
    if (eq[3 * v] >= 0) node[eq[3 * v] / 3] = v;
  for (int64_t r = 0; r < n; ++r)
    for (int64_t q = ptr[r]; q < ptr[r + 1]; ++q)
      val[q] = fc::assembly::entry(box, node[r / 3], (int)(r % 3), node[idx[q] / 3], idx[q] % 3, ke.data());
  return FC_FEM_OK;
}

// Not part of the public ABI: the reactions at the held DOFs (zero elsewhere) for the free
// equations' solution q and the loads f over every DOF, with the device assembly's code, for tests.
int fc_test_fem_reactions_host(int nx, int ny, int nz, double lx, double ly, double lz, const int64_t *eq,
                               const double *young, double poisson, const double *q, const double *f, double *r) {
  const fc::assembly::Box box{nx, ny, nz, lx, ly, lz};
  const int64_t elements = (int64_t)nx * ny * nz, nodes = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
  std::vector<double> ke((size_t)elements * 576);
  for (int64_t e = 0; e < elements; ++e) {
    double x[24];
    fc::assembly::element_corners(box, e, x);
    if (!fc::hex8::stiffness(x, young[e], poisson, ke.data() + e * 576)) return FC_FEM_INVALID;
  }
  for (int64_t d = 0; d < 3 * nodes; ++d)
    r[d] = eq[d] >= 0 ? 0.0 : fc::assembly::reaction(box, d / 3, (int)(d % 3), eq, q, f[d], ke.data());
  return FC_FEM_OK;
}

// Not part of the public ABI: stress recovery with the device code (host/stress.hpp) on the host,
// for tests. u over every DOF (3 nodes); points[elements * 48], nodal_node[nodes * 6] (the mean
// over the elements holding each node), von_mises[nodes].
int fc_test_fem_stresses_host(int nx, int ny, int nz, double lx, double ly, double lz, const double *young,
                              double poisson, const double *u, double *points, double *nodal_node,
                              double *von_mises) {
  const fc::assembly::Box box{nx, ny, nz, lx, ly, lz};
  const int64_t elements = (int64_t)nx * ny * nz, nodes = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
  const int64_t px = nx + 1, py = ny + 1;
  std::vector<double> nodal((size_t)elements * 48);
  for (int64_t e = 0; e < elements; ++e) {
    double x[24], ue[24];
    fc::assembly::element_corners(box, e, x);
    const int64_t ex = e % nx, ey = (e / nx) % ny, ez = e / ((int64_t)nx * ny);
    const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    for (int c = 0; c < 8; ++c) {
      const int64_t v = (ex + off[c][0]) + px * ((ey + off[c][1]) + py * (ez + off[c][2]));
      for (int a = 0; a < 3; ++a) ue[3 * c + a] = u[3 * v + a];
    }
    if (!fc::stress::element_stresses(x, young[e], poisson, ue, points + e * 48, nodal.data() + e * 48))
      return FC_FEM_INVALID;
  }
  for (int64_t v = 0; v < nodes; ++v) {
    fc::stress::nodal_mean(box, v, nodal.data(), nodal_node + v * 6);
    von_mises[v] = fc::stress::von_mises(nodal_node + v * 6);
  }
  return FC_FEM_OK;
}

int fc_hex8_stiffness(const double *xyz24, double young, double poisson, double *out576) {
  if (!xyz24 || !out576) return FC_FEM_INVALID;
  return hex8_stiffness(xyz24, young, poisson, out576) ? FC_FEM_OK : FC_FEM_INVALID;
}

int fc_nested_dissection(int64_t n, const double *xyz, const int64_t *adj_ptr, const int32_t *adj_idx,
                         int64_t *order) {
  if (n < 0 || (n > 0 && (!xyz || !adj_ptr || !adj_idx || !order))) return FC_FEM_INVALID;
  try {
    auto o = nested_dissection(Graph{n, adj_ptr, adj_idx}, xyz);
    std::copy(o.begin(), o.end(), order);
  } catch (const std::bad_alloc &) {
    return FC_FEM_NOMEM;
  }
  return FC_FEM_OK;
}

int fc_graph_dissection(int64_t n, const int64_t *adj_ptr, const int32_t *adj_idx, int64_t *order) {
  if (n < 0 || (n > 0 && (!adj_ptr || !adj_idx || !order))) return FC_FEM_INVALID;
  try {
    auto o = graph_dissection(Graph{n, adj_ptr, adj_idx});
    std::copy(o.begin(), o.end(), order);
  } catch (const std::bad_alloc &) {
    return FC_FEM_NOMEM;
  }
  return FC_FEM_OK;
}

int fc_fill_reducing_order(int64_t n, const double *xyz, const int64_t *adj_ptr, const int32_t *adj_idx,
                           int64_t *order) {
  if (n < 0 || (n > 0 && (!xyz || !adj_ptr || !adj_idx || !order))) return FC_FEM_INVALID;
  try {
    auto o = fill_reducing(Graph{n, adj_ptr, adj_idx}, xyz);
    std::copy(o.begin(), o.end(), order);
  } catch (const std::bad_alloc &) {
    return FC_FEM_NOMEM;
  }
  return FC_FEM_OK;
}

int64_t fc_fill(int64_t n, const int64_t *adj_ptr, const int32_t *adj_idx, const int64_t *order) {
  if (n < 0 || (n > 0 && (!adj_ptr || !adj_idx || !order))) return -1;
  try {
    return fill_of(Graph{n, adj_ptr, adj_idx}, order);
  } catch (const std::bad_alloc &) {
    return -1;
  }
}

int fc_fem_box(int nx, int ny, int nz, double lx, double ly, double lz, const double *young, double poisson,
               const unsigned char *clamped, int threads, fc_problem **out) {
  if (!out || nx <= 0 || ny <= 0 || nz <= 0 || !young || !clamped || !(lx > 0 && ly > 0 && lz > 0))
    return FC_FEM_INVALID;
  *out = nullptr;
  try {
    auto p = new fc_problem();
    const int64_t px = nx + 1, py = ny + 1, pz = nz + 1;
    const int64_t nodes = px * py * pz, elements = (int64_t)nx * ny * nz;
    p->nodes = nodes;
    std::vector<double> xyz(3 * nodes);
    for (int64_t k = 0; k < pz; ++k)
      for (int64_t j = 0; j < py; ++j)
        for (int64_t i = 0; i < px; ++i) {
          int64_t v = i + px * (j + py * k);
          xyz[3 * v + 0] = lx * (double)i / (double)nx;
          xyz[3 * v + 1] = ly * (double)j / (double)ny;
          xyz[3 * v + 2] = lz * (double)k / (double)nz;
        }
    auto element_nodes = [&](int64_t e, int64_t *nd) {
      int64_t i = e % nx, j = (e / nx) % ny, k = e / ((int64_t)nx * ny);
      static const int corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                       {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
      for (int c = 0; c < 8; ++c)
        nd[c] = (i + corner[c][0]) + px * ((j + corner[c][1]) + py * (k + corner[c][2]));
    };
    // Node graph: every node a hex shares with it, itself included, sorted (sparse.rs:99-126).
    // On a structured grid that is the 27-point neighbourhood clipped to the box.
    std::vector<int64_t> aptr(nodes + 1, 0);
    std::vector<int32_t> aidx;
    aidx.reserve(27 * nodes);
    for (int64_t k = 0; k < pz; ++k)
      for (int64_t j = 0; j < py; ++j)
        for (int64_t i = 0; i < px; ++i) {
          int64_t v = i + px * (j + py * k);
          for (int64_t dk = -1; dk <= 1; ++dk)
            for (int64_t dj = -1; dj <= 1; ++dj)
              for (int64_t di = -1; di <= 1; ++di) {
                int64_t a = i + di, b = j + dj, c = k + dk;
                if (a < 0 || b < 0 || c < 0 || a >= px || b >= py || c >= pz) continue;
                aidx.push_back((int32_t)(a + px * (b + py * c)));
              }
          aptr[v + 1] = (int64_t)aidx.size();
        }
    Graph g{nodes, aptr.data(), aidx.data()};
    p->order = fill_reducing(g, xyz.data());
    // Free equations node by node in the fill-reducing order (constraints.rs:755-767).
    p->eq.assign(3 * nodes, -1);
    std::vector<int64_t> pos(nodes, -1);
    int64_t nfree = 0;
    for (int64_t v : p->order)
      if (!clamped[v]) {
        pos[v] = nfree;
        for (int a = 0; a < 3; ++a) p->eq[3 * v + a] = 3 * nfree + a;
        ++nfree;
      }
    p->n = 3 * nfree;
    // K_ff pattern: for a free node, its free neighbours by position, three columns each.
    std::vector<std::vector<int64_t>> nbr(nodes);
    std::vector<int64_t> rowptr(p->n + 1, 0);
    for (int64_t v = 0; v < nodes; ++v) {
      if (pos[v] < 0) continue;
      for (const int32_t *w = g.begin(v); w != g.end(v); ++w)
        if (pos[*w] >= 0) nbr[v].push_back(*w);
      std::sort(nbr[v].begin(), nbr[v].end(), [&](int64_t a, int64_t b) { return pos[a] < pos[b]; });
    }
    {
      std::vector<int64_t> cnt(p->n, 0);
      for (int64_t v = 0; v < nodes; ++v)
        if (pos[v] >= 0)
          for (int a = 0; a < 3; ++a) cnt[3 * pos[v] + a] = 3 * (int64_t)nbr[v].size();
      for (int64_t r = 0; r < p->n; ++r) rowptr[r + 1] = rowptr[r] + cnt[r];
    }
    const int64_t nnz = rowptr[p->n];
    p->idx.resize(nnz);
    p->val.assign(nnz, 0.0);
    for (int64_t v = 0; v < nodes; ++v) {
      if (pos[v] < 0) continue;
      for (int a = 0; a < 3; ++a) {
        int64_t r = 3 * pos[v] + a, at = rowptr[r];
        for (int64_t w : nbr[v])
          for (int b = 0; b < 3; ++b) p->idx[at++] = (int32_t)(3 * pos[w] + b);
      }
    }
    p->ptr = std::move(rowptr);
    // Element matrices in rounds, computed in parallel and added in element order
    // (analysis.rs:199-234): every entry's sum runs over the elements in label order.
    const int64_t ROUND = 4096;
    const int nt = hardware_threads(threads);
    std::vector<double> ke(ROUND * 576);
    std::atomic<bool> bad{false};
    for (int64_t r0 = 0; r0 < elements; r0 += ROUND) {
      const int64_t r1 = std::min(elements, r0 + ROUND);
      auto work = [&](int t) {
        for (int64_t e = r0 + t; e < r1; e += nt) {
          int64_t nd[8];
          element_nodes(e, nd);
          double x[24];
          for (int c = 0; c < 8; ++c)
            for (int b = 0; b < 3; ++b) x[3 * c + b] = xyz[3 * nd[c] + b];
          if (!hex8_stiffness(x, young[e], poisson, &ke[(e - r0) * 576])) bad = true;
        }
      };
      if (nt > 1 && r1 - r0 > 64) {
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t) pool.emplace_back(work, t);
        for (auto &th : pool) th.join();
      } else {
        for (int t = 0; t < nt; ++t) work(t);
      }
      if (bad) {
        delete p;
        return FC_FEM_INVALID;
      }
      for (int64_t e = r0; e < r1; ++e) {
        int64_t nd[8];
        element_nodes(e, nd);
        const double *k = &ke[(e - r0) * 576];
        for (int i = 0; i < 8; ++i) {
          if (pos[nd[i]] < 0) continue;
          const auto &row_nodes = nbr[nd[i]];
          for (int j = 0; j < 8; ++j) {
            if (pos[nd[j]] < 0) continue;
            // position of node j among node i's free neighbours (sorted by position)
            auto it = std::lower_bound(row_nodes.begin(), row_nodes.end(), nd[j],
                                       [&](int64_t a, int64_t b) { return pos[a] < pos[b]; });
            const int64_t at = it - row_nodes.begin();
            for (int r = 0; r < 3; ++r) {
              const int64_t row = 3 * pos[nd[i]] + r;
              double *dst = &p->val[p->ptr[row] + 3 * at];
              for (int c = 0; c < 3; ++c) dst[c] += k[(3 * i + r) * 24 + 3 * j + c];
            }
          }
        }
      }
    }
    *out = p;
  } catch (const std::bad_alloc &) {
    return FC_FEM_NOMEM;
  }
  return FC_FEM_OK;
}

void fc_fem_free(fc_problem *p) { delete p; }
int64_t fc_fem_n(const fc_problem *p) { return p ? p->n : -1; }
int64_t fc_fem_nnz(const fc_problem *p) { return p ? (int64_t)p->idx.size() : -1; }
int64_t fc_fem_nodes(const fc_problem *p) { return p ? p->nodes : -1; }

int fc_fem_csr(const fc_problem *p, int64_t *ptr, int32_t *idx, double *val) {
  if (!p) return FC_FEM_INVALID;
  if (ptr) std::copy(p->ptr.begin(), p->ptr.end(), ptr);
  if (idx) std::copy(p->idx.begin(), p->idx.end(), idx);
  if (val) std::copy(p->val.begin(), p->val.end(), val);
  return FC_FEM_OK;
}

int fc_fem_order(const fc_problem *p, int64_t *order) {
  if (!p || !order) return FC_FEM_INVALID;
  std::copy(p->order.begin(), p->order.end(), order);
  return FC_FEM_OK;
}

int fc_fem_equations(const fc_problem *p, int64_t *eq) {
  if (!p || !eq) return FC_FEM_INVALID;
  std::copy(p->eq.begin(), p->eq.end(), eq);
  return FC_FEM_OK;
}

}  // extern "C"
