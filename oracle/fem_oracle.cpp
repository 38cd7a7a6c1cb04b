// ORACLE — test infrastructure, not product code. The oracle's own input builder: structured
// boxes of hex8 elements assembled into the free-DOF stiffness K_ff the way the reference's
// linear static analysis builds it, so the timed CPU reference and the checks never depend on
// the product's builder. Restated from:
//   - node graph and fill-reducing order: crates/solver/src/sparse.rs:99-120 (NodeGraph::new),
//     crates/solver/src/ordering.rs:28-98 (nested_dissection), :102-110 (fill_reducing_order),
//     :117-153 (level_structure, clear), :156-250 (graph_dissection), :254-275 (fill);
//   - hex8 stiffness: crates/fem/src/shape.rs:51-52, 95-103 (corners, trilinear shape),
//     crates/fem/src/quadrature.rs:28-44, 78-90 (2-point Gauss, xi fastest), crates/fem/src/
//     material.rs:22-27, 40-53 (isotropic D), crates/fem/src/element.rs:300-324 (Jacobian,
//     gradients), :396-425 (stiffness), :713-715, :745-774 (B blocks, symmetric accumulation),
//     crates/fem/src/dense.rs:91-116, 169-172 and crates/model/src/mesh.rs:257-269 (inverse,
//     determinant, admissible Jacobian);
//   - assembly: crates/solver/src/analysis.rs:199-234 (elements added in label order),
//     crates/solver/src/sparse.rs:178-226 (Block, add_block);
//   - free equations and K_ff: crates/solver/src/constraints.rs:755-767 (numbering node by
//     node in the fill-reducing order), :820-900 (the plain selection T_f^T K T_f).
// The mesh is the reference's grid helper (crates/solver/tests/common/mod.rs:23-98) for hex8:
// node v = i + (nx+1)(j + (ny+1)k) at (lx i/nx, ly j/ny, lz k/nz), element labels with x
// fastest, corners in the order of shape.rs:51-52. Built with -ffp-contract=off like the rest
// of the oracle: every product and sum rounded on its own, as the reference's Rust.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <new>
#include <thread>
#include <vector>

extern "C" int or_tree_counts(int64_t n, const int64_t *ptr, const int32_t *idx, int by_columns, int64_t *parent,
                              int64_t *counts);

namespace {

using Rows = std::vector<std::vector<int64_t>>;
constexpr size_t LEAF = 16;               // ordering.rs:25
constexpr int PERIPHERAL_SEARCHES = 8;    // ordering.rs:114
constexpr int64_t UNSET = std::numeric_limits<int64_t>::max();

// ---- fill-reducing order ------------------------------------------------------------------

std::vector<int64_t> plane_dissection(const std::vector<double> &xyz, const Rows &adj) {
  const int64_t n = (int64_t)adj.size();
  std::vector<int64_t> order;
  order.reserve(n);
  std::vector<uint8_t> side(n, 0);
  // (emit?, nodes): a part to split, or a separator to emit after its parts
  std::vector<std::pair<bool, std::vector<int64_t>>> todo;
  std::vector<int64_t> everything(n);
  for (int64_t v = 0; v < n; ++v) everything[v] = v;
  todo.emplace_back(false, std::move(everything));
  while (!todo.empty()) {
    auto [emit, part] = std::move(todo.back());
    todo.pop_back();
    if (emit || part.size() <= LEAF) {
      order.insert(order.end(), part.begin(), part.end());
      continue;
    }
    double lo[3], hi[3];
    for (int k = 0; k < 3; ++k) lo[k] = INFINITY, hi[k] = -INFINITY;
    for (int64_t v : part)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::fmin(lo[k], xyz[3 * v + k]);
        hi[k] = std::fmax(hi[k], xyz[3 * v + k]);
      }
    int axis = 0;
    for (int k = 0; k < 3; ++k) axis = (hi[k] - lo[k] > hi[axis] - lo[axis]) ? k : axis;
    std::sort(part.begin(), part.end(), [&](int64_t a, int64_t b) {
      const double x = xyz[3 * a + axis], y = xyz[3 * b + axis];
      return x != y ? x < y : a < b;
    });
    const size_t half = part.size() / 2;
    for (size_t q = 0; q < part.size(); ++q) side[part[q]] = q < half ? 1 : 2;
    auto meets = [&](int64_t v, uint8_t other) {
      for (int64_t w : adj[v])
        if (side[w] == other) return true;
      return false;
    };
    std::vector<int64_t> left_edge, right_edge;
    for (size_t q = 0; q < part.size(); ++q) {
      if (q < half && meets(part[q], 2)) left_edge.push_back(part[q]);
      if (q >= half && meets(part[q], 1)) right_edge.push_back(part[q]);
    }
    std::vector<int64_t> &sep = left_edge.size() <= right_edge.size() ? left_edge : right_edge;
    for (int64_t v : part) side[v] = 0;
    for (int64_t v : sep) side[v] = 3;
    std::vector<int64_t> a, b;
    for (size_t q = 0; q < part.size(); ++q)
      if (side[part[q]] != 3) (q < half ? a : b).push_back(part[q]);
    for (int64_t v : sep) side[v] = 0;
    todo.emplace_back(true, std::move(sep));
    todo.emplace_back(false, std::move(b));
    todo.emplace_back(false, std::move(a));
  }
  return order;
}

Rows levels_from(const Rows &adj, int64_t root, int64_t token, const std::vector<int64_t> &owner,
                 std::vector<int64_t> &level) {
  Rows out{{root}};
  level[root] = 0;
  for (;;) {
    std::vector<int64_t> next;
    const int64_t depth = (int64_t)out.size();
    for (int64_t v : out.back())
      for (int64_t w : adj[v])
        if (owner[w] == token && level[w] == UNSET) {
          level[w] = depth;
          next.push_back(w);
        }
    if (next.empty()) return out;
    out.push_back(std::move(next));
  }
}

void unmark(std::vector<int64_t> &level, const Rows &s) {
  for (const auto &l : s)
    for (int64_t v : l) level[v] = UNSET;
}

std::vector<int64_t> graph_dissection(const Rows &adj) {
  const int64_t n = (int64_t)adj.size();
  std::vector<int64_t> order, owner(n, 0), level(n, UNSET);
  order.reserve(n);
  int64_t token = 0;
  std::vector<std::pair<bool, std::vector<int64_t>>> todo;
  std::vector<int64_t> everything(n);
  for (int64_t v = 0; v < n; ++v) everything[v] = v;
  todo.emplace_back(false, std::move(everything));
  while (!todo.empty()) {
    auto [emit, part] = std::move(todo.back());
    todo.pop_back();
    if (emit) {
      order.insert(order.end(), part.begin(), part.end());
      continue;
    }
    if (part.empty()) continue;
    if (part.size() <= LEAF) {
      order.insert(order.end(), part.begin(), part.end());
      continue;
    }
    ++token;
    for (int64_t v : part) owner[v] = token;
    auto degree = [&](int64_t v) {
      int64_t d = 0;
      for (int64_t w : adj[v]) d += owner[w] == token;
      return d;
    };
    Rows s = levels_from(adj, part.front(), token, owner, level);
    for (int t = 0; t < PERIPHERAL_SEARCHES; ++t) {
      if (s.back().empty()) break;
      int64_t cand = s.back().front(), cd = degree(cand);
      for (int64_t v : s.back()) {
        const int64_t d = degree(v);
        if (d < cd || (d == cd && v < cand)) cand = v, cd = d;
      }
      unmark(level, s);
      Rows deeper = levels_from(adj, cand, token, owner, level);
      if (deeper.size() <= s.size()) {
        unmark(level, deeper);
        for (size_t d = 0; d < s.size(); ++d)
          for (int64_t v : s[d]) level[v] = (int64_t)d;
        break;
      }
      s = std::move(deeper);
    }
    size_t reached = 0;
    for (const auto &l : s) reached += l.size();
    if (reached < part.size()) {
      std::vector<int64_t> rest, comp;
      for (int64_t v : part)
        if (level[v] == UNSET) rest.push_back(v);
      unmark(level, s);
      for (const auto &l : s) comp.insert(comp.end(), l.begin(), l.end());
      std::sort(comp.begin(), comp.end());
      todo.emplace_back(false, std::move(rest));
      todo.emplace_back(false, std::move(comp));
      continue;
    }
    if (s.size() < 3) {
      unmark(level, s);
      order.insert(order.end(), part.begin(), part.end());
      continue;
    }
    size_t middle = 1, count = 0;
    for (size_t d = 1; d < s.size(); ++d) {
      count += s[d].size();
      if (2 * count >= part.size()) {
        middle = std::min(d, s.size() - 2);
        break;
      }
    }
    std::vector<int64_t> before, sep, after;
    for (size_t d = 0; d < middle; ++d) before.insert(before.end(), s[d].begin(), s[d].end());
    for (int64_t v : s[middle]) {
      bool next = false;
      for (int64_t w : adj[v])
        if (owner[w] == token && level[w] == (int64_t)middle + 1) {
          next = true;
          break;
        }
      (next ? sep : before).push_back(v);
    }
    for (size_t d = middle + 1; d < s.size(); ++d) after.insert(after.end(), s[d].begin(), s[d].end());
    unmark(level, s);
    std::sort(before.begin(), before.end());
    std::sort(sep.begin(), sep.end());
    std::sort(after.begin(), after.end());
    todo.emplace_back(true, std::move(sep));
    todo.emplace_back(false, std::move(after));
    todo.emplace_back(false, std::move(before));
  }
  return order;
}

// Entries of the Cholesky factor of the node graph eliminated in `order` (ordering.rs:254-275,
// cholesky.rs:216-218).
int64_t fill_of(const Rows &adj, const std::vector<int64_t> &order) {
  const int64_t n = (int64_t)adj.size();
  std::vector<int64_t> at(n), ptr{0};
  std::vector<int32_t> idx;
  for (int64_t k = 0; k < n; ++k) at[order[k]] = k;
  std::vector<int64_t> col;
  for (int64_t k = 0; k < n; ++k) {
    col.clear();
    for (int64_t w : adj[order[k]])
      if (at[w] < k) col.push_back(at[w]);
    col.push_back(k);
    std::sort(col.begin(), col.end());
    col.erase(std::unique(col.begin(), col.end()), col.end());
    for (int64_t r : col) idx.push_back((int32_t)r);
    ptr.push_back((int64_t)idx.size());
  }
  std::vector<int64_t> parent(n), counts(n);
  or_tree_counts(n, ptr.data(), idx.data(), 0, parent.data(), counts.data());
  int64_t total = 0;
  for (int64_t c : counts) total += c;
  return total;
}

std::vector<int64_t> fill_reducing(const std::vector<double> &xyz, const Rows &adj) {
  std::vector<int64_t> planes = plane_dissection(xyz, adj);
  if (adj.size() <= LEAF) return planes;
  std::vector<int64_t> graph = graph_dissection(adj);
  return fill_of(adj, graph) < fill_of(adj, planes) ? graph : planes;
}

// ---- hex8 element ---------------------------------------------------------------------------

const double HEX[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                          {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

double det3(const double m[3][3]) {
  return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
         m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

bool admissible(const double j[3][3]) {
  const double det = j[0][0] * (j[1][1] * j[2][2] - j[1][2] * j[2][1]) -
                     j[0][1] * (j[1][0] * j[2][2] - j[1][2] * j[2][0]) +
                     j[0][2] * (j[1][0] * j[2][1] - j[1][1] * j[2][0]);
  double norms = 1.0;
  for (int r = 0; r < 3; ++r) norms *= std::sqrt(j[r][0] * j[r][0] + j[r][1] * j[r][1] + j[r][2] * j[r][2]);
  double q = det / norms;
  q = std::isfinite(q) ? std::min(1.0, std::max(-1.0, q)) : 0.0;
  return q > 1e-12;
}

// 24 x 24 row-major stiffness of a hex8 with corners x[8][3]; false when the material or an
// integration point's Jacobian is not admissible.
bool hex8_stiffness(const double x[8][3], double young, double nu, double *k) {
  if (!(young > 0.0 && std::isfinite(young) && nu > -1.0 && nu < 0.5)) return false;
  const double lambda = young * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  const double mu = young / (2.0 * (1.0 + nu));
  double D[6][6];
  std::memset(D, 0, sizeof D);
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) D[i][j] = lambda;
    D[i][i] = lambda + 2.0 * mu;
    D[i + 3][i + 3] = mu;
  }
  std::fill(k, k + 576, 0.0);
  const double abscissa[2] = {-0.5773502691896258, 0.5773502691896258};
  for (int pz = 0; pz < 2; ++pz)
    for (int py = 0; py < 2; ++py)
      for (int px = 0; px < 2; ++px) {
        const double xi[3] = {abscissa[px], abscissa[py], abscissa[pz]};
        const double weight = (1.0 * 1.0) * 1.0;
        double dn[8][3];
        for (int a = 0; a < 8; ++a) {
          double f[3];
          for (int q = 0; q < 3; ++q) f[q] = 1.0 + xi[q] * HEX[a][q];
          dn[a][0] = HEX[a][0] * f[1] * f[2] / 8.0;
          dn[a][1] = HEX[a][1] * f[0] * f[2] / 8.0;
          dn[a][2] = HEX[a][2] * f[0] * f[1] / 8.0;
        }
        double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int a = 0; a < 8; ++a)
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) J[r][c] += dn[a][r] * x[a][c];
        if (!admissible(J)) return false;
        const double det = det3(J);
        if (!(std::fabs(det) > 0.0 && std::isfinite(det))) return false;
        double inv[3][3];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            inv[i][j] = (J[j1][i1] * J[j2][i2] - J[j1][i2] * J[j2][i1]) / det;
          }
        double g[8][3];
        for (int a = 0; a < 8; ++a)
          for (int b = 0; b < 3; ++b) g[a][b] = inv[b][0] * dn[a][0] + inv[b][1] * dn[a][1] + inv[b][2] * dn[a][2];
        const double w = det * weight;
        for (int j = 0; j < 8; ++j) {
          const double Bj[6][3] = {{g[j][0], 0, 0}, {0, g[j][1], 0},       {0, 0, g[j][2]},
                                   {g[j][1], g[j][0], 0}, {g[j][2], 0, g[j][0]}, {0, g[j][2], g[j][1]}};
          double DB[6][3];
          for (int s = 0; s < 6; ++s)
            for (int c = 0; c < 3; ++c) {
              double sum = 0.0;
              for (int t = 0; t < 6; ++t) sum += D[s][t] * Bj[t][c];
              DB[s][c] = sum;
            }
          for (int i = 0; i <= j; ++i) {
            const double Bi[6][3] = {{g[i][0], 0, 0}, {0, g[i][1], 0},       {0, 0, g[i][2]},
                                     {g[i][1], g[i][0], 0}, {g[i][2], 0, g[i][0]}, {0, g[i][2], g[i][1]}};
            for (int r = 0; r < 3; ++r)
              for (int c = i == j ? r : 0; c < 3; ++c) {
                double sum = 0.0;
                for (int s = 0; s < 6; ++s) sum += Bi[s][r] * DB[s][c];
                const double v = w * sum;
                const int row = 3 * i + r, col = 3 * j + c;
                k[row * 24 + col] += v;
                if (row != col) k[col * 24 + row] += v;
              }
          }
        }
      }
  return true;
}

}  // namespace

extern "C" {

// A box of nx x ny x nz hex8 elements of size lx x ly x lz; young[e] per element label order
// (e = i + nx (j + ny k)); clamped[v] holds all three DOFs of node v. Outputs: *n free equations,
// K_ff by rows (ptr[n+1], idx/val sized by *nnz: call first with null ptr/idx/val to size them),
// the node elimination order (order[nodes]) and each mesh DOF's equation (eq[3 nodes], -1 held).
// Returns 0, or -1 for an element that is not admissible, -2 on allocation failure.
struct or_fem;
struct or_fem {
  int64_t n = 0;
  std::vector<int64_t> ptr, order, eq;
  std::vector<int32_t> idx;
  std::vector<double> val;
};

int or_fem_box(int64_t nx, int64_t ny, int64_t nz, double lx, double ly, double lz, const double *young, double nu,
               const uint8_t *clamped, int threads, or_fem **out) {
  *out = nullptr;
  try {
    const int64_t px = nx + 1, py = ny + 1, pz = nz + 1, nodes = px * py * pz, elements = nx * ny * nz;
    std::vector<double> xyz(3 * nodes);
    for (int64_t k = 0; k < pz; ++k)
      for (int64_t j = 0; j < py; ++j)
        for (int64_t i = 0; i < px; ++i) {
          const int64_t v = i + px * (j + py * k);
          xyz[3 * v] = lx * (double)i / (double)nx;
          xyz[3 * v + 1] = ly * (double)j / (double)ny;
          xyz[3 * v + 2] = lz * (double)k / (double)nz;
        }
    const int64_t offs[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    std::vector<int64_t> conn(8 * elements);
    for (int64_t k = 0; k < nz; ++k)
      for (int64_t j = 0; j < ny; ++j)
        for (int64_t i = 0; i < nx; ++i) {
          const int64_t e = i + nx * (j + ny * k);
          for (int c = 0; c < 8; ++c)
            conn[8 * e + c] = (i + offs[c][0]) + px * ((j + offs[c][1]) + py * (k + offs[c][2]));
        }
    // the node graph (sparse.rs:104-120): each node's row holds every node of its elements
    Rows adj(nodes);
    for (int64_t e = 0; e < elements; ++e)
      for (int c = 0; c < 8; ++c) adj[conn[8 * e + c]].insert(adj[conn[8 * e + c]].end(), &conn[8 * e], &conn[8 * e + 8]);
    for (auto &row : adj) {
      std::sort(row.begin(), row.end());
      row.erase(std::unique(row.begin(), row.end()), row.end());
    }
    auto f = new or_fem();
    f->order = fill_reducing(xyz, adj);
    // the matrix over every mesh DOF on the node graph's pattern (3 DOFs a node, x y z)
    const int64_t dofs = 3 * nodes;
    std::vector<int64_t> kptr(dofs + 1, 0);
    for (int64_t v = 0; v < nodes; ++v)
      for (int r = 0; r < 3; ++r) kptr[3 * v + r + 1] = kptr[3 * v + r] + 3 * (int64_t)adj[v].size();
    std::vector<double> kval(kptr[dofs], 0.0);
    // element matrices in parallel, added in label order (analysis.rs:199-234)
    std::vector<double> ke(576 * (size_t)elements);
    std::vector<uint8_t> ok(elements, 1);
    {
      const int T = std::max(1, threads);
      std::vector<std::thread> pool;
      for (int t = 0; t < T; ++t)
        pool.emplace_back([&, t] {
          for (int64_t e = t; e < elements; e += T) {
            double corner[8][3];
            for (int c = 0; c < 8; ++c)
              for (int q = 0; q < 3; ++q) corner[c][q] = xyz[3 * conn[8 * e + c] + q];
            ok[e] = hex8_stiffness(corner, young[e], nu, &ke[576 * (size_t)e]);
          }
        });
      for (auto &th : pool) th.join();
    }
    for (int64_t e = 0; e < elements; ++e) {
      if (!ok[e]) {
        delete f;
        return -1;
      }
      const int64_t *en = &conn[8 * e];
      const double *m = &ke[576 * (size_t)e];
      for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 8; ++b) {
          const auto &row = adj[en[a]];
          const int64_t at = std::lower_bound(row.begin(), row.end(), en[b]) - row.begin();
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) kval[kptr[3 * en[a] + r] + 3 * at + c] += m[(3 * a + r) * 24 + 3 * b + c];
        }
    }
    // free equations node by node in the elimination order (constraints.rs:755-767)
    f->eq.assign(dofs, -1);
    std::vector<int64_t> eq_dof;
    for (int64_t v : f->order)
      for (int r = 0; r < 3; ++r)
        if (!clamped[v]) {
          f->eq[3 * v + r] = (int64_t)eq_dof.size();
          eq_dof.push_back(3 * v + r);
        }
    // K_ff = T_f^T K T_f for a plain selection (constraints.rs:820-900): row e takes the free
    // columns of its DOF's row, in increasing equation order
    f->n = (int64_t)eq_dof.size();
    f->ptr.assign(1, 0);
    std::vector<std::pair<int64_t, double>> row;
    for (int64_t e = 0; e < f->n; ++e) {
      const int64_t d = eq_dof[e];
      row.clear();
      for (int64_t q = kptr[d]; q < kptr[d + 1]; ++q) {
        const int64_t node = adj[d / 3][(q - kptr[d]) / 3], col = 3 * node + (q - kptr[d]) % 3;
        if (f->eq[col] >= 0) row.emplace_back(f->eq[col], 1.0 * kval[q] * 1.0);
      }
      std::sort(row.begin(), row.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
      for (const auto &x : row) {
        f->idx.push_back((int32_t)x.first);
        f->val.push_back(x.second);
      }
      f->ptr.push_back((int64_t)f->idx.size());
    }
    *out = f;
    return 0;
  } catch (const std::bad_alloc &) {
    return -2;
  }
}

int64_t or_fem_info(const or_fem *f, int what) {
  switch (what) {
    case 0: return f->n;
    case 1: return (int64_t)f->idx.size();
    case 2: return (int64_t)f->order.size();
    default: return -1;
  }
}

void or_fem_export(const or_fem *f, int64_t *ptr, int32_t *idx, double *val, int64_t *order, int64_t *eq) {
  if (ptr) std::copy(f->ptr.begin(), f->ptr.end(), ptr);
  if (idx) std::copy(f->idx.begin(), f->idx.end(), idx);
  if (val) std::copy(f->val.begin(), f->val.end(), val);
  if (order) std::copy(f->order.begin(), f->order.end(), order);
  if (eq) std::copy(f->eq.begin(), f->eq.end(), eq);
}

void or_fem_free(or_fem *f) { delete f; }

}  // extern "C"
