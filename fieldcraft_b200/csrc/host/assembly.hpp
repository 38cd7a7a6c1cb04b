// Assembly of a structured hex8 box's K_ff entry by entry, written once for the host test hook and
// the device kernel: entry (v, a; w, c) is the sum over the elements holding both nodes, in
// element label order from zero, of their stiffness entries, which is the order in which the
// host builder (crates/solver/src/analysis.rs:199-234, sparse.rs add_block) adds the element
// matrices, so every entry has the builder's bits.
#pragma once

#include <cstdint>

#include "hex8.hpp"

namespace fc {
namespace assembly {

// The box: nx x ny x nz elements, (nx + 1)(ny + 1)(nz + 1) nodes numbered x fastest; element
// (ex, ey, ez) is label ex + nx (ey + ny ez) with corners in the reference's order.
struct Box {
  int nx, ny, nz;
  double lx, ly, lz;
};

// The local corner (0..7) at offset (dx, dy, dz) in {0, 1}^3 from an element's first node.
FC_HEX8_FN int corner_of(int dx, int dy, int dz) {
  const int table[2][2][2] = {{{0, 4}, {3, 7}}, {{1, 5}, {2, 6}}};  // [dx][dy][dz]
  return table[dx][dy][dz];
}

// Element e's corner coordinates (xyz[8 x 3]) as the builder places the nodes.
FC_HEX8_FN void element_corners(const Box &b, int64_t e, double *xyz) {
  const int64_t ex = e % b.nx, ey = (e / b.nx) % b.ny, ez = e / ((int64_t)b.nx * b.ny);
  const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  for (int c = 0; c < 8; ++c) {
    xyz[3 * c + 0] = hex8::mul(b.lx, (double)(ex + off[c][0])) / (double)b.nx;
    xyz[3 * c + 1] = hex8::mul(b.ly, (double)(ey + off[c][1])) / (double)b.ny;
    xyz[3 * c + 2] = hex8::mul(b.lz, (double)(ez + off[c][2])) / (double)b.nz;
  }
}

// Entry (3 v + a, 3 w + c) of K over all nodes (the free part takes its rows and columns), from
// the element matrices ke[e * 576 + row * 24 + col].
FC_HEX8_FN double entry(const Box &b, int64_t v, int a, int64_t w, int c, const double *ke) {
  const int64_t px = b.nx + 1, py = b.ny + 1;
  const int64_t iv = v % px, jv = (v / px) % py, kv = v / (px * py);
  const int64_t iw = w % px, jw = (w / px) % py, kw = w / (px * py);
  auto lo = [](int64_t p, int64_t q) { return (p > q ? p : q) - 1 > 0 ? (p > q ? p : q) - 1 : 0; };
  auto hi = [](int64_t p, int64_t q, int n) { const int64_t m = p < q ? p : q; return m < n - 1 ? m : n - 1; };
  double acc = 0.0;
  for (int64_t ez = lo(kv, kw); ez <= hi(kv, kw, b.nz); ++ez)
    for (int64_t ey = lo(jv, jw); ey <= hi(jv, jw, b.ny); ++ey)
      for (int64_t ex = lo(iv, iw); ex <= hi(iv, iw, b.nx); ++ex) {
        const int64_t e = ex + b.nx * (ey + (int64_t)b.ny * ez);
        const int i = corner_of((int)(iv - ex), (int)(jv - ey), (int)(kv - ez));
        const int j = corner_of((int)(iw - ex), (int)(jw - ey), (int)(kw - ez));
        acc = hex8::add(acc, ke[e * 576 + (3 * i + a) * 24 + 3 * j + c]);
      }
  return acc;
}

// u over every DOF from the free equations' values q: eq[3 v + a] its equation or -1 (a held
// DOF, zero motion) (Reduction::expand, crates/solver/src/constraints.rs:929-939).
FC_HEX8_FN double expanded(const int64_t *eq, const double *q, int64_t dof) {
  const int64_t e = eq[dof];
  return e >= 0 ? q[e] : 0.0;
}

// The reaction at DOF (v, a): row 3 v + a of the whole K times u (over every DOF, held ones at
// zero), the row's entries in column order, less the applied load f_va (Reduction::reactions,
// constraints.rs:1001-1015, a plain clamp's T_p row). The row's columns are the DOFs of the nodes
// sharing an element with v, by node index then direction.
FC_HEX8_FN double reaction(const Box &b, int64_t v, int a, const int64_t *eq, const double *q, double f_va,
                           const double *ke) {
  const int64_t px = b.nx + 1, py = b.ny + 1, pz = b.nz + 1;
  const int64_t iv = v % px, jv = (v / px) % py, kv = v / (px * py);
  double ku = 0.0;
  for (int64_t dk = -1; dk <= 1; ++dk)
    for (int64_t dj = -1; dj <= 1; ++dj)
      for (int64_t di = -1; di <= 1; ++di) {
        const int64_t i = iv + di, j = jv + dj, k = kv + dk;
        if (i < 0 || j < 0 || k < 0 || i >= px || j >= py || k >= pz) continue;
        const int64_t w = i + px * (j + py * k);
        for (int c = 0; c < 3; ++c) ku = hex8::add(ku, hex8::mul(entry(b, v, a, w, c, ke), expanded(eq, q, 3 * w + c)));
      }
  return hex8::sub(ku, f_va);
}

}  // namespace assembly
}  // namespace fc
