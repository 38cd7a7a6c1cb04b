// Stress recovery of hex8 elements after the solve (crates/solver/src/analysis.rs:478-540;
// crates/fem/src/element.rs:587-670, 775-860; material.rs:88-93, 118-124), written once for the
// host and the device: per element the stress D epsilon at the 2 x 2 x 2 Gauss points, the points'
// values extrapolated to the corners (the least-squares map of the corner functions, which for
// eight points on a box is the exact inverse: each corner takes the corner functions at sqrt(3)
// times its natural coordinates), then per node the mean over the elements holding it (in
// element label order) and its von Mises stress. Products and sums are rounded one by one.
#pragma once

#include <cstdint>

#include "assembly.hpp"
#include "hex8.hpp"

namespace fc {
namespace stress {

using hex8::add;
using hex8::mul;
using hex8::sub;

// Element e's stresses: at its Gauss points (points[8][6], xi fastest) and extrapolated to its
// corners (nodal[8][6]), for the element's nodal displacements ue[8][3]. Components xx yy zz xy
// xz yz (engineering shear strains in D epsilon). False for a material or a Jacobian out of range.
FC_HEX8_FN bool element_stresses(const double *xyz, double young, double nu, const double *ue, double *points,
                                 double *nodal) {
  const double corners[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  const double gauss = 0.5773502691896258;
  if (!(young > 0.0) || !(nu > -1.0 && nu < 0.5)) return false;
  const double lambda = mul(young, nu) / mul(add(1.0, nu), sub(1.0, mul(2.0, nu)));
  const double mu = young / mul(2.0, add(1.0, nu));
  double d[6][6] = {};
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) d[i][j] = lambda;
    d[i][i] = add(lambda, mul(2.0, mu));
    d[i + 3][i + 3] = mu;
  }
  const double g[2] = {-gauss, gauss};
  int p = 0;
  for (int pz = 0; pz < 2; ++pz)
    for (int py = 0; py < 2; ++py)
      for (int px = 0; px < 2; ++px, ++p) {
        const double xi[3] = {g[px], g[py], g[pz]};
        double dn[8][3];
        for (int i = 0; i < 8; ++i) {
          const double *c = corners[i];
          const double f[3] = {add(1.0, mul(xi[0], c[0])), add(1.0, mul(xi[1], c[1])), add(1.0, mul(xi[2], c[2]))};
          dn[i][0] = mul(mul(c[0], f[1]), f[2]) / 8.0;
          dn[i][1] = mul(mul(c[1], f[0]), f[2]) / 8.0;
          dn[i][2] = mul(mul(c[2], f[0]), f[1]) / 8.0;
        }
        double jm[3][3] = {};
        for (int i = 0; i < 8; ++i)
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) jm[a][b] = add(jm[a][b], mul(dn[i][a], xyz[3 * i + b]));
        const double t1 = mul(jm[0][0], sub(mul(jm[1][1], jm[2][2]), mul(jm[1][2], jm[2][1])));
        const double t2 = mul(jm[0][1], sub(mul(jm[1][0], jm[2][2]), mul(jm[1][2], jm[2][0])));
        const double t3 = mul(jm[0][2], sub(mul(jm[1][0], jm[2][1]), mul(jm[1][1], jm[2][0])));
        const double det = add(sub(t1, t2), t3);
        if (!(det > 0.0) || !hex8::finite(det)) return false;
        double inv[3][3];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            const int j1 = (j + 1) % 3, j2 = (j + 2) % 3, i1 = (i + 1) % 3, i2 = (i + 2) % 3;
            inv[i][j] = sub(mul(jm[j1][i1], jm[j2][i2]), mul(jm[j1][i2], jm[j2][i1])) / det;
          }
        // grad[c][b] = sum over nodes of u_c dN/dx_b, node by node
        double grad[3][3] = {};
        for (int i = 0; i < 8; ++i) {
          double dx[3];
          for (int b = 0; b < 3; ++b)
            dx[b] = add(add(mul(inv[b][0], dn[i][0]), mul(inv[b][1], dn[i][1])), mul(inv[b][2], dn[i][2]));
          for (int c = 0; c < 3; ++c)
            for (int b = 0; b < 3; ++b) grad[c][b] = add(grad[c][b], mul(ue[3 * i + c], dx[b]));
        }
        const double strain[6] = {grad[0][0], grad[1][1], grad[2][2], add(grad[0][1], grad[1][0]),
                                  add(grad[0][2], grad[2][0]), add(grad[1][2], grad[2][1])};
        for (int s = 0; s < 6; ++s) {
          double acc = 0.0;
          for (int t = 0; t < 6; ++t) acc = add(acc, mul(d[s][t], strain[t]));
          points[6 * p + s] = acc;
        }
      }
  // corner n takes sum over points q of N_q(sqrt(3) xi_n) sigma_q, the corner functions of the
  // points' box (point q's corner signs are corners[q] in the same order)
  const double r3 = 1.7320508075688772;
  for (int n = 0; n < 8; ++n) {
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (int q = 0; q < 8; ++q) {
      double w = 1.0;
      for (int a = 0; a < 3; ++a) w = mul(w, add(1.0, mul(mul(r3, corners[n][a]), corners[q][a])));
      w = w / 8.0;
      for (int s = 0; s < 6; ++s) v[s] = add(v[s], mul(w, points[6 * q + s]));
    }
    for (int s = 0; s < 6; ++s) nodal[6 * n + s] = v[s];
  }
  return true;
}

// The von Mises stress of xx yy zz xy xz yz (material.rs:88-93).
FC_HEX8_FN double von_mises(const double *s) {
  const double normal = add(add(mul(sub(s[0], s[1]), sub(s[0], s[1])), mul(sub(s[1], s[2]), sub(s[1], s[2]))),
                            mul(sub(s[2], s[0]), sub(s[2], s[0])));
  const double shear = add(add(mul(s[3], s[3]), mul(s[4], s[4])), mul(s[5], s[5]));
  return sqrt(add(mul(0.5, normal), mul(3.0, shear)));
}

// Node v's stress: the mean over the elements holding it, in element label order, of their
// corner values at v (nodal_all[e * 48 + corner * 6 + s]); out[6].
FC_HEX8_FN void nodal_mean(const assembly::Box &b, int64_t v, const double *nodal_all, double *out) {
  const int64_t px = b.nx + 1, py = b.ny + 1;
  const int64_t iv = v % px, jv = (v / px) % py, kv = v / (px * py);
  double sum[6] = {0, 0, 0, 0, 0, 0};
  int count = 0;
  for (int64_t ez = kv - 1; ez <= kv; ++ez)
    for (int64_t ey = jv - 1; ey <= jv; ++ey)
      for (int64_t ex = iv - 1; ex <= iv; ++ex) {
        if (ex < 0 || ey < 0 || ez < 0 || ex >= b.nx || ey >= b.ny || ez >= b.nz) continue;
        const int64_t e = ex + b.nx * (ey + (int64_t)b.ny * ez);
        const int c = assembly::corner_of((int)(iv - ex), (int)(jv - ey), (int)(kv - ez));
        for (int s = 0; s < 6; ++s) sum[s] = add(sum[s], nodal_all[e * 48 + c * 6 + s]);
        count += 1;
      }
  for (int s = 0; s < 6; ++s) out[s] = count > 0 ? sum[s] / (double)count : 0.0;
}

}  // namespace stress
}  // namespace fc
