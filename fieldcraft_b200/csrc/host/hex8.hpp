// The hex8 element's stiffness matrix (crates/fem/src/element.rs:397-425, 745-774; shape.rs,
// quadrature.rs, material.rs), written once for the host builder and for the device assembly:
// every product and sum is rounded on its own (no fused multiply-add on the device), so both
// give the same bits.
#pragma once

#if defined(__CUDACC__)
#define FC_HEX8_FN __host__ __device__ __forceinline__
#else
#include <cmath>
#define FC_HEX8_FN inline
#endif

namespace fc {
namespace hex8 {

FC_HEX8_FN double mul(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
FC_HEX8_FN double add(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
FC_HEX8_FN double sub(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
FC_HEX8_FN bool finite(double x) {
#if defined(__CUDA_ARCH__)
  return isfinite(x);
#else
  return std::isfinite(x);
#endif
}

// k[24 x 24] (row-major; unknowns node by node, x y z) of a hex8 element with corners xyz[8 x 3]
// (the reference's corner order), Young's modulus `young` and Poisson's ratio `nu`, by 2 x 2 x 2
// Gauss points; false for a material or a Jacobian out of range.
FC_HEX8_FN bool stiffness(const double *xyz, double young, double nu, double *k) {
  // natural coordinates of the corners (shape.rs:51-52) and the two-point abscissa (quadrature.rs:31)
  const double corners[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  const double gauss = 0.5773502691896258;
  if (!(young > 0.0) || !(nu > -1.0 && nu < 0.5)) return false;
  // isotropic elasticity (material.rs:40-53)
  const double lambda = mul(young, nu) / mul(add(1.0, nu), sub(1.0, mul(2.0, nu)));
  const double mu = young / mul(2.0, add(1.0, nu));
  double d[6][6] = {};
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) d[i][j] = lambda;
    d[i][i] = add(lambda, mul(2.0, mu));
    d[i + 3][i + 3] = mu;
  }
  for (int q = 0; q < 576; ++q) k[q] = 0.0;
  const double g[2] = {-gauss, gauss};
  // points with xi fastest, then eta, then zeta; every weight is 1 (quadrature.rs:78-90)
  for (int pz = 0; pz < 2; ++pz)
    for (int py = 0; py < 2; ++py)
      for (int px = 0; px < 2; ++px) {
        const double xi[3] = {g[px], g[py], g[pz]};
        const double weight = 1.0;
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
        if (!(det > 0.0) || !finite(det)) return false;
        double inv[3][3];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            const int j1 = (j + 1) % 3, j2 = (j + 2) % 3, i1 = (i + 1) % 3, i2 = (i + 2) % 3;
            inv[i][j] = sub(mul(jm[j1][i1], jm[j2][i2]), mul(jm[j1][i2], jm[j2][i1])) / det;
          }
        double dx[8][3];
        for (int i = 0; i < 8; ++i)
          for (int b = 0; b < 3; ++b)
            dx[i][b] = add(add(mul(inv[b][0], dn[i][0]), mul(inv[b][1], dn[i][1])), mul(inv[b][2], dn[i][2]));
        const double w = mul(det, weight);
        // upper blocks j >= i, mirrored, so K is exactly symmetric (element.rs:745-774)
        for (int j = 0; j < 8; ++j) {
          const double *gj = dx[j];
          const double bj[6][3] = {{gj[0], 0, 0}, {0, gj[1], 0}, {0, 0, gj[2]},
                                   {gj[1], gj[0], 0}, {gj[2], 0, gj[0]}, {0, gj[2], gj[1]}};
          double db[6][3];
          for (int s = 0; s < 6; ++s)
            for (int c = 0; c < 3; ++c) {
              double acc = 0.0;
              for (int t = 0; t < 6; ++t) acc = add(acc, mul(d[s][t], bj[t][c]));
              db[s][c] = acc;
            }
          for (int i = 0; i <= j; ++i) {
            const double *gi = dx[i];
            const double bi[6][3] = {{gi[0], 0, 0}, {0, gi[1], 0}, {0, 0, gi[2]},
                                     {gi[1], gi[0], 0}, {gi[2], 0, gi[0]}, {0, gi[2], gi[1]}};
            for (int r = 0; r < 3; ++r)
              for (int c = (i == j ? r : 0); c < 3; ++c) {
                double acc = 0.0;
                for (int s = 0; s < 6; ++s) acc = add(acc, mul(bi[s][r], db[s][c]));
                const double v = mul(w, acc);
                const int row = 3 * i + r, col = 3 * j + c;
                k[row * 24 + col] = add(k[row * 24 + col], v);
                if (row != col) k[col * 24 + row] = add(k[col * 24 + row], v);
              }
          }
        }
      }
  return true;
}

}  // namespace hex8
}  // namespace fc
