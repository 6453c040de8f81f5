// SUPG quasi-compressible element arithmetic, matrix-free (one thread = one
// element).
//
// Reference: src/femSUPGExplicitFluidSolver.cpp:1095-1498.  Per Gauss point
// the reference builds L, U, S, US, B, D, DB, H and accumulates five 24x24
// matrices (Mass, K1, K1+, K2, K3, K4), then forms k = -dt (K1+K2+K3+K4) u_e.
// Here each K_i u_e is evaluated directly from the Gauss-point quantities:
//   (K1 u)[a][c] += rho N_a (u.grad) u_c w                    (Bubnov convection)
//   (K2 u)[a][c] += sum_r B[r][a,c] (D(lambda, mu) B u)_r w   (viscous + penalty)
//   (K3 u)[a][c] += rho tau (u.grad N_a) (u.grad) u_c w       (SUPG)
//   (K4 u)[a][c] += rho nu_C dN_a/dx_c (div u) w              (grad-div)
// with w = detJ * weight, tau and nu_C from eval_stabilization (src lines
// 336-377) and lambda from eval_bulk_modulus (src lines 382-441).  The Mass
// and K1+ matrices do not reach the update (src lines 1325-1327, 806) and the
// Frobenius norms of K are diagnostics; none of them is formed.
#pragma once
#include "fm_device.cuh"

namespace fm {

// irSecondOrder rule (src/femIntegrationRule.cpp): tet4 4 points, weight
// (1/6)(1/4); hexa8 2x2x2 points at +-1/sqrt(3) in the reference's order,
// weight 1.
template <int NPE>
struct GaussRule;
template <>
struct GaussRule<4> {
  static constexpr int n = 4;
  __device__ static void point(int g, double q[3]) {
    const double a = 0.58541020, b = 0.13819660;
    q[0] = (g == 0) ? a : b;
    q[1] = (g == 1) ? a : b;
    q[2] = (g == 2) ? a : b;
  }
  __device__ static double weight() { return (1.0 / 6.0) * (1.0 / 4.0); }
};
template <>
struct GaussRule<8> {
  static constexpr int n = 8;
  __device__ static void point(int g, double q[3]) {
    const double s = 0.57735026918962573;  // 1/sqrt(3), correctly rounded
    const double sx[8] = {-s, s, s, -s, -s, s, s, -s};
    const double sy[8] = {-s, -s, s, s, -s, -s, s, s};
    const double sz[8] = {s, s, s, s, -s, -s, -s, -s};
    q[0] = sx[g];
    q[1] = sy[g];
    q[2] = sz[g];
  }
  __device__ static double weight() { return 8.0 * (1.0 / 8.0); }
};

// Shape functions and local derivatives (femTetra4.cpp:295-330,
// femHexa8.cpp:13-42).
template <int NPE>
__device__ __forceinline__ void shape(const double q[3], double N[NPE], double dN[NPE][3]) {
  if (NPE == 4) {
    N[0] = q[0]; N[1] = q[1]; N[2] = q[2]; N[3] = 1.0 - q[0] - q[1] - q[2];
    dN[0][0] = 1.0; dN[0][1] = 0.0; dN[0][2] = 0.0;
    dN[1][0] = 0.0; dN[1][1] = 1.0; dN[1][2] = 0.0;
    dN[2][0] = 0.0; dN[2][1] = 0.0; dN[2][2] = 1.0;
    dN[3][0] = -1.0; dN[3][1] = -1.0; dN[3][2] = -1.0;
  } else {
    const double c1[8] = {-1.0, 1.0, 1.0, -1.0, -1.0, 1.0, 1.0, -1.0};
    const double c2[8] = {-1.0, -1.0, 1.0, 1.0, -1.0, -1.0, 1.0, 1.0};
    const double c3[8] = {-1.0, -1.0, -1.0, -1.0, 1.0, 1.0, 1.0, 1.0};
#pragma unroll
    for (int a = 0; a < NPE; ++a) {
      const double fx = 1.0 + q[0] * c1[a], fy = 1.0 + q[1] * c2[a], fz = 1.0 + q[2] * c3[a];
      N[a] = 0.125 * fx * fy * fz;
      dN[a][0] = 0.125 * c1[a] * fy * fz;
      dN[a][1] = 0.125 * c2[a] * fx * fz;
      dN[a][2] = 0.125 * c3[a] * fx * fy;
    }
  }
}

// Shape values and local derivatives at the Gauss points, tabulated once per
// CTA in shared memory with the same expressions as shape<NPE> (identical
// values); the Gauss-point loops read them at warp-uniform addresses.
template <int NPE, typename T>
struct ShapeTable {
  T N[GaussRule<NPE>::n][NPE];
  T dN[GaussRule<NPE>::n][NPE][3];
};

template <int NPE, typename T>
__device__ __forceinline__ void fill_shape_table(ShapeTable<NPE, T>* t) {
  for (int g = threadIdx.x; g < GaussRule<NPE>::n; g += blockDim.x) {
    double q[3], Nf[NPE], dN[NPE][3];
    GaussRule<NPE>::point(g, q);
    shape<NPE>(q, Nf, dN);
#pragma unroll
    for (int a = 0; a < NPE; ++a) {
      t->N[g][a] = (T)Nf[a];
#pragma unroll
      for (int c = 0; c < 3; ++c) t->dN[g][a][c] = (T)dN[a][c];
    }
  }
}

// Jacobian J[a][b] = sum_n dN[n][a] x[n][b] (femElement.cpp:104-127), its
// cofactor inverse (femUtils.cpp:716-770), global derivatives
// gd[n][b] = sum_c inv[b][c] dN[n][c] (femElement.cpp:345-352) and the
// geometric matrix G[a][b] = sum_c inv[c][a] inv[c][b] (femElement.cpp:222-230).
// The local derivatives are read through dN(n, a): a register array, or a
// shared-memory table read where used.
template <int NPE, class DN>
__device__ __forceinline__ double jacobian_at(DN dN, const double* sx, const double* sy, const double* sz, const int ln[NPE],
                                              double inv[3][3]) {
  double J[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double j0 = 0.0, j1 = 0.0, j2 = 0.0;
#pragma unroll
    for (int n = 0; n < NPE; ++n) {
      const double d = dN(n, a);
      j0 += d * sx[ln[n]];
      j1 += d * sy[ln[n]];
      j2 += d * sz[ln[n]];
    }
    J[a][0] = j0; J[a][1] = j1; J[a][2] = j2;
  }
  const double m00 = J[0][0], m01 = J[0][1], m02 = J[0][2], m10 = J[1][0], m11 = J[1][1], m12 = J[1][2], m20 = J[2][0],
               m21 = J[2][1], m22 = J[2][2];
  const double det = m00 * (m11 * m22 - m21 * m12) - m01 * (m10 * m22 - m12 * m20) + m02 * (m10 * m21 - m11 * m20);
  const double id = 1.0 / det;
  inv[0][0] = (m11 * m22 - m21 * m12) * id;
  inv[0][1] = (m02 * m21 - m01 * m22) * id;
  inv[0][2] = (m01 * m12 - m02 * m11) * id;
  inv[1][0] = (m12 * m20 - m10 * m22) * id;
  inv[1][1] = (m00 * m22 - m02 * m20) * id;
  inv[1][2] = (m10 * m02 - m00 * m12) * id;
  inv[2][0] = (m10 * m21 - m20 * m11) * id;
  inv[2][1] = (m20 * m01 - m00 * m21) * id;
  inv[2][2] = (m00 * m11 - m10 * m01) * id;
  return det;
}

template <int NPE>
__device__ __forceinline__ double jacobian(const double dN[NPE][3], const double* sx, const double* sy, const double* sz,
                                           const int ln[NPE], double inv[3][3]) {
  return jacobian_at<NPE>([&](int n, int a) { return dN[n][a]; }, sx, sy, sz, ln, inv);
}

// Per Gauss point (per element for tet4): G = J^-T J^-1
// (femElement.cpp:192-232), the G:G term of tau, (mu/rho)^2 cI G:G
// (eval_stabilization, src lines 336-377), and G's cofactor inverse
// (eval_bulk_modulus, src lines 382-441).
__device__ __forceinline__ void tet_metric(const double inv[3][3], double nu, double cI, double G[3][3], double& t3,
                                           double iG[3][3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) G[a][b] = inv[0][a] * inv[0][b] + inv[1][a] * inv[1][b] + inv[2][a] * inv[2][b];
  t3 = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) t3 += G[a][0] * G[a][0] + G[a][1] * G[a][1] + G[a][2] * G[a][2];
  t3 = t3 * nu * nu * cI;
  const double m00 = G[0][0], m01 = G[0][1], m02 = G[0][2], m10 = G[1][0], m11 = G[1][1], m12 = G[1][2],
               m20 = G[2][0], m21 = G[2][1], m22 = G[2][2];
  const double dG = m00 * (m11 * m22 - m21 * m12) - m01 * (m10 * m22 - m12 * m20) + m02 * (m10 * m21 - m11 * m20);
  const double idg = 1.0 / dG;
  iG[0][0] = (m11 * m22 - m21 * m12) * idg;
  iG[0][1] = (m02 * m21 - m01 * m22) * idg;
  iG[0][2] = (m01 * m12 - m02 * m11) * idg;
  iG[1][0] = (m12 * m20 - m10 * m22) * idg;
  iG[1][1] = (m00 * m22 - m02 * m20) * idg;
  iG[1][2] = (m10 * m02 - m00 * m12) * idg;
  iG[2][0] = (m10 * m21 - m20 * m11) * idg;
  iG[2][1] = (m20 * m01 - m00 * m21) * idg;
  iG[2][2] = (m00 * m11 - m10 * m01) * idg;
}

// Gauss-point geometry of one hexa8 element, formed once per placement and
// kept in HBM: per point g the inverse Jacobian (9 entries) and det J, entry
// q of point g at geo[(g * FM_GEO_PER_GP + q) * E + e] (coalesced over the
// tile's consecutive element slots).  The mesh does not move, so these are
// the values the element loop would form at every step from the same
// coordinates with the same expressions.
__device__ __forceinline__ double geo_at(const double* geo, int64_t E, int g, double inv[3][3]) {
  const double* q = geo + (int64_t)g * FM_GEO_PER_GP * E;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) inv[a][b] = __ldg(q + (a * 3 + b) * E);
  return __ldg(q + 9 * E);
}

// Requests point g's ten entries into L1 ahead of their use (the loads of a
// warp cover consecutive element slots: one or two 128-byte lines an entry).
template <typename T>
__device__ __forceinline__ void geo_prefetch(const T* geo, int64_t E, int g) {
  const T* q = geo + (int64_t)g * FM_GEO_PER_GP * E;
#pragma unroll
  for (int k = 0; k < FM_GEO_PER_GP; ++k) asm volatile("prefetch.global.L1 [%0];" ::"l"(q + k * E));
}

// The mixed form's copy: the same FP64 values rounded to FP32.
__device__ __forceinline__ float geo_at_f(const float* geo, int64_t E, int g, float inv[3][3]) {
  const float* q = geo + (int64_t)g * FM_GEO_PER_GP * E;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) inv[a][b] = __ldg(q + (a * 3 + b) * E);
  return __ldg(q + 9 * E);
}

// One element: k[a][c] = -dt (sum of the enabled K_i u_e)[a][c].  Coordinates
// and velocities are read from the tile's shared-memory node arrays through
// the local ids ln[]; with GEO the Gauss-point inverse Jacobians and
// determinants are read from the stored geometry instead (geo = the
// element's first entry, E = the row stride).  Also returns the element's
// lambda (volume average) and regime (average of the Gauss-point regimes)
// for output.
template <int NPE, bool GEO = false>
__device__ __forceinline__ void supg_element(const DevProb& P, const ShapeTable<NPE, double>& tab, const double* sx,
                                             const double* sy, const double* sz, const double* su, const double* sv,
                                             const double* sw, const int ln[NPE], double k[NPE][3], double& lam_el,
                                             double& reg_el, const double* geo = nullptr, int64_t E = 0) {
  const double rho = P.rho, mu = P.mu, alpha = P.alpha, cI = P.c_i;
  const double nu = mu / rho;
  const bool bbar = (P.ex_mask & 2) != 0;
  const bool iK1 = (P.ex_mask & 4) != 0, iK2 = (P.ex_mask & 8) != 0, iK3 = (P.ex_mask & 16) != 0,
             iK4 = (P.ex_mask & 32) != 0;
  const double wq = GaussRule<NPE>::weight();
#pragma unroll
  for (int a = 0; a < NPE; ++a) k[a][0] = k[a][1] = k[a][2] = 0.0;
  // B-bar (eval_avg_shapeDeriv, src lines 660-707, and the B matrix rows
  // 0-2, src lines 234-256).  With sd0[a][c] = sum_g w_g gd_g[a][c] / V the
  // volume-averaged derivatives, B1 = (sd0[a][0] - gd[a][0]) / 3, B2 =
  // gd[a][0] - B1 and likewise B3/B4, B5/B6 for y and z, the sums over the
  // nodes are
  //   strain:  eps_c = gr_cc - 2 d_c + (d_0 + d_1 + d_2),
  //            d_c = (Dbar_c - gr_cc) / 3,  Dbar_c = sum_a sd0[a][c] u_c(a)
  //   force:   r_c(a) w = gd[a][c] (w sig_c - q_c) + sd0[a][c] q_c,
  //            q_c = w (sig_0 + sig_1 + sig_2 - 2 sig_c) / 3,
  // so sd0 enters only through the element constants Dbar_c = sum_g w_g
  // gr_g[c][c] / V (before the Gauss loop) and sd0[a][c] Q_c, Q_c = sum_g q_c
  // (after it): the 24 averaged derivatives are never held in registers.
  auto jac_inv = [&](int g, double inv[3][3]) -> double {
    if constexpr (GEO) return geo_at(geo, E, g, inv);
    return jacobian_at<NPE>([&](int n, int c) { return tab.dN[g][n][c]; }, sx, sy, sz, ln, inv);
  };
  double Dbar[3] = {0.0, 0.0, 0.0}, Qb[3] = {0.0, 0.0, 0.0}, bden = 0.0;
  if (NPE == 8 && bbar) {
    double dsum[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
    for (int g = 0; g < GaussRule<NPE>::n; ++g) {
      double inv[3][3];
      const double w = jac_inv(g, inv) * wq;
      bden += w;
      double g0 = 0.0, g1 = 0.0, g2 = 0.0;
#pragma unroll
      for (int a = 0; a < NPE; ++a) {
        const double d0 = tab.dN[g][a][0], d1 = tab.dN[g][a][1], d2 = tab.dN[g][a][2];
        g0 += (inv[0][0] * d0 + inv[0][1] * d1 + inv[0][2] * d2) * su[ln[a]];
        g1 += (inv[1][0] * d0 + inv[1][1] * d1 + inv[1][2] * d2) * sv[ln[a]];
        g2 += (inv[2][0] * d0 + inv[2][1] * d1 + inv[2][2] * d2) * sw[ln[a]];
      }
      dsum[0] += w * g0; dsum[1] += w * g1; dsum[2] += w * g2;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) Dbar[c] = dsum[c] / bden;
  }
  // tet4: the local derivatives are constant, so the Jacobian, its inverse,
  // G = J^-T J^-1, the G:G term of tau and G's inverse are element constants;
  // they are formed once here (the same expressions as at every Gauss point,
  // hence the same values) instead of at each of the 4 points
  auto dN4 = [](int a, int c) -> double { return a == 3 ? -1.0 : (a == c ? 1.0 : 0.0); };
  double inv4[3][3], det4 = 0.0, G4[3][3], t3_4 = 0.0, iG4[3][3];
  if constexpr (NPE == 4) {
    det4 = jacobian_at<NPE>(dN4, sx, sy, sz, ln, inv4);
    tet_metric(inv4, nu, cI, G4, t3_4, iG4);
  }
  double vol = 0.0, lam_int = 0.0, reg = 0.0;
  if constexpr (GEO) {
    geo_prefetch(geo, E, 0);
    geo_prefetch(geo, E, 1);
  }
#pragma unroll 1
  for (int g = 0; g < GaussRule<NPE>::n; ++g) {
    // shape values and local derivatives: tet4 in closed form (constant
    // derivatives), hexa8 read from the shared-memory table where used; the
    // global derivatives are formed where used too (no register arrays)
    double Nq[NPE];
    if (NPE == 4) {
      double q[3];
      GaussRule<NPE>::point(g, q);
      Nq[0] = q[0]; Nq[1] = q[1]; Nq[2] = q[2]; Nq[3 % NPE] = 1.0 - q[0] - q[1] - q[2];
    }
    auto Nv = [&](int a) -> double { return NPE == 4 ? Nq[a] : tab.N[g][a]; };
    auto dNv = [&](int a, int c) -> double {
      if (NPE == 4) return dN4(a, c);
      return tab.dN[g][a][c];
    };
    double inv[3][3], G[3][3], t3 = 0.0, iG[3][3];
    double det;
    if constexpr (NPE == 4) {
      det = det4;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          inv[a][b] = inv4[a][b];
          G[a][b] = G4[a][b];
          iG[a][b] = iG4[a][b];
        }
      t3 = t3_4;
    } else {
      if constexpr (GEO) {
        if (g + 2 < GaussRule<NPE>::n) geo_prefetch(geo, E, g + 2);
      }
      det = jac_inv(g, inv);
      tet_metric(inv, nu, cI, G, t3, iG);
    }
    auto gdv = [&](int a, int b) -> double {
      return inv[b][0] * dNv(a, 0) + inv[b][1] * dNv(a, 1) + inv[b][2] * dNv(a, 2);
    };
    // velocity, gradient, divergence at the point.  hexa8: the gradient in
    // local coordinates first, Lg[c][k] = sum_a dN[a][k] u_a[c], then
    // gr[c][d] = sum_k inv[d][k] Lg[c][k] (the same sum over the nodes as
    // sum_a gd[a][d] u_a[c], 99 instead of 144 FLOP a point); tet4's
    // derivatives are constants, so its global ones cost nothing to form
    double u[3] = {0.0, 0.0, 0.0}, gr[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    if constexpr (NPE == 8) {
      double Lg[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
#pragma unroll
      for (int a = 0; a < NPE; ++a) {
        const double ua[3] = {su[ln[a]], sv[ln[a]], sw[ln[a]]};
        const double Na = Nv(a);
        const double da[3] = {dNv(a, 0), dNv(a, 1), dNv(a, 2)};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          u[c] += Na * ua[c];
#pragma unroll
          for (int kk = 0; kk < 3; ++kk) Lg[c][kk] += da[kk] * ua[c];
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) gr[c][d] = inv[d][0] * Lg[c][0] + inv[d][1] * Lg[c][1] + inv[d][2] * Lg[c][2];
    } else {
#pragma unroll
      for (int a = 0; a < NPE; ++a) {
        const double ua[3] = {su[ln[a]], sv[ln[a]], sw[ln[a]]};
        const double ga[3] = {gdv(a, 0), gdv(a, 1), gdv(a, 2)};
        const double Na = Nv(a);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          u[c] += Na * ua[c];
#pragma unroll
          for (int d = 0; d < 3; ++d) gr[c][d] += ga[d] * ua[c];
        }
      }
    }
    const double div = gr[0][0] + gr[1][1] + gr[2][2];
    // eval_stabilization (dt term removed in the reference)
    const double trG = G[0][0] + G[1][1] + G[2][2];
    double t2 = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) t2 += u[a] * (G[a][0] * u[0] + G[a][1] * u[1] + G[a][2] * u[2]);
    const double tau = 1.0 / sqrt(t2 + t3);
    const double nuC = 1.0 / (trG * tau);
    // eval_bulk_modulus: lambda = alpha * max(mu/rho, sqrt(u^T G^-1 u))
    double lam, regime;
    {
      const double l2 = sqrt((iG[0][0] * u[0] + iG[0][1] * u[1] + iG[0][2] * u[2]) * u[0] +
                             (iG[1][0] * u[0] + iG[1][1] * u[1] + iG[1][2] * u[2]) * u[1] +
                             (iG[2][0] * u[0] + iG[2][1] * u[1] + iG[2][2] * u[2]) * u[2]);
      const double l1 = nu;
      lam = alpha * ((l1 < l2) ? l2 : l1);  // std::max(limit_1, limit_2)
      regime = (l1 > l2) ? 1.0 : 2.0;
    }
    const double w = det * wq;
    vol += w;
    lam_int += lam * w;
    reg += regime;
    double conv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) conv[c] = u[0] * gr[c][0] + u[1] * gr[c][1] + u[2] * gr[c][2];
    // strain (B u) and stress (D B u)
    double eps[6];
    if (NPE == 8 && bbar) {
      const double d0 = (1.0 / 3.0) * (Dbar[0] - gr[0][0]), d1 = (1.0 / 3.0) * (Dbar[1] - gr[1][1]),
                   d2 = (1.0 / 3.0) * (Dbar[2] - gr[2][2]);
      eps[0] = gr[0][0] - d0 + d1 + d2;
      eps[1] = d0 + gr[1][1] - d1 + d2;
      eps[2] = d0 + d1 + gr[2][2] - d2;
    } else {
      eps[0] = gr[0][0]; eps[1] = gr[1][1]; eps[2] = gr[2][2];
    }
    eps[3] = gr[0][1] + gr[1][0];
    eps[4] = gr[1][2] + gr[2][1];
    eps[5] = gr[0][2] + gr[2][0];
    const double l2m = lam + 2 * mu;
    const double sig[6] = {l2m * eps[0] + lam * eps[1] + lam * eps[2], lam * eps[0] + l2m * eps[1] + lam * eps[2],
                           lam * eps[0] + lam * eps[1] + l2m * eps[2], mu * eps[3], mu * eps[4], mu * eps[5]};
    const double c1w = rho * w, c3w = rho * tau * w, c4w = rho * nuC * div * w;
    // normal-stress parts of K2: w sig_c multiplies gd[a][c]; with B-bar less
    // q_c, whose sd0 part is added after the loop
    double sd[3] = {sig[0] * w, sig[1] * w, sig[2] * w};
    if (NPE == 8 && bbar && iK2) {
      const double st = sig[0] + sig[1] + sig[2];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double q = (1.0 / 3.0) * w * (st - 2.0 * sig[c]);
        Qb[c] += q;
        sd[c] -= q;
      }
    }
    if constexpr (NPE == 8) {
      // hexa8: every term is linear in gd[a] = inv dN[a] (K2: S gd[a] with S
      // the symmetric matrix of the stress terms above; K4: c4w gd[a]; K3:
      // u.gd[a]), so inv is folded into one 3x3 matrix and one vector a
      // point, T = (S + c4w I) inv and ut = inv^T u, and each node takes
      // T dN[a] and ut.dN[a] (17 instead of ~36 FLOP a node)
      double S[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
      if (iK2) {
        S[0][0] = sd[0]; S[1][1] = sd[1]; S[2][2] = sd[2];
        S[0][1] = S[1][0] = sig[3] * w;
        S[1][2] = S[2][1] = sig[4] * w;
        S[0][2] = S[2][0] = sig[5] * w;
      }
      if (iK4) {
#pragma unroll
        for (int c = 0; c < 3; ++c) S[c][c] += c4w;
      }
      double T[3][3], ut[3];
#pragma unroll
      for (int kk = 0; kk < 3; ++kk) {
#pragma unroll
        for (int c = 0; c < 3; ++c) T[c][kk] = S[c][0] * inv[0][kk] + S[c][1] * inv[1][kk] + S[c][2] * inv[2][kk];
        ut[kk] = u[0] * inv[0][kk] + u[1] * inv[1][kk] + u[2] * inv[2][kk];
      }
#pragma unroll
      for (int a = 0; a < NPE; ++a) {
        const double da[3] = {dNv(a, 0), dNv(a, 1), dNv(a, 2)};
        double sa = 0.0;
        if (iK1) sa = c1w * Nv(a);
        if (iK3) sa += c3w * (ut[0] * da[0] + ut[1] * da[1] + ut[2] * da[2]);
#pragma unroll
        for (int c = 0; c < 3; ++c) k[a][c] += T[c][0] * da[0] + T[c][1] * da[1] + T[c][2] * da[2] + sa * conv[c];
      }
    } else {
#pragma unroll
    for (int a = 0; a < NPE; ++a) {
      const double ga[3] = {gdv(a, 0), gdv(a, 1), gdv(a, 2)};
      const double Aa = u[0] * ga[0] + u[1] * ga[1] + u[2] * ga[2];
      double f[3] = {0.0, 0.0, 0.0};
      if (iK1) {
        const double Na = Nv(a);
#pragma unroll
        for (int c = 0; c < 3; ++c) f[c] += c1w * Na * conv[c];
      }
      if (iK3) {
#pragma unroll
        for (int c = 0; c < 3; ++c) f[c] += c3w * Aa * conv[c];
      }
      if (iK4) {
#pragma unroll
        for (int c = 0; c < 3; ++c) f[c] += c4w * ga[c];
      }
      if (iK2) {
        f[0] += ga[0] * sd[0] + (ga[1] * sig[3] + ga[2] * sig[5]) * w;
        f[1] += ga[1] * sd[1] + (ga[0] * sig[3] + ga[2] * sig[4]) * w;
        f[2] += ga[2] * sd[2] + (ga[1] * sig[4] + ga[0] * sig[5]) * w;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) k[a][c] += f[c];
    }
    }
  }
  if (NPE == 8 && bbar && iK2) {
    // k[a][c] += sd0[a][c] Q_c, sd0 formed again Gauss point by Gauss point
#pragma unroll
    for (int c = 0; c < 3; ++c) Qb[c] /= bden;
#pragma unroll 1
    for (int g = 0; g < GaussRule<NPE>::n; ++g) {
      double inv[3][3];
      const double w = jac_inv(g, inv) * wq;
      const double s0 = w * Qb[0], s1 = w * Qb[1], s2 = w * Qb[2];
#pragma unroll
      for (int a = 0; a < NPE; ++a) {
        const double d0 = tab.dN[g][a][0], d1 = tab.dN[g][a][1], d2 = tab.dN[g][a][2];
        k[a][0] += (inv[0][0] * d0 + inv[0][1] * d1 + inv[0][2] * d2) * s0;
        k[a][1] += (inv[1][0] * d0 + inv[1][1] * d1 + inv[1][2] * d2) * s1;
        k[a][2] += (inv[2][0] * d0 + inv[2][1] * d1 + inv[2][2] * d2) * s2;
      }
    }
  }
  const double mdt = -P.dt;
#pragma unroll
  for (int a = 0; a < NPE; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) k[a][c] *= mdt;
  lam_el = lam_int / vol;
  reg_el = reg / (double)GaussRule<NPE>::n;
}

}  // namespace fm

namespace fm {

// ---------------------------------------------------------------------------
// Mixed precision SUPG element (FM_MIXED): the Gauss-point work in FP32,
// k = -dt K u_e converted to FP64 for the nodal accumulation, the AB2 history
// and the update, which stay FP64.  Coordinates and velocities enter FP32 as
// differences to the element's node 0, formed in FP64 (Xr, Ud; Xr[0] = Ud[0]
// = 0), so the Jacobian and the velocity gradient lose no digits to
// cancellation.  Elements flagged `precise` (aspect ratio above
// FM_MIXED_ASPECT_LIMIT) form the Jacobian and its inverse in FP64 from the
// staged FP64 coordinates.  The Jacobian, the global derivatives, the
// velocity and its gradient and the nodal terms run two components at a time
// in paired FP32 arithmetic (sm_100 FFMA2 / FMUL2; 5% off the mixed tile
// kernel for tet4 and hexa8).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float rcp_f(float x) {
  const float y = ptx_rcp_approx(x);
  return fmaf(y, fmaf(-x, y, 1.0f), y);  // one Newton step: full FP32 accuracy
}
__device__ __forceinline__ float rsqrt_f(float x) {
  const float y = ptx_rsqrt_approx(x);
  return y * fmaf(-0.5f * x, y * y, 1.5f);
}

// FP32 form of tet_metric.
__device__ __forceinline__ void metric_f(const float inv[3][3], float nu, float cI, float G[3][3], float& t3,
                                         float iG[3][3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) G[a][b] = inv[0][a] * inv[0][b] + inv[1][a] * inv[1][b] + inv[2][a] * inv[2][b];
  t3 = 0.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) t3 += G[a][0] * G[a][0] + G[a][1] * G[a][1] + G[a][2] * G[a][2];
  t3 = t3 * nu * nu * cI;
  const float m00 = G[0][0], m01 = G[0][1], m02 = G[0][2], m10 = G[1][0], m11 = G[1][1], m12 = G[1][2],
              m20 = G[2][0], m21 = G[2][1], m22 = G[2][2];
  const float dG = m00 * (m11 * m22 - m21 * m12) - m01 * (m10 * m22 - m12 * m20) + m02 * (m10 * m21 - m11 * m20);
  const float idg = rcp_f(dG);
  iG[0][0] = (m11 * m22 - m21 * m12) * idg;
  iG[0][1] = (m02 * m21 - m01 * m22) * idg;
  iG[0][2] = (m01 * m12 - m02 * m11) * idg;
  iG[1][0] = (m12 * m20 - m10 * m22) * idg;
  iG[1][1] = (m00 * m22 - m02 * m20) * idg;
  iG[1][2] = (m10 * m02 - m00 * m12) * idg;
  iG[2][0] = (m10 * m21 - m20 * m11) * idg;
  iG[2][1] = (m20 * m01 - m00 * m21) * idg;
  iG[2][2] = (m00 * m11 - m10 * m01) * idg;
}

template <int NPE, bool GEO = false>
__device__ __forceinline__ void supg_element_mixed(const DevProb& P, const ShapeTable<NPE, float>& tab,
                                                   const ShapeTable<NPE, double>& tabd, const float Xr[NPE][3],
                                                   const float U0[3], const float Ud[NPE][3], bool precise,
                                                   const double* sx, const double* sy, const double* sz,
                                                   const int ln[NPE], double k[NPE][3], double& lam_el,
                                                   double& reg_el, const float* geo = nullptr, int64_t E = 0) {
  const float rho = (float)P.rho, mu = (float)P.mu, alpha = (float)P.alpha, cI = (float)P.c_i;
  const float nu = (float)(P.mu / P.rho);
  const bool bbar = (P.ex_mask & 2) != 0;
  const bool iK1 = (P.ex_mask & 4) != 0, iK2 = (P.ex_mask & 8) != 0, iK3 = (P.ex_mask & 16) != 0,
             iK4 = (P.ex_mask & 32) != 0;
  const float wq = (float)GaussRule<NPE>::weight();
  float kf[NPE][3];
#pragma unroll
  for (int a = 0; a < NPE; ++a) kf[a][0] = kf[a][1] = kf[a][2] = 0.0f;
  // shape values / local derivatives at Gauss point g: tet4 in closed form
  // (constant derivatives), hexa8 from the shared-memory table
  auto dNv = [&](int g, int a, int c) -> float {
    if (NPE == 4) return a == 3 ? -1.0f : (a == c ? 1.0f : 0.0f);
    return tab.dN[g][a][c];
  };
  auto Nv = [&](int g, int a) -> float {
    if (NPE == 4) {
      double q[3];
      GaussRule<NPE>::point(g, q);
      return a < 3 ? (float)q[a] : (float)(1.0 - q[0] - q[1] - q[2]);
    }
    return tab.N[g][a];
  };
  // per Gauss point: inverse Jacobian and det, FP32 or (precise) FP64; with
  // GEO read from the stored geometry (formed in FP64 for every element)
  auto geometry = [&](int g, float inv[3][3]) -> float {
    if constexpr (GEO) return geo_at_f(geo, E, g, inv);
    if (precise) {
      double dN[NPE][3], invd[3][3];
#pragma unroll
      for (int a = 0; a < NPE; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) dN[a][c] = tabd.dN[g][a][c];
      const double det = jacobian<NPE>(dN, sx, sy, sz, ln, invd);
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) inv[i][j] = (float)invd[i][j];
      return (float)det;
    }
    float J[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      // (J[a][0], J[a][1]) as one pair, J[a][2] alone
      float2 s01 = make_float2(0.0f, 0.0f);
      float s2 = 0.0f;
#pragma unroll
      for (int n = 1; n < NPE; ++n) {
        const float d = dNv(g, n, a);
        s01 = __ffma2_rn(make_float2(d, d), make_float2(Xr[n][0], Xr[n][1]), s01);
        s2 += d * Xr[n][2];
      }
      J[a][0] = s01.x; J[a][1] = s01.y; J[a][2] = s2;
    }
    const float c00 = J[1][1] * J[2][2] - J[2][1] * J[1][2], c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2],
                c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    const float det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
    const float id = rcp_f(det);
    inv[0][0] = c00 * id;
    inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
    inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
    inv[1][0] = c01 * id;
    inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
    inv[1][2] = (J[1][0] * J[0][2] - J[0][0] * J[1][2]) * id;
    inv[2][0] = c02 * id;
    inv[2][1] = (J[2][0] * J[0][1] - J[0][0] * J[2][1]) * id;
    inv[2][2] = (J[0][0] * J[1][1] - J[1][0] * J[0][1]) * id;
    return det;
  };
  // volume-averaged derivatives for B-bar (eval_avg_shapeDeriv, src lines 660-707)
  float sd0[NPE][3];
  if (NPE == 8 && bbar) {
    float num[NPE][3], den = 0.0f;
#pragma unroll
    for (int a = 0; a < NPE; ++a) num[a][0] = num[a][1] = num[a][2] = 0.0f;
#pragma unroll 1
    for (int g = 0; g < GaussRule<NPE>::n; ++g) {
      float inv[3][3];
      const float w = geometry(g, inv) * wq;
      den += w;
#pragma unroll
      for (int a = 0; a < NPE; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
          num[a][b] += (inv[b][0] * dNv(g, a, 0) + inv[b][1] * dNv(g, a, 1) + inv[b][2] * dNv(g, a, 2)) * w;
    }
    const float iden = rcp_f(den);
#pragma unroll
    for (int a = 0; a < NPE; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) sd0[a][b] = num[a][b] * iden;
  }
  // tet4: inverse Jacobian, G, its G:G term and G's inverse are element
  // constants, formed once (the same values as at every Gauss point)
  float inv4[3][3], det4 = 0.0f, G4[3][3], t3_4 = 0.0f, iG4[3][3];
  if constexpr (NPE == 4) {
    det4 = geometry(0, inv4);
    metric_f(inv4, nu, cI, G4, t3_4, iG4);
  }
  float vol = 0.0f, lam_int = 0.0f, reg = 0.0f;
  if constexpr (GEO) {
    geo_prefetch(geo, E, 0);
    geo_prefetch(geo, E, 1);
  }
#pragma unroll 1
  for (int g = 0; g < GaussRule<NPE>::n; ++g) {
    float inv[3][3], G[3][3], t3, iG[3][3];
    float det;
    if constexpr (NPE == 4) {
      det = det4;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          inv[a][b] = inv4[a][b];
          G[a][b] = G4[a][b];
          iG[a][b] = iG4[a][b];
        }
      t3 = t3_4;
    } else {
      if constexpr (GEO) {
        if (g + 2 < GaussRule<NPE>::n) geo_prefetch(geo, E, g + 2);
      }
      det = geometry(g, inv);
      metric_f(inv, nu, cI, G, t3, iG);
    }
    float gd[NPE][3];
    {
      const float2 i0 = make_float2(inv[0][0], inv[1][0]), i1 = make_float2(inv[0][1], inv[1][1]),
                   i2 = make_float2(inv[0][2], inv[1][2]);
#pragma unroll
      for (int a = 0; a < NPE; ++a) {
        const float d0 = dNv(g, a, 0), d1 = dNv(g, a, 1), d2 = dNv(g, a, 2);
        float2 q = __fmul2_rn(i0, make_float2(d0, d0));
        q = __ffma2_rn(i1, make_float2(d1, d1), q);
        q = __ffma2_rn(i2, make_float2(d2, d2), q);
        gd[a][0] = q.x; gd[a][1] = q.y;
        gd[a][2] = inv[2][0] * d0 + inv[2][1] * d1 + inv[2][2] * d2;
      }
    }
    float u[3], gr[3][3];
    {
      // (u0, u1) and (gr[c][0], gr[c][1]) as pairs
      float2 u01 = make_float2(U0[0], U0[1]);
      float u2 = U0[2];
      float2 g01[3] = {make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f)};
      float g2[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int a = 1; a < NPE; ++a) {
        const float Na = Nv(g, a);
        u01 = __ffma2_rn(make_float2(Na, Na), make_float2(Ud[a][0], Ud[a][1]), u01);
        u2 += Na * Ud[a][2];
        const float2 ga = make_float2(gd[a][0], gd[a][1]);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          g01[c] = __ffma2_rn(ga, make_float2(Ud[a][c], Ud[a][c]), g01[c]);
          g2[c] += gd[a][2] * Ud[a][c];
        }
      }
      u[0] = u01.x; u[1] = u01.y; u[2] = u2;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        gr[c][0] = g01[c].x; gr[c][1] = g01[c].y; gr[c][2] = g2[c];
      }
    }
    const float div = gr[0][0] + gr[1][1] + gr[2][2];
    // eval_stabilization (dt term removed in the reference)
    const float trG = G[0][0] + G[1][1] + G[2][2];
    float t2 = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a) t2 += u[a] * (G[a][0] * u[0] + G[a][1] * u[1] + G[a][2] * u[2]);
    const float tau = rsqrt_f(t2 + t3);
    const float nuC = rcp_f(trG * tau);
    // eval_bulk_modulus: lambda = alpha * max(mu/rho, sqrt(u^T G^-1 u))
    float lam, regime;
    {
      const float q2 = (iG[0][0] * u[0] + iG[0][1] * u[1] + iG[0][2] * u[2]) * u[0] +
                       (iG[1][0] * u[0] + iG[1][1] * u[1] + iG[1][2] * u[2]) * u[1] +
                       (iG[2][0] * u[0] + iG[2][1] * u[1] + iG[2][2] * u[2]) * u[2];
      const float l2 = q2 > 0.0f ? q2 * rsqrt_f(q2) : sqrtf(q2);  // sqrt; NaN for negative input as sqrt
      const float l1 = nu;
      lam = alpha * ((l1 < l2) ? l2 : l1);  // std::max(limit_1, limit_2)
      regime = (l1 > l2) ? 1.0f : 2.0f;
    }
    const float w = det * wq;
    vol += w;
    lam_int += lam * w;
    reg += regime;
    float conv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) conv[c] = u[0] * gr[c][0] + u[1] * gr[c][1] + u[2] * gr[c][2];
    float eps[6];
    if (NPE == 8 && bbar) {
      float e0 = 0.0f, e1 = 0.0f, e2 = 0.0f;
#pragma unroll
      for (int a = 1; a < NPE; ++a) {
        const float B1 = (1.0f / 3.0f) * (sd0[a][0] - gd[a][0]), B2 = gd[a][0] - B1;
        const float B3 = (1.0f / 3.0f) * (sd0[a][1] - gd[a][1]), B4 = gd[a][1] - B3;
        const float B5 = (1.0f / 3.0f) * (sd0[a][2] - gd[a][2]), B6 = gd[a][2] - B5;
        e0 += B2 * Ud[a][0] + B3 * Ud[a][1] + B5 * Ud[a][2];
        e1 += B1 * Ud[a][0] + B4 * Ud[a][1] + B5 * Ud[a][2];
        e2 += B1 * Ud[a][0] + B3 * Ud[a][1] + B6 * Ud[a][2];
      }
      // the node-0 term: B-bar rows sum to zero over the nodes, so the
      // differences to node 0 give the same strain
      eps[0] = e0; eps[1] = e1; eps[2] = e2;
    } else {
      eps[0] = gr[0][0]; eps[1] = gr[1][1]; eps[2] = gr[2][2];
    }
    eps[3] = gr[0][1] + gr[1][0];
    eps[4] = gr[1][2] + gr[2][1];
    eps[5] = gr[0][2] + gr[2][0];
    const float l2m = lam + 2.0f * mu;
    const float sig[6] = {l2m * eps[0] + lam * eps[1] + lam * eps[2], lam * eps[0] + l2m * eps[1] + lam * eps[2],
                          lam * eps[0] + lam * eps[1] + l2m * eps[2], mu * eps[3], mu * eps[4], mu * eps[5]};
    const float c1w = rho * w, c3w = rho * tau * w, c4w = rho * nuC * div * w;
    const float2 conv01 = make_float2(conv[0], conv[1]);
#pragma unroll
    for (int a = 0; a < NPE; ++a) {
      const float Aa = u[0] * gd[a][0] + u[1] * gd[a][1] + u[2] * gd[a][2];
      // (f0, f1) as a pair, f2 alone
      float2 f01 = make_float2(0.0f, 0.0f);
      float f2v = 0.0f;
      if (iK1) {
        const float t = c1w * Nv(g, a);
        f01 = __ffma2_rn(make_float2(t, t), conv01, f01);
        f2v += t * conv[2];
      }
      if (iK3) {
        const float t = c3w * Aa;
        f01 = __ffma2_rn(make_float2(t, t), conv01, f01);
        f2v += t * conv[2];
      }
      if (iK4) {
        f01 = __ffma2_rn(make_float2(c4w, c4w), make_float2(gd[a][0], gd[a][1]), f01);
        f2v += c4w * gd[a][2];
      }
      float f[3] = {f01.x, f01.y, f2v};
      if (iK2) {
        float r0, r1, r2;
        if (NPE == 8 && bbar) {
          const float B1 = (1.0f / 3.0f) * (sd0[a][0] - gd[a][0]), B2 = gd[a][0] - B1;
          const float B3 = (1.0f / 3.0f) * (sd0[a][1] - gd[a][1]), B4 = gd[a][1] - B3;
          const float B5 = (1.0f / 3.0f) * (sd0[a][2] - gd[a][2]), B6 = gd[a][2] - B5;
          r0 = B2 * sig[0] + B1 * sig[1] + B1 * sig[2];
          r1 = B3 * sig[0] + B4 * sig[1] + B3 * sig[2];
          r2 = B5 * sig[0] + B5 * sig[1] + B6 * sig[2];
        } else {
          r0 = gd[a][0] * sig[0];
          r1 = gd[a][1] * sig[1];
          r2 = gd[a][2] * sig[2];
        }
        // (f0, f1) as a pair
        float2 t01 = __ffma2_rn(make_float2(gd[a][1], gd[a][0]), make_float2(sig[3], sig[3]), make_float2(r0, r1));
        t01 = __ffma2_rn(make_float2(gd[a][2], gd[a][2]), make_float2(sig[5], sig[4]), t01);
        const float2 n01 = __ffma2_rn(t01, make_float2(w, w), make_float2(f[0], f[1]));
        f[0] = n01.x; f[1] = n01.y;
        f[2] += (r2 + gd[a][1] * sig[4] + gd[a][0] * sig[5]) * w;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) kf[a][c] += f[c];
    }
  }
  const double mdt = -P.dt;
#pragma unroll
  for (int a = 0; a < NPE; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) k[a][c] = mdt * (double)kf[a][c];
  lam_el = (double)lam_int / (double)vol;
  reg_el = (double)reg / (double)GaussRule<NPE>::n;
}

}  // namespace fm
