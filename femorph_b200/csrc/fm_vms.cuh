// VMS tet4 element arithmetic (one thread = one element).
//
// Reference: src/femVMSExplicitFluidSolver.cpp.  The P1 structure is used to
// evaluate the reference's Gauss-point loops in closed form: the velocity
// gradient and the shape-function gradients are element constants, the
// weights are all V/4, and the Gauss-point shape values lN[g][a] are
// ALPHA on the diagonal and BETA elsewhere, so every sum over Gauss points of
// lN[g][a] * f_g equals BETA * sum_g f_g + (ALPHA - BETA) * f_a.  The result
// is the same algebraic expression as the reference; only the rounding order
// differs.
#pragma once
#include "fm_device.cuh"

namespace fm {

#define FM_VA 0.58541020
#define FM_VB 0.13819660
// Gauss-point projection coefficients (see vms_subscale_update):
// S = ALPHA + 3 BETA, FM_PR = BETA (S + ALPHA - BETA) / S,
// FM_PG1 = (ALPHA - BETA)^2 / S - 1.
#define FM_VS (FM_VA + 3.0 * FM_VB)
#define FM_PR (FM_VB * (FM_VS + (FM_VA - FM_VB)) / FM_VS)
#define FM_PG1 ((FM_VA - FM_VB) * (FM_VA - FM_VB) / FM_VS - 1.0)

// Element geometry: initial_assemble (src lines 21-91).  The cofactors and
// the determinant round each product individually, as the reference's
// uncontracted expressions do.  DN and V can still differ from the
// reference's in the last bit: 1/det comes from rcp_nr (within about one ulp
// of the correctly rounded 1.0 / detJ of src line 64) and V = det * (1/6)
// where the reference divides detJ / 6.0 (src line 73).
struct TetGeom {
  double DN[3][4];
  double V;
};

__device__ __forceinline__ void tet_geometry(const double X[4][3], TetGeom& g) {
  double j[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) j[i][k] = X[k + 1][i] - X[0][i];
  double c00 = __dsub_rn(__dmul_rn(j[1][1], j[2][2]), __dmul_rn(j[2][1], j[1][2]));
  double c01 = __dsub_rn(__dmul_rn(j[2][0], j[1][2]), __dmul_rn(j[1][0], j[2][2]));
  double c02 = __dsub_rn(__dmul_rn(j[1][0], j[2][1]), __dmul_rn(j[2][0], j[1][1]));
  double c10 = __dsub_rn(__dmul_rn(j[2][1], j[0][2]), __dmul_rn(j[0][1], j[2][2]));
  double c11 = __dsub_rn(__dmul_rn(j[0][0], j[2][2]), __dmul_rn(j[2][0], j[0][2]));
  double c12 = __dsub_rn(__dmul_rn(j[2][0], j[0][1]), __dmul_rn(j[0][0], j[2][1]));
  double c20 = __dsub_rn(__dmul_rn(j[0][1], j[1][2]), __dmul_rn(j[1][1], j[0][2]));
  double c21 = __dsub_rn(__dmul_rn(j[1][0], j[0][2]), __dmul_rn(j[0][0], j[1][2]));
  double c22 = __dsub_rn(__dmul_rn(j[0][0], j[1][1]), __dmul_rn(j[1][0], j[0][1]));
  double det = __dadd_rn(__dadd_rn(__dmul_rn(j[0][0], c00), __dmul_rn(j[0][1], c01)), __dmul_rn(j[0][2], c02));
  double id = rcp_nr(det);
  // invJac[i][k] = cof[k][i] / det ; DN[i][0] = -(inv[0][i]) - inv[1][i] - inv[2][i]
  double inv[3][3];
  inv[0][0] = __dmul_rn(c00, id); inv[0][1] = __dmul_rn(c10, id); inv[0][2] = __dmul_rn(c20, id);
  inv[1][0] = __dmul_rn(c01, id); inv[1][1] = __dmul_rn(c11, id); inv[1][2] = __dmul_rn(c21, id);
  inv[2][0] = __dmul_rn(c02, id); inv[2][1] = __dmul_rn(c12, id); inv[2][2] = __dmul_rn(c22, id);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    g.DN[i][0] = __dsub_rn(__dsub_rn(-inv[0][i], inv[1][i]), inv[2][i]);
    g.DN[i][1] = inv[0][i];
    g.DN[i][2] = inv[1][i];
    g.DN[i][3] = inv[2][i];
  }
  g.V = det * (1.0 / 6.0);
}

// Pending subscale update of the previous dual iteration:
// assemble_projRes_explicit (src lines 406-588) followed by
// update_subscales_explicit (src lines 593-646), with include_sg_p = false
// and the element-local projection (proj_res_at_nodes = false).
//   U   : nodal velocity after the dual update, before BCs (src line 1134)
//   pq  : pressures of the problem's nodes 0..3 (src line 489 reads
//         sol_n[i][3] with the local index i)
//   sdu : in = subscales at the 4 Gauss points, out = updated subscales
//   G, Us (out): velocity gradient and nodal velocity sum of U, which the
//         residual reuses when U equals the post-BC state (no BC node)
template <typename T>
__device__ __forceinline__ void vms_subscale_update(const TetGeom& geo, const T U[4][3], const T pq[4], T sdu[4][3],
                                                    T inv_dt, T c1nu, T c2, T ih, T G[3][3], T Us[3]) {
  const T Bt = (T)FM_VB, AB = (T)(FM_VA - FM_VB);
  T gp[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j)
      G[i][j] = (T)geo.DN[j][0] * U[0][i] + (T)geo.DN[j][1] * U[1][i] + (T)geo.DN[j][2] * U[2][i] +
                (T)geo.DN[j][3] * U[3][i];
    gp[i] = (T)geo.DN[i][0] * pq[0] + (T)geo.DN[i][1] * pq[1] + (T)geo.DN[i][2] * pq[2] + (T)geo.DN[i][3] * pq[3];
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) Us[i] = (U[0][i] + U[1][i]) + (U[2][i] + U[3][i]);
  T r[4][3];
  T maxa2 = (T)0;
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    T hah[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) hah[i] = Bt * Us[i] + AB * U[g][i] + sdu[g][i];
    T a2 = hah[0] * hah[0] + hah[1] * hah[1] + hah[2] * hah[2];
    maxa2 = a2 > maxa2 ? a2 : maxa2;
#pragma unroll
    for (int i = 0; i < 3; ++i) r[g][i] = G[i][0] * hah[0] + G[i][1] * hah[1] + G[i][2] * hah[2] + gp[i];
  }
  // Element-local L2 projection of r onto P1, P_a = sum_g lN[g][a] r_g / S
  // (S = sum_g lN[g][a] = ALPHA + 3 BETA), evaluated back at the Gauss
  // points: sum_a lN[g][a] P_a = BETA sum_a P_a + (ALPHA - BETA) P_g, and
  // sum_a P_a = R = sum_g r_g, so the projection at g is FM_PR R + FM_PG r_g.
  T tau_u_inv = c1nu * ih * ih + c2 * sqrt_nr(maxa2) * ih;
  T tau1 = rcp_nr(inv_dt + tau_u_inv);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const T R = (r[0][i] + r[1][i]) + (r[2][i] + r[3][i]);
    const T cR = (T)FM_PR * R;
#pragma unroll
    for (int g = 0; g < 4; ++g) sdu[g][i] = (sdu[g][i] * inv_dt + ((T)FM_PG1 * r[g][i] + cR)) * tau1;
  }
}

// Element residual: assemble_RHS (src lines 93-399) with hdu = U (current
// dual state after BCs), u_prev = Up (previous dual state), forcing 0
// (femNode::force is never set) and subgrid pressure 0 (include_sg_p =
// false).  Writes the 16 nodal residual entries lRes[a][0..3].
// G, Us: velocity gradient and nodal velocity sum of U when have_G (from the
// subscale update), else computed here.
template <typename T, bool HAS_PREV>
__device__ __forceinline__ void vms_residual(const TetGeom& geo, const T U[4][3], const T P[4], const T Up[4][3],
                                             const T sdu[4][3], T nu4, T inv_eps, T inv_dt, T G[3][3], T Us[3],
                                             bool have_G, double lRes[4][4]) {
  const T Bt = (T)FM_VB, AB = (T)(FM_VA - FM_VB);
  const T S = (T)FM_VA + (T)3 * Bt;
  if (!have_G) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
      for (int j = 0; j < 3; ++j)
        G[i][j] = (T)geo.DN[j][0] * U[0][i] + (T)geo.DN[j][1] * U[1][i] + (T)geo.DN[j][2] * U[2][i] +
                  (T)geo.DN[j][3] * U[3][i];
      Us[i] = (U[0][i] + U[1][i]) + (U[2][i] + U[3][i]);
    }
  }
  const T tr = (G[0][0] + G[1][1]) + G[2][2];
  T Ups[3];
  if (HAS_PREV) {
#pragma unroll
    for (int i = 0; i < 3; ++i) Ups[i] = (Up[0][i] + Up[1][i]) + (Up[2][i] + Up[3][i]);
  }
  const T Psum = (P[0] + P[1]) + (P[2] + P[3]);
  // X_g = (a_g . grad) u (+ acceleration); M2[i][k] = sum_g sdu_g[i] a_g[k]
  T X[4][3], M2[3][3], Ssdu[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    Ssdu[i] = (T)0;
#pragma unroll
    for (int k = 0; k < 3; ++k) M2[i][k] = (T)0;
  }
  T Hs = (T)0;
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    T ug[3], hah[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      ug[i] = Bt * Us[i] + AB * U[g][i];
      hah[i] = ug[i] + sdu[g][i];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      X[g][i] = G[i][0] * hah[0] + G[i][1] * hah[1] + G[i][2] * hah[2];
      if (HAS_PREV) {
        T upg = Bt * Ups[i] + AB * Up[g][i];
        X[g][i] += (ug[i] - upg) * inv_dt;
      }
      Ssdu[i] += sdu[g][i];
#pragma unroll
      for (int k = 0; k < 3; ++k) M2[i][k] += sdu[g][i] * hah[k];
    }
  }
  // sum_g (BETA Psum + (ALPHA - BETA) P_g) = S Psum
  Hs = S * Psum;
  // K'[i][k] = 4 nu G[i][k] - M2[i][k] - Hs delta_ik ; lRes[a][i] = V/4 (lumped terms + K'.DN)
  T Kp[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) Kp[i][k] = nu4 * G[i][k] - M2[i][k] - (i == k ? Hs : (T)0);
  const double w = geo.V * 0.25;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    T Xs = (X[0][i] + X[1][i]) + (X[2][i] + X[3][i]);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      T v = Bt * Xs + AB * X[a][i] + Kp[i][0] * (T)geo.DN[0][a] + Kp[i][1] * (T)geo.DN[1][a] +
            Kp[i][2] * (T)geo.DN[2][a];
      lRes[a][i] = w * (double)v;
    }
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    T v = tr * S - (Ssdu[0] * (T)geo.DN[0][a] + Ssdu[1] * (T)geo.DN[1][a] + Ssdu[2] * (T)geo.DN[2][a]);
    lRes[a][3] = w * (double)(inv_eps * v);
  }
}

// ---------------------------------------------------------------------------
// Mixed precision (FM_MIXED).  Gauss-point work in FP32; kept in FP64: the
// element volume (it weights the FP64 nodal accumulation), the Jacobian
// inverse of badly shaped elements (aspect ratio above FM_MIXED_ASPECT_LIMIT,
// flagged on the host), the pressure-gradient term, the nodal accumulation,
// the lumped-mass division and the state.  Nodal velocities enter FP32 as
// differences to the element's first node (formed in FP64), so the velocity
// gradient does not lose digits to cancellation.
// ---------------------------------------------------------------------------
struct TetGeomF {
  float DN[3][4];
  double V;
};

__device__ __forceinline__ void tet_geometry_mixed(const double X[4][3], bool precise, TetGeomF& g) {
  double j[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) j[i][k] = X[k + 1][i] - X[0][i];
  const double c00 = j[1][1] * j[2][2] - j[2][1] * j[1][2];
  const double c01 = j[2][0] * j[1][2] - j[1][0] * j[2][2];
  const double c02 = j[1][0] * j[2][1] - j[2][0] * j[1][1];
  const double det = j[0][0] * c00 + j[0][1] * c01 + j[0][2] * c02;
  g.V = det * (1.0 / 6.0);
  float inv[3][3];
  if (precise) {
    const double id = rcp_nr(det);
    const double c10 = j[2][1] * j[0][2] - j[0][1] * j[2][2];
    const double c11 = j[0][0] * j[2][2] - j[2][0] * j[0][2];
    const double c12 = j[2][0] * j[0][1] - j[0][0] * j[2][1];
    const double c20 = j[0][1] * j[1][2] - j[1][1] * j[0][2];
    const double c21 = j[1][0] * j[0][2] - j[0][0] * j[1][2];
    const double c22 = j[0][0] * j[1][1] - j[1][0] * j[0][1];
    inv[0][0] = (float)(c00 * id); inv[0][1] = (float)(c10 * id); inv[0][2] = (float)(c20 * id);
    inv[1][0] = (float)(c01 * id); inv[1][1] = (float)(c11 * id); inv[1][2] = (float)(c21 * id);
    inv[2][0] = (float)(c02 * id); inv[2][1] = (float)(c12 * id); inv[2][2] = (float)(c22 * id);
  } else {
    float f[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int k = 0; k < 3; ++k) f[i][k] = (float)j[i][k];
    const float d00 = f[1][1] * f[2][2] - f[2][1] * f[1][2];
    const float d01 = f[2][0] * f[1][2] - f[1][0] * f[2][2];
    const float d02 = f[1][0] * f[2][1] - f[2][0] * f[1][1];
    const float d10 = f[2][1] * f[0][2] - f[0][1] * f[2][2];
    const float d11 = f[0][0] * f[2][2] - f[2][0] * f[0][2];
    const float d12 = f[2][0] * f[0][1] - f[0][0] * f[2][1];
    const float d20 = f[0][1] * f[1][2] - f[1][1] * f[0][2];
    const float d21 = f[1][0] * f[0][2] - f[0][0] * f[1][2];
    const float d22 = f[0][0] * f[1][1] - f[1][0] * f[0][1];
    const float id = ptx_rcp_approx((float)det);
    inv[0][0] = d00 * id; inv[0][1] = d10 * id; inv[0][2] = d20 * id;
    inv[1][0] = d01 * id; inv[1][1] = d11 * id; inv[1][2] = d21 * id;
    inv[2][0] = d02 * id; inv[2][1] = d12 * id; inv[2][2] = d22 * id;
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    g.DN[i][0] = -inv[0][i] - inv[1][i] - inv[2][i];
    g.DN[i][1] = inv[0][i];
    g.DN[i][2] = inv[1][i];
    g.DN[i][3] = inv[2][i];
  }
}

// Subscale update, FP32.  U0: velocity of node 0; Ud[a] = U[a] - U0 (Ud[0] = 0);
// pqd[a] = pq[a] - pq[0].
// G, Ds (out): gradient and difference sum of Ud, reused by the residual
// when there is no BC node.
__device__ __forceinline__ void vms_subscale_update_mixed(const TetGeomF& geo, const float U0[3], const float Ud[4][3],
                                                          const float pqd[4], float sdu[4][3], float inv_dt, float c1nu,
                                                          float c2, float ih, float G[3][3], float Ds[3]) {
  const float A = (float)FM_VA, Bt = (float)FM_VB, AB = (float)(FM_VA - FM_VB);
  const float S = A + 3.0f * Bt;
  float gp[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) G[i][j] = geo.DN[j][1] * Ud[1][i] + geo.DN[j][2] * Ud[2][i] + geo.DN[j][3] * Ud[3][i];
    gp[i] = geo.DN[i][1] * pqd[1] + geo.DN[i][2] * pqd[2] + geo.DN[i][3] * pqd[3];
    Ds[i] = Ud[1][i] + Ud[2][i] + Ud[3][i];
  }
  float r[4][3];
  float maxa2 = 0.0f;
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    float hah[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) hah[i] = S * U0[i] + Bt * Ds[i] + AB * Ud[g][i] + sdu[g][i];
    const float a2 = hah[0] * hah[0] + hah[1] * hah[1] + hah[2] * hah[2];
    maxa2 = fmaxf(a2, maxa2);
#pragma unroll
    for (int i = 0; i < 3; ++i) r[g][i] = G[i][0] * hah[0] + G[i][1] * hah[1] + G[i][2] * hah[2] + gp[i];
  }
  const float tau1 = ptx_rcp_approx(inv_dt + c1nu * ih * ih + c2 * (maxa2 > 0.0f ? maxa2 * ptx_rsqrt_approx(maxa2) : 0.0f) * ih);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float R = (r[0][i] + r[1][i]) + (r[2][i] + r[3][i]);
    const float cR = (float)FM_PR * R;
#pragma unroll
    for (int g = 0; g < 4; ++g) sdu[g][i] = (sdu[g][i] * inv_dt + ((float)FM_PG1 * r[g][i] + cR)) * tau1;
  }
}

// Paired FP32 arithmetic (sm_100 FFMA2 / FADD2 / FMUL2: two IEEE FP32
// operations in one instruction): the residual works on two Gauss points or
// two nodes at a time (the mixed tile kernel 3% faster at 96^3; the sums
// round like the scalar ones up to the order of the fused products).
__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 f2s(float x) { return make_float2(x, x); }

// Element residual, FP32 Gauss-point work with FP64 output.  P: nodal
// pressures (FP64, the pressure-gradient term is formed in FP64); Dacc[a] =
// U[a] - Uprev[a] (only with HAS_PREV).
template <bool HAS_PREV>
__device__ __forceinline__ void vms_residual_mixed(const TetGeomF& geo, const float U0[3], const float Ud[4][3],
                                                   const double P[4], const float Dacc[4][3], const float sdu[4][3],
                                                   float nu4, float inv_eps, float inv_dt, float G[3][3], float Ds[3],
                                                   bool have_G, double lRes[4][4]) {
  const float A = (float)FM_VA, Bt = (float)FM_VB, AB = (float)(FM_VA - FM_VB);
  const float S = A + 3.0f * Bt;
  if (!have_G) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      // G[i][0..1] as one pair, G[i][2] alone
      float2 g01 = __fmul2_rn(f2(geo.DN[0][1], geo.DN[1][1]), f2s(Ud[1][i]));
      g01 = __ffma2_rn(f2(geo.DN[0][2], geo.DN[1][2]), f2s(Ud[2][i]), g01);
      g01 = __ffma2_rn(f2(geo.DN[0][3], geo.DN[1][3]), f2s(Ud[3][i]), g01);
      G[i][0] = g01.x; G[i][1] = g01.y;
      G[i][2] = geo.DN[2][1] * Ud[1][i] + geo.DN[2][2] * Ud[2][i] + geo.DN[2][3] * Ud[3][i];
      Ds[i] = Ud[1][i] + Ud[2][i] + Ud[3][i];
    }
  }
  const float tr = (G[0][0] + G[1][1]) + G[2][2];
  float2 X2[2][3];   // X2[h][i] = (X[2h][i], X[2h+1][i])
  float2 M01[3];     // (M2[i][0], M2[i][1])
  float M2z[3], Ssdu[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    Ssdu[i] = 0.0f;
    M01[i] = f2s(0.0f);
    M2z[i] = 0.0f;
  }
  float Dsum[3];
  if (HAS_PREV) {
#pragma unroll
    for (int i = 0; i < 3; ++i) Dsum[i] = (Dacc[0][i] + Dacc[1][i]) + (Dacc[2][i] + Dacc[3][i]);
  }
  float base[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) base[i] = S * U0[i] + Bt * Ds[i];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    // Gauss points 2h and 2h+1 side by side
    float2 hah[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
      hah[i] = __fadd2_rn(__ffma2_rn(f2s(AB), f2(Ud[2 * h][i], Ud[2 * h + 1][i]), f2s(base[i])),
                          f2(sdu[2 * h][i], sdu[2 * h + 1][i]));
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float2 x = __fmul2_rn(f2s(G[i][0]), hah[0]);
      x = __ffma2_rn(f2s(G[i][1]), hah[1], x);
      x = __ffma2_rn(f2s(G[i][2]), hah[2], x);
      if (HAS_PREV) {
        const float2 d = __ffma2_rn(f2s(AB), f2(Dacc[2 * h][i], Dacc[2 * h + 1][i]), f2s(Bt * Dsum[i]));
        x = __ffma2_rn(d, f2s(inv_dt), x);
      }
      X2[h][i] = x;
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int g = 2 * h + q;
      const float hk0 = q ? hah[0].y : hah[0].x, hk1 = q ? hah[1].y : hah[1].x, hk2 = q ? hah[2].y : hah[2].x;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        Ssdu[i] += sdu[g][i];
        M01[i] = __ffma2_rn(f2s(sdu[g][i]), f2(hk0, hk1), M01[i]);
        M2z[i] += sdu[g][i] * hk2;
      }
    }
  }
  float Kp[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    Kp[i][0] = nu4 * G[i][0] - M01[i].x;
    Kp[i][1] = nu4 * G[i][1] - M01[i].y;
    Kp[i][2] = nu4 * G[i][2] - M2z[i];
  }
  const double w = geo.V * 0.25;
  const double Hs = (double)S * ((P[0] + P[1]) + (P[2] + P[3]));
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float Xs = (X2[0][i].x + X2[0][i].y) + (X2[1][i].x + X2[1][i].y);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      // nodes 2h and 2h+1
      float2 v = __ffma2_rn(f2s(AB), X2[h][i], f2s(Bt * Xs));
      v = __ffma2_rn(f2s(Kp[i][0]), f2(geo.DN[0][2 * h], geo.DN[0][2 * h + 1]), v);
      v = __ffma2_rn(f2s(Kp[i][1]), f2(geo.DN[1][2 * h], geo.DN[1][2 * h + 1]), v);
      v = __ffma2_rn(f2s(Kp[i][2]), f2(geo.DN[2][2 * h], geo.DN[2][2 * h + 1]), v);
      lRes[2 * h][i] = w * ((double)v.x - Hs * (double)geo.DN[i][2 * h]);
      lRes[2 * h + 1][i] = w * ((double)v.y - Hs * (double)geo.DN[i][2 * h + 1]);
    }
  }
  const float trS = tr * S;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    float2 s = __fmul2_rn(f2s(Ssdu[0]), f2(geo.DN[0][2 * h], geo.DN[0][2 * h + 1]));
    s = __ffma2_rn(f2s(Ssdu[1]), f2(geo.DN[1][2 * h], geo.DN[1][2 * h + 1]), s);
    s = __ffma2_rn(f2s(Ssdu[2]), f2(geo.DN[2][2 * h], geo.DN[2][2 * h + 1]), s);
    const float2 v = __fmul2_rn(f2s(inv_eps), __fadd2_rn(f2s(trS), make_float2(-s.x, -s.y)));
    lRes[2 * h][3] = w * (double)v.x;
    lRes[2 * h + 1][3] = w * (double)v.y;
  }
}

}  // namespace fm
