// SUPG explicit step kernels (tet4 and hexa8): supg_tile_kernel +
// supg_iface_kernel per time step, and the output-only pressure pass.
//
// Same tile scheme as the VMS kernels: nodes staged in shared memory,
// element forces added colour by colour (fixed order, no atomics), interior
// nodes updated in place, interface nodes through per-tile partials.
// Node update (src lines 1509-1521): u^{n+1} = u^n + (1/l_M) acc with
// acc = sum of -dt K u_e (forward Euler, or 1.5 k^n - 0.5 k^{n-1} for AB2
// after the first step), then setNodeVelocity and setDirichletBC.  Global
// fixed dofs (src lines 1527-1561) are applied on read: the stored state
// keeps the values compute_pressure sees (it runs before the zeroing).
#include <cuda_runtime.h>

#include "fm_device.cuh"
#include "fm_supg.cuh"

namespace fm {

template <int NPE>
__global__ void supg_stats_kernel(DevBatch B, int tile0, int tn_max, double* out);

__device__ __forceinline__ void mask_fixed(int gf, double& u, double& v, double& w) {
  if (gf & FM_FIX_X) u = 0.0;
  if (gf & FM_FIX_Y) v = 0.0;
  if (gf & FM_FIX_Z) w = 0.0;
}

__device__ __forceinline__ void supg_node_update(const DevBatch& B, const DevProb& P, double time, int64_t g,
                                                 const double old[3], const double acc[3], int32_t* status,
                                                 double* max_u2) {
  const double im = 1.0 / B.mass[g];
  double s[4] = {old[0] + im * acc[0], old[1] + im * acc[1], old[2] + im * acc[2], 0.0};
  const int32_t rec = B.node_bc[g];
  if (rec >= 0) apply_bc(B, rec, time, s, status);
  B.su[g] = s[0];
  B.sv[g] = s[1];
  B.sw[g] = s[2];
  mask_fixed(P.glob_fixed, s[0], s[1], s[2]);
  const double u2 = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
  if (!isfinite(u2)) *status = FM_ERR_DIVERGED;
  if (u2 > *max_u2) *max_u2 = u2;
}

// get_solution_extrema + EXITCOND (src lines 1594-1643): max |u| above the
// threshold stops the solve.
__device__ __forceinline__ void check_exit(const DevBatch& B, const DevProb& P, int pidx, double max_u2, int32_t status) {
  if (P.exit_cond > 0.0 && sqrt(max_u2) > P.exit_cond) status = FM_ERR_DIVERGED;
  if (status != FM_OK) B.pstate[pidx].status = status;
}

// MIXED: Gauss-point work in FP32 (supg_element_mixed).  All 128-thread
// kernels are held to 168 registers a thread so that three CTAs fit an SM
// (FP64 tet4: a small spill, 12% faster than two CTAs at 241 registers;
// FP64 hexa8 with the stored geometry: ~500 bytes of spill, faster than two
// CTAs at 255 registers, while forming the geometry in the kernel it spilled
// 1 KB at three CTAs and ran 30% slower; mixed hexa8 with the stored
// geometry: no spill, and 2% faster than four CTAs at 128 registers).
//
// Accumulation of the element contributions into the tile's nodes, in the
// order of the elements (colour-sorted) in both schemes, so both give the
// same sums:
//  - tet4 (GATHER): element threads write their 12 entries to shared memory,
//    then each node's owner thread adds the entries of this chunk's elements
//    from the node's incidence list (two barriers a chunk; the one that
//    frees the staged entries sits after the next chunk's element work);
//  - hexa8: one round per colour present in the chunk (elements of one
//    colour share no node), a barrier after each; the 24 entries a hexa
//    would stage cost more shared memory than the barriers cost time.
//
// The hexa8 kernels (GEO) read each Gauss point's inverse Jacobian and det J
// from the geometry stored at placement (supg_geo_kernel; FP64, or rounded
// to FP32 for the mixed form) instead of forming them from the staged
// coordinates at every step, and stage no coordinates.
template <int NPE, int THREADS, bool MIXED>
__global__ void __launch_bounds__(THREADS, THREADS == 128 ? 3 : 1)
    supg_tile_kernel(DevBatch B, int tn_max, int inc_max) {
  constexpr bool GATHER = NPE == 4;
  constexpr bool GEO = NPE == 8;
  extern __shared__ double sm[];
  double* s_x = sm;
  double* s_y = s_x + tn_max;
  double* s_z = s_y + tn_max;
  double* s_u = s_z + tn_max;
  double* s_v = s_u + tn_max;
  double* s_w = s_v + tn_max;
  double* s_a0 = s_w + tn_max;
  double* s_a1 = s_a0 + tn_max;
  double* s_a2 = s_a1 + tn_max;
  double* R = s_a2 + tn_max;                                        // GATHER: [NPE * 3][THREADS]
  int32_t* s_col = (int32_t*)(R + (GATHER ? NPE * 3 * THREADS : 0));  // colour offsets (<= 129)
  uint16_t* s_inc = (uint16_t*)(s_col + 130);                      // GATHER: incidence entries
  uint16_t* s_off = s_inc + (GATHER ? inc_max : 0);                // GATHER: per-node offsets
  uint16_t* s_cur = s_off + (GATHER ? tn_max + 1 : 0);             // GATHER: per-node cursors
  __shared__ ShapeTable<NPE, double> s_shape;
  __shared__ ShapeTable<NPE, float> s_shape_f;

  const TileMeta tm = B.tiles[blockIdx.x];
  const int pidx = tm.problem;
  if (pidx < 0) return;  // free tile slot
  const DevProbState st = B.pstate[pidx];
  if (st.iter >= B.target[pidx] || st.status != FM_OK) return;
  const DevProb& P = B.probs[pidx];
  const bool euler = (P.ex_mask & 1) || st.iter == 0;
  const bool ab2 = !(P.ex_mask & 1);
  const int tid = threadIdx.x;
  for (int ln = tid; ln < tm.n_node; ln += THREADS) {
    const int g = B.tile_nodes[tm.node_begin + ln];
    if (!GEO) {
      s_x[ln] = B.x[g]; s_y[ln] = B.y[g]; s_z[ln] = B.z[g];
    }
    double u = B.su[g], v = B.sv[g], w = B.sw[g];
    mask_fixed(P.glob_fixed, u, v, w);
    s_u[ln] = u; s_v[ln] = v; s_w[ln] = w;
    s_a0[ln] = 0.0; s_a1[ln] = 0.0; s_a2[ln] = 0.0;
  }
  for (int c = tid; c <= tm.n_col; c += THREADS) s_col[c] = B.tile_cols[tm.col_begin + c];
  if (GATHER) {
    for (int i = tid; i <= tm.n_node; i += THREADS) {
      const uint16_t o = B.tile_off[tm.off_begin + i];
      s_off[i] = o;
      if (i < tm.n_node) s_cur[i] = o;
    }
    const int ninc = tm.n_elem * NPE;
    for (int i = tid; i < ninc; i += THREADS) s_inc[i] = B.tile_inc[tm.inc_begin + i];
  }
  fill_shape_table<NPE, double>(&s_shape);
  if (MIXED) fill_shape_table<NPE, float>(&s_shape_f);
  __syncthreads();
  const int64_t E = B.E;
  // one lane asks L2 for a later tile's connectivity, incidence entries, AB2
  // history rows and interior-node ranges (see vms_tile_kernel)
  if (B.l2_ahead > 0 && tid == THREADS - 32 && blockIdx.x + B.l2_ahead < (unsigned)B.n_tiles) {
    const TileMeta tn = B.tiles[blockIdx.x + B.l2_ahead];
    if (tn.problem >= 0 && tn.n_elem > 0) {
      const int64_t e0 = tn.elem_begin;  // multiple of 32 slots: 16-byte aligned rows
      const uint32_t cb = ((uint32_t)tn.n_elem * NPE * 2u + 15u) & ~15u;
      bulk_prefetch_l2(B.conn + e0 * NPE, cb);
      if (GATHER) bulk_prefetch_l2(B.tile_inc + tn.inc_begin, cb);
      if (B.sdus) {
#pragma unroll 1
        for (int q = 0; q < 3 * NPE; ++q) bulk_prefetch_l2(B.sdus + (int64_t)q * E + e0, ((uint32_t)tn.n_elem * 8u + 15u) & ~15u);
      }
      if (tn.n_int > 0 && tn.node0 >= 0) {
        const int64_t g0 = tn.node0 & ~1, g1 = ((int64_t)tn.node0 + tn.n_int + 1) & ~1ll;
        const uint32_t nb = (uint32_t)(g1 - g0) * 8u;
        if (!GEO) {
          bulk_prefetch_l2(B.x + g0, nb); bulk_prefetch_l2(B.y + g0, nb); bulk_prefetch_l2(B.z + g0, nb);
        }
        bulk_prefetch_l2(B.su + g0, nb); bulk_prefetch_l2(B.sv + g0, nb); bulk_prefetch_l2(B.sw + g0, nb);
        bulk_prefetch_l2(B.mass + g0, nb);
        const int64_t h0 = tn.node0 & ~3, h1 = ((int64_t)tn.node0 + tn.n_int + 3) & ~3ll;
        bulk_prefetch_l2(B.node_bc + h0, (uint32_t)(h1 - h0) * 4u);
      }
    }
  }
  int c_lo = 0;
  for (int base = 0; base < tm.n_elem; base += THREADS) {
    const int le = base + tid;
    const bool active = le < tm.n_elem;
    double k[NPE][3];
    int ln[NPE];
    if (active) {
      const int64_t e = tm.elem_begin + le;
      if (NPE == 4) {
        const uint2 cw = __ldg(reinterpret_cast<const uint2*>(B.conn) + e);
        ln[0] = cw.x & 0xffff; ln[1] = cw.x >> 16; ln[2] = cw.y & 0xffff; ln[3] = cw.y >> 16;
      } else {
        const uint4 cw = __ldg(reinterpret_cast<const uint4*>(B.conn) + e);
        ln[0] = cw.x & 0xffff; ln[1] = cw.x >> 16; ln[2] = cw.y & 0xffff; ln[3] = cw.y >> 16;
        ln[4 % NPE] = cw.z & 0xffff; ln[5 % NPE] = cw.z >> 16; ln[6 % NPE] = cw.w & 0xffff; ln[7 % NPE] = cw.w >> 16;
      }
      double lam, reg;
      if constexpr (MIXED) {
        // bit 15 of the first id flags an element whose Jacobian stays FP64
        const bool precise = (ln[0] & 0x8000) != 0;
        ln[0] &= 0x7fff;
        float Xr[NPE][3], U0[3], Ud[NPE][3];
        const double u0 = s_u[ln[0]], v0 = s_v[ln[0]], w0 = s_w[ln[0]];
        U0[0] = (float)u0; U0[1] = (float)v0; U0[2] = (float)w0;
        if (!GEO) {
          const double x0 = s_x[ln[0]], y0 = s_y[ln[0]], z0 = s_z[ln[0]];
#pragma unroll
          for (int a = 0; a < NPE; ++a) {
            Xr[a][0] = (float)(s_x[ln[a]] - x0); Xr[a][1] = (float)(s_y[ln[a]] - y0);
            Xr[a][2] = (float)(s_z[ln[a]] - z0);
          }
        }
#pragma unroll
        for (int a = 0; a < NPE; ++a) {
          Ud[a][0] = (float)(s_u[ln[a]] - u0); Ud[a][1] = (float)(s_v[ln[a]] - v0); Ud[a][2] = (float)(s_w[ln[a]] - w0);
        }
        supg_element_mixed<NPE, GEO>(P, s_shape_f, s_shape, Xr, U0, Ud, precise, s_x, s_y, s_z, ln, k, lam, reg,
                                     GEO ? B.geo32 + e : nullptr, E);
      } else {
        supg_element<NPE, GEO>(P, s_shape, s_x, s_y, s_z, s_u, s_v, s_w, ln, k, lam, reg, GEO ? B.geo + e : nullptr, E);
      }
      B.el_lam[e] = lam;
      B.el_reg[e] = reg;
      if (ab2) {
#pragma unroll
        for (int a = 0; a < NPE; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            double* h = B.sdus + (int64_t)(a * 3 + c) * E + e;
            const double kp = k[a][c];
            if (!euler) k[a][c] = (3.0 / 2.0) * kp - (1.0 / 2.0) * __ldcs(h);
            __stcs(h, kp);
          }
      }
    }
    if constexpr (GATHER) {
      // the barrier that frees R (owners of the previous chunk done) comes
      // after this chunk's element work, not at the end of the accumulation
      if (base > 0) __syncthreads();
      if (active) {
#pragma unroll
        for (int a = 0; a < NPE; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c) R[(a * 3 + c) * THREADS + tid] = k[a][c];
      }
      __syncthreads();
      // owners add this chunk's entries to their nodes, in element order
      for (int n = tid; n < tm.n_node; n += THREADS) {
        int c = s_cur[n];
        const int ce = s_off[n + 1];
        if (c >= ce) continue;
        double a0 = s_a0[n], a1 = s_a1[n], a2 = s_a2[n];
        while (c < ce) {
          const int ent = s_inc[c];
          const int col = ent / NPE - base;
          if (col >= THREADS) break;
          const double* Rp = R + (ent % NPE) * 3 * THREADS + col;
          a0 += Rp[0];
          a1 += Rp[THREADS];
          a2 += Rp[2 * THREADS];
          ++c;
        }
        s_cur[n] = (uint16_t)c;
        s_a0[n] = a0; s_a1[n] = a1; s_a2[n] = a2;
      }
    } else {
      while (c_lo < tm.n_col && s_col[c_lo + 1] <= base) ++c_lo;
      for (int c = c_lo; c < tm.n_col && s_col[c] < base + THREADS; ++c) {
        if (active && le >= s_col[c] && le < s_col[c + 1]) {
#pragma unroll
          for (int a = 0; a < NPE; ++a) {
            s_a0[ln[a]] += k[a][0];
            s_a1[ln[a]] += k[a][1];
            s_a2[ln[a]] += k[a][2];
          }
        }
        __syncthreads();
      }
    }
  }
  __syncthreads();
  int32_t status = FM_OK;
  double max_u2 = 0.0;
  for (int l2 = tid; l2 < tm.n_node; l2 += THREADS) {
    const double acc[3] = {s_a0[l2], s_a1[l2], s_a2[l2]};
    if (l2 < tm.n_int) {
      const int g = B.tile_nodes[tm.node_begin + l2];
      const double old[3] = {s_u[l2], s_v[l2], s_w[l2]};
      supg_node_update(B, P, st.time, g, old, acc, &status, &max_u2);
    } else {
      const int s = tm.slot_base + (l2 - tm.n_int);
      B.part[2 * s] = make_double2(acc[0], acc[1]);
      B.part[2 * s + 1] = make_double2(acc[2], 0.0);
    }
  }
  check_exit(B, P, pidx, max_u2, status);
}

// Stored Gauss-point geometry of the hexa8 tiles [tile0, tile0 + gridDim.x)
// (geo_at's layout): the tile's coordinates staged in shared memory, then per
// element and Gauss point the Jacobian inverse and determinant by
// jacobian_at over the same shape table the element loop reads, stored in
// FP64 (B.geo) or rounded to FP32 (B.geo32, mixed form).  Run once when a
// problem is placed in a batch.
__global__ void supg_geo_kernel(DevBatch B, int tile0) {
  extern __shared__ double sm[];
  __shared__ ShapeTable<8, double> s_shape;
  const TileMeta tm = B.tiles[tile0 + blockIdx.x];
  if (tm.problem < 0) return;
  double* s_x = sm;
  double* s_y = s_x + tm.n_node;
  double* s_z = s_y + tm.n_node;
  for (int ln = threadIdx.x; ln < tm.n_node; ln += blockDim.x) {
    const int g = B.tile_nodes[tm.node_begin + ln];
    s_x[ln] = B.x[g]; s_y[ln] = B.y[g]; s_z[ln] = B.z[g];
  }
  fill_shape_table<8, double>(&s_shape);
  __syncthreads();
  const int64_t E = B.E;
  for (int le = threadIdx.x; le < tm.n_elem; le += blockDim.x) {
    const int64_t e = tm.elem_begin + le;
    const uint4 cw = __ldg(reinterpret_cast<const uint4*>(B.conn) + e);
    // bit 15 of the first id is the mixed form's FP64-Jacobian flag
    const int ln[8] = {(int)(cw.x & 0x7fff), (int)(cw.x >> 16), (int)(cw.y & 0xffff), (int)(cw.y >> 16),
                       (int)(cw.z & 0xffff), (int)(cw.z >> 16), (int)(cw.w & 0xffff), (int)(cw.w >> 16)};
#pragma unroll 1
    for (int g = 0; g < 8; ++g) {
      double inv[3][3];
      const double det = jacobian_at<8>([&](int n, int c) { return s_shape.dN[g][n][c]; }, s_x, s_y, s_z, ln, inv);
      const int64_t q0 = (int64_t)g * FM_GEO_PER_GP * E + e;
      if (B.geo) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b) B.geo[q0 + (a * 3 + b) * E] = inv[a][b];
        B.geo[q0 + 9 * E] = det;
      }
      if (B.geo32) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int b = 0; b < 3; ++b) B.geo32[q0 + (a * 3 + b) * E] = (float)inv[a][b];
        B.geo32[q0 + 9 * E] = (float)det;
      }
    }
  }
}

__global__ void supg_iface_kernel(DevBatch B) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B.n_iface; i += gridDim.x * blockDim.x) {
    // entry fields load together with the problem id (see vms_iface_kernel)
    const int pidx = B.iface_prob[i];
    const int g = B.iface_node[i];
    const int k0 = B.iface_slot_beg[i], k1 = k0 + B.iface_slot_cnt[i];
    if (pidx < 0) continue;  // free interface entry
    // partials loaded before the state check (see vms_iface_kernel); the
    // fourth component is not used
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    sum_partials(B, k0, k1, acc);
    const DevProbState st = B.pstate[pidx];
    if (st.iter >= B.target[pidx] || st.status != FM_OK) continue;
    const DevProb& P = B.probs[pidx];
    double old[3] = {B.su[g], B.sv[g], B.sw[g]};
    mask_fixed(P.glob_fixed, old[0], old[1], old[2]);
    int32_t status = FM_OK;
    double max_u2 = 0.0;
    supg_node_update(B, P, st.time, g, old, acc, &status, &max_u2);
    check_exit(B, P, pidx, max_u2, status);
  }
  finish_iteration(B);
}

// Partition parts: the interface pass in two halves around the exchange
// (see vms_xpack_kernel / vms_xupdate_kernel).
__global__ void supg_xpack_kernel(DevBatch B) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B.n_iface; i += gridDim.x * blockDim.x) {
    const int pidx = B.iface_prob[i];
    if (pidx < 0) continue;
    const DevProbState st = B.pstate[pidx];
    if (st.iter >= B.target[pidx] || st.status != FM_OK) continue;
    const DevProb& P = B.probs[pidx];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};  // the fourth component is not used
    sum_partials(B, B.iface_slot_beg[i], B.iface_slot_beg[i] + B.iface_slot_cnt[i], acc);
    const int xi = B.iface_xidx[i];
    if (xi >= 0) {
      double* d = B.xsend + ((int64_t)P.xslice * B.x_n + xi) * 4;
      d[0] = acc[0]; d[1] = acc[1]; d[2] = acc[2]; d[3] = 0.0;
      continue;
    }
    const int g = B.iface_node[i];
    double old[3] = {B.su[g], B.sv[g], B.sw[g]};
    mask_fixed(P.glob_fixed, old[0], old[1], old[2]);
    int32_t status = FM_OK;
    double max_u2 = 0.0;
    supg_node_update(B, P, st.time, g, old, acc, &status, &max_u2);
    check_exit(B, P, pidx, max_u2, status);
  }
}

__global__ void supg_xupdate_kernel(DevBatch B) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < B.n_xentries; j += gridDim.x * blockDim.x) {
    const int i = B.x_entries[j];
    const int pidx = B.iface_prob[i];
    if (pidx < 0) continue;
    const DevProbState st = B.pstate[pidx];
    if (st.iter >= B.target[pidx] || st.status != FM_OK) continue;
    const DevProb& P = B.probs[pidx];
    const int xi = B.iface_xidx[i];
    const double acc[3] = {exchange_sum(B, xi, 0), exchange_sum(B, xi, 1), exchange_sum(B, xi, 2)};
    const int g = B.iface_node[i];
    double old[3] = {B.su[g], B.sv[g], B.sw[g]};
    mask_fixed(P.glob_fixed, old[0], old[1], old[2]);
    int32_t status = FM_OK;
    double max_u2 = 0.0;
    supg_node_update(B, P, st.time, g, old, acc, &status, &max_u2);
    check_exit(B, P, pidx, max_u2, status);
  }
  finish_iteration(B);
}

// compute_pressure (src lines 446-501): p_e = -lambda_e * (int div u) / (int 1),
// on the stored (pre-zeroing) state.  Output only.
template <int NPE>
__global__ void supg_pressure_kernel(DevBatch B, int tn_max, double* pres) {
  extern __shared__ double sm[];
  double* s_x = sm;
  double* s_y = s_x + tn_max;
  double* s_z = s_y + tn_max;
  double* s_u = s_z + tn_max;
  double* s_v = s_u + tn_max;
  double* s_w = s_v + tn_max;
  const TileMeta tm = B.tiles[blockIdx.x];
  if (tm.problem < 0) return;  // free tile slot
  for (int ln = threadIdx.x; ln < tm.n_node; ln += blockDim.x) {
    const int g = B.tile_nodes[tm.node_begin + ln];
    s_x[ln] = B.x[g]; s_y[ln] = B.y[g]; s_z[ln] = B.z[g];
    s_u[ln] = B.su[g]; s_v[ln] = B.sv[g]; s_w[ln] = B.sw[g];
  }
  __syncthreads();
  for (int le = threadIdx.x; le < tm.n_elem; le += blockDim.x) {
    const int64_t e = tm.elem_begin + le;
    int ln[NPE];
    for (int a = 0; a < NPE; ++a) ln[a] = B.conn[e * NPE + a] & 0x7fff;  // bit 15: mixed-form flag
    double num = 0.0, den = 0.0;
    for (int g = 0; g < GaussRule<NPE>::n; ++g) {
      double q[3], Nf[NPE], dN[NPE][3], inv[3][3];
      GaussRule<NPE>::point(g, q);
      shape<NPE>(q, Nf, dN);
      const double det = jacobian<NPE>(dN, s_x, s_y, s_z, ln, inv);
      double div = 0.0;
      for (int a = 0; a < NPE; ++a) {
        const double ua[3] = {s_u[ln[a]], s_v[ln[a]], s_w[ln[a]]};
        for (int c = 0; c < 3; ++c)
          div += (inv[c][0] * dN[a][0] + inv[c][1] * dN[a][1] + inv[c][2] * dN[a][2]) * ua[c];
      }
      num += div * det * GaussRule<NPE>::weight();
      den += det * GaussRule<NPE>::weight();
    }
    pres[e] = -B.el_lam[e] * (num / den);
  }
}

size_t supg_smem_bytes(int tn_max, int inc_max, int npe, int threads) {
  const bool gather = npe == 4;
  return (size_t)tn_max * 9 * sizeof(double) + (gather ? (size_t)npe * 3 * threads * sizeof(double) : 0) +
         130 * sizeof(int32_t) + (gather ? ((size_t)inc_max + 2 * (size_t)tn_max + 1) * sizeof(uint16_t) : 0);
}

// Sets kernel k's dynamic shared-memory limit to the device's opt-in
// maximum less the kernel's static shared memory.
template <typename K>
static cudaError_t raise_dyn_smem(K k, int optin) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, k);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

// Raises the kernels' dynamic shared-memory limit to the device's opt-in
// maximum (the attribute is per kernel and process-wide, so a batch with
// small tiles must not lower it below what another batch launches with; the
// shared-memory carve-out still follows each launch's actual size).
cudaError_t supg_configure(size_t smem, int npe) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  (void)smem;  // checked against the limit by the caller
  if (npe == 4) {
    e = raise_dyn_smem(supg_tile_kernel<4, 128, false>, optin);
    if (e == cudaSuccess) e = raise_dyn_smem(supg_tile_kernel<4, 256, false>, optin);
    if (e == cudaSuccess) e = raise_dyn_smem(supg_tile_kernel<4, 128, true>, optin);
    if (e == cudaSuccess) e = raise_dyn_smem(supg_tile_kernel<4, 256, true>, optin);
    if (e == cudaSuccess) e = raise_dyn_smem(supg_pressure_kernel<4>, optin);
    if (e == cudaSuccess) e = raise_dyn_smem(supg_stats_kernel<4>, optin);
  } else {
    e = raise_dyn_smem(supg_geo_kernel, optin);
    if (e == cudaSuccess) e = raise_dyn_smem(supg_tile_kernel<8, 128, false>, optin);
    if (e == cudaSuccess) e = raise_dyn_smem(supg_tile_kernel<8, 256, false>, optin);
    if (e == cudaSuccess) e = raise_dyn_smem(supg_tile_kernel<8, 128, true>, optin);
    if (e == cudaSuccess) e = raise_dyn_smem(supg_tile_kernel<8, 256, true>, optin);
    if (e == cudaSuccess) e = raise_dyn_smem(supg_pressure_kernel<8>, optin);
    if (e == cudaSuccess) e = raise_dyn_smem(supg_stats_kernel<8>, optin);
  }
  return e;
}

template <int NPE, bool MIXED>
static void launch_supg_tile(const DevBatch& B, int tn_max, int inc_max, int threads, size_t smem, cudaStream_t s) {
  if (threads == 256)
    supg_tile_kernel<NPE, 256, MIXED><<<B.n_tiles, 256, smem, s>>>(B, tn_max, inc_max);
  else
    supg_tile_kernel<NPE, 128, MIXED><<<B.n_tiles, 128, smem, s>>>(B, tn_max, inc_max);
}

cudaError_t launch_supg_step(const DevBatch& B, int tn_max, int inc_max, int threads, int iface_blocks, int npe,
                             bool mixed, bool xpack, cudaStream_t s, cudaEvent_t* ev) {
  const size_t smem = supg_smem_bytes(tn_max, inc_max, npe, threads);
  if (ev) cudaEventRecord(ev[0], s);
  if (npe == 4) {
    if (mixed) launch_supg_tile<4, true>(B, tn_max, inc_max, threads, smem, s);
    else launch_supg_tile<4, false>(B, tn_max, inc_max, threads, smem, s);
  } else {
    if (mixed) launch_supg_tile<8, true>(B, tn_max, inc_max, threads, smem, s);
    else launch_supg_tile<8, false>(B, tn_max, inc_max, threads, smem, s);
  }
  if (ev) cudaEventRecord(ev[1], s);
  if (xpack)
    supg_xpack_kernel<<<iface_blocks, 256, 0, s>>>(B);
  else
    supg_iface_kernel<<<iface_blocks, 256, 0, s>>>(B);
  if (ev) cudaEventRecord(ev[2], s);
  return cudaGetLastError();
}

cudaError_t launch_supg_geo(const DevBatch& B, int tile0, int ntiles, int tn_max, cudaStream_t s) {
  if (ntiles <= 0) return cudaSuccess;
  supg_geo_kernel<<<ntiles, 128, (size_t)tn_max * 3 * sizeof(double), s>>>(B, tile0);
  return cudaGetLastError();
}

cudaError_t launch_supg_xupdate(const DevBatch& B, int blocks, cudaStream_t s) {
  supg_xupdate_kernel<<<blocks, 256, 0, s>>>(B);
  return cudaGetLastError();
}

cudaError_t launch_supg_pressure(const DevBatch& B, int tn_max, int npe, double* pres, cudaStream_t s) {
  const size_t smem = (size_t)tn_max * 6 * sizeof(double);
  if (npe == 4)
    supg_pressure_kernel<4><<<B.n_tiles, 128, smem, s>>>(B, tn_max, pres);
  else
    supg_pressure_kernel<8><<<B.n_tiles, 128, smem, s>>>(B, tn_max, pres);
  return cudaGetLastError();
}

}  // namespace fm

namespace fm {

// ---------------------------------------------------------------------------
// Per-step log quantities of the SUPG solver (output only).
//
// supg_stats_kernel: one CTA per tile of one problem, on the state about to
// be stepped (the one the reference's element loop sees): per Gauss point
// tau_SUPG (eval_stabilization), lambda (eval_bulk_modulus), the element
// length 2 sqrt(u^T G^-1 u) / |u| (get_el_lengths_from_G, src lines 756-790;
// NaN for u = 0 as there) and the advective |u_x| dt / l, viscous
// 2 nu dt / l^2 and lambda 2 lambda dt / l^2 CFL numbers; per element E and
// nu of the volume-averaged lambda (src lines 1180-1245, 1430-1459).  A value
// enters a minimum or maximum only by a strict comparison, as in the
// reference, so NaNs never do.  Each CTA writes its 11 partial results:
// min/max tau, min/max lambda, max viscous / advective / lambda CFL,
// min/max E, min/max nu.
//
// velocity_extrema_kernel: min/max of each velocity component and max |u|
// over one problem's nodes (get_solution_extrema, src lines 604-655), global
// fixed dofs masked; each CTA writes 7 partial results.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void upd_min(double& m, double v) { if (v < m) m = v; }
__device__ __forceinline__ void upd_max(double& m, double v) { if (v > m) m = v; }

template <int NPE>
__global__ void supg_stats_kernel(DevBatch B, int tile0, int tn_max, double* out) {
  extern __shared__ double sm[];
  double* s_x = sm;
  double* s_y = s_x + tn_max;
  double* s_z = s_y + tn_max;
  double* s_u = s_z + tn_max;
  double* s_v = s_u + tn_max;
  double* s_w = s_v + tn_max;
  __shared__ double s_red[11][32];
  const TileMeta tm = B.tiles[tile0 + blockIdx.x];
  const DevProb& P = B.probs[tm.problem];
  for (int ln = threadIdx.x; ln < tm.n_node; ln += blockDim.x) {
    const int g = B.tile_nodes[tm.node_begin + ln];
    s_x[ln] = B.x[g]; s_y[ln] = B.y[g]; s_z[ln] = B.z[g];
    double u = B.su[g], v = B.sv[g], w = B.sw[g];
    if (P.glob_fixed & FM_FIX_X) u = 0.0;
    if (P.glob_fixed & FM_FIX_Y) v = 0.0;
    if (P.glob_fixed & FM_FIX_Z) w = 0.0;
    s_u[ln] = u; s_v[ln] = v; s_w[ln] = w;
  }
  __syncthreads();
  const double big = 1.7976931348623157e308;
  double r[11] = {big, -big, big, -big, 0.0, 0.0, 0.0, big, -big, big, -big};
  const double rho = P.rho, mu = P.mu, nu = mu / rho, alpha = P.alpha, cI = P.c_i, dt = P.dt;
  for (int le = threadIdx.x; le < tm.n_elem; le += blockDim.x) {
    const int64_t e = tm.elem_begin + le;
    int ln[NPE];
    for (int a = 0; a < NPE; ++a) ln[a] = B.conn[e * NPE + a] & 0x7fff;
    double vol = 0.0, lam_int = 0.0;
    for (int g = 0; g < GaussRule<NPE>::n; ++g) {
      double q[3], Nf[NPE], dN[NPE][3], inv[3][3];
      GaussRule<NPE>::point(g, q);
      shape<NPE>(q, Nf, dN);
      const double det = jacobian<NPE>(dN, s_x, s_y, s_z, ln, inv);
      double u[3] = {0.0, 0.0, 0.0};
      for (int a = 0; a < NPE; ++a) {
        u[0] += Nf[a] * s_u[ln[a]];
        u[1] += Nf[a] * s_v[ln[a]];
        u[2] += Nf[a] * s_w[ln[a]];
      }
      double G[3][3];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) G[a][b] = inv[0][a] * inv[0][b] + inv[1][a] * inv[1][b] + inv[2][a] * inv[2][b];
      double t2 = 0.0, t3 = 0.0;
      for (int a = 0; a < 3; ++a) {
        t2 += u[a] * (G[a][0] * u[0] + G[a][1] * u[1] + G[a][2] * u[2]);
        t3 += G[a][0] * G[a][0] + G[a][1] * G[a][1] + G[a][2] * G[a][2];
      }
      const double tau = 1.0 / sqrt(t2 + t3 * nu * nu * cI);
      const double m00 = G[0][0], m01 = G[0][1], m02 = G[0][2], m10 = G[1][0], m11 = G[1][1], m12 = G[1][2],
                   m20 = G[2][0], m21 = G[2][1], m22 = G[2][2];
      const double dG = m00 * (m11 * m22 - m21 * m12) - m01 * (m10 * m22 - m12 * m20) + m02 * (m10 * m21 - m11 * m20);
      const double idg = 1.0 / dG;
      const double iG[3][3] = {{(m11 * m22 - m21 * m12) * idg, (m02 * m21 - m01 * m22) * idg, (m01 * m12 - m02 * m11) * idg},
                               {(m12 * m20 - m10 * m22) * idg, (m00 * m22 - m02 * m20) * idg, (m10 * m02 - m00 * m12) * idg},
                               {(m10 * m21 - m20 * m11) * idg, (m20 * m01 - m00 * m21) * idg, (m00 * m11 - m10 * m01) * idg}};
      const double l2 = sqrt((iG[0][0] * u[0] + iG[0][1] * u[1] + iG[0][2] * u[2]) * u[0] +
                             (iG[1][0] * u[0] + iG[1][1] * u[1] + iG[1][2] * u[2]) * u[1] +
                             (iG[2][0] * u[0] + iG[2][1] * u[1] + iG[2][2] * u[2]) * u[2]);
      const double lam = alpha * ((nu < l2) ? l2 : nu);
      const double un = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
      const double o[3] = {u[0] / un, u[1] / un, u[2] / un};
      double el = 0.0;
      for (int a = 0; a < 3; ++a) el += (iG[a][0] * o[0] + iG[a][1] * o[1] + iG[a][2] * o[2]) * o[a];
      el = 2.0 * sqrt(el);
      const double w = det * GaussRule<NPE>::weight();
      vol += w;
      lam_int += lam * w;
      upd_min(r[0], tau); upd_max(r[1], tau);
      upd_min(r[2], lam); upd_max(r[3], lam);
      upd_max(r[4], 2.0 * nu * (dt / (el * el)));
      upd_max(r[5], fabs(u[0] * dt) / el);
      upd_max(r[6], 2.0 * lam * (dt / (el * el)));
    }
    const double lam_el = lam_int / vol;
    const double E = (mu * (3 * lam_el + 2 * mu)) / (lam_el + mu);
    const double nue = lam_el / (2 * (lam_el + mu));
    upd_min(r[7], E); upd_max(r[8], E);
    upd_min(r[9], nue); upd_max(r[10], nue);
  }
  // block reduction (warp results through shared memory, then warp 0)
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = (blockDim.x + 31) >> 5;
  for (int k = 0; k < 11; ++k) {
    const bool isMin = (k == 0 || k == 2 || k == 7 || k == 9);
    double v = r[k];
    for (int off = 16; off > 0; off >>= 1) {
      const double o2 = __shfl_down_sync(0xffffffffu, v, off);
      if (isMin) upd_min(v, o2); else upd_max(v, o2);
    }
    if (lane == 0) s_red[k][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 11) {
    const int k = threadIdx.x;
    const bool isMin = (k == 0 || k == 2 || k == 7 || k == 9);
    double v = s_red[k][0];
    for (int i = 1; i < nwarp; ++i) {
      if (isMin) upd_min(v, s_red[k][i]); else upd_max(v, s_red[k][i]);
    }
    out[(int64_t)blockIdx.x * 11 + k] = v;
  }
}

__global__ void velocity_extrema_kernel(DevBatch B, int64_t node_begin, int64_t n_nodes, int glob_fixed, double* out) {
  __shared__ double s_red[7][32];
  const double big = 1.7976931348623157e308;
  double r[7] = {big, -big, big, -big, big, -big, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_nodes; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = node_begin + i;
    double u[3] = {B.su[g], B.sv[g], B.sw[g]};
    if (glob_fixed & FM_FIX_X) u[0] = 0.0;
    if (glob_fixed & FM_FIX_Y) u[1] = 0.0;
    if (glob_fixed & FM_FIX_Z) u[2] = 0.0;
    upd_max(r[6], sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
    for (int c = 0; c < 3; ++c) {
      upd_min(r[2 * c], u[c]);
      upd_max(r[2 * c + 1], u[c]);
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = (blockDim.x + 31) >> 5;
  for (int k = 0; k < 7; ++k) {
    const bool isMin = (k == 0 || k == 2 || k == 4);
    double v = r[k];
    for (int off = 16; off > 0; off >>= 1) {
      const double o2 = __shfl_down_sync(0xffffffffu, v, off);
      if (isMin) upd_min(v, o2); else upd_max(v, o2);
    }
    if (lane == 0) s_red[k][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    const int k = threadIdx.x;
    const bool isMin = (k == 0 || k == 2 || k == 4);
    double v = s_red[k][0];
    for (int i = 1; i < nwarp; ++i) {
      if (isMin) upd_min(v, s_red[k][i]); else upd_max(v, s_red[k][i]);
    }
    out[(int64_t)blockIdx.x * 7 + k] = v;
  }
}

cudaError_t launch_supg_stats(const DevBatch& B, int tile0, int ntiles, int tn_max, int npe, double* out,
                              cudaStream_t s) {
  const size_t smem = (size_t)tn_max * 6 * sizeof(double);
  if (ntiles <= 0) return cudaSuccess;
  if (npe == 4)
    supg_stats_kernel<4><<<ntiles, 128, smem, s>>>(B, tile0, tn_max, out);
  else
    supg_stats_kernel<8><<<ntiles, 128, smem, s>>>(B, tile0, tn_max, out);
  return cudaGetLastError();
}

cudaError_t launch_velocity_extrema(const DevBatch& B, int64_t node_begin, int64_t n_nodes, int glob_fixed, int blocks,
                                    double* out, cudaStream_t s) {
  velocity_extrema_kernel<<<blocks, 256, 0, s>>>(B, node_begin, n_nodes, glob_fixed, out);
  return cudaGetLastError();
}

}  // namespace fm
