// VMS explicit step kernels: one launch of vms_tile_kernel (all tiles of
// all problems) plus one of vms_iface_kernel per dual iteration.
//
// vms_tile_kernel, one CTA per tile:
//   1. stage the tile's nodes (coordinates, state, BC index) in shared memory;
//   2. per element (one thread each, chunks of blockDim.x):
//      geometry from the staged coordinates, the pending subscale update of
//      the previous iteration (assemble_projRes_explicit +
//      update_subscales_explicit), the element residual (assemble_RHS);
//   3. add the 16 residual entries to shared-memory node accumulators, one
//      colour at a time (elements of a colour share no node), so every node
//      receives its contributions in a fixed order - no atomics;
//   4. nodes interior to the tile are complete: dual update
//      (update_dual_solution), BCs (setNodeVelocity, apply_zeroTraction,
//      setDirichletBC) and store; interface nodes store their tile partial.
// vms_iface_kernel sums each interface node's partials in tile order and
// applies the same node update, then advances the problems' iteration.
#include <cuda_runtime.h>

#include "fm_device.cuh"
#include "fm_vms.cuh"

namespace fm {

// update_dual_solution (src lines 754-772) + BCs (src lines 1179-1197).
// post: state after the previous iteration's BCs; pre: before them (only
// differs at BC nodes).  The dual update starts from sol_n, which is the
// post-BC state at the first dual iteration of a step (update_solution,
// src lines 726-752) and the pre-BC state afterwards.
__device__ __forceinline__ void vms_node_update(const DevBatch& B, const DevProb& P, int pidx, int iter, double time,
                                                int64_t g, const double post[4], const double acc[4], bool first_dual,
                                                int32_t* status) {
  const int32_t rec = B.node_bc[g];
  double s[4];
  if (!first_dual && rec >= 0) {
    s[0] = B.pu[g]; s[1] = B.pv[g]; s[2] = B.pw[g]; s[3] = B.pp[g];
  } else {
    s[0] = post[0]; s[1] = post[1]; s[2] = post[2]; s[3] = post[3];
  }
  const double m = B.mass[g];
#pragma unroll
  for (int d = 0; d < 4; ++d) s[d] = __dsub_rn(s[d], __ddiv_rn(__dmul_rn(P.ds, acc[d]), m));
  if (!(isfinite(s[0]) && isfinite(s[1]) && isfinite(s[2]) && isfinite(s[3]))) *status = FM_ERR_DIVERGED;
#pragma unroll
  for (int i = 0; i < 4; ++i)
    if (P.q1[i] == g) B.q1p[pidx * 8 + (iter & 1) * 4 + i] = s[3];
  if (rec >= 0) {
    B.pu[g] = s[0]; B.pv[g] = s[1]; B.pw[g] = s[2]; B.pp[g] = s[3];
    apply_bc(B, rec, time, s, status);
  }
  B.su[g] = s[0]; B.sv[g] = s[1]; B.sw[g] = s[2]; B.sp[g] = s[3];
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 2) vms_tile_kernel(DevBatch B, int tn_max) {
  extern __shared__ double sm[];
  double* s_x = sm;
  double* s_y = s_x + tn_max;
  double* s_z = s_y + tn_max;
  double* s_u = s_z + tn_max;
  double* s_v = s_u + tn_max;
  double* s_w = s_v + tn_max;
  double* s_p = s_w + tn_max;
  double* s_qu = s_p + tn_max;   // pre-BC velocity
  double* s_qv = s_qu + tn_max;
  double* s_qw = s_qv + tn_max;
  double* s_a0 = s_qw + tn_max;
  double* s_a1 = s_a0 + tn_max;
  double* s_a2 = s_a1 + tn_max;
  double* s_a3 = s_a2 + tn_max;
  int32_t* s_col = (int32_t*)(s_a3 + tn_max);   // colour offsets (<= 129)

  const TileMeta tm = B.tiles[blockIdx.x];
  const int pidx = tm.problem;
  const DevProbState st = B.pstate[pidx];
  if (st.iter >= B.target[pidx]) return;
  const DevProb& P = B.probs[pidx];
  const int per_step = P.ndual + 1;
  const bool first_dual = (st.iter % per_step) == 0;
  const bool pending = st.iter > 0;
  const int tid = threadIdx.x;

  for (int ln = tid; ln < tm.n_node; ln += THREADS) {
    const int g = B.tile_nodes[tm.node_begin + ln];
    s_x[ln] = B.x[g]; s_y[ln] = B.y[g]; s_z[ln] = B.z[g];
    const double u = B.su[g], v = B.sv[g], w = B.sw[g];
    s_u[ln] = u; s_v[ln] = v; s_w[ln] = w; s_p[ln] = B.sp[g];
    if (B.node_bc[g] >= 0) {
      s_qu[ln] = B.pu[g]; s_qv[ln] = B.pv[g]; s_qw[ln] = B.pw[g];
    } else {
      s_qu[ln] = u; s_qv[ln] = v; s_qw[ln] = w;
    }
    s_a0[ln] = 0.0; s_a1[ln] = 0.0; s_a2[ln] = 0.0; s_a3[ln] = 0.0;
  }
  for (int c = tid; c <= tm.n_col; c += THREADS) s_col[c] = B.tile_cols[tm.col_begin + c];
  double pq[4];
  {
    const double* q = B.q1p + pidx * 8 + ((st.iter - 1) & 1) * 4;
    pq[0] = q[0]; pq[1] = q[1]; pq[2] = q[2]; pq[3] = q[3];
  }
  const double inv_dt = 1.0 / P.dt;
  const double c1nu = P.c1 * P.nu;
  const double nu4 = 4.0 * P.nu;
  __syncthreads();

  const int64_t E = B.E;
  int c_lo = 0;
  for (int base = 0; base < tm.n_elem; base += THREADS) {
    const int le = base + tid;
    const bool active = le < tm.n_elem;
    double lres[4][4];
    int ln[4];
    if (active) {
      const int64_t e = tm.elem_begin + le;
      const uint2 cw = __ldg(reinterpret_cast<const uint2*>(B.conn) + e);
      ln[0] = cw.x & 0xffff; ln[1] = cw.x >> 16; ln[2] = cw.y & 0xffff; ln[3] = cw.y >> 16;
      double X[4][3], U[4][3], Pn[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        X[a][0] = s_x[ln[a]]; X[a][1] = s_y[ln[a]]; X[a][2] = s_z[ln[a]];
      }
      TetGeom geo;
      tet_geometry(X, geo);
      const double ih = rcbrt(6.0 * geo.V);
      double sdu[4][3];
#pragma unroll
      for (int g = 0; g < 4; ++g)
#pragma unroll
        for (int i = 0; i < 3; ++i) sdu[g][i] = __ldcs(B.sdus + (int64_t)(g * 3 + i) * E + e);
      double Q[4][3];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        Q[a][0] = s_qu[ln[a]]; Q[a][1] = s_qv[ln[a]]; Q[a][2] = s_qw[ln[a]];
      }
      if (pending) {
        vms_subscale_update<double>(geo, Q, pq, sdu, inv_dt, c1nu, P.c2, ih);
#pragma unroll
        for (int g = 0; g < 4; ++g)
#pragma unroll
          for (int i = 0; i < 3; ++i) __stcs(B.sdus + (int64_t)(g * 3 + i) * E + e, sdu[g][i]);
      }
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        U[a][0] = s_u[ln[a]]; U[a][1] = s_v[ln[a]]; U[a][2] = s_w[ln[a]]; Pn[a] = s_p[ln[a]];
      }
      if (first_dual)
        vms_residual<double, false>(geo, U, Pn, U, sdu, nu4, P.inv_eps, inv_dt, lres);
      else
        vms_residual<double, true>(geo, U, Pn, Q, sdu, nu4, P.inv_eps, inv_dt, lres);
    }
    // colour rounds over this chunk
    while (c_lo < tm.n_col && s_col[c_lo + 1] <= base) ++c_lo;
    for (int c = c_lo; c < tm.n_col && s_col[c] < base + THREADS; ++c) {
      if (active && le >= s_col[c] && le < s_col[c + 1]) {
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          s_a0[ln[a]] += lres[a][0];
          s_a1[ln[a]] += lres[a][1];
          s_a2[ln[a]] += lres[a][2];
          s_a3[ln[a]] += lres[a][3];
        }
      }
      __syncthreads();
    }
  }
  __syncthreads();
  int32_t status = FM_OK;
  for (int ln2 = tid; ln2 < tm.n_node; ln2 += THREADS) {
    const double acc[4] = {s_a0[ln2], s_a1[ln2], s_a2[ln2], s_a3[ln2]};
    if (ln2 < tm.n_int) {
      const int g = B.tile_nodes[tm.node_begin + ln2];
      const double post[4] = {s_u[ln2], s_v[ln2], s_w[ln2], s_p[ln2]};
      vms_node_update(B, P, pidx, st.iter, st.time, g, post, acc, first_dual, &status);
    } else {
      const int s = tm.slot_base + (ln2 - tm.n_int);
      B.part0[s] = acc[0]; B.part1[s] = acc[1]; B.part2[s] = acc[2]; B.part3[s] = acc[3];
    }
  }
  if (status != FM_OK) B.pstate[pidx].status = status;
}

__global__ void vms_iface_kernel(DevBatch B) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B.n_iface; i += gridDim.x * blockDim.x) {
    const int pidx = B.iface_prob[i];
    const DevProbState st = B.pstate[pidx];
    if (st.iter >= B.target[pidx]) continue;
    const DevProb& P = B.probs[pidx];
    const bool first_dual = (st.iter % (P.ndual + 1)) == 0;
    const int g = B.iface_node[i];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = B.iface_slot_beg[i]; k < B.iface_slot_beg[i + 1]; ++k) {
      const int s = B.iface_slots[k];
      acc[0] += B.part0[s]; acc[1] += B.part1[s]; acc[2] += B.part2[s]; acc[3] += B.part3[s];
    }
    const double post[4] = {B.su[g], B.sv[g], B.sw[g], B.sp[g]};
    int32_t status = FM_OK;
    vms_node_update(B, P, pidx, st.iter, st.time, g, post, acc, first_dual, &status);
    if (status != FM_OK) B.pstate[pidx].status = status;
  }
  finish_iteration(B);
}

size_t vms_smem_bytes(int tn_max) { return (size_t)tn_max * 14 * sizeof(double) + 130 * sizeof(int32_t); }

cudaError_t launch_vms_iteration(const DevBatch& B, int tn_max, int threads, int iface_blocks, cudaStream_t s) {
  const size_t smem = vms_smem_bytes(tn_max);
  if (threads == 256) {
    vms_tile_kernel<256><<<B.n_tiles, 256, smem, s>>>(B, tn_max);
  } else {
    vms_tile_kernel<128><<<B.n_tiles, 128, smem, s>>>(B, tn_max);
  }
  vms_iface_kernel<<<iface_blocks, 256, 0, s>>>(B);
  return cudaGetLastError();
}

cudaError_t vms_configure(size_t smem) {
  cudaError_t e = cudaFuncSetAttribute(vms_tile_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(vms_tile_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

}  // namespace fm
