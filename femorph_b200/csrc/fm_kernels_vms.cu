// VMS explicit step kernels: one launch of vms_tile_kernel (all tiles of
// all problems) plus one of vms_iface_kernel per dual iteration.
//
// vms_tile_kernel, one CTA per tile:
//   1. stage the tile's nodes (coordinates, state, BC index) in shared memory;
//   2. per element (one thread each, chunks of blockDim.x):
//      geometry from the staged coordinates, the pending subscale update of
//      the previous iteration (assemble_projRes_explicit +
//      update_subscales_explicit), the element residual (assemble_RHS);
//   3. stage the chunk's 16 residual entries an element in shared memory;
//      after one barrier each thread adds, for the nodes it owns, the
//      chunk's contributions to its shared-memory accumulators, walking the
//      node's incidence list in element order, so every node receives its
//      contributions in a fixed order - no atomics;
//   4. nodes interior to the tile are complete: dual update
//      (update_dual_solution), BCs (setNodeVelocity, apply_zeroTraction,
//      setDirichletBC) and store; interface nodes store their tile partial.
// vms_iface_kernel sums each interface node's partials in tile order and
// applies the same node update, then advances the problems' iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "fm_device.cuh"
#include "fm_vms.cuh"

namespace fm {

// update_dual_solution (src lines 754-772) + BCs (src lines 1179-1197).
// post: state after the previous iteration's BCs; pre: before them (only
// differs at BC nodes).  The dual update starts from sol_n, which is the
// post-BC state at the first dual iteration of a step (update_solution,
// src lines 726-752) and the pre-BC state afterwards.
// The problem constants the element and node passes read, copied into
// registers once per CTA (read through the DevProb in global memory they
// would be reloaded for every element: the compiler cannot prove that the
// kernel's own stores leave them unchanged).
struct VmsConsts {
  double ds, c2, inv_eps;
  int32_t q1[4];
};
__device__ __forceinline__ VmsConsts vms_consts(const DevProb& P) {
  VmsConsts c;
  c.ds = P.ds;
  c.c2 = P.c2;
  c.inv_eps = P.inv_eps;
  c.q1[0] = P.q1[0]; c.q1[1] = P.q1[1]; c.q1[2] = P.q1[2]; c.q1[3] = P.q1[3];
  return c;
}

template <class PROB>  // DevProb or VmsConsts: reads ds and q1[]
__device__ __forceinline__ void vms_node_update(const DevBatch& B, const PROB& P, int pidx, int iter, double time,
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

// Node records in shared memory: four 16-byte pieces per node, (x, y)
// (z, u) (v, w) (p, tag), piece k of node ln stored at position
// k ^ ((ln >> 1) & 3).  With 64-byte records the unswizzled piece k of every
// node falls in one of only two 4-bank groups, so a warp's 16-byte loads of
// 32 different nodes serialise up to 16-fold; the swizzle spreads them over
// all eight groups.
__device__ __forceinline__ int rec_index(int ln, int k) { return ln * 4 + (k ^ ((ln >> 1) & 3)); }

// Brings the line holding *p into L1 (no data returned).
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// Node record piece 3 = (p, tag): tag = batch node id, with bit 62 set when
// the node carries a BC (its pre-BC values are then read from memory).
constexpr long long FM_TAG_BC = 1ll << 62;

// Per-element VMS work for one chunk slot: pending subscale update (written
// back to global memory) and the element residual lres.  S: subscale storage
// type (double, or float in the mixed form).
template <bool MIXED, typename S>
__device__ __forceinline__ void vms_element(const DevBatch& B, const VmsConsts& P, int64_t e, const int ln[4],
                                            bool precise, const double2* s_rec, const S sd_in[12],
                                            const double pq[4], bool pending, bool first_dual, double inv_dt,
                                            double c1nu, double nu4, double lres[4][4]) {
  const int64_t E = B.E;
  // Pass 1 reads the coordinates and Q, the velocity before the last BC
  // application (it differs from the staged state only at BC nodes, whose
  // tag has FM_TAG_BC set beside the node's batch id, and is read from
  // memory there).  FP64: pass 2
  // re-reads the post-BC velocity U and pressure from shared memory, so the
  // two velocity sets are never held in registers at the same time (the
  // FP32 form, with fewer live registers, reads them in pass 1).
  // Node record: (x, y) (z, u) (v, w) (p, tag).
  double X[4][3], Q[4][3], U[4][3], Pn[4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const double2 r0 = s_rec[rec_index(ln[a], 0)], r1 = s_rec[rec_index(ln[a], 1)],
                  r2 = s_rec[rec_index(ln[a], 2)], r3 = s_rec[rec_index(ln[a], 3)];
    X[a][0] = r0.x; X[a][1] = r0.y; X[a][2] = r1.x;
    if constexpr (MIXED) {
      U[a][0] = r1.y; U[a][1] = r2.x; U[a][2] = r2.y;
      Pn[a] = r3.x;
    }
    const long long tag = __double_as_longlong(r3.y);
    if (tag & FM_TAG_BC) {
      const long long g = tag & 0x7fffffffll;
      Q[a][0] = B.pu[g]; Q[a][1] = B.pv[g]; Q[a][2] = B.pw[g];
    } else {
      Q[a][0] = r1.y; Q[a][1] = r2.x; Q[a][2] = r2.y;
    }
  }
  auto load_post = [&]() {
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const double2 r1 = s_rec[rec_index(ln[a], 1)], r2 = s_rec[rec_index(ln[a], 2)], r3 = s_rec[rec_index(ln[a], 3)];
      U[a][0] = r1.y; U[a][1] = r2.x; U[a][2] = r2.y;
      Pn[a] = r3.x;
    }
  };
  if constexpr (MIXED) {
    TetGeomF geo;
    tet_geometry_mixed(X, precise, geo);
    const float ih = rcbrt_nr((float)(6.0 * geo.V));
    float sdu[4][3];
#pragma unroll
    for (int q = 0; q < 12; ++q) sdu[q / 3][q % 3] = sd_in[q];
    float G[3][3], Ds[3];
    if (pending) {
      // velocities enter FP32 as differences to node 0, formed in FP64
      float Q0[3], Qd[4][3], pqd[4];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        Q0[i] = (float)Q[0][i];
#pragma unroll
        for (int a = 0; a < 4; ++a) Qd[a][i] = (float)(Q[a][i] - Q[0][i]);
      }
#pragma unroll
      for (int a = 0; a < 4; ++a) pqd[a] = (float)(pq[a] - pq[0]);
      vms_subscale_update_mixed(geo, Q0, Qd, pqd, sdu, (float)inv_dt, (float)c1nu, (float)P.c2, ih, G, Ds);
#pragma unroll
      for (int q = 0; q < 12; ++q) __stcs(B.sdus32 + (int64_t)q * E + e, sdu[q / 3][q % 3]);
    }
    float U0[3], Ud[4][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      U0[i] = (float)U[0][i];
#pragma unroll
      for (int a = 0; a < 4; ++a) Ud[a][i] = (float)(U[a][i] - U[0][i]);
    }
    if (first_dual) {
      vms_residual_mixed<false>(geo, U0, Ud, Pn, Ud, sdu, (float)nu4, (float)P.inv_eps, (float)inv_dt, G, Ds, false,
                                lres);
    } else {
      float Dacc[4][3];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int i = 0; i < 3; ++i) Dacc[a][i] = (float)(U[a][i] - Q[a][i]);
      vms_residual_mixed<true>(geo, U0, Ud, Pn, Dacc, sdu, (float)nu4, (float)P.inv_eps, (float)inv_dt, G, Ds, false,
                               lres);
    }
  } else {
    (void)precise;
    TetGeom geo;
    tet_geometry(X, geo);
    const double ih = rcbrt_nr(6.0 * geo.V);
    double sdu[4][3];
#pragma unroll
    for (int q = 0; q < 12; ++q) sdu[q / 3][q % 3] = sd_in[q];
    double G[3][3], Gs[3];
    if (pending) {
      vms_subscale_update<double>(geo, Q, pq, sdu, inv_dt, c1nu, P.c2, ih, G, Gs);
#pragma unroll
      for (int q = 0; q < 12; ++q) __stcs(B.sdus + (int64_t)q * E + e, sdu[q / 3][q % 3]);
    }
    load_post();
    if (first_dual)
      vms_residual<double, false>(geo, U, Pn, U, sdu, nu4, P.inv_eps, inv_dt, G, Gs, false, lres);
    else
      vms_residual<double, true>(geo, U, Pn, Q, sdu, nu4, P.inv_eps, inv_dt, G, Gs, false, lres);
  }
}

// Shared memory of one tile CTA, in this order:
//  node records: 8 doubles x tn_pad (rec_index layout), then four residual
//    accumulators of tn_pad doubles; tn_pad = tn_max rounded up to even so
//    every later region is 16-byte aligned;
//  chunk stage: two buffers, each 12 subscale rows + 1 connectivity row of
//    THREADS slots (bulk-copy targets).  FP64: each buffer is sized to 16 rows
//    of THREADS doubles because a thread overwrites its own column with its 16
//    residual entries once it has read its inputs; mixed: a separate
//    16 x THREADS double region holds the residual entries;
//  incidence entries (uint16 x inc_max), incidence offsets (uint16 x tn_pad+2).
template <int THREADS, bool MIXED>
__host__ __device__ constexpr size_t vms_stage_bytes() {
  return MIXED ? 2 * ((size_t)12 * THREADS * sizeof(float) + (size_t)THREADS * 8) + (size_t)16 * THREADS * 8
               : 2 * (size_t)16 * THREADS * 8;
}
template <int THREADS, bool MIXED>
__host__ __device__ constexpr size_t vms_stage_buffer_bytes() {
  return MIXED ? (size_t)12 * THREADS * sizeof(float) + (size_t)THREADS * 8 : (size_t)16 * THREADS * 8;
}

// MINB: resident CTAs an SM the variant is compiled for (its register budget).
template <int THREADS, bool MIXED, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) vms_tile_kernel(DevBatch B, int tn_max, int inc_max) {
  using S = typename std::conditional<MIXED, float, double>::type;
  extern __shared__ __align__(16) double sm[];
  const int tn_pad = (tn_max + 1) & ~1;
  double2* s_rec = reinterpret_cast<double2*>(sm);  // per node: (x,y) (z,u) (v,w) (p,tag)
  double* s_a0 = sm + 8 * tn_pad;  // residual accumulators (each node owned by one thread)
  double* s_a1 = s_a0 + tn_pad;
  double* s_a2 = s_a1 + tn_pad;
  double* s_a3 = s_a2 + tn_pad;
  char* stage = reinterpret_cast<char*>(s_a3 + tn_pad);
  constexpr size_t BUF = vms_stage_buffer_bytes<THREADS, MIXED>();
  double* s_lres_mixed = reinterpret_cast<double*>(stage + 2 * BUF);  // mixed only
  uint16_t* s_inc = reinterpret_cast<uint16_t*>(stage + vms_stage_bytes<THREADS, MIXED>());  // inc_max (multiple of 8)
  uint16_t* s_off = s_inc + inc_max;
  __shared__ uint64_t bars[2];
  __shared__ int s_abort;

  const TileMeta tm = B.tiles[blockIdx.x];
  const int pidx = tm.problem;
  if (pidx < 0) return;  // free tile slot
  const int tid = threadIdx.x;
  // this thread's staged nodes: their ids are loaded before the problem
  // state is checked, so both round trips overlap
  constexpr int MAXOWN = FM_MAX_TILE_NODES / THREADS;  // the host caps tile_nodes
  int gid[MAXOWN];
#pragma unroll
  for (int j = 0; j < MAXOWN; ++j) {
    const int ln = tid + j * THREADS;
    gid[j] = ln < tm.n_node ? B.tile_nodes[tm.node_begin + ln] : -1;
  }
  const DevProbState st = B.pstate[pidx];
  if (st.iter >= B.target[pidx] || st.status != FM_OK) return;
  const DevProb& P = B.probs[pidx];
  const VmsConsts PC = vms_consts(P);
  const int per_step = P.ndual + 1;
  const bool first_dual = (st.iter % per_step) == 0;
  const bool pending = st.iter > 0;
  const int64_t E = B.E;
  const S* sdus_g = MIXED ? reinterpret_cast<const S*>(B.sdus32) : reinterpret_cast<const S*>(B.sdus);
  const uint2* conn_g = reinterpret_cast<const uint2*>(B.conn);
  const int nchunks = (tm.n_elem + THREADS - 1) / THREADS;

  // one thread issues the bulk copies of chunk k into stage buffer k & 1
  auto issue = [&](int k) {
    const int b = k & 1;
    const int base = k * THREADS;
    const int nch = min(THREADS, tm.n_elem - base);
    const int64_t e0 = tm.elem_begin + base;  // multiple of 32 elements
    const uint32_t rs = MIXED ? ((nch + 3) & ~3) : ((nch + 1) & ~1);  // 16-byte multiples
    const uint32_t bytes_s = rs * (uint32_t)sizeof(S);
    const uint32_t bytes_c = (uint32_t)((nch + 1) & ~1) * 8u;
    S* bs = reinterpret_cast<S*>(stage + b * BUF);
    mbar_arrive_expect_tx(&bars[b], 12u * bytes_s + bytes_c);
#pragma unroll 1
    for (int q = 0; q < 12; ++q) bulk_load(bs + q * THREADS, sdus_g + (int64_t)q * E + e0, bytes_s, &bars[b]);
    bulk_load(bs + 12 * THREADS, conn_g + e0, bytes_c, &bars[b]);
  };

  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
    s_abort = 0;
    // the first chunk's copies overlap the node staging below (they target
    // the stage buffers, which the staging does not touch)
    if (nchunks > 0) issue(0);
  }
  // node staging: the gathers of this thread's (up to FM_MAX_TILE_NODES /
  // THREADS) nodes overlap
  {
#pragma unroll
    for (int j = 0; j < MAXOWN; ++j) {
      const int ln = tid + j * THREADS;
      const int g = gid[j];
      if (g >= 0) {
        const long long tag = (long long)g | (B.node_bc[g] >= 0 ? FM_TAG_BC : 0ll);
        s_rec[rec_index(ln, 0)] = make_double2(B.x[g], B.y[g]);
        s_rec[rec_index(ln, 1)] = make_double2(B.z[g], B.su[g]);
        s_rec[rec_index(ln, 2)] = make_double2(B.sv[g], B.sw[g]);
        s_rec[rec_index(ln, 3)] = make_double2(B.sp[g], __longlong_as_double(tag));
        s_a0[ln] = 0.0; s_a1[ln] = 0.0; s_a2[ln] = 0.0; s_a3[ln] = 0.0;
      }
    }
  }
  for (int i = tid; i <= tm.n_node; i += THREADS) s_off[i] = B.tile_off[tm.off_begin + i];
  {
    const int ninc = tm.n_elem * 4;
    const uint4* src = reinterpret_cast<const uint4*>(B.tile_inc + tm.inc_begin);  // 16-byte aligned
    uint4* dst = reinterpret_cast<uint4*>(s_inc);
    for (int i = tid; i < (ninc + 7) / 8; i += THREADS) dst[i] = src[i];
  }
  double pq[4];
  {
    const double* q = B.q1p + pidx * 8 + ((st.iter - 1) & 1) * 4;
    pq[0] = q[0]; pq[1] = q[1]; pq[2] = q[2]; pq[3] = q[3];
  }
  const double inv_dt = 1.0 / P.dt;
  const double c1nu = P.c1 * P.nu;
  const double nu4 = 4.0 * P.nu;
  __syncthreads();
  // one lane asks L2 for a later tile's element rows and interior-node
  // ranges (contiguous), so that tile's bulk copies and gathers hit L2; the
  // round-up to 16 bytes reads at most 12 bytes past an array, inside the
  // batch's single device allocation (another array or the carve padding)
  if (B.l2_ahead > 0 && tid == THREADS - 32 && blockIdx.x + B.l2_ahead < (unsigned)B.n_tiles) {
    const TileMeta tn = B.tiles[blockIdx.x + B.l2_ahead];
    if (tn.problem >= 0 && tn.n_elem > 0) {
      const int64_t e0 = tn.elem_begin;  // multiple of 32 slots: 16-byte aligned rows
      const uint32_t bs = ((uint32_t)tn.n_elem * (uint32_t)sizeof(S) + 15u) & ~15u;
#pragma unroll 1
      for (int q = 0; q < 12; ++q) bulk_prefetch_l2(sdus_g + (int64_t)q * E + e0, bs);
      bulk_prefetch_l2(conn_g + e0, ((uint32_t)tn.n_elem * 8u + 15u) & ~15u);
      bulk_prefetch_l2(B.tile_inc + tn.inc_begin, ((uint32_t)tn.n_elem * 8u + 15u) & ~15u);
      if (tn.n_int > 0 && tn.node0 >= 0) {
        const int64_t g0 = tn.node0 & ~1, g1 = ((int64_t)tn.node0 + tn.n_int + 1) & ~1ll;
        const uint32_t nb = (uint32_t)(g1 - g0) * 8u;
        bulk_prefetch_l2(B.x + g0, nb); bulk_prefetch_l2(B.y + g0, nb); bulk_prefetch_l2(B.z + g0, nb);
        bulk_prefetch_l2(B.su + g0, nb); bulk_prefetch_l2(B.sv + g0, nb); bulk_prefetch_l2(B.sw + g0, nb);
        bulk_prefetch_l2(B.sp + g0, nb); bulk_prefetch_l2(B.mass + g0, nb);
        const int64_t h0 = tn.node0 & ~3, h1 = ((int64_t)tn.node0 + tn.n_int + 3) & ~3ll;
        bulk_prefetch_l2(B.node_bc + h0, (uint32_t)(h1 - h0) * 4u);
      }
    }
  }

  // nodes owned by this thread for the accumulation: j * THREADS + tid;
  // cur/end walk each one's incidence list in element order, nxt holds the
  // entry at cur (loaded one step ahead, so the walk's shared-memory loads
  // do not wait on each other)
  auto owned_node = [](int t, int j) { return j * THREADS + t; };
  int cur[MAXOWN], endi[MAXOWN], nxt[MAXOWN];
#pragma unroll
  for (int j = 0; j < MAXOWN; ++j) {
    const int ln = owned_node(tid, j);
    cur[j] = ln < tm.n_node ? s_off[ln] : 0;
    endi[j] = ln < tm.n_node ? s_off[ln + 1] : 0;
    nxt[j] = cur[j] < endi[j] ? s_inc[cur[j]] : 0;
  }
  int k = 0;
  for (; k < nchunks; ++k) {
    if (tid == 0 && k + 1 < nchunks) {
      fence_proxy_async_smem();  // buffer (k+1)&1 was last read before the previous barrier
      issue(k + 1);
    }
    if (k + 1 == nchunks) {
      // the node update after the last chunk reads the mass and BC index of
      // this thread's interior nodes: fetch them into L1 now
#pragma unroll
      for (int j = 0; j < MAXOWN; ++j) {
        const int ln2 = tid + j * THREADS;
        if (ln2 < tm.n_int) {
          const int g = (int)(__double_as_longlong(s_rec[rec_index(ln2, 3)].y) & 0x7fffffffll);
          prefetch_l1(B.mass + g);
          prefetch_l1(B.node_bc + g);
        }
      }
    }
    // each thread waits for the chunk itself (the mbarrier phase makes the
    // bulk-copied bytes visible to it); a timed-out wait skips the chunk and
    // is agreed on at the end-of-chunk barrier
    const bool arrived = mbar_wait_bounded(&bars[k & 1], (uint32_t)((k >> 1) & 1), B.wait_limit);
    const int base = k * THREADS;
    const int le = base + tid;
    const bool active = arrived && le < tm.n_elem;
    char* buf = stage + (k & 1) * BUF;
    // residual entries.  FP64: [16][THREADS] in the stage buffer, each thread
    // overwriting its own column (its inputs, already read).  Mixed (own
    // region): per element 8 16-byte pieces (corner, component pair), piece p
    // of element col at col * 8 + (p ^ (col & 7)), so that the owners'
    // scattered 16-byte reads spread over all bank groups (1.5% faster
    // there; in the FP64 stage buffer it would need one more barrier a chunk,
    // which costs more than it gains)
    double* R = MIXED ? s_lres_mixed : reinterpret_cast<double*>(buf);
    double2* R2 = reinterpret_cast<double2*>(R);
    double lres[4][4];
    if (active) {
      const S* bs = reinterpret_cast<const S*>(buf);
      const uint2 cw = reinterpret_cast<const uint2*>(bs + 12 * THREADS)[tid];
      int ln[4];
      // bit 15 of the first id flags (mixed form) an element whose Jacobian
      // inverse stays in FP64
      const bool precise = (cw.x & 0x8000u) != 0;
      ln[0] = cw.x & 0x7fff; ln[1] = cw.x >> 16; ln[2] = cw.y & 0xffff; ln[3] = cw.y >> 16;
      S sd_in[12];
#pragma unroll
      for (int q = 0; q < 12; ++q) sd_in[q] = bs[q * THREADS + tid];
      vms_element<MIXED, S>(B, PC, tm.elem_begin + le, ln, precise, s_rec, sd_in, pq, pending, first_dual, inv_dt,
                            c1nu, nu4, lres);
      if (B.diag_res) {
#pragma unroll
        for (int r = 0; r < 16; ++r) B.diag_res[(int64_t)r * E + tm.elem_begin + le] = lres[r >> 2][r & 3];
      }
    }
    if constexpr (MIXED) {
      // the mixed form's residual region is its own, so the barrier that lets
      // it be overwritten (owners of the previous chunk done) comes after
      // this chunk's element work: warps that finish the previous chunk's
      // accumulation early go on with their elements instead of waiting
      if (k > 0) __syncthreads();
      if (active) {
        double2* Rt = R2 + tid * 8;
#pragma unroll
        for (int q = 0; q < 8; ++q)
          Rt[q ^ (tid & 7)] = make_double2(lres[q >> 1][2 * (q & 1)], lres[q >> 1][2 * (q & 1) + 1]);
      }
      // any timed-out wait aborts here, before the accumulation
      if (__syncthreads_or(!arrived)) {
        if (tid == 0) s_abort = 1;
        break;
      }
    } else {
      if (active) {
#pragma unroll
        for (int r = 0; r < 16; ++r) R[r * THREADS + tid] = lres[r >> 2][r & 3];
      }
      __syncthreads();
    }
    // owners add this chunk's contributions to their nodes, in element order
#pragma unroll
    for (int j = 0; j < MAXOWN; ++j) {
      const int ln = owned_node(tid, j);
      int c = cur[j];
      const int ce = endi[j];
      int ent = nxt[j];
      // nodes without an entry in this chunk leave their accumulators alone
      if (c < ce && (ent >> 2) - base < THREADS) {
        double a0 = s_a0[ln], a1 = s_a1[ln], a2 = s_a2[ln], a3 = s_a3[ln];
        // the residual entries of incidence entry e (of this chunk)
        auto fetch = [&](int e, double v[4]) {
          const int col = (e >> 2) - base;
          if constexpr (MIXED) {
            const double2* Rc = R2 + col * 8;
            const int q0i = 2 * (e & 3), sw = col & 7;
            const double2 q0 = Rc[q0i ^ sw], q1 = Rc[(q0i + 1) ^ sw];
            v[0] = q0.x; v[1] = q0.y; v[2] = q1.x; v[3] = q1.y;
          } else {
            const double* Rp = R + (e & 3) * 4 * THREADS + col;  // rows 4*corner .. 4*corner+3
            v[0] = Rp[0]; v[1] = Rp[THREADS]; v[2] = Rp[2 * THREADS]; v[3] = Rp[3 * THREADS];
          }
        };
        // two entries a pass (their loads overlap), added in element order;
        // the entries after them are loaded one pass ahead
        while (true) {
          const int ent1 = s_inc[c + 1 < ce ? c + 1 : c];
          const int ent2 = s_inc[c + 2 < ce ? c + 2 : c];
          const bool two = c + 1 < ce && (ent1 >> 2) - base < THREADS;
          double v[4], w[4];
          fetch(ent, v);
          fetch(two ? ent1 : ent, w);
          a0 += v[0]; a1 += v[1]; a2 += v[2]; a3 += v[3];
          if (!two) {
            ++c;
            ent = ent1;
            break;
          }
          a0 += w[0]; a1 += w[1]; a2 += w[2]; a3 += w[3];
          c += 2;
          ent = ent2;
          if (c >= ce || (ent >> 2) - base >= THREADS) break;
        }
        cur[j] = c;
        nxt[j] = ent;
        s_a0[ln] = a0; s_a1[ln] = a1; s_a2[ln] = a2; s_a3[ln] = a3;
      }
    }
    // FP64 end of chunk: stage buffer k&1 (holding this chunk's residuals) is
    // free again; any timed-out wait aborts
    if constexpr (!MIXED) {
      if (__syncthreads_or(!arrived)) {
        if (tid == 0) s_abort = 1;
        break;
      }
    }
  }
  __syncthreads();
  if (s_abort) {
    // a copy never completed: wait (bounded) for the copies this CTA issued,
    // report, and leave the tile's nodes untouched
    if (tid == 0) {
      for (int j = k; j < nchunks && j <= k + 1; ++j)
        mbar_wait_bounded(&bars[j & 1], (uint32_t)((j >> 1) & 1), FM_DRAIN_LIMIT);
      B.pstate[pidx].status = FM_ERR_TIMEOUT;
    }
    return;
  }
  int32_t status = FM_OK;
#pragma unroll
  for (int j = 0; j < MAXOWN; ++j) {
    const int ln2 = tid + j * THREADS;
    if (ln2 >= tm.n_node) break;
    const double acc[4] = {s_a0[ln2], s_a1[ln2], s_a2[ln2], s_a3[ln2]};
    if (ln2 < tm.n_int) {
      const double2 r1 = s_rec[rec_index(ln2, 1)], r2 = s_rec[rec_index(ln2, 2)], r3 = s_rec[rec_index(ln2, 3)];
      const int g = (int)(__double_as_longlong(r3.y) & 0x7fffffffll);
      const double post[4] = {r1.y, r2.x, r2.y, r3.x};
      vms_node_update(B, PC, pidx, st.iter, st.time, g, post, acc, first_dual, &status);
    } else {
      const int s = tm.slot_base + (ln2 - tm.n_int);
      B.part[2 * s] = make_double2(acc[0], acc[1]);
      B.part[2 * s + 1] = make_double2(acc[2], acc[3]);
    }
  }
  if (status != FM_OK) B.pstate[pidx].status = status;
}

__global__ void vms_iface_kernel(DevBatch B) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B.n_iface; i += gridDim.x * blockDim.x) {
    // the entry's fields load together with its problem id (a free entry's
    // are read but not used), so they do not wait for the state check
    const int pidx = B.iface_prob[i];
    const int g = B.iface_node[i];
    const int k0 = B.iface_slot_beg[i], k1 = k0 + B.iface_slot_cnt[i];
    if (pidx < 0) continue;  // free interface entry
    // the partials are loaded before the state check (an active entry's
    // slots are valid whatever the problem's state)
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    sum_partials(B, k0, k1, acc);
    const DevProbState st = B.pstate[pidx];
    if (st.iter >= B.target[pidx] || st.status != FM_OK) continue;
    const DevProb& P = B.probs[pidx];
    const bool first_dual = (st.iter % (P.ndual + 1)) == 0;
    const double post[4] = {B.su[g], B.sv[g], B.sw[g], B.sp[g]};
    int32_t status = FM_OK;
    vms_node_update(B, P, pidx, st.iter, st.time, g, post, acc, first_dual, &status);
    if (status != FM_OK) B.pstate[pidx].status = status;
  }
  finish_iteration(B);
}

// Partition parts, first half of the interface pass: interface nodes that
// are not shared with other parts are updated as in vms_iface_kernel; the
// shared ones put their sums into the part's slice of the exchange buffer.
__global__ void vms_xpack_kernel(DevBatch B) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B.n_iface; i += gridDim.x * blockDim.x) {
    const int pidx = B.iface_prob[i];
    if (pidx < 0) continue;
    const DevProbState st = B.pstate[pidx];
    if (st.iter >= B.target[pidx] || st.status != FM_OK) continue;
    const DevProb& P = B.probs[pidx];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    sum_partials(B, B.iface_slot_beg[i], B.iface_slot_beg[i] + B.iface_slot_cnt[i], acc);
    const int xi = B.iface_xidx[i];
    if (xi >= 0) {
      double* d = B.xsend + ((int64_t)P.xslice * B.x_n + xi) * 4;
      d[0] = acc[0]; d[1] = acc[1]; d[2] = acc[2]; d[3] = acc[3];
      continue;
    }
    const bool first_dual = (st.iter % (P.ndual + 1)) == 0;
    const int g = B.iface_node[i];
    const double post[4] = {B.su[g], B.sv[g], B.sw[g], B.sp[g]};
    int32_t status = FM_OK;
    vms_node_update(B, P, pidx, st.iter, st.time, g, post, acc, first_dual, &status);
    if (status != FM_OK) B.pstate[pidx].status = status;
  }
}

// Second half: the shared nodes, from the sums over all parts; then the
// iteration is complete.
__global__ void vms_xupdate_kernel(DevBatch B) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < B.n_xentries; j += gridDim.x * blockDim.x) {
    const int i = B.x_entries[j];
    const int pidx = B.iface_prob[i];
    if (pidx < 0) continue;
    const DevProbState st = B.pstate[pidx];
    if (st.iter >= B.target[pidx] || st.status != FM_OK) continue;
    const DevProb& P = B.probs[pidx];
    const int xi = B.iface_xidx[i];
    const double acc[4] = {exchange_sum(B, xi, 0), exchange_sum(B, xi, 1), exchange_sum(B, xi, 2), exchange_sum(B, xi, 3)};
    const bool first_dual = (st.iter % (P.ndual + 1)) == 0;
    const int g = B.iface_node[i];
    const double post[4] = {B.su[g], B.sv[g], B.sw[g], B.sp[g]};
    int32_t status = FM_OK;
    vms_node_update(B, P, pidx, st.iter, st.time, g, post, acc, first_dual, &status);
    if (status != FM_OK) B.pstate[pidx].status = status;
  }
  finish_iteration(B);
}

// ---- diagnostics of the reference's VMS log line and res_v / res_p output ----
// eval_centroid_residuals (src/femVMSExplicitFluidSolver.cpp:699-711) reads
// the nodal residual right after each element's assembly, so element e sees,
// at each of its nodes, the sum of the contributions of the elements up to e
// in the reference's element order.  ent lists, per problem node, its
// (batch element slot * 4 + corner) entries in that order; cres receives the
// running sum at every entry.
__global__ void vms_diag_prefix_kernel(const double* res, int64_t E, const int32_t* off, const int32_t* ent,
                                       int32_t n_nodes, double* cres) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += gridDim.x * blockDim.x) {
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (int j = off[i]; j < off[i + 1]; ++j) {
      const int32_t q = ent[j];
      const int64_t k = q >> 2;
      const int c = q & 3;
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        a[d] += res[(int64_t)(c * 4 + d) * E + k];
        cres[(k * 4 + c) * 4 + d] = a[d];
      }
    }
  }
}

// Centroid residuals (the quarter-weighted running sums at the element's four
// nodes, in corner order) into el (problem element order, 4 values each), and
// the block maxima of |res_u| and |res_p| (eval_residual_norms, src lines
// 774-793) into blk[2 * block].
__global__ void vms_diag_centroid_kernel(const double* cres, const int32_t* eo, int64_t eb, int64_t ec, double* el,
                                         double* blk) {
  __shared__ double s_u[256], s_p[256];
  double mu = 0.0, mp = 0.0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < ec; k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t e = eo[k];
    if (e < 0) continue;
    double r[4] = {0.0, 0.0, 0.0, 0.0};
    const double* c = cres + (eb + k) * 16;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int d = 0; d < 4; ++d) r[d] += c[a * 4 + d] * 0.25;
#pragma unroll
    for (int d = 0; d < 4; ++d) el[(int64_t)e * 4 + d] = r[d];
    const double nu = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    mu = nu > mu ? nu : mu;
    mp = fabs(r[3]) > mp ? fabs(r[3]) : mp;
  }
  s_u[threadIdx.x] = mu;
  s_p[threadIdx.x] = mp;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s_u[threadIdx.x] = fmax(s_u[threadIdx.x], s_u[threadIdx.x + w]);
      s_p[threadIdx.x] = fmax(s_p[threadIdx.x], s_p[threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    blk[2 * blockIdx.x] = s_u[0];
    blk[2 * blockIdx.x + 1] = s_p[0];
  }
}

// Largest nodal velocity magnitude of the state before BCs (the CFL of the
// reference's log line reads sol_n after update_dual_solution, src lines
// 1202-1208); block maxima into blk[block].
__global__ void vms_diag_vmax_kernel(DevBatch B, int64_t nb, int64_t n, double* blk) {
  __shared__ double s_m[256];
  double m = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = nb + i;
    const bool bc = B.node_bc[g] >= 0;
    const double u = bc ? B.pu[g] : B.su[g], v = bc ? B.pv[g] : B.sv[g], w = bc ? B.pw[g] : B.sw[g];
    const double a = sqrt(u * u + v * v + w * w);
    m = a > m ? a : m;
  }
  s_m[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s_m[threadIdx.x] = fmax(s_m[threadIdx.x], s_m[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) blk[blockIdx.x] = s_m[0];
}

// One problem's diagnostics after an iteration: out[0 .. 2*blocks) the
// centroid maxima per block, out[2*blocks .. 3*blocks) the velocity maxima.
cudaError_t launch_vms_diagnostics(const DevBatch& B, const double* cres_buf, const int32_t* off, const int32_t* ent,
                                   int32_t n_nodes, const int32_t* eo, int64_t eb, int64_t ec, int64_t nb,
                                   double* el, double* out, int blocks, cudaStream_t s) {
  const int pb = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)n_nodes + 255) / 256, 148 * 8));
  vms_diag_prefix_kernel<<<pb, 256, 0, s>>>(B.diag_res, B.E, off, ent, n_nodes, const_cast<double*>(cres_buf));
  vms_diag_centroid_kernel<<<blocks, 256, 0, s>>>(cres_buf, eo, eb, ec, el, out);
  vms_diag_vmax_kernel<<<blocks, 256, 0, s>>>(B, nb, n_nodes, out + 2 * blocks);
  return cudaGetLastError();
}

size_t vms_smem_bytes(int tn_max, int inc_max, int threads, bool mixed) {
  const size_t tn_pad = (size_t)((tn_max + 1) & ~1);
  const size_t stage = threads == 256 ? (mixed ? vms_stage_bytes<256, true>() : vms_stage_bytes<256, false>())
                                      : (mixed ? vms_stage_bytes<128, true>() : vms_stage_bytes<128, false>());
  return tn_pad * 12 * sizeof(double) + stage + (size_t)inc_max * sizeof(uint16_t) + (tn_pad + 2) * sizeof(uint16_t);
}

// Register-budget variants of the tile kernel: (threads, mixed, CTAs an SM).
// The first variant of each (threads, mixed) pair is the default.
#define FM_VMS_VARIANTS(X) \
  X(128, false, 3) X(128, false, 4) X(128, true, 4) X(128, true, 5) X(256, false, 1) X(256, false, 2) X(256, true, 2)

int vms_default_ctas(int threads, bool mixed) { return threads == 256 ? (mixed ? 2 : 1) : (mixed ? 4 : 3); }

bool vms_variant_exists(int threads, bool mixed, int ctas) {
#define FM_VMS_HAS(T, M, C) \
  if (threads == T && mixed == M && ctas == C) return true;
  FM_VMS_VARIANTS(FM_VMS_HAS)
#undef FM_VMS_HAS
  return false;
}

// One dual iteration: tile kernel, then the interface pass (xpack: its first
// half for a batch of partition parts; launch_vms_xupdate completes it).
cudaError_t launch_vms_iteration(const DevBatch& B, int tn_max, int inc_max, int threads, int ctas, int iface_blocks,
                                 bool mixed, bool xpack, cudaStream_t s, cudaEvent_t* ev) {
  const size_t smem = vms_smem_bytes(tn_max, inc_max, threads, mixed);
  if (ctas <= 0) ctas = vms_default_ctas(threads, mixed);
  if (ev) cudaEventRecord(ev[0], s);
  bool launched = false;
#define FM_VMS_LAUNCH(T, M, C)                                                       \
  if (!launched && threads == T && mixed == M && ctas == C) {                        \
    vms_tile_kernel<T, M, C><<<B.n_tiles, T, smem, s>>>(B, tn_max, inc_max);         \
    launched = true;                                                                 \
  }
  FM_VMS_VARIANTS(FM_VMS_LAUNCH)
#undef FM_VMS_LAUNCH
  if (!launched) return cudaErrorInvalidValue;
  if (ev) cudaEventRecord(ev[1], s);
  if (xpack)
    vms_xpack_kernel<<<iface_blocks, 256, 0, s>>>(B);
  else
    vms_iface_kernel<<<iface_blocks, 256, 0, s>>>(B);
  if (ev) cudaEventRecord(ev[2], s);
  return cudaGetLastError();
}

cudaError_t launch_vms_xupdate(const DevBatch& B, int blocks, cudaStream_t s) {
  vms_xupdate_kernel<<<blocks, 256, 0, s>>>(B);
  return cudaGetLastError();
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

// Raises the tile kernels' dynamic shared-memory limit to the device's
// opt-in maximum (the attribute is per kernel and process-wide, so a batch
// with small tiles must not lower it below what another batch launches with;
// the shared-memory carve-out still follows each launch's actual size).
cudaError_t vms_configure(int tn_max, int inc_max) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  (void)tn_max;  // sizes are checked against the limit by the caller
  (void)inc_max;
#define FM_VMS_RAISE(T, M, C) \
  if (e == cudaSuccess) e = raise_dyn_smem(vms_tile_kernel<T, M, C>, optin);
  FM_VMS_VARIANTS(FM_VMS_RAISE)
#undef FM_VMS_RAISE
  return e;
}

}  // namespace fm
