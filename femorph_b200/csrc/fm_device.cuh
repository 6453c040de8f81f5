// Device-side batch view and helpers shared by the VMS and SUPG kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fm_internal.hpp"

namespace fm {

// Pointers of one device-resident batch (all in batch numbering).
struct DevBatch {
  // nodes
  const double *x, *y, *z;        // coordinates
  double *su, *sv, *sw, *sp;      // state after BCs
  double *pu, *pv, *pw, *pp;      // state before BCs (read only at BC nodes)
  const double* mass;             // VMS nd_mass / SUPG row-sum mass (one per node)
  const int32_t* node_bc;         // BC record or -1
  const BCRec* recs;
  const int32_t* tab_off;
  const int32_t* tab_len;
  const double* tab_rows;
  // elements
  const uint16_t* conn;           // local node ids, n_elems x npe
  double* sdus;                   // VMS subscales [12][E] ; SUPG AB2 history [24][E]
  float* sdus32;                  // VMS mixed: FP32 subscales [12][E]
  double* el_lam;                 // SUPG per-element lambda / regime (diagnostics)
  double* el_reg;
  double* diag_res;               // VMS diagnostics on: [16][E] residual entries of the last iteration (else null)
  double* geo;                    // SUPG hexa8 FP64: [8 * FM_GEO_PER_GP][E] Gauss-point geometry (else null)
  float* geo32;                   // SUPG hexa8 mixed: the same, rounded to FP32 (else null)
  int64_t E;
  // tiles
  const TileMeta* tiles;
  int32_t n_tiles;
  const int32_t* tile_nodes;
  const int32_t* tile_cols;
  const uint16_t* tile_inc;       // per tile: node -> (element*npe + corner) entries, element order
  const uint16_t* tile_off;       // per tile: n_node+1 offsets into tile_inc
  // interface
  double2* part;                  // [slot][2]: (c0, c1) (c2, c3), one 32-byte sector a slot
  const int32_t* iface_node;
  const int32_t* iface_slot_beg;  // first partial-slot entry of each interface node
  const int32_t* iface_slot_cnt;  // number of entries
  const int32_t* iface_slots;
  const int32_t* iface_prob;      // problem slot, -1 for a free entry
  int32_t n_iface;
  // problems
  const DevProb* probs;
  DevProbState* pstate;
  const int32_t* target;         // [prob] iteration count to reach
  double* q1p;                    // [prob][2][4] pre-BC pressures of nodes 0..3
  int32_t n_probs;
  unsigned int* done;             // block counter of the interface pass
  // partition exchange (null / 0 in a batch without partition parts)
  const int32_t* iface_xidx;      // exchange index of each interface entry (-1: none)
  const int32_t* x_entries;       // the interface entries that have one
  int32_t n_xentries;
  int32_t x_n;                    // length of the partition's exchange list
  int32_t x_slices;               // one slice per part in the batch
  double* xsend;                  // [x_slices][x_n][4] partial sums of this batch's parts
  const double* xrecv;            // the same, summed over all processes (xsend when all parts are here)
  // polls of a tile CTA's wait for one chunk's bulk copies before it gives
  // up with FM_ERR_TIMEOUT (FM_WAIT_LIMIT unless fm_batch_set_wait_limit)
  uint32_t wait_limit;
  // tile CTAs ask L2 for tile blockIdx.x + l2_ahead's element rows and
  // interior-node ranges (0: off)
  int32_t l2_ahead;
};

// Sum over the part slices of exchange entry xi (component c).
__device__ __forceinline__ double exchange_sum(const DevBatch& B, int xi, int c) {
  double a = 0.0;
  for (int q = 0; q < B.x_slices; ++q) a += B.xrecv[((int64_t)q * B.x_n + xi) * 4 + c];
  return a;
}

// ---- bulk asynchronous copies global -> shared (cp.async.bulk, sm_90+) ----
// Plain (non-multicast) 1D bulk copies completing on a CTA-local mbarrier.
// Addresses must be 16-byte aligned and sizes a multiple of 16 bytes.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// orders this thread's prior generic-proxy shared accesses (after a CTA
// barrier: every thread's) before later async-proxy writes
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Asks L2 for bytes (a multiple of 16) from a 16-byte aligned global
// address; nothing waits for it.
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  if (bytes) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Polls at most `limit` times (each try_wait may itself suspend for a
// bounded, hardware-defined time); false when the phase did not complete.
// FM_WAIT_LIMIT (fm_internal.hpp) is the default limit of the chunk waits.
constexpr uint32_t FM_DRAIN_LIMIT = 1u << 16;  // a timed-out CTA's wait for its own copies
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// ---- reciprocal, inverse cube root and square root ----
// Seeds from the PTX approximate FP32 instructions (rcp/lg2/ex2/rsqrt
// .approx, relative error below 2^-21), then one correction in FP64.  With
// e = 1 - x y0 (reciprocal) or e = 1 - x y0^3 (inverse cube root) the exact
// result is y0 / (1 - e) = y0 (1 + e + e^2 + ...), resp.
// y0 (1 - e)^(-1/3) = y0 (1 + e/3 + 2 e^2 / 9 + 14 e^3 / 81 + ...); the
// series is cut after the e^2 term (Householder's third-order step), which
// with |e| < 2^-19 leaves a truncation below 2^-57, so the result is within
// about one ulp of the correctly rounded value in one dependent step less
// than two Newton steps.  The square root takes a Newton step on its inverse
// and one on the root itself.
__device__ __forceinline__ float ptx_rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ptx_lg2_approx(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ptx_ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ptx_rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// 1/x; the seed path needs |x| inside the FP32 normal range, other values
// take the IEEE division.
__device__ __forceinline__ double rcp_nr(double x) {
  const double ax = fabs(x);
  if (!(ax > 1e-37 && ax < 1e37)) return 1.0 / x;
  const double y = (double)ptx_rcp_approx((float)x);
  const double e = fma(-x, y, 1.0);
  return fma(y, fma(e, e, e), y);
}
// x^(-1/3) for x > 0 (third-order step above); the FP32 form below takes
// one Newton step, y <- y + y (1 - x y^3) / 3.
__device__ __forceinline__ double rcbrt_nr(double x) {
  if (!(x > 1e-37 && x < 1e37)) return rcbrt(x);
  const double y = (double)ptx_ex2_approx(ptx_lg2_approx((float)x) * (-1.0f / 3.0f));
  const double e = fma(-x, y * y * y, 1.0);
  return fma(y, e * fma(e, 2.0 / 9.0, 1.0 / 3.0), y);
}
__device__ __forceinline__ float rcbrt_nr(float x) {
  float y = ptx_ex2_approx(ptx_lg2_approx(x) * (-1.0f / 3.0f));
  const float e = fmaf(-x, y * y * y, 1.0f);
  return fmaf(y * (1.0f / 3.0f), e, y);
}
// sqrt(x) for x >= 0: one Newton step on y = 1/sqrt(x),
// y <- y (3 - x y^2) / 2 (relative error ~2^-44), then s = x y and one
// Newton step on s itself with the exact residual x - s^2 (an FMA),
// s <- s + (x - s^2) y / 2, which leaves s within an ulp of sqrt(x).
__device__ __forceinline__ double sqrt_nr(double x) {
  if (!(x > 0.0)) return 0.0;
  if (!(x > 1e-37 && x < 1e37)) return sqrt(x);
  double y = (double)ptx_rsqrt_approx((float)x);
  y = y * fma(-0.5 * x, y * y, 1.5);
  const double s = x * y;
  return fma(fma(-s, s, x), 0.5 * y, s);
}

// femUtils.cpp:830-871 (interpTableData) with femUtils.cpp:818-828
// (interpVelocity).  Returns false when the time lies before the table.
__device__ __forceinline__ bool interp_table(double t, const double* tab, int n, double v[3]) {
  if (t >= tab[(n - 1) * 4 + 3]) {
    v[0] = tab[(n - 1) * 4 + 0];
    v[1] = tab[(n - 1) * 4 + 1];
    v[2] = tab[(n - 1) * 4 + 2];
    return true;
  }
  int count = 1;
  bool found = false;
  while (!found && count < n) {
    found = (t >= tab[(count - 1) * 4 + 3]) && (t < tab[count * 4 + 3]);
    if (!found) count++;
  }
  if (!found) return false;
  double t1 = tab[(count - 1) * 4 + 3], t2 = tab[count * 4 + 3];
  for (int c = 0; c < 3; ++c) {
    double v1 = tab[(count - 1) * 4 + c], v2 = tab[count * 4 + c];
    v[c] = __dadd_rn(v1, __dmul_rn(__ddiv_rn(__dsub_rn(v2, v1), __dsub_rn(t2, t1)), __dsub_rn(t, t1)));
  }
  return true;
}

// Applies a node's resolved BC to (u, v, w, p) at time t.
__device__ __forceinline__ void apply_bc(const DevBatch& B, int32_t rec, double t, double s[4], int32_t* status) {
  BCRec r = B.recs[rec];
  if (r.tab >= 0) {
    double v[3];
    if (interp_table(t, B.tab_rows + (int64_t)B.tab_off[r.tab] * 4, B.tab_len[r.tab], v)) {
      if (r.mask & BC_VX) s[0] = v[0];
      if (r.mask & BC_VY) s[1] = v[1];
      if (r.mask & BC_VZ) s[2] = v[2];
    } else {
      *status = FM_ERR_TABLE;
    }
  }
  if (r.mask & BC_PRES) s[3] = r.p;
  if (r.mask & BC_DIR) {
    s[0] = r.d[0];
    s[1] = r.d[1];
    s[2] = r.d[2];
  }
}

// Adds the tile partials of interface slots [k0, k1) to acc in slot (tile)
// order.  The slot ids, and then the partials, are loaded four at a time
// (past k1 the first id is loaded again and not added), so that their round
// trips overlap instead of following one another slot by slot.
__device__ __forceinline__ void sum_partials(const DevBatch& B, int k0, int k1, double acc[4]) {
  for (int k = k0; k < k1; k += 4) {
    int s[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) s[i] = B.iface_slots[k + i < k1 ? k + i : k];
    double2 q[4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      q[i][0] = B.part[2 * s[i]];
      q[i][1] = B.part[2 * s[i] + 1];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (k + i < k1) {
        acc[0] += q[i][0].x;
        acc[1] += q[i][0].y;
        acc[2] += q[i][1].x;
        acc[3] += q[i][1].y;
      }
  }
}

// Marks the end of one pass over the interface nodes.  The last block to
// finish (counter pattern: fence, ticket, no waiting) advances every active
// problem by one iteration and its time at the start of a new step.  A
// problem with a device error (status != FM_OK) stops where it is: the
// kernels skip it from then on, so its state stays that of the failed
// iteration.
__device__ __forceinline__ void finish_iteration(const DevBatch& B) {
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned int ticket = atomicAdd(B.done, 1u);
    s_last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (int p = threadIdx.x; p < B.n_probs; p += blockDim.x) {
    DevProbState st = B.pstate[p];
    if (st.iter < B.target[p] && st.status == FM_OK) {
      const int per_step = B.probs[p].ndual + 1;
      st.iter += 1;
      if (st.iter % per_step == 0) st.time = st.time + B.probs[p].dt;
      B.pstate[p].iter = st.iter;
      B.pstate[p].time = st.time;
    }
  }
  if (threadIdx.x == 0) *B.done = 0u;
}

}  // namespace fm
