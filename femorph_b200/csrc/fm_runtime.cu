// Device runtime and C ABI of femorph_b200.
//
// A batch owns device pools (nodes, element slots, tiles, interface entries,
// partial-sum slots, BC records, problem slots).  A problem is prepared on
// the host (its own tile layout, fm_problem_prepare) and placed into free
// ranges of the pools with its indices relocated (fm_batch_add); removing it
// marks its tiles and interface entries inactive and frees its ranges.  The
// kernels run over the pools' high-water marks and skip inactive entries, so
// problems can join and leave between launches (continuous batching) while
// every resident problem keeps its state on the device.  fm_batch_create
// sizes the pools exactly for a fixed set of problems.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "fm_device.cuh"
#include "fm_internal.hpp"

namespace fm {
const char* last_error();
size_t vms_smem_bytes(int tn_max, int inc_max, int threads, bool mixed);
cudaError_t vms_configure(int tn_max, int inc_max);
cudaError_t launch_vms_iteration(const DevBatch& B, int tn_max, int inc_max, int threads, int ctas, int iface_blocks,
                                 bool mixed, bool xpack, cudaStream_t s, cudaEvent_t* ev);
int vms_default_ctas(int threads, bool mixed);
bool vms_variant_exists(int threads, bool mixed, int ctas);
cudaError_t launch_vms_xupdate(const DevBatch& B, int blocks, cudaStream_t s);
cudaError_t launch_vms_diagnostics(const DevBatch& B, const double* cres_buf, const int32_t* off, const int32_t* ent,
                                   int32_t n_nodes, const int32_t* eo, int64_t eb, int64_t ec, int64_t nb,
                                   double* el, double* out, int blocks, cudaStream_t s);
size_t supg_smem_bytes(int tn_max, int inc_max, int npe, int threads);
cudaError_t supg_configure(size_t smem, int npe);
cudaError_t launch_supg_step(const DevBatch& B, int tn_max, int inc_max, int threads, int iface_blocks, int npe, bool mixed,
                             bool xpack, cudaStream_t s, cudaEvent_t* ev);
cudaError_t launch_supg_xupdate(const DevBatch& B, int blocks, cudaStream_t s);
cudaError_t launch_supg_geo(const DevBatch& B, int tile0, int ntiles, int tn_max, cudaStream_t s);
cudaError_t launch_supg_pressure(const DevBatch& B, int tn_max, int npe, double* pres, cudaStream_t s);
cudaError_t launch_supg_stats(const DevBatch& B, int tile0, int ntiles, int tn_max, int npe, double* out,
                              cudaStream_t s);
cudaError_t launch_velocity_extrema(const DevBatch& B, int64_t node_begin, int64_t n_nodes, int glob_fixed, int blocks,
                                    double* out, cudaStream_t s);

// Aspect ratio h_max / (2 sqrt(6) r_in) of a tet (1 for the regular tet,
// about 1.7 for a Kuhn tet); r_in = 3V / (sum of face areas).
static double tet_aspect_ratio(const double* X, const int32_t* c) {
  double p[4][3];
  for (int a = 0; a < 4; ++a)
    for (int k = 0; k < 3; ++k) p[a][k] = X[(int64_t)c[a] * 3 + k];
  auto sub = [](const double* a, const double* b, double* r) {
    for (int k = 0; k < 3; ++k) r[k] = a[k] - b[k];
  };
  auto cross_norm = [](const double* u, const double* v) {
    double x = u[1] * v[2] - u[2] * v[1], y = u[2] * v[0] - u[0] * v[2], z = u[0] * v[1] - u[1] * v[0];
    return std::sqrt(x * x + y * y + z * z);
  };
  double hmax = 0.0;
  for (int a = 0; a < 4; ++a)
    for (int b2 = a + 1; b2 < 4; ++b2) {
      double d[3];
      sub(p[a], p[b2], d);
      hmax = std::max(hmax, std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]));
    }
  double e1[3], e2[3], e3[3];
  sub(p[1], p[0], e1);
  sub(p[2], p[0], e2);
  sub(p[3], p[0], e3);
  const double vol6 = std::fabs(e1[0] * (e2[1] * e3[2] - e2[2] * e3[1]) - e1[1] * (e2[0] * e3[2] - e2[2] * e3[0]) +
                                e1[2] * (e2[0] * e3[1] - e2[1] * e3[0]));
  static const int f[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
  double area = 0.0;
  for (int k = 0; k < 4; ++k) {
    double u[3], v[3];
    sub(p[f[k][1]], p[f[k][0]], u);
    sub(p[f[k][2]], p[f[k][0]], v);
    area += 0.5 * cross_norm(u, v);
  }
  if (!(vol6 > 0.0)) return 1e300;
  const double r_in = 3.0 * (vol6 / 6.0) / area;
  return hmax / (2.0 * std::sqrt(6.0) * r_in);
}

// Aspect ratio of a hexa8 (corner order of femHexa8: bottom face 0-3, top
// face 4-7): longest over shortest of its 12 edges (1 for a cube).
static double hexa_aspect_ratio(const double* X, const int32_t* c) {
  static const int ed[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  double lo = 1e300, hi = 0.0;
  for (int k = 0; k < 12; ++k) {
    double s = 0.0;
    for (int d = 0; d < 3; ++d) {
      const double v = X[(int64_t)c[ed[k][0]] * 3 + d] - X[(int64_t)c[ed[k][1]] * 3 + d];
      s += v * v;
    }
    lo = std::min(lo, s);
    hi = std::max(hi, s);
  }
  if (!(lo > 0.0)) return 1e300;
  return std::sqrt(hi / lo);
}

// First-fit range allocator over [0, cap) with coalescing free list.
struct Pool {
  int64_t cap = 0, hwm = 0;
  std::map<int64_t, int64_t> free;  // offset -> length
  void init(int64_t c) {
    cap = c;
    hwm = 0;
    free.clear();
    if (c > 0) free[0] = c;
  }
  bool alloc(int64_t len, int64_t align, int64_t* off) {
    if (len <= 0) {
      *off = 0;
      return true;
    }
    for (auto it = free.begin(); it != free.end(); ++it) {
      const int64_t o = it->first, l = it->second;
      const int64_t a = (o + align - 1) / align * align;
      if (a + len <= o + l) {
        free.erase(it);
        if (a > o) free[o] = a - o;
        if (a + len < o + l) free[a + len] = o + l - (a + len);
        *off = a;
        hwm = std::max(hwm, a + len);
        return true;
      }
    }
    return false;
  }
  void release(int64_t off, int64_t len) {
    if (len <= 0) return;
    auto it = free.emplace(off, len).first;
    auto nx = std::next(it);
    if (nx != free.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free.erase(nx);
    }
    if (it != free.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free.erase(it);
      }
    }
    // the high-water mark drops when the top of the pool is free again
    auto last = free.empty() ? free.end() : std::prev(free.end());
    if (last != free.end() && last->first + last->second == cap) hwm = std::min(hwm, last->first);
  }
};

enum PoolId { P_NODE, P_ELEM, P_TILE, P_TNODE, P_TCOL, P_TINC, P_TOFF, P_SLOT, P_IFACE, P_ISLOT, P_REC, P_TAB, P_ROW, P_PROB,
              P_COUNT };

struct Placement {
  fm_problem* p = nullptr;
  int64_t off[P_COUNT] = {0};
  int64_t len[P_COUNT] = {0};
  int32_t tn_max = 0, inc_max = 0;
  std::shared_ptr<Layout> L;  // the problem's layout (node and element numbering)
  // VMS diagnostics (device, own allocations): per problem node its
  // (element slot * 4 + corner) entries in the problem's element order, the
  // problem element of each slot, and the centroid residuals (E x 4)
  int32_t *dg_off = nullptr, *dg_ent = nullptr, *dg_eo = nullptr;
  double* dg_el = nullptr;
};

// Blocks of the diagnostics reductions.
constexpr int DIAG_BLOCKS = 148 * 4;

}  // namespace fm

using namespace fm;

struct fm_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  int solver = 0, npe = 4, precision = 0;
  fm_tuning tune{};
  Pool pools[P_COUNT];
  std::vector<Placement> slots;     // by problem slot (P_PROB offset)
  DevBatch D{};
  std::vector<void*> allocs;
  int tn_max = 0, inc_max = 0, threads = 128, iface_blocks = 1, graph_steps = 0;
  int configured_tn = 0, configured_inc = 0;
  bool has_history = false;
  std::vector<int32_t> iters;       // host copy of each slot's completed iterations
  int32_t* h_targets = nullptr;     // pinned staging of the target array
  cudaEvent_t ev_tgt = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int64_t last_launches = 0;
  bool timed = false;
  cudaGraphExec_t graph = nullptr;
  int graph_iters = 0;
  double* d_scratch = nullptr;
  double* d_stats = nullptr;   // per-CTA partial results of the log reductions
  // partition parts (fm_problem_partition): the batch holds x_slices parts
  // of one partition; external when the others live in other processes,
  // whose partial sums the caller adds between fm_batch_exchange_begin and
  // fm_batch_exchange_end
  bool exchange = false, x_external = false, x_open = false;
  bool x_free_targets = false;      // device targets left open by fm_batch_exchange_begin
  int32_t x_slices = 0, x_blocks = 1;
  int64_t x_n = 0;
  std::vector<int32_t> x_slice_of;  // by problem slot
  // VMS diagnostics (fm_batch_set_diagnostics): residual entries of the last
  // iteration (16 x element slots), running sums (element slots x 16),
  // per-block maxima and their pinned host copy
  bool diag = false;
  double *d_diag_res = nullptr, *d_cres = nullptr, *d_diag_out = nullptr, *h_diag = nullptr;
};

#define CK(x)                                                                                     \
  do {                                                                                            \
    cudaError_t _e = (x);                                                                         \
    if (_e != cudaSuccess) return fail(FM_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)); \
  } while (0)

static int dalloc(fm_batch* b, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(e == cudaErrorMemoryAllocation ? FM_ERR_OOM : FM_ERR_CUDA,
                std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  b->allocs.push_back(*p);
  return FM_OK;
}

static void release_all(fm_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  for (void* p : b->allocs) cudaFree(p);
  b->allocs.clear();
  if (b->h_targets) cudaFreeHost(b->h_targets);
  if (b->ev_tgt) cudaEventDestroy(b->ev_tgt);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
}

template <class T>
static int put(T* dev_base, int64_t off, const T* src, int64_t n, cudaStream_t s) {
  if (n <= 0) return FM_OK;
  CK(cudaMemcpyAsync(dev_base + off, src, sizeof(T) * (size_t)n, cudaMemcpyHostToDevice, s));
  return FM_OK;
}

// Default launch shape (measured on the 96^3 cavity and the hexa channel):
// VMS FP64 1024-tet tiles (3 CTAs/SM, register bound), VMS mixed 512-tet
// tiles (4 CTAs/SM fit the shared memory), SUPG hexa8 384 elements.
static void default_tuning(int solver, int npe, int precision, fm_tuning& t) {
  if (t.threads != 128 && t.threads != 256) t.threads = 128;
  const bool vms_mixed = solver == FM_SOLVER_VMS && precision == FM_MIXED;
  if (t.tile_elems <= 0) t.tile_elems = (npe == 8) ? 384 : (vms_mixed ? 512 : 1024);
  if (t.tile_nodes <= 0) t.tile_nodes = (npe == 8) ? 640 : (vms_mixed ? 256 : 512);
  if (t.tile_nodes > 4096) t.tile_nodes = 4096;
  if (solver == FM_SOLVER_VMS && t.tile_nodes > FM_MAX_TILE_NODES) t.tile_nodes = FM_MAX_TILE_NODES;
  if (t.graph_steps < 0) t.graph_steps = 0;
}

// Builds (or reuses) the problem's own tile layout for the given tile sizes.
// Touches only this problem, so different problems may be prepared on
// different host threads while a batch runs.
static int prepare(fm_problem* p, int te, int tn, std::shared_ptr<Layout>* out) {
  if (p->layout && p->layout_te == te && p->layout_tn == tn) {
    *out = p->layout;
    return FM_OK;
  }
  std::shared_ptr<Layout> L = std::make_shared<Layout>();
  fm_problem* arr[1] = {p};
  int r = build_layout(arr, 1, te, tn, *L);
  if (r) return r;
  if (p->params.precision == FM_MIXED) {
    // mixed form: elements whose Jacobian inverse stays in FP64 (aspect ratio
    // above the limit) are flagged in bit 15 of their first tile-local node id
    const int npe = p->etype;
    const int64_t EC = L->elem_count[0];
    const int nw = (int)std::max<int64_t>(1, std::min<int64_t>({32, (int64_t)std::thread::hardware_concurrency(),
                                                                  EC / 16384}));
    std::vector<std::thread> th;
    for (int w = 0; w < nw; ++w)
      th.emplace_back([&, w] {
        for (int64_t k = EC * w / nw; k < EC * (w + 1) / nw; ++k) {
          const int32_t oe = L->elem_old[0][k];
          if (oe < 0) continue;
          const int32_t* c = &p->conn[(int64_t)oe * npe];
          const double ar =
              npe == 4 ? tet_aspect_ratio(p->coords.data(), c) : hexa_aspect_ratio(p->coords.data(), c);
          if (ar > FM_MIXED_ASPECT_LIMIT) L->conn_local[(size_t)k * npe] |= 0x8000;
        }
      });
    for (auto& x : th) x.join();
  }
  p->layout = L;
  p->layout_te = te;
  p->layout_tn = tn;
  *out = L;
  return FM_OK;
}

// Sizes of one prepared problem in each pool.
static void pool_sizes(const fm_problem* p, const Layout& L, int64_t len[P_COUNT]) {
  len[P_NODE] = p->N;
  len[P_ELEM] = L.n_elems;  // includes the trailing over-read padding
  len[P_TILE] = (int64_t)L.tiles.size();
  len[P_TNODE] = (int64_t)L.tile_nodes.size();
  len[P_TCOL] = (int64_t)L.tile_cols.size();
  len[P_TINC] = (int64_t)L.tile_inc.size();
  len[P_TOFF] = (int64_t)L.tile_off.size();
  len[P_SLOT] = L.n_slots;
  len[P_IFACE] = (int64_t)L.iface_node.size();
  len[P_ISLOT] = (int64_t)L.iface_slots.size();
  len[P_REC] = (int64_t)p->recs.size();
  len[P_TAB] = (int64_t)p->tab_off.size();
  len[P_ROW] = (int64_t)p->tab_rows.size() / 4;
  len[P_PROB] = 1;
}
static const int64_t kAlign[P_COUNT] = {1, ELEM_ALIGN, 1, 1, 1, 8, 1, 1, 1, 1, 1, 1, 1, 1};

// Allocates the device arrays for the given pool capacities.
static int allocate(fm_batch* b, const int64_t cap[P_COUNT]) {
  for (int k = 0; k < P_COUNT; ++k) b->pools[k].init(cap[k]);
  DevBatch& D = b->D;
  memset(&D, 0, sizeof(D));
  // element rows (subscales, connectivity) are bulk-copied from row q at
  // q * NE + (multiple of 32): NE must be a multiple of 32 too, so every row
  // start stays 16-byte aligned for FP32 and FP64 rows alike
  const int64_t NN = std::max<int64_t>(cap[P_NODE], 1);
  const int64_t NE = (std::max<int64_t>(cap[P_ELEM], 1) + ELEM_ALIGN - 1) / ELEM_ALIGN * ELEM_ALIGN;
  // one device allocation carved into every array (256-byte aligned): the
  // carving runs once to size the block and once to hand out the pointers
  double *x, *y, *z, *su, *sv, *sw, *sp, *pu, *pv, *pw, *pp, *ms;
  int32_t* nbc;
  uint16_t* conn;
  TileMeta* tiles;
  int32_t *tnodes, *tcols;
  uint16_t *tinc, *toff;
  int32_t *inode, *isb, *isc, *iprob, *islots;
  BCRec* recs;
  int32_t *toffs, *tlens;
  double* rows;
  DevProb* dp;
  DevProbState* ds;
  int32_t* tg;
  double* q1;
  uint32_t* done;
  int32_t* ixidx = nullptr;
  const int64_t NP = std::max<int64_t>(cap[P_PROB], 1);
  const int64_t xcount = b->exchange ? (int64_t)b->x_slices * b->x_n * 4 : 0;
  char* block = nullptr;
  size_t total = 0;
  auto A = [&](void** p, size_t bytes) {
    const size_t off = (total + 255) & ~(size_t)255;
    total = off + (bytes ? bytes : 16);
    *p = block ? block + off : nullptr;
  };
  auto carve = [&]() {
    total = 0;
    for (double** q : {&x, &y, &z, &su, &sv, &sw, &sp, &pu, &pv, &pw, &pp, &ms}) A((void**)q, NN * sizeof(double));
    A((void**)&nbc, NN * sizeof(int32_t));
    A((void**)&conn, (size_t)NE * b->npe * sizeof(uint16_t));
    if (b->solver == FM_SOLVER_VMS && b->precision == FM_MIXED) {
      A((void**)&D.sdus32, (size_t)NE * 12 * sizeof(float));
    } else if (b->solver == FM_SOLVER_VMS || b->has_history) {
      A((void**)&D.sdus, (size_t)NE * (b->solver == FM_SOLVER_VMS ? 12 : 3 * b->npe) * sizeof(double));
    }
    if (b->solver == FM_SOLVER_SUPG && b->npe == 8 && b->precision != FM_MIXED)
      A((void**)&D.geo, (size_t)NE * 8 * FM_GEO_PER_GP * sizeof(double));
    if (b->solver == FM_SOLVER_SUPG && b->npe == 8 && b->precision == FM_MIXED)
      A((void**)&D.geo32, (size_t)NE * 8 * FM_GEO_PER_GP * sizeof(float));
    if (b->solver == FM_SOLVER_SUPG) {
      A((void**)&D.el_lam, NE * sizeof(double));
      A((void**)&D.el_reg, NE * sizeof(double));
      A((void**)&b->d_scratch, NE * sizeof(double));
    }
    A((void**)&tiles, std::max<int64_t>(cap[P_TILE], 1) * sizeof(TileMeta));
    A((void**)&tnodes, std::max<int64_t>(cap[P_TNODE], 1) * sizeof(int32_t));
    A((void**)&tcols, std::max<int64_t>(cap[P_TCOL], 1) * sizeof(int32_t));
    A((void**)&tinc, std::max<int64_t>(cap[P_TINC], 8) * sizeof(uint16_t));
    A((void**)&toff, std::max<int64_t>(cap[P_TOFF], 1) * sizeof(uint16_t));
    A((void**)&D.part, std::max<int64_t>(cap[P_SLOT], 1) * 4 * sizeof(double));
    for (int32_t** q : {&inode, &isb, &isc, &iprob}) A((void**)q, std::max<int64_t>(cap[P_IFACE], 1) * sizeof(int32_t));
    A((void**)&islots, std::max<int64_t>(cap[P_ISLOT], 1) * sizeof(int32_t));
    A((void**)&recs, std::max<int64_t>(cap[P_REC], 1) * sizeof(BCRec));
    A((void**)&toffs, std::max<int64_t>(cap[P_TAB], 1) * sizeof(int32_t));
    A((void**)&tlens, std::max<int64_t>(cap[P_TAB], 1) * sizeof(int32_t));
    A((void**)&rows, std::max<int64_t>(cap[P_ROW], 1) * 4 * sizeof(double));
    A((void**)&dp, NP * sizeof(DevProb));
    A((void**)&ds, NP * sizeof(DevProbState));
    A((void**)&tg, NP * sizeof(int32_t));
    A((void**)&q1, NP * 8 * sizeof(double));
    A((void**)&done, sizeof(uint32_t));
    A((void**)&b->d_stats, std::max<int64_t>(cap[P_TILE], 256) * 11 * sizeof(double));
    if (b->exchange) {
      A((void**)&ixidx, std::max<int64_t>(cap[P_IFACE], 1) * sizeof(int32_t));
      A((void**)&D.xsend, std::max<int64_t>(xcount, 1) * sizeof(double));
      if (b->x_external) A((void**)&D.xrecv, std::max<int64_t>(xcount, 1) * sizeof(double));
    }
  };
  carve();
  int r = dalloc(b, (void**)&block, total);
  if (r) return r;
  carve();
  if (b->exchange) {
    D.iface_xidx = ixidx;
    D.x_n = (int32_t)b->x_n;
    D.x_slices = b->x_slices;
    if (!b->x_external) D.xrecv = D.xsend;
    CK(cudaMemset(ixidx, 0xff, std::max<int64_t>(cap[P_IFACE], 1) * sizeof(int32_t)));
    CK(cudaMemset(D.xsend, 0, std::max<int64_t>(xcount, 1) * sizeof(double)));
    if (b->x_external) CK(cudaMemset(const_cast<double*>(D.xrecv), 0, std::max<int64_t>(xcount, 1) * sizeof(double)));
  }
  D.x = x; D.y = y; D.z = z; D.su = su; D.sv = sv; D.sw = sw; D.sp = sp;
  D.pu = pu; D.pv = pv; D.pw = pw; D.pp = pp; D.mass = ms; D.node_bc = nbc;
  D.conn = conn; D.E = NE;
  D.tiles = tiles; D.tile_nodes = tnodes; D.tile_cols = tcols; D.tile_inc = tinc; D.tile_off = toff;
  D.iface_node = inode; D.iface_slot_beg = isb; D.iface_slot_cnt = isc; D.iface_prob = iprob; D.iface_slots = islots;
  D.recs = recs; D.tab_off = toffs; D.tab_len = tlens; D.tab_rows = rows;
  D.probs = dp; D.pstate = ds; D.target = tg; D.q1p = q1; D.done = done;
  D.wait_limit = FM_WAIT_LIMIT;
  // tile CTAs ask L2 for a tile this many CTAs ahead (measured: mixed VMS
  // two SM-counts, 0.460 -> 0.444 ms a step at 96^3; SUPG one SM-count, tet4
  // 96^3 0.797 -> 0.770 ms FP64 and 0.537 -> 0.511 ms mixed, hexa8 channel
  // -0.3% FP64 and -1.2% mixed; the FP64 VMS form gains nothing and keeps it
  // off)
  {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      sms = 148;
    if (b->solver == FM_SOLVER_SUPG) D.l2_ahead = sms;
    else if (b->precision == FM_MIXED) D.l2_ahead = 2 * sms;
  }
  // every slot starts inactive
  CK(cudaMemset(tiles, 0xff, std::max<int64_t>(cap[P_TILE], 1) * sizeof(TileMeta)));
  CK(cudaMemset(iprob, 0xff, std::max<int64_t>(cap[P_IFACE], 1) * sizeof(int32_t)));
  CK(cudaMemset(ds, 0, NP * sizeof(DevProbState)));
  CK(cudaMemset(tg, 0, NP * sizeof(int32_t)));
  CK(cudaMemset(q1, 0, NP * 8 * sizeof(double)));
  CK(cudaMemset(done, 0, sizeof(uint32_t)));
  b->iters.assign(NP, 0);
  b->slots.assign(NP, Placement());
  CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&b->ev0));
  CK(cudaEventCreate(&b->ev1));
  CK(cudaEventCreateWithFlags(&b->ev_tgt, cudaEventDisableTiming));
  CK(cudaMallocHost((void**)&b->h_targets, sizeof(int32_t) * NP));
  return FM_OK;
}

// Makes the kernels' shared-memory limits cover the current tile maxima.
static int configure(fm_batch* b) {
  if (b->tn_max <= b->configured_tn && b->inc_max <= b->configured_inc) return FM_OK;
  const int tn = std::max(b->tn_max, b->configured_tn), inc = std::max(b->inc_max, b->configured_inc);
  size_t smem = b->solver == FM_SOLVER_VMS ? vms_smem_bytes(tn, inc, b->threads, b->precision == FM_MIXED)
                                           : supg_smem_bytes(tn, inc, b->npe, b->threads);
  // 227 KB opt-in limit per block, less room for the kernels' static shared memory
  if (smem + 1024 > 227 * 1024) return fail(FM_ERR_INVALID, "tile too large for shared memory; lower tile_nodes");
  cudaError_t ce = b->solver == FM_SOLVER_VMS ? vms_configure(tn, inc) : supg_configure(smem, b->npe);
  if (ce != cudaSuccess) return fail(FM_ERR_CUDA, std::string("kernel attribute: ") + cudaGetErrorString(ce));
  b->configured_tn = tn;
  b->configured_inc = inc;
  return FM_OK;
}

static void refresh_extent(fm_batch* b) {
  DevBatch& D = b->D;
  D.n_tiles = (int32_t)b->pools[P_TILE].hwm;
  D.n_iface = (int32_t)b->pools[P_IFACE].hwm;
  D.n_probs = (int32_t)b->pools[P_PROB].hwm;
  b->iface_blocks = (int)std::max<int64_t>(1, std::min<int64_t>((D.n_iface + 255) / 256, 148 * 8));
  int tn = 0, inc = 0;
  for (const Placement& pl : b->slots)
    if (pl.p) {
      tn = std::max(tn, pl.tn_max);
      inc = std::max(inc, pl.inc_max);
    }
  b->tn_max = tn;
  b->inc_max = inc;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
}

// Places a prepared problem into the pools; FM_ERR_OOM if some pool has no
// room (nothing is changed then).
// ---- VMS diagnostics resources ----
static void diag_free_problem(Placement& pl) {
  cudaFree(pl.dg_off);
  cudaFree(pl.dg_ent);
  cudaFree(pl.dg_eo);
  cudaFree(pl.dg_el);
  pl.dg_off = pl.dg_ent = pl.dg_eo = nullptr;
  pl.dg_el = nullptr;
}

static void diag_free(fm_batch* b) {
  for (Placement& pl : b->slots) diag_free_problem(pl);
  cudaFree(b->d_diag_res);
  cudaFree(b->d_cres);
  cudaFree(b->d_diag_out);
  if (b->h_diag) cudaFreeHost(b->h_diag);
  b->d_diag_res = b->d_cres = b->d_diag_out = b->h_diag = nullptr;
  b->D.diag_res = nullptr;
  b->diag = false;
}

// The problem's reference-order incidence lists and output array.
static int diag_prepare_problem(Placement& pl) {
  const fm_problem* p = pl.p;
  const Layout& L = *pl.L;
  const auto& eo = L.elem_old[0];
  const int64_t N = p->N, E = p->E, EC = (int64_t)eo.size();
  if ((pl.off[P_ELEM] + EC) * 4 >= (int64_t)INT32_MAX)
    return fail(FM_ERR_INVALID, "diagnostics index element slots in 32 bits: batch too large");
  std::vector<int32_t> slot_of(E, -1), off(N + 1, 0), ent((size_t)E * 4), eo32(EC);
  for (int64_t k = 0; k < EC; ++k) {
    eo32[k] = eo[k];
    if (eo[k] >= 0) slot_of[eo[k]] = (int32_t)(pl.off[P_ELEM] + k);
  }
  for (int64_t q = 0; q < E * 4; ++q) off[p->conn[q] + 1]++;
  for (int64_t i = 0; i < N; ++i) off[i + 1] += off[i];
  std::vector<int32_t> pos(off.begin(), off.end() - 1);
  for (int64_t e = 0; e < E; ++e)
    for (int a = 0; a < 4; ++a) ent[pos[p->conn[e * 4 + a]]++] = slot_of[e] * 4 + a;
  // smallest pow(6 V, 1/3) over the elements (src/femVMSExplicitFluidSolver.cpp:947-952)
  double hmin = std::numeric_limits<double>::max();
  for (int64_t e = 0; e < E; ++e) {
    const double* x0 = &p->coords[(size_t)p->conn[e * 4] * 3];
    double j[3][3];
    for (int k = 0; k < 3; ++k) {
      const double* xk = &p->coords[(size_t)p->conn[e * 4 + k + 1] * 3];
      for (int i = 0; i < 3; ++i) j[i][k] = xk[i] - x0[i];
    }
    const double det = j[0][0] * (j[1][1] * j[2][2] - j[2][1] * j[1][2]) +
                       j[0][1] * (j[2][0] * j[1][2] - j[1][0] * j[2][2]) +
                       j[0][2] * (j[1][0] * j[2][1] - j[2][0] * j[1][1]);
    hmin = std::min(hmin, std::pow(6.0 * (det / 6.0), 1.0 / 3.0));
  }
  pl.p->diag_min_h = hmin;
  pl.p->diag_step = -1;
  auto al = [&](void** q, size_t bytes) { return cudaMalloc(q, bytes ? bytes : 16); };
  cudaError_t e = al((void**)&pl.dg_off, (N + 1) * sizeof(int32_t));
  if (e == cudaSuccess) e = al((void**)&pl.dg_ent, (size_t)E * 4 * sizeof(int32_t));
  if (e == cudaSuccess) e = al((void**)&pl.dg_eo, EC * sizeof(int32_t));
  if (e == cudaSuccess) e = al((void**)&pl.dg_el, (size_t)E * 4 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(pl.dg_off, off.data(), (N + 1) * sizeof(int32_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(pl.dg_ent, ent.data(), (size_t)E * 4 * sizeof(int32_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(pl.dg_eo, eo32.data(), EC * sizeof(int32_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(pl.dg_el, 0, (size_t)E * 4 * sizeof(double));
  if (e != cudaSuccess) {
    diag_free_problem(pl);
    return fail(e == cudaErrorMemoryAllocation ? FM_ERR_OOM : FM_ERR_CUDA,
                std::string("diagnostics: ") + cudaGetErrorString(e));
  }
  return FM_OK;
}

static int place(fm_batch* b, fm_problem* p, const std::shared_ptr<Layout>& Lp) {
  const Layout& L = *Lp;
  Placement pl;
  pl.p = p;
  pl.L = Lp;
  pool_sizes(p, L, pl.len);
  int k = 0;
  for (; k < P_COUNT; ++k)
    if (!b->pools[k].alloc(pl.len[k], kAlign[k], &pl.off[k])) break;
  if (k < P_COUNT) {
    for (int j = 0; j < k; ++j) b->pools[j].release(pl.off[j], pl.len[j]);
    return fail(FM_ERR_OOM, "batch capacity exhausted");
  }
  const int ps = (int)pl.off[P_PROB];
  const int64_t noff = pl.off[P_NODE], eoff = pl.off[P_ELEM], soff = pl.off[P_SLOT];
  cudaStream_t s = b->stream;
  DevBatch& D = b->D;
  const int npe = b->npe;
  int r = 0;
  // node data: coordinates, initial state after the time-0 BCs, mass, BC records
  const std::vector<int32_t>& nn = L.node_new[0];
  const int64_t N = p->N;
  hvec<double> hx(N), hy(N), hz(N), hu(N), hv(N), hw(N), hp(N), hm(N);
  hvec<int32_t> hbc(N);
  const bool has_init = !p->init.empty();
  std::atomic<bool> table_miss{false};
  // every node writes its own batch slot: in parallel on the host threads
  parallel_blocks(N, [&](int64_t ib, int64_t ie, int) {
  for (int64_t i = ib; i < ie; ++i) {
    const int64_t g = nn[i];
    hx[g] = p->coords[i * 3 + 0];
    hy[g] = p->coords[i * 3 + 1];
    hz[g] = p->coords[i * 3 + 2];
    double st[4] = {0.0, 0.0, 0.0, 0.0};
    if (has_init)
      for (int c = 0; c < 4; ++c) st[c] = p->init[i * 4 + c];
    if (b->solver == FM_SOLVER_SUPG) st[3] = 0.0;
    hbc[g] = -1;
    if (p->node_rec[i] >= 0) {
      const BCRec& rr = p->recs[p->node_rec[i]];
      hbc[g] = (int32_t)pl.off[P_REC] + p->node_rec[i];
      if (rr.tab >= 0) {
        const double* tab = p->tab_rows.data() + (int64_t)p->tab_off[rr.tab] * 4;
        const int nrow = p->tab_len[rr.tab];
        double v[3];
        if (0.0 >= tab[(nrow - 1) * 4 + 3]) {
          for (int c = 0; c < 3; ++c) v[c] = tab[(nrow - 1) * 4 + c];
        } else {
          int cnt = 1;
          bool found = false;
          while (!found && cnt < nrow) {
            found = (0.0 >= tab[(cnt - 1) * 4 + 3]) && (0.0 < tab[cnt * 4 + 3]);
            if (!found) cnt++;
          }
          if (!found) {
            table_miss = true;
            continue;
          }
          const double t1 = tab[(cnt - 1) * 4 + 3], t2 = tab[cnt * 4 + 3];
          for (int c = 0; c < 3; ++c)
            v[c] = tab[(cnt - 1) * 4 + c] + ((tab[cnt * 4 + c] - tab[(cnt - 1) * 4 + c]) / (t2 - t1)) * (0.0 - t1);
        }
        if (rr.mask & BC_VX) st[0] = v[0];
        if (rr.mask & BC_VY) st[1] = v[1];
        if (rr.mask & BC_VZ) st[2] = v[2];
      }
      if (rr.mask & BC_PRES) st[3] = rr.p;
      if (rr.mask & BC_DIR) {
        st[0] = rr.d[0];
        st[1] = rr.d[1];
        st[2] = rr.d[2];
      }
    }
    hu[g] = st[0];
    hv[g] = st[1];
    hw[g] = st[2];
    hp[g] = st[3];
    hm[g] = p->mass[i];
  }
  }, 1 << 14);
  if (table_miss) {
    for (int j = 0; j < P_COUNT; ++j) b->pools[j].release(pl.off[j], pl.len[j]);
    return fail(FM_ERR_TABLE, "Could not find time in femUtils::interpTableData.");
  }
  r = r ? r : put(const_cast<double*>(D.x), noff, hx.data(), N, s);
  r = r ? r : put(const_cast<double*>(D.y), noff, hy.data(), N, s);
  r = r ? r : put(const_cast<double*>(D.z), noff, hz.data(), N, s);
  // post-BC state uploaded once, the pre-BC copies filled on the device
  r = r ? r : put(D.su, noff, hu.data(), N, s);
  r = r ? r : put(D.sv, noff, hv.data(), N, s);
  r = r ? r : put(D.sw, noff, hw.data(), N, s);
  r = r ? r : put(D.sp, noff, hp.data(), N, s);
  if (!r)
    for (int q = 0; q < 4; ++q) {
      const double* src = q == 0 ? D.su : q == 1 ? D.sv : q == 2 ? D.sw : D.sp;
      double* dst = q == 0 ? D.pu : q == 1 ? D.pv : q == 2 ? D.pw : D.pp;
      CK(cudaMemcpyAsync(dst + noff, src + noff, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
    }
  r = r ? r : put(const_cast<double*>(D.mass), noff, hm.data(), N, s);
  r = r ? r : put(const_cast<int32_t*>(D.node_bc), noff, hbc.data(), N, s);
  {
    std::vector<BCRec> recs(p->recs);
    for (BCRec& q : recs)
      if (q.tab >= 0) q.tab += (int32_t)pl.off[P_TAB];
    std::vector<int32_t> toffs(p->tab_off);
    for (int32_t& q : toffs) q += (int32_t)pl.off[P_ROW];
    r = r ? r : put(const_cast<BCRec*>(D.recs), pl.off[P_REC], recs.data(), (int64_t)recs.size(), s);
    r = r ? r : put(const_cast<int32_t*>(D.tab_off), pl.off[P_TAB], toffs.data(), (int64_t)toffs.size(), s);
    r = r ? r : put(const_cast<int32_t*>(D.tab_len), pl.off[P_TAB], p->tab_len.data(), (int64_t)p->tab_len.size(), s);
    r = r ? r : put(const_cast<double*>(D.tab_rows), pl.off[P_ROW] * 4, p->tab_rows.data(), (int64_t)p->tab_rows.size(), s);
  }
  // element data: connectivity (mixed: FP64-inverse flags set by prepare()), zero history
  {
    const auto& conn = L.conn_local;
    r = r ? r : put(const_cast<uint16_t*>(D.conn), eoff * npe, conn.data(), (int64_t)conn.size(), s);
    const int64_t ne = pl.len[P_ELEM];
    if (D.sdus32)
      for (int q = 0; q < 12; ++q) CK(cudaMemsetAsync(D.sdus32 + (int64_t)q * D.E + eoff, 0, ne * sizeof(float), s));
    if (D.sdus) {
      const int nh = b->solver == FM_SOLVER_VMS ? 12 : 3 * npe;
      for (int q = 0; q < nh; ++q) CK(cudaMemsetAsync(D.sdus + (int64_t)q * D.E + eoff, 0, ne * sizeof(double), s));
    }
    if (D.el_lam) {
      CK(cudaMemsetAsync(D.el_lam + eoff, 0, ne * sizeof(double), s));
      CK(cudaMemsetAsync(D.el_reg + eoff, 0, ne * sizeof(double), s));
    }
  }
  // tiles and their lists, relocated
  {
    std::vector<TileMeta> tiles(L.tiles);
    for (TileMeta& tm : tiles) {
      tm.elem_begin += (int32_t)eoff;
      tm.node_begin += (int32_t)pl.off[P_TNODE];
      tm.slot_base += (int32_t)soff;
      tm.col_begin += (int32_t)pl.off[P_TCOL];
      tm.inc_begin += (int32_t)pl.off[P_TINC];
      tm.off_begin += (int32_t)pl.off[P_TOFF];
      // the look-ahead prefetch reads node0 .. node0 + n_int - 1: checked to
      // be the tile's interior nodes (consecutive by construction), else -1
      // (no node prefetch for the tile)
      {
        const int32_t* tn = L.tile_nodes.data() + (tm.node_begin - (int32_t)pl.off[P_TNODE]);
        bool consecutive = tm.n_int > 0;
        for (int32_t j = 1; j < tm.n_int && consecutive; ++j) consecutive = tn[j] == tn[0] + j;
        tm.node0 = consecutive ? tn[0] + (int32_t)noff : -1;
      }
      tm.problem = ps;
      pl.tn_max = std::max(pl.tn_max, tm.n_node);
    }
    pl.inc_max = (L.max_tile_elems * npe + 7) / 8 * 8;
    r = r ? r : put(const_cast<TileMeta*>(D.tiles), pl.off[P_TILE], tiles.data(), (int64_t)tiles.size(), s);
    if (noff == 0) {  // node ids need no relocation
      r = r ? r : put(const_cast<int32_t*>(D.tile_nodes), pl.off[P_TNODE], L.tile_nodes.data(),
                      (int64_t)L.tile_nodes.size(), s);
    } else {
      std::vector<int32_t> tnodes(L.tile_nodes.begin(), L.tile_nodes.end());
      for (int32_t& q : tnodes) q += (int32_t)noff;
      r = r ? r : put(const_cast<int32_t*>(D.tile_nodes), pl.off[P_TNODE], tnodes.data(), (int64_t)tnodes.size(), s);
      CK(cudaStreamSynchronize(s));  // tnodes goes out of scope
    }
    r = r ? r : put(const_cast<int32_t*>(D.tile_cols), pl.off[P_TCOL], L.tile_cols.data(), (int64_t)L.tile_cols.size(), s);
    r = r ? r : put(const_cast<uint16_t*>(D.tile_inc), pl.off[P_TINC], L.tile_inc.data(), (int64_t)L.tile_inc.size(), s);
    r = r ? r : put(const_cast<uint16_t*>(D.tile_off), pl.off[P_TOFF], L.tile_off.data(), (int64_t)L.tile_off.size(), s);
  }
  // interface entries
  {
    const int64_t ni = (int64_t)L.iface_node.size();
    std::vector<int32_t> inode(ni), isb(ni), isc(ni), iprob(ni, ps), islots(L.iface_slots);
    for (int64_t i = 0; i < ni; ++i) {
      inode[i] = L.iface_node[i] + (int32_t)noff;
      isb[i] = L.iface_slot_beg[i] + (int32_t)pl.off[P_ISLOT];
      isc[i] = L.iface_slot_beg[i + 1] - L.iface_slot_beg[i];
    }
    for (int32_t& q : islots) q += (int32_t)soff;
    r = r ? r : put(const_cast<int32_t*>(D.iface_node), pl.off[P_IFACE], inode.data(), ni, s);
    r = r ? r : put(const_cast<int32_t*>(D.iface_slot_beg), pl.off[P_IFACE], isb.data(), ni, s);
    r = r ? r : put(const_cast<int32_t*>(D.iface_slot_cnt), pl.off[P_IFACE], isc.data(), ni, s);
    r = r ? r : put(const_cast<int32_t*>(D.iface_slots), pl.off[P_ISLOT], islots.data(), (int64_t)islots.size(), s);
    r = r ? r : put(const_cast<int32_t*>(D.iface_prob), pl.off[P_IFACE], iprob.data(), ni, s);
    if (D.iface_xidx) r = r ? r : put(const_cast<int32_t*>(D.iface_xidx), pl.off[P_IFACE], L.iface_xidx.data(), ni, s);
  }
  // problem constants and progress
  {
    DevProb d;
    memset(&d, 0, sizeof(d));
    const fm_params& pr = p->params;
    d.rho = pr.props[0];
    d.mu = pr.props[1];
    d.nu = pr.props[1] / pr.props[0];
    d.inv_eps = pr.props[2];
    d.alpha = pr.props[2];
    d.c1 = pr.props[3];
    d.c_i = pr.props[3];
    d.c2 = pr.props[4];
    d.dt = pr.time_step;
    d.ds = pr.dual_step;
    d.exit_cond = pr.exit_condition;
    d.ndual = b->solver == FM_SOLVER_VMS ? std::max(0, pr.tot_dual_steps) : 0;
    d.solver = b->solver;
    d.precision = b->precision;
    d.npe = npe;
    for (int q = 0; q < 6; ++q)
      if (pr.ex_opts[q]) d.ex_mask |= (1 << q);
    d.glob_fixed = pr.glob_fixed;
    for (int q = 0; q < 4; ++q) d.q1[q] = (q < p->N) ? (int32_t)(noff + nn[q]) : -1;
    d.xslice = -1;
    if (b->exchange && p->part >= 0) {
      if ((int)b->x_slice_of.size() <= ps) b->x_slice_of.resize(ps + 1, -1);
      int used = 0;
      for (int32_t v : b->x_slice_of) used += (v >= 0);
      b->x_slice_of[ps] = used;
      d.xslice = used;
    }
    d.node_begin = noff;
    d.n_nodes = p->N;
    d.elem_begin = eoff;
    d.n_elems = p->E;
    DevProbState st;
    memset(&st, 0, sizeof(st));
    st.time = 0.0 + pr.time_step;
    const double z8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int32_t zero = 0;
    r = r ? r : put(const_cast<DevProb*>(D.probs), ps, &d, 1, s);
    r = r ? r : put(D.pstate, ps, &st, 1, s);
    r = r ? r : put(const_cast<int32_t*>(D.target), ps, &zero, 1, s);
    r = r ? r : put(D.q1p, (int64_t)ps * 8, z8, 8, s);
  }
  CK(cudaStreamSynchronize(s));  // host staging vectors go out of scope
  if (r) {
    for (int j = 0; j < P_COUNT; ++j) b->pools[j].release(pl.off[j], pl.len[j]);
    return r;
  }
  b->iters[ps] = 0;
  p->batch = b;
  p->index = ps;
  p->steps_done = 0;
  b->slots[ps] = std::move(pl);
  refresh_extent(b);
  if (b->diag) {
    r = diag_prepare_problem(b->slots[ps]);
    if (r) return r;
  }
  r = configure(b);
  if (!r && (D.geo || D.geo32)) {
    // the problem's Gauss-point geometry, ahead of its first step on the stream
    cudaError_t e = launch_supg_geo(D, (int)b->slots[ps].off[P_TILE], (int)L.tiles.size(), b->slots[ps].tn_max, s);
    if (e != cudaSuccess) r = fail(FM_ERR_CUDA, std::string("geometry: ") + cudaGetErrorString(e));
  }
  return r;
}

// Pool capacities of fm_batch_create_empty for the given maxima.  Tiles hold
// about tile_elems elements (at least half that unless tile_nodes binds
// first); each tile start is padded to a multiple of 32 element slots;
// tile-boundary nodes appear once per tile that touches them (about 1.4 N
// for tet tiles of 1024 elements) and own one interface partial slot each;
// BC records exist for boundary nodes only.  A problem that needs more than
// what is left gets FM_ERR_OOM from fm_batch_add.
static void capacity_pools(const fm_capacity* cap, int te, int64_t c[P_COUNT]) {
  const int64_t E = cap->max_elems, N = cap->max_nodes, P = cap->max_problems, npe = cap->elem_type;
  c[P_NODE] = N;
  c[P_TILE] = E / std::max<int64_t>(1, te / 2) + 2 * P;
  c[P_ELEM] = E + 2 * P * ELEM_ALIGN + c[P_TILE] * ELEM_ALIGN;
  c[P_TNODE] = 2 * N + 16 * c[P_TILE];
  c[P_TCOL] = c[P_TILE] * 130;
  c[P_TINC] = npe * E + 16 * c[P_TILE] + 16 * P;
  c[P_TOFF] = c[P_TNODE] + c[P_TILE];
  c[P_SLOT] = 2 * N + 32 * c[P_TILE];
  c[P_IFACE] = N;
  c[P_ISLOT] = c[P_SLOT];
  c[P_REC] = N / 2 + 64 * P;
  c[P_TAB] = c[P_REC];
  c[P_ROW] = cap->max_table_rows > 0 ? cap->max_table_rows : c[P_REC];
  c[P_PROB] = P;
}

// Device bytes allocate() takes for these pool capacities.
static int64_t pool_bytes(const int64_t cap[P_COUNT], int solver, int npe, int prec, bool history) {
  const int64_t NN = std::max<int64_t>(cap[P_NODE], 1);
  const int64_t NE = (std::max<int64_t>(cap[P_ELEM], 1) + ELEM_ALIGN - 1) / ELEM_ALIGN * ELEM_ALIGN;
  auto at_least = [](int64_t v, int64_t m) { return std::max<int64_t>(v, m); };
  int64_t b = NN * (12 * 8 + 4) + NE * npe * 2;
  if (solver == FM_SOLVER_VMS && prec == FM_MIXED) b += NE * 12 * 4;
  else if (solver == FM_SOLVER_VMS || history) b += NE * (solver == FM_SOLVER_VMS ? 12 : 3 * npe) * 8;
  if (solver == FM_SOLVER_SUPG) b += NE * 3 * 8;
  if (solver == FM_SOLVER_SUPG && npe == 8) b += NE * 8 * FM_GEO_PER_GP * (prec == FM_MIXED ? 4 : 8);
  b += at_least(cap[P_TILE], 1) * (int64_t)sizeof(TileMeta) + at_least(cap[P_TNODE], 1) * 4 +
       at_least(cap[P_TCOL], 1) * 4 + at_least(cap[P_TINC], 8) * 2 + at_least(cap[P_TOFF], 1) * 2;
  b += at_least(cap[P_SLOT], 1) * 4 * 8 + at_least(cap[P_IFACE], 1) * 4 * 4 + at_least(cap[P_ISLOT], 1) * 4;
  b += at_least(cap[P_REC], 1) * (int64_t)sizeof(BCRec) + at_least(cap[P_TAB], 1) * 2 * 4 + at_least(cap[P_ROW], 1) * 32;
  const int64_t NP = at_least(cap[P_PROB], 1);
  b += NP * ((int64_t)sizeof(DevProb) + (int64_t)sizeof(DevProbState) + 4 + 64);
  return b;
}

extern "C" {

const char* fm_strerror(int code) {
  switch (code) {
    case FM_OK: return "ok";
    case FM_ERR_INVALID: return "invalid argument or input";
    case FM_ERR_OOM: return "out of memory";
    case FM_ERR_CUDA: return "CUDA runtime error";
    case FM_ERR_DIVERGED: return "solution diverged (NaN/Inf or velocity above EXITCOND)";
    case FM_ERR_TIMEOUT: return "device wait timed out";
    case FM_ERR_TABLE: return "Could not find time in femUtils::interpTableData.";
    case FM_ERR_IO: return "file I/O error";
    case FM_ERR_NODEVICE: return "no usable CUDA device";
    default: return "unknown error";
  }
}

const char* fm_last_error_message(void) { return last_error(); }
int fm_version(void) { return 101; }

int fm_problem_create(const fm_mesh* m, const fm_bc* bc, const fm_params* prm, const double* init, fm_problem** out) {
  NvtxRange nvtx_range("fm_problem_create");
  if (!m || !prm || !out) return fail(FM_ERR_INVALID, "null argument");
  *out = nullptr;
  if (m->elem_type != FM_TET4 && m->elem_type != FM_HEXA8) return fail(FM_ERR_INVALID, "elem_type must be 4 or 8");
  if (m->n_nodes <= 0 || m->n_elems <= 0 || !m->coords || !m->conn) return fail(FM_ERR_INVALID, "empty mesh");
  if (prm->solver != FM_SOLVER_VMS && prm->solver != FM_SOLVER_SUPG) return fail(FM_ERR_INVALID, "bad solver");
  if (prm->solver == FM_SOLVER_VMS && m->elem_type != FM_TET4)
    return fail(FM_ERR_INVALID, "the VMS solver is tet4-only (femVMSExplicitFluidSolver.cpp hard-codes 4 nodes)");
  if (prm->solver == FM_SOLVER_SUPG && m->elem_type == FM_TET4 && prm->ex_opts[1])
    return fail(FM_ERR_INVALID, "B-bar (EXOPTS 2nd field) is hexa8-only; the reference reads out of bounds on tet4");
  if (prm->precision != FM_FP64 && prm->precision != FM_MIXED) return fail(FM_ERR_INVALID, "bad precision");
  if (!(prm->time_step > 0)) return fail(FM_ERR_INVALID, "time_step must be positive");
  if (prm->props[0] == 0.0) return fail(FM_ERR_INVALID, "density must be non-zero");
  fm_problem* p = new fm_problem();
  p->etype = m->elem_type;
  p->N = m->n_nodes;
  p->E = m->n_elems;
  // copies and the connectivity check on the host threads
  p->coords.resize(m->n_nodes * 3);
  p->conn.resize(m->n_elems * m->elem_type);
  parallel_blocks((int64_t)p->coords.size(), [&](int64_t b, int64_t e, int) {
    std::copy(m->coords + b, m->coords + e, p->coords.begin() + b);
  }, 1 << 16);
  std::atomic<bool> bad{false};
  parallel_blocks((int64_t)p->conn.size(), [&](int64_t b, int64_t e, int) {
    bool any = false;
    for (int64_t i = b; i < e; ++i) {
      const int32_t c = m->conn[i];
      p->conn[i] = c;
      any |= (c < 0 || c >= p->N);
    }
    if (any) bad = true;
  }, 1 << 16);
  if (bad) {
    delete p;
    return fail(FM_ERR_INVALID, "connectivity out of range");
  }
  p->params = *prm;
  if (bc) {
    if (bc->n_vel_rows) {
      p->vel_node.assign(bc->vel_node, bc->vel_node + bc->n_vel_rows);
      p->vel_vals.assign(bc->vel_vals, bc->vel_vals + bc->n_vel_rows * 4);
      p->vel_dir.assign(bc->vel_dir, bc->vel_dir + bc->n_vel_rows);
    }
    if (bc->n_dir) {
      p->dir_node.assign(bc->dir_node, bc->dir_node + bc->n_dir);
      p->dir_vals.assign(bc->dir_vals, bc->dir_vals + bc->n_dir * 3);
    }
    if (bc->n_pres) {
      p->pres_node.assign(bc->pres_node, bc->pres_node + bc->n_pres);
      p->pres_vals.assign(bc->pres_vals, bc->pres_vals + bc->n_pres);
    }
  }
  if (init) p->init.assign(init, init + p->N * 4);
  int r = resolve_bcs(p);
  if (r) {
    delete p;
    return r;
  }
  compute_mass(p);
  *out = p;
  return FM_OK;
}

int fm_problem_destroy(fm_problem* p) {
  if (!p) return FM_OK;
  if (p->batch) fm_batch_remove(p->batch, p);
  delete p;
  return FM_OK;
}

int fm_problem_info(const fm_problem* p, int64_t* nn, int64_t* ne, int32_t* et, int32_t* solver, int64_t* steps) {
  if (!p) return fail(FM_ERR_INVALID, "null problem");
  if (nn) *nn = p->N;
  if (ne) *ne = p->E;
  if (et) *et = p->etype;
  if (solver) *solver = p->params.solver;
  if (steps) *steps = p->steps_done;
  return FM_OK;
}

int fm_problem_get_mass(fm_problem* p, double* mass) {
  if (!p || !mass) return fail(FM_ERR_INVALID, "null argument");
  if (p->params.solver == FM_SOLVER_VMS) {
    memcpy(mass, p->mass.data(), sizeof(double) * p->N);
  } else {
    for (int64_t i = 0; i < p->N; ++i)
      for (int c = 0; c < 3; ++c) mass[i * 3 + c] = p->mass[i];
  }
  return FM_OK;
}

int fm_problem_prepare(fm_problem* p, const fm_tuning* tuning) {
  NvtxRange nvtx_range("fm_problem_prepare");
  if (!p) return fail(FM_ERR_INVALID, "null problem");
  fm_tuning t;
  memset(&t, 0, sizeof(t));
  if (tuning) t = *tuning;
  default_tuning(p->params.solver, p->etype, p->params.precision, t);
  std::shared_ptr<Layout> L;
  return prepare(p, t.tile_elems, t.tile_nodes, &L);
}

int fm_problem_check_layout(fm_problem* p, const fm_tuning* tuning) {
  NvtxRange nvtx_range("fm_problem_check_layout");
  if (!p) return fail(FM_ERR_INVALID, "null problem");
  fm_tuning t;
  memset(&t, 0, sizeof(t));
  if (tuning) t = *tuning;
  default_tuning(p->params.solver, p->etype, p->params.precision, t);
  std::shared_ptr<Layout> L;
  int r = prepare(p, t.tile_elems, t.tile_nodes, &L);
  if (r) return r;
  return check_layout(p, *L);
}

int fm_batch_estimate_bytes(fm_problem* const* probs, int32_t n, const fm_tuning* tuning, int64_t* bytes) {
  if (!probs || n <= 0 || !bytes) return fail(FM_ERR_INVALID, "null argument");
  int64_t N = 0, E = 0;
  int npe = probs[0]->etype;
  for (int i = 0; i < n; ++i) {
    N += probs[i]->N;
    E += probs[i]->E;
  }
  (void)tuning;
  const bool vms = probs[0]->params.solver == FM_SOLVER_VMS;
  const bool mixed = probs[0]->params.precision == FM_MIXED;
  // nodes: 12 FP64 arrays + BC index; elements: connectivity + history;
  // tiles, incidence lists and interface partials: ~40 B per element
  const int64_t per_e = (int64_t)npe * 2 + (vms ? (mixed ? 48 : 96) : (3 * npe * 8 + 24)) + 40 +
                        (!vms && npe == 8 ? 8 * FM_GEO_PER_GP * (mixed ? 4 : 8) : 0);
  *bytes = N * 100 + E * per_e + (16 << 20);
  return FM_OK;
}

static int check_same(fm_problem* const* probs, int n, int* solver, int* npe, int* prec) {
  *solver = probs[0]->params.solver;
  *npe = probs[0]->etype;
  *prec = probs[0]->params.precision;
  for (int i = 0; i < n; ++i) {
    if (!probs[i]) return fail(FM_ERR_INVALID, "null problem");
    if (probs[i]->batch) return fail(FM_ERR_INVALID, "problem already belongs to a batch");
    if (probs[i]->params.solver != *solver || probs[i]->etype != *npe || probs[i]->params.precision != *prec)
      return fail(FM_ERR_INVALID, "all problems of a batch must share solver, element type and precision");
  }
  return FM_OK;
}

static int new_batch(int solver, int npe, int prec, const fm_tuning* tuning, int32_t device, fm_batch** out) {
  if (tuning && tuning->ctas_per_sm != 0 && solver == FM_SOLVER_VMS) {
    const int th = tuning->threads == 256 ? 256 : 128;
    if (!vms_variant_exists(th, prec == FM_MIXED, tuning->ctas_per_sm))
      return fail(FM_ERR_INVALID, "no VMS tile kernel variant for this ctas_per_sm, threads and precision");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FM_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(FM_ERR_INVALID, "bad device ordinal");
  CK(cudaSetDevice(device));
  fm_batch* b = new fm_batch();
  memset(&b->tune, 0, sizeof(b->tune));
  if (tuning) b->tune = *tuning;
  default_tuning(solver, npe, prec, b->tune);
  b->device = device;
  b->solver = solver;
  b->npe = npe;
  b->precision = prec;
  b->threads = b->tune.threads;
  if (solver == FM_SOLVER_VMS && b->tune.ctas_per_sm == 0) b->tune.ctas_per_sm = vms_default_ctas(b->threads, prec == FM_MIXED);
  b->graph_steps = b->tune.graph_steps;
  *out = b;
  return FM_OK;
}

int fm_batch_create(fm_problem* const* probs, int32_t n, const fm_tuning* tuning, int32_t device, fm_batch** out) {
  NvtxRange nvtx_range("fm_batch_create");
  if (!probs || n <= 0 || !out) return fail(FM_ERR_INVALID, "null argument");
  *out = nullptr;
  int solver, npe, prec;
  int r = check_same(probs, n, &solver, &npe, &prec);
  if (r) return r;
  // partition parts: all of one partition (same part count and exchange
  // list), each part once
  int nparts = 0;
  for (int i = 0; i < n; ++i) nparts += (probs[i]->part >= 0);
  if (nparts > 0) {
    if (nparts != n) return fail(FM_ERR_INVALID, "a batch of partition parts takes no other problems");
    std::vector<char> seen(probs[0]->n_parts, 0);
    for (int i = 0; i < n; ++i) {
      if (probs[i]->n_parts != probs[0]->n_parts || probs[i]->x_total != probs[0]->x_total)
        return fail(FM_ERR_INVALID, "partition parts of different partitions in one batch");
      if (seen[probs[i]->part]++) return fail(FM_ERR_INVALID, "the same partition part twice in one batch");
    }
    if (probs[0]->x_total > INT32_MAX / 4) return fail(FM_ERR_INVALID, "partition exchange list too long");
  }
  fm_batch* b = nullptr;
  r = new_batch(solver, npe, prec, tuning, device, &b);
  if (r) return r;
  if (nparts > 0) {
    b->exchange = true;
    b->x_slices = n;
    b->x_n = probs[0]->x_total;
    b->x_external = n < probs[0]->n_parts;
  }
  // exact pool sizes from the prepared layouts
  int64_t cap[P_COUNT] = {0};
  std::vector<std::shared_ptr<Layout>> preps(n);
  for (int i = 0; i < n; ++i) {
    r = prepare(probs[i], b->tune.tile_elems, b->tune.tile_nodes, &preps[i]);
    if (r) {
      delete b;
      return r;
    }
    int64_t len[P_COUNT];
    pool_sizes(probs[i], *preps[i], len);
    for (int k = 0; k < P_COUNT; ++k) cap[k] += len[k] + (kAlign[k] > 1 ? kAlign[k] : 0);
    b->has_history |= (solver == FM_SOLVER_SUPG && probs[i]->params.ex_opts[0] == 0);
  }
  r = allocate(b, cap);
  for (int i = 0; i < n && !r; ++i) r = place(b, probs[i], preps[i]);
  if (!r && b->exchange) {
    // the interface entries of the shared nodes, for the second half of the pass
    std::vector<int32_t> xe;
    for (const Placement& pl : b->slots)
      if (pl.p)
        for (int64_t k = 0; k < pl.len[P_IFACE]; ++k)
          if (pl.L->iface_xidx[k] >= 0) xe.push_back((int32_t)(pl.off[P_IFACE] + k));
    int32_t* d = nullptr;
    r = dalloc(b, (void**)&d, std::max<size_t>(xe.size(), 1) * sizeof(int32_t));
    if (!r) r = put(d, 0, xe.data(), (int64_t)xe.size(), b->stream);
    if (!r && cudaStreamSynchronize(b->stream) != cudaSuccess) r = fail(FM_ERR_CUDA, "exchange entry upload");
    b->D.x_entries = d;
    b->D.n_xentries = (int32_t)xe.size();
    b->x_blocks = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)xe.size() + 255) / 256, 148 * 8));
  }
  if (r) {
    for (int i = 0; i < n; ++i)
      if (probs[i]->batch == b) {
        probs[i]->batch = nullptr;
        probs[i]->index = -1;
      }
    release_all(b);
    delete b;
    return r;
  }
  *out = b;
  return FM_OK;
}

int fm_batch_create_empty(const fm_capacity* cap, const fm_tuning* tuning, int32_t device, fm_batch** out) {
  NvtxRange nvtx_range("fm_batch_create_empty");
  if (!cap || !out) return fail(FM_ERR_INVALID, "null argument");
  if (cap->elem_type != FM_TET4 && cap->elem_type != FM_HEXA8) return fail(FM_ERR_INVALID, "bad element type");
  if (cap->max_elems <= 0 || cap->max_nodes <= 0 || cap->max_problems <= 0) return fail(FM_ERR_INVALID, "bad capacity");
  *out = nullptr;
  fm_batch* b = nullptr;
  int r = new_batch(cap->solver, cap->elem_type, cap->precision, tuning, device, &b);
  if (r) return r;
  b->has_history = cap->solver == FM_SOLVER_SUPG;
  int64_t c[P_COUNT];
  capacity_pools(cap, b->tune.tile_elems, c);
  r = allocate(b, c);
  if (r) {
    release_all(b);
    delete b;
    return r;
  }
  *out = b;
  return FM_OK;
}

int fm_batch_capacity_bytes(const fm_capacity* cap, const fm_tuning* tuning, int64_t* bytes) {
  if (!cap || !bytes) return fail(FM_ERR_INVALID, "null argument");
  if (cap->elem_type != FM_TET4 && cap->elem_type != FM_HEXA8) return fail(FM_ERR_INVALID, "bad element type");
  fm_tuning t;
  memset(&t, 0, sizeof(t));
  if (tuning) t = *tuning;
  default_tuning(cap->solver, cap->elem_type, cap->precision, t);
  int64_t c[P_COUNT];
  capacity_pools(cap, t.tile_elems, c);
  *bytes = pool_bytes(c, cap->solver, cap->elem_type, cap->precision, cap->solver == FM_SOLVER_SUPG);
  return FM_OK;
}

int fm_batch_add(fm_batch* b, fm_problem* p) {
  NvtxRange nvtx_range("fm_batch_add");
  if (!b || !p) return fail(FM_ERR_INVALID, "null argument");
  if (p->batch) return fail(FM_ERR_INVALID, "problem already belongs to a batch");
  if (p->part >= 0 || b->exchange)
    return fail(FM_ERR_INVALID, "partition parts are batched together by fm_batch_create, with no other problems");
  if (p->params.solver != b->solver || p->etype != b->npe || p->params.precision != b->precision)
    return fail(FM_ERR_INVALID, "problem does not match the batch's solver, element type and precision");
  if (b->solver == FM_SOLVER_SUPG && p->params.ex_opts[0] == 0 && !b->has_history)
    return fail(FM_ERR_INVALID, "batch was created without AB2 history");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  std::shared_ptr<Layout> L;
  int r = prepare(p, b->tune.tile_elems, b->tune.tile_nodes, &L);
  if (r) return r;
  return place(b, p, L);
}

int fm_batch_remove(fm_batch* b, fm_problem* p) {
  NvtxRange nvtx_range("fm_batch_remove");
  if (!b || !p || p->batch != b) return fail(FM_ERR_INVALID, "problem is not in this batch");
  if (b->exchange) return fail(FM_ERR_INVALID, "partition parts stay in their batch until it is destroyed");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  const int ps = p->index;
  Placement& pl = b->slots[ps];
  DevBatch& D = b->D;
  // mark the problem's tiles and interface entries inactive, park its slot
  CK(cudaMemset(const_cast<TileMeta*>(D.tiles) + pl.off[P_TILE], 0xff, pl.len[P_TILE] * sizeof(TileMeta)));
  CK(cudaMemset(const_cast<int32_t*>(D.iface_prob) + pl.off[P_IFACE], 0xff, pl.len[P_IFACE] * sizeof(int32_t)));
  CK(cudaMemset(const_cast<int32_t*>(D.target) + ps, 0, sizeof(int32_t)));
  CK(cudaMemset(D.pstate + ps, 0, sizeof(DevProbState)));
  for (int k = 0; k < P_COUNT; ++k) b->pools[k].release(pl.off[k], pl.len[k]);
  b->iters[ps] = 0;
  diag_free_problem(pl);
  pl = Placement();
  p->batch = nullptr;
  p->index = -1;
  refresh_extent(b);
  return FM_OK;
}

int fm_batch_destroy(fm_batch* b) {
  if (!b) return FM_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (Placement& pl : b->slots)
    if (pl.p) {
      pl.p->batch = nullptr;
      pl.p->index = -1;
    }
  diag_free(b);
  release_all(b);
  delete b;
  return FM_OK;
}

}  // extern "C"

// One iteration (dual iteration for VMS, step for SUPG): tile kernel +
// interface kernel.
// A batch of partition parts runs the interface pass in two halves (shared
// nodes packed, then updated from the sums over all parts); when every part
// is in the batch the second half follows directly (ev[2] is then recorded
// again after it).
static cudaError_t launch_first(fm_batch* b, cudaStream_t s, cudaEvent_t* ev) {
  if (b->solver == FM_SOLVER_VMS)
    return launch_vms_iteration(b->D, b->tn_max, b->inc_max, b->threads, b->tune.ctas_per_sm, b->iface_blocks,
                                b->precision == FM_MIXED, b->exchange, s, ev);
  return launch_supg_step(b->D, b->tn_max, b->inc_max, b->threads, b->iface_blocks, b->npe, b->precision == FM_MIXED,
                          b->exchange,
                          s, ev);
}
static cudaError_t launch_second(fm_batch* b, cudaStream_t s) {
  return b->solver == FM_SOLVER_VMS ? launch_vms_xupdate(b->D, b->x_blocks, s) : launch_supg_xupdate(b->D, b->x_blocks, s);
}
static cudaError_t launch_one(fm_batch* b, cudaStream_t s, cudaEvent_t* ev) {
  cudaError_t e = launch_first(b, s, ev);
  if (e != cudaSuccess || !b->exchange) return e;
  e = launch_second(b, s);
  if (ev) cudaEventRecord(ev[2], s);
  return e;
}

// VMS diagnostics after iteration `it` of a launch sequence: for every
// problem that took part, the reference's log row (step, dual iteration,
// time, max centroid |res_u|, max |res_p|, CFL) is queued on the problem.
static int record_diagnostics(fm_batch* b, const std::vector<int32_t>& add_iters, int it, cudaStream_t s) {
  const int n = (int)add_iters.size();
  for (int i = 0; i < n; ++i) {
    Placement& pl = b->slots[i];
    fm_problem* p = pl.p;
    if (!p || it >= add_iters[i] || !pl.dg_el) continue;
    const int64_t EC = (int64_t)pl.L->elem_old[0].size();
    cudaError_t e = launch_vms_diagnostics(b->D, b->d_cres, pl.dg_off, pl.dg_ent, (int32_t)p->N, pl.dg_eo,
                                           pl.off[P_ELEM], EC, pl.off[P_NODE], pl.dg_el, b->d_diag_out, DIAG_BLOCKS, s);
    if (e != cudaSuccess) return fail(FM_ERR_CUDA, std::string("diagnostics: ") + cudaGetErrorString(e));
    CK(cudaMemcpyAsync(b->h_diag, b->d_diag_out, 3 * DIAG_BLOCKS * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    double mu = 0.0, mp = 0.0, mv = 0.0;
    for (int k = 0; k < DIAG_BLOCKS; ++k) {
      mu = std::max(mu, b->h_diag[2 * k]);
      mp = std::max(mp, b->h_diag[2 * k + 1]);
      mv = std::max(mv, b->h_diag[2 * DIAG_BLOCKS + k]);
    }
    // the iteration just done; the step's time accumulates like the
    // reference's currentTime (src/femVMSExplicitFluidSolver.cpp:1028)
    const int64_t per = std::max(0, p->params.tot_dual_steps) + 1;
    const int64_t idx = (int64_t)b->iters[i] + it;
    const int64_t step = idx / per;
    const double dt = p->params.time_step;
    if (step != p->diag_step) {
      if (step == p->diag_step + 1 && p->diag_step >= 0) {
        p->diag_time += dt;
      } else {
        double t = 0.0;
        for (int64_t q = 0; q <= step; ++q) t += dt;
        p->diag_time = t;
      }
      p->diag_step = step;
    }
    const double row[6] = {(double)step, (double)(idx % per + 1), p->diag_time, mu, mp, mv * dt / p->diag_min_h};
    p->diag_rows.insert(p->diag_rows.end(), row, row + 6);
  }
  return FM_OK;
}

// Sets per-slot targets (iterations) and launches enough iterations.  With
// prof != nullptr every kernel is bracketed by CUDA events and the per-kernel
// device times are summed into prof[0] (tile kernel) and prof[1] (interface
// kernel), in milliseconds.
static int run_iterations(fm_batch* b, const std::vector<int32_t>& add_iters, cudaStream_t s, double* prof = nullptr) {
  NvtxRange nvtx_range("fm_batch_step");
  if (b->x_external)
    return fail(FM_ERR_INVALID,
                "the batch holds partition parts whose other parts run elsewhere: advance it with "
                "fm_batch_exchange_begin / fm_batch_exchange_end");
  const int n = (int)b->pools[P_PROB].hwm;
  int32_t maxit = 0;
  for (int i = 0; i < n; ++i) maxit = std::max(maxit, add_iters[i]);
  if (b->exchange)
    for (int i = 0; i < n; ++i)
      if (b->slots[i].p && add_iters[i] != maxit)
        return fail(FM_ERR_INVALID, "the parts of a partition advance together: give them the same step count");
  if (maxit == 0 || b->D.n_tiles == 0) return FM_OK;
  // new targets (the host tracks every slot's iteration count exactly)
  b->x_free_targets = false;
  CK(cudaEventSynchronize(b->ev_tgt));  // staging buffer free again
  for (int i = 0; i < n; ++i) b->h_targets[i] = b->iters[i] + add_iters[i];
  CK(cudaMemcpyAsync(const_cast<int32_t*>(b->D.target), b->h_targets, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
  CK(cudaEventRecord(b->ev_tgt, s));
  CK(cudaEventRecord(b->ev0, s));
  int64_t launches = 0;
  std::vector<cudaEvent_t> evs;
  if (prof) {
    evs.resize((size_t)maxit * 3);
    for (auto& e : evs) CK(cudaEventCreate(&e));
  }
  int it = 0;
  // whole blocks of graph_steps iterations replay one captured CUDA graph
  // (the per-slot targets live in device memory, so the same graph serves
  // every block and every ragged step pattern; it is re-captured when the
  // batch's extent changes)
  if (!prof && !b->diag && b->graph_steps > 0 && maxit >= b->graph_steps) {
    if (!b->graph) {
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      cudaError_t e = cudaSuccess;
      for (int i = 0; i < b->graph_steps && e == cudaSuccess; ++i) e = launch_one(b, s, nullptr);
      cudaError_t e2 = cudaStreamEndCapture(s, &g);
      if (e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(FM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
      }
      e = cudaGraphInstantiate(&b->graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return fail(FM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
      b->graph_iters = b->graph_steps;
    }
    for (; it + b->graph_iters <= maxit; it += b->graph_iters) {
      CK(cudaGraphLaunch(b->graph, s));
      launches += (b->exchange ? 3 : 2) * (int64_t)b->graph_iters;
    }
  }
  for (; it < maxit; ++it) {
    cudaEvent_t* ev = prof ? &evs[(size_t)it * 3] : nullptr;
    cudaError_t e = launch_one(b, s, ev);
    if (e != cudaSuccess) return fail(FM_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    launches += b->exchange ? 3 : 2;
    if (b->diag) {
      int r = record_diagnostics(b, add_iters, it, s);
      if (r) return r;
    }
  }
  CK(cudaEventRecord(b->ev1, s));
  if (prof) {
    CK(cudaEventSynchronize(b->ev1));
    prof[0] = prof[1] = 0.0;
    for (int i = 0; i < maxit; ++i) {
      float a = 0.f, c = 0.f;
      CK(cudaEventElapsedTime(&a, evs[i * 3], evs[i * 3 + 1]));
      CK(cudaEventElapsedTime(&c, evs[i * 3 + 1], evs[i * 3 + 2]));
      prof[0] += a;
      prof[1] += c;
    }
    for (auto& e : evs) cudaEventDestroy(e);
  }
  b->last_launches = launches;
  b->timed = true;
  for (int i = 0; i < n; ++i) b->iters[i] += add_iters[i];
  return FM_OK;
}

static void iters_for(fm_batch* b, const int32_t* nsteps_per_slot, std::vector<int32_t>& add) {
  const int n = (int)b->pools[P_PROB].hwm;
  add.assign(n, 0);
  for (int i = 0; i < n; ++i) {
    const Placement& pl = b->slots[i];
    if (!pl.p) continue;
    const int per = b->solver == FM_SOLVER_VMS ? std::max(0, pl.p->params.tot_dual_steps) + 1 : 1;
    add[i] = nsteps_per_slot[i] * per;
  }
}

extern "C" {

int fm_batch_step_ragged(fm_batch* b, const int32_t* nsteps, void* stream) {
  if (!b || !nsteps) return fail(FM_ERR_INVALID, "null argument");
  CK(cudaSetDevice(b->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : b->stream;
  // nsteps is indexed by the problems' order of addition to the batch: map
  // to slots through each problem's index
  const int n = (int)b->pools[P_PROB].hwm;
  std::vector<int32_t> per_slot(n, 0);
  int k = 0;
  for (int i = 0; i < n; ++i)
    if (b->slots[i].p) {
      if (nsteps[k] < 0) return fail(FM_ERR_INVALID, "negative step count");
      per_slot[i] = nsteps[k++];
    }
  std::vector<int32_t> add;
  iters_for(b, per_slot.data(), add);
  int r = run_iterations(b, add, s);
  if (r) return r;
  for (int i = 0; i < n; ++i)
    if (b->slots[i].p) b->slots[i].p->steps_done += per_slot[i];
  return FM_OK;
}

int fm_batch_step_problems(fm_batch* b, fm_problem* const* probs, const int32_t* nsteps, int32_t count, void* stream) {
  if (!b || (count > 0 && (!probs || !nsteps))) return fail(FM_ERR_INVALID, "null argument");
  CK(cudaSetDevice(b->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : b->stream;
  const int n = (int)b->pools[P_PROB].hwm;
  std::vector<int32_t> per_slot(n, 0);
  for (int i = 0; i < count; ++i) {
    if (!probs[i] || probs[i]->batch != b || nsteps[i] < 0) return fail(FM_ERR_INVALID, "bad problem or step count");
    per_slot[probs[i]->index] = nsteps[i];
  }
  std::vector<int32_t> add;
  iters_for(b, per_slot.data(), add);
  int r = run_iterations(b, add, s);
  if (r) return r;
  for (int i = 0; i < count; ++i) probs[i]->steps_done += nsteps[i];
  return FM_OK;
}

int fm_batch_step(fm_batch* b, int32_t nsteps, void* stream) {
  if (!b) return fail(FM_ERR_INVALID, "null batch");
  std::vector<int32_t> v(b->pools[P_PROB].hwm + 1, nsteps);
  return fm_batch_step_ragged(b, v.data(), stream);
}

int fm_batch_exchange_buffers(fm_batch* b, double** send, double** recv, int64_t* count) {
  if (!b) return fail(FM_ERR_INVALID, "null batch");
  if (!b->exchange) return fail(FM_ERR_INVALID, "the batch holds no partition parts");
  if (send) *send = b->D.xsend;
  if (recv) *recv = const_cast<double*>(b->D.xrecv);
  if (count) *count = (int64_t)b->x_slices * b->x_n * 4;
  return FM_OK;
}

int fm_batch_iterations_per_step(fm_batch* b, int32_t* per_step) {
  if (!b || !per_step) return fail(FM_ERR_INVALID, "null argument");
  *per_step = 1;
  for (const Placement& pl : b->slots)
    if (pl.p) {
      if (b->solver == FM_SOLVER_VMS) *per_step = std::max(0, pl.p->params.tot_dual_steps) + 1;
      break;
    }
  return FM_OK;
}

}  // extern "C"

// Host bookkeeping of `k` completed iterations of every part in the batch.
static void count_iterations(fm_batch* b, int k) {
  const int n = (int)b->pools[P_PROB].hwm;
  for (int i = 0; i < n; ++i) {
    fm_problem* p = b->slots[i].p;
    if (!p) continue;
    const int per = b->solver == FM_SOLVER_VMS ? std::max(0, p->params.tot_dual_steps) + 1 : 1;
    for (int j = 0; j < k; ++j) {
      b->iters[i] += 1;
      if (b->iters[i] % per == 0) p->steps_done += 1;
    }
  }
}

extern "C" {

int fm_batch_exchange_begin(fm_batch* b, void* stream) {
  NvtxRange nvtx_range("fm_batch_exchange_begin");
  if (!b) return fail(FM_ERR_INVALID, "null batch");
  if (!b->exchange) return fail(FM_ERR_INVALID, "the batch holds no partition parts");
  if (b->x_open) return fail(FM_ERR_INVALID, "fm_batch_exchange_begin called twice without fm_batch_exchange_end");
  CK(cudaSetDevice(b->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : b->stream;
  // every part advances by one iteration per begin/end pair: the device
  // targets are opened once (no per-iteration copy or host wait, so the
  // host can run ahead of the GPU)
  if (!b->x_free_targets) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(s, &cs));
    if (cs != cudaStreamCaptureStatusNone)
      return fail(FM_ERR_INVALID, "run one fm_batch_exchange_begin/end pair before capturing them in a CUDA graph");
    const int n = (int)b->pools[P_PROB].hwm;
    CK(cudaEventSynchronize(b->ev_tgt));
    for (int i = 0; i < n; ++i) b->h_targets[i] = b->slots[i].p ? INT32_MAX : 0;
    CK(cudaMemcpyAsync(const_cast<int32_t*>(b->D.target), b->h_targets, sizeof(int32_t) * n, cudaMemcpyHostToDevice,
                       s));
    CK(cudaEventRecord(b->ev_tgt, s));
    b->x_free_targets = true;
  }
  cudaError_t e = launch_first(b, s, nullptr);
  if (e != cudaSuccess) return fail(FM_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  b->x_open = true;
  return FM_OK;
}

int fm_batch_exchange_end(fm_batch* b, void* stream) {
  NvtxRange nvtx_range("fm_batch_exchange_end");
  if (!b) return fail(FM_ERR_INVALID, "null batch");
  if (!b->x_open) return fail(FM_ERR_INVALID, "fm_batch_exchange_end called without fm_batch_exchange_begin");
  CK(cudaSetDevice(b->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : b->stream;
  cudaError_t e = launch_second(b, s);
  b->x_open = false;
  if (e != cudaSuccess) return fail(FM_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  // a pair recorded into a CUDA graph has not run: its iterations are
  // counted when the graph is replayed (fm_batch_exchange_account)
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(s, &cs));
  if (cs == cudaStreamCaptureStatusNone) count_iterations(b, 1);
  return FM_OK;
}

int fm_batch_exchange_account(fm_batch* b, int32_t iterations) {
  if (!b || iterations < 0) return fail(FM_ERR_INVALID, "bad argument");
  if (!b->exchange) return fail(FM_ERR_INVALID, "the batch holds no partition parts");
  count_iterations(b, iterations);
  return FM_OK;
}

int fm_batch_profile(fm_batch* b, int32_t nsteps, double* kernel_ms, int64_t* launches) {
  NvtxRange nvtx_range("fm_batch_profile");
  if (!b || nsteps < 0) return fail(FM_ERR_INVALID, "bad argument");
  CK(cudaSetDevice(b->device));
  const int n = (int)b->pools[P_PROB].hwm;
  std::vector<int32_t> per_slot(n, nsteps), add;
  iters_for(b, per_slot.data(), add);
  int64_t per_kernel = 0;
  for (int32_t a : add) per_kernel = std::max<int64_t>(per_kernel, a);
  double prof[2] = {0.0, 0.0};
  int r = run_iterations(b, add, b->stream, prof);
  if (r) return r;
  for (int i = 0; i < n; ++i)
    if (b->slots[i].p) b->slots[i].p->steps_done += nsteps;
  if (kernel_ms) {
    kernel_ms[0] = prof[0];
    kernel_ms[1] = prof[1];
  }
  if (launches) {
    launches[0] = per_kernel;
    launches[1] = per_kernel;
  }
  return FM_OK;
}

int fm_batch_sync(fm_batch* b) {
  if (!b) return fail(FM_ERR_INVALID, "null batch");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  CK(cudaDeviceSynchronize());
  const int n = (int)b->pools[P_PROB].hwm;
  std::vector<DevProbState> st(std::max(n, 1));
  if (n > 0) CK(cudaMemcpy(st.data(), b->D.pstate, sizeof(DevProbState) * n, cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; ++i)
    if (b->slots[i].p && st[i].status != FM_OK) return fail(st[i].status, fm_strerror(st[i].status));
  return FM_OK;
}

int fm_problem_status(fm_problem* p) {
  if (!p || !p->batch) return fail(FM_ERR_INVALID, "problem is not in a batch");
  fm_batch* b = p->batch;
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  DevProbState st;
  CK(cudaMemcpy(&st, b->D.pstate + p->index, sizeof(st), cudaMemcpyDeviceToHost));
  return st.status;
}

int fm_problem_velocity_extrema(fm_problem* p, double* out) {
  if (!p || !out) return fail(FM_ERR_INVALID, "null argument");
  fm_batch* b = p->batch;
  if (!b) return fail(FM_ERR_INVALID, "problem is not in a batch");
  CK(cudaSetDevice(b->device));
  const Placement& pl = b->slots[p->index];
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(256, (p->N + 255) / 256));
  const int gf = b->solver == FM_SOLVER_SUPG ? p->params.glob_fixed : 0;
  cudaError_t e = launch_velocity_extrema(b->D, pl.off[P_NODE], p->N, gf, blocks, b->d_stats, b->stream);
  if (e != cudaSuccess) return fail(FM_ERR_CUDA, cudaGetErrorString(e));
  std::vector<double> h((size_t)blocks * 7);
  CK(cudaMemcpyAsync(h.data(), b->d_stats, h.size() * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  for (int k = 0; k < 7; ++k) out[k] = h[k];
  for (int i = 1; i < blocks; ++i)
    for (int k = 0; k < 7; ++k) {
      const double v = h[(size_t)i * 7 + k];
      const bool isMin = (k == 0 || k == 2 || k == 4);
      if (isMin ? v < out[k] : v > out[k]) out[k] = v;
    }
  return FM_OK;
}

int fm_problem_supg_log_stats(fm_problem* p, double* out) {
  if (!p || !out) return fail(FM_ERR_INVALID, "null argument");
  fm_batch* b = p->batch;
  if (!b) return fail(FM_ERR_INVALID, "problem is not in a batch");
  if (b->solver != FM_SOLVER_SUPG) return fail(FM_ERR_INVALID, "log statistics are those of the SUPG solver");
  CK(cudaSetDevice(b->device));
  const Placement& pl = b->slots[p->index];
  const int nt = (int)pl.len[P_TILE];
  cudaError_t e = launch_supg_stats(b->D, (int)pl.off[P_TILE], nt, pl.tn_max, b->npe, b->d_stats, b->stream);
  if (e != cudaSuccess) return fail(FM_ERR_CUDA, cudaGetErrorString(e));
  std::vector<double> h((size_t)nt * 11);
  CK(cudaMemcpyAsync(h.data(), b->d_stats, h.size() * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  for (int k = 0; k < 11; ++k) out[k] = h[k];
  for (int i = 1; i < nt; ++i)
    for (int k = 0; k < 11; ++k) {
      const double v = h[(size_t)i * 11 + k];
      const bool isMin = (k == 0 || k == 2 || k == 7 || k == 9);
      if (isMin ? v < out[k] : v > out[k]) out[k] = v;
    }
  return FM_OK;
}

int fm_batch_last_timing(fm_batch* b, double* ms, int64_t* launches) {
  if (!b) return fail(FM_ERR_INVALID, "null batch");
  if (!b->timed) {
    if (ms) *ms = 0.0;
    if (launches) *launches = 0;
    return FM_OK;
  }
  float f = 0.f;
  CK(cudaEventSynchronize(b->ev1));
  CK(cudaEventElapsedTime(&f, b->ev0, b->ev1));
  if (ms) *ms = f;
  if (launches) *launches = b->last_launches;
  return FM_OK;
}

int fm_batch_layout(fm_batch* b, int64_t* nt, int64_t* ni, int32_t* mc, int64_t* ns) {
  if (!b) return fail(FM_ERR_INVALID, "null batch");
  int64_t t = 0, i = 0, s = 0;
  int32_t c = 0;
  for (const Placement& pl : b->slots)
    if (pl.p) {
      t += pl.len[P_TILE];
      i += pl.len[P_IFACE];
      s += pl.len[P_SLOT];
      c = std::max(c, pl.L->max_colors);
    }
  if (nt) *nt = t;
  if (ni) *ni = i;
  if (mc) *mc = c;
  if (ns) *ns = s;
  return FM_OK;
}

int fm_batch_resident(fm_batch* b, int32_t* problems, int64_t* elems, int64_t* free_elems) {
  if (!b) return fail(FM_ERR_INVALID, "null batch");
  int32_t np = 0;
  int64_t ne = 0;
  for (const Placement& pl : b->slots)
    if (pl.p) {
      ++np;
      ne += pl.p->E;
    }
  if (problems) *problems = np;
  if (elems) *elems = ne;
  if (free_elems) {
    int64_t f = 0;
    for (auto& kv : b->pools[P_ELEM].free) f = std::max(f, kv.second);
    *free_elems = f;
  }
  return FM_OK;
}

int fm_problem_get_state(fm_problem* p, double* u, double* pres, double* elem3, double* sdus) {
  NvtxRange nvtx_range("fm_problem_get_state");
  if (!p) return fail(FM_ERR_INVALID, "null problem");
  fm_batch* b = p->batch;
  if (!b) return fail(FM_ERR_INVALID, "problem is not in a batch");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  const Placement& pl = b->slots[p->index];
  const int64_t nb = pl.off[P_NODE], eb = pl.off[P_ELEM];
  const int64_t N = p->N, E = p->E;
  const std::vector<int32_t>& nn = pl.L->node_new[0];
  const auto& eo = pl.L->elem_old[0];
  const int64_t EC = (int64_t)eo.size();
  std::vector<double> tmp(N);
  double* cols[4] = {b->D.su, b->D.sv, b->D.sw, b->D.sp};
  if (u) {
    for (int c = 0; c < 3; ++c) {
      CK(cudaMemcpy(tmp.data(), cols[c] + nb, sizeof(double) * N, cudaMemcpyDeviceToHost));
      for (int64_t i = 0; i < N; ++i) u[i * 3 + c] = tmp[nn[i]];
    }
    if (b->solver == FM_SOLVER_SUPG && p->params.glob_fixed)
      for (int64_t i = 0; i < N; ++i)
        for (int c = 0; c < 3; ++c)
          if (p->params.glob_fixed & (1 << c)) u[i * 3 + c] = 0.0;
  }
  if (b->solver == FM_SOLVER_VMS) {
    if (pres) {
      CK(cudaMemcpy(tmp.data(), cols[3] + nb, sizeof(double) * N, cudaMemcpyDeviceToHost));
      for (int64_t i = 0; i < N; ++i) pres[i] = tmp[nn[i]];
    }
    if (elem3 || sdus) {
      std::vector<double> h((size_t)E * 12), col(EC);
      std::vector<float> colf(b->D.sdus32 ? EC : 0);
      for (int q = 0; q < 12; ++q) {
        if (b->D.sdus32) {
          CK(cudaMemcpy(colf.data(), b->D.sdus32 + (int64_t)q * b->D.E + eb, sizeof(float) * EC,
                        cudaMemcpyDeviceToHost));
          for (int64_t k = 0; k < EC; ++k) col[k] = colf[k];
        } else {
          CK(cudaMemcpy(col.data(), b->D.sdus + (int64_t)q * b->D.E + eb, sizeof(double) * EC,
                        cudaMemcpyDeviceToHost));
        }
        for (int64_t k = 0; k < EC; ++k)
          if (eo[k] >= 0) h[(size_t)eo[k] * 12 + q] = col[k];
      }
      if (sdus) memcpy(sdus, h.data(), sizeof(double) * E * 12);
      if (elem3)
        for (int64_t e = 0; e < E; ++e)
          for (int c = 0; c < 3; ++c) {
            // eval_centroid_subgrid (src lines 713-724): sum_a sdu[a][c]*0.25
            double s = 0.0;
            for (int g = 0; g < 4; ++g) s += h[(size_t)e * 12 + g * 3 + c] * 0.25;
            elem3[e * 3 + c] = s;
          }
    }
  } else {
    if (pres) {
      cudaError_t e = launch_supg_pressure(b->D, b->tn_max, b->npe, b->d_scratch, b->stream);
      if (e != cudaSuccess) return fail(FM_ERR_CUDA, cudaGetErrorString(e));
      CK(cudaStreamSynchronize(b->stream));
      std::vector<double> col(EC);
      CK(cudaMemcpy(col.data(), b->d_scratch + eb, sizeof(double) * EC, cudaMemcpyDeviceToHost));
      for (int64_t k = 0; k < EC; ++k)
        if (eo[k] >= 0) pres[eo[k]] = col[k];
    }
    if (elem3) {
      std::vector<double> c1(EC), c2(EC);
      CK(cudaMemcpy(c1.data(), b->D.el_lam + eb, sizeof(double) * EC, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(c2.data(), b->D.el_reg + eb, sizeof(double) * EC, cudaMemcpyDeviceToHost));
      for (int64_t k = 0; k < EC; ++k) {
        if (eo[k] < 0) continue;
        elem3[(int64_t)eo[k] * 2 + 0] = c1[k];
        elem3[(int64_t)eo[k] * 2 + 1] = c2[k];
      }
    }
  }
  return FM_OK;
}

}  // extern "C"

// ---- checkpoint / restart ----
// File layout (little-endian): CkptHeader, then in the problem's own
// numbering
//   8 node columns of n_nodes doubles: u v w p after BCs, u v w p before BCs;
//   n_sd_cols element columns of n_elems values of sd_bytes each (VMS: the
//     12 Gauss-point subscales [gp*3+c], FP32 in the mixed form; SUPG: the
//     3*npe AB2 history columns of a problem without EXOPTS euler);
//   n_diag_cols element columns of n_elems doubles (SUPG: lambda, regime).
namespace {
struct CkptHeader {
  char magic[8];  // "FMSTATE1"
  int32_t version, solver, precision, npe;
  int64_t n_nodes, n_elems;
  int32_t n_sd_cols, sd_bytes, n_diag_cols, iter;
  int32_t status, reserved;
  int64_t steps_done;
  double time, max_u2;
  double q1p[8];  // pre-BC pressures of nodes 0..3, both iteration parities
  uint64_t setup_hash;  // setup_hash(): mesh, parameters, BCs
};
static_assert(sizeof(CkptHeader) == 160, "checkpoint header size");

// FNV-1a over the 64-bit words of the coordinates, then the connectivity,
// then everything else that shapes the solve: the physical and time-stepping
// parameters and the BC records and tables.  A checkpoint restores only into
// a problem with the same hash.
uint64_t setup_hash(const fm_problem* p) {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](uint64_t w) { h = (h ^ w) * 1099511628211ull; };
  auto mixd = [&](double d) {
    uint64_t w;
    memcpy(&w, &d, 8);
    mix(w);
  };
  auto mixbytes = [&](const void* data, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < n; ++i) mix(c[i]);
  };
  for (int64_t i = 0; i < p->N * 3; ++i) mixd(p->coords[i]);
  const int64_t nc = p->E * p->etype;
  for (int64_t i = 0; i < nc; ++i) mix((uint64_t)(uint32_t)p->conn[i]);
  mix((uint64_t)p->N);
  mix((uint64_t)p->E);
  const fm_params& q = p->params;
  for (int i = 0; i < 5; ++i) mixd(q.props[i]);
  mixd(q.time_step);
  mixd(q.dual_step);
  mixd(q.exit_condition);
  mix((uint64_t)(uint32_t)q.tot_dual_steps);
  for (int i = 0; i < 6; ++i) mix((uint64_t)(uint32_t)q.ex_opts[i]);
  mix((uint64_t)(uint32_t)q.glob_fixed);
  mixbytes(p->node_rec.data(), p->node_rec.size() * sizeof(int32_t));
  mixbytes(p->recs.data(), p->recs.size() * sizeof(BCRec));
  mixbytes(p->tab_off.data(), p->tab_off.size() * sizeof(int32_t));
  mixbytes(p->tab_len.data(), p->tab_len.size() * sizeof(int32_t));
  for (double d : p->tab_rows) mixd(d);
  return h;
}

struct CkptCols {
  int n_sd = 0, sd_bytes = 8, n_diag = 0;
};
CkptCols ckpt_cols(const fm_batch* b, const fm_problem* p) {
  CkptCols c;
  if (b->solver == FM_SOLVER_VMS) {
    c.n_sd = 12;
    c.sd_bytes = b->D.sdus32 ? 4 : 8;
  } else {
    c.n_sd = p->params.ex_opts[0] == 0 ? 3 * b->npe : 0;  // only AB2 reads its history
    c.n_diag = 2;
  }
  return c;
}

// Device address of element column q of slot range eb (subscales or
// history first, then lambda and regime).
void* ckpt_elem_col(const fm_batch* b, const CkptCols& cc, int q, int64_t eb) {
  if (q >= cc.n_sd) return (q == cc.n_sd ? b->D.el_lam : b->D.el_reg) + eb;
  if (cc.sd_bytes == 4) return b->D.sdus32 + (int64_t)q * b->D.E + eb;
  return b->D.sdus + (int64_t)q * b->D.E + eb;
}

struct FileCloser {
  FILE* f;
  ~FileCloser() {
    if (f) fclose(f);
  }
};
}  // namespace

extern "C" {

int fm_problem_checkpoint(fm_problem* p, const char* path) {
  NvtxRange nvtx_range("fm_problem_checkpoint");
  if (!p || !path) return fail(FM_ERR_INVALID, "null argument");
  fm_batch* b = p->batch;
  if (!b) return fail(FM_ERR_INVALID, "problem is not in a batch");
  if (b->x_open) return fail(FM_ERR_INVALID, "an exchange is open: checkpoint after fm_batch_exchange_end");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  const int ps = p->index;
  const Placement& pl = b->slots[ps];
  const int64_t nb = pl.off[P_NODE], eb = pl.off[P_ELEM];
  const int64_t N = p->N, E = p->E;
  const std::vector<int32_t>& nn = pl.L->node_new[0];
  const auto& eo = pl.L->elem_old[0];
  const int64_t EC = (int64_t)eo.size();
  const CkptCols cc = ckpt_cols(b, p);

  CkptHeader h;
  memset(&h, 0, sizeof(h));
  memcpy(h.magic, "FMSTATE1", 8);
  h.version = 2;
  h.solver = b->solver;
  h.precision = b->precision;
  h.npe = b->npe;
  h.n_nodes = N;
  h.n_elems = E;
  h.n_sd_cols = cc.n_sd;
  h.sd_bytes = cc.sd_bytes;
  h.n_diag_cols = cc.n_diag;
  DevProbState st;
  CK(cudaMemcpy(&st, b->D.pstate + ps, sizeof(st), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(h.q1p, b->D.q1p + (int64_t)ps * 8, sizeof(h.q1p), cudaMemcpyDeviceToHost));
  h.iter = st.iter;
  h.status = st.status;
  h.time = st.time;
  h.max_u2 = st.max_u2;
  h.steps_done = p->steps_done;
  h.setup_hash = setup_hash(p);

  // written to path.tmp and renamed over path once complete, so a failed or
  // short write never replaces an earlier good checkpoint
  const std::string tmp_path = std::string(path) + ".tmp";
  FileCloser fc{fopen(tmp_path.c_str(), "wb")};
  if (!fc.f) return fail(FM_ERR_IO, std::string("cannot open ") + tmp_path);
  bool ok = fwrite(&h, sizeof(h), 1, fc.f) == 1;
  std::vector<double> tmp(N), out(N);
  double* cols[8] = {b->D.su, b->D.sv, b->D.sw, b->D.sp, b->D.pu, b->D.pv, b->D.pw, b->D.pp};
  for (int c = 0; c < 8 && ok; ++c) {
    CK(cudaMemcpy(tmp.data(), cols[c] + nb, sizeof(double) * N, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < N; ++i) out[i] = tmp[nn[i]];
    ok = fwrite(out.data(), sizeof(double), N, fc.f) == (size_t)N;
  }
  // element columns: device slot k holds problem element eo[k] (padding < 0)
  std::vector<char> col((size_t)EC * 8), eout((size_t)E * 8);
  for (int q = 0; q < cc.n_sd + cc.n_diag && ok; ++q) {
    const int bytes = q < cc.n_sd ? cc.sd_bytes : 8;
    CK(cudaMemcpy(col.data(), ckpt_elem_col(b, cc, q, eb), (size_t)EC * bytes, cudaMemcpyDeviceToHost));
    for (int64_t k = 0; k < EC; ++k)
      if (eo[k] >= 0) memcpy(&eout[(size_t)eo[k] * bytes], &col[(size_t)k * bytes], bytes);
    ok = fwrite(eout.data(), bytes, E, fc.f) == (size_t)E;
  }
  ok = ok && fflush(fc.f) == 0;
  ok = (fclose(fc.f) == 0) && ok;
  fc.f = nullptr;
  if (!ok || rename(tmp_path.c_str(), path) != 0) {
    remove(tmp_path.c_str());
    return fail(FM_ERR_IO, std::string("cannot write ") + path);
  }
  return FM_OK;
}

int fm_problem_restore(fm_problem* p, const char* path) {
  NvtxRange nvtx_range("fm_problem_restore");
  if (!p || !path) return fail(FM_ERR_INVALID, "null argument");
  fm_batch* b = p->batch;
  if (!b) return fail(FM_ERR_INVALID, "problem is not in a batch");
  if (b->x_open) return fail(FM_ERR_INVALID, "an exchange is open: restore after fm_batch_exchange_end");
  FileCloser fc{fopen(path, "rb")};
  if (!fc.f) return fail(FM_ERR_IO, std::string("cannot open ") + path);
  CkptHeader h;
  if (fread(&h, sizeof(h), 1, fc.f) != 1 || memcmp(h.magic, "FMSTATE1", 8) != 0 || h.version != 2)
    return fail(FM_ERR_INVALID, std::string(path) + " is not a femorph_b200 checkpoint");
  const CkptCols cc = ckpt_cols(b, p);
  if (h.solver != b->solver || h.precision != b->precision || h.npe != b->npe)
    return fail(FM_ERR_INVALID, "checkpoint of another solver, precision or element type");
  if (h.n_nodes != p->N || h.n_elems != p->E || h.setup_hash != setup_hash(p))
    return fail(FM_ERR_INVALID, "checkpoint of another mesh, parameter set or BC set");
  if (h.n_sd_cols != cc.n_sd || h.sd_bytes != cc.sd_bytes || h.n_diag_cols != cc.n_diag)
    return fail(FM_ERR_INVALID, "checkpoint element columns differ (SUPG AB2 history or not)");
  if (h.iter < 0 || h.steps_done < 0) return fail(FM_ERR_INVALID, "checkpoint counters out of range");
  const int64_t N = p->N, E = p->E;
  // read everything before touching the device, so a bad file leaves the
  // problem's state as it was
  std::vector<double> nodes((size_t)N * 8);
  if (fread(nodes.data(), sizeof(double), nodes.size(), fc.f) != nodes.size())
    return fail(FM_ERR_IO, std::string("truncated checkpoint ") + path);
  const int ncols = cc.n_sd + cc.n_diag;
  std::vector<std::vector<char>> ecols(ncols);
  for (int q = 0; q < ncols; ++q) {
    const int bytes = q < cc.n_sd ? cc.sd_bytes : 8;
    ecols[q].resize((size_t)E * bytes);
    if (fread(ecols[q].data(), bytes, E, fc.f) != (size_t)E)
      return fail(FM_ERR_IO, std::string("truncated checkpoint ") + path);
  }
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  const int ps = p->index;
  const Placement& pl = b->slots[ps];
  const int64_t nb = pl.off[P_NODE], eb = pl.off[P_ELEM];
  const std::vector<int32_t>& nn = pl.L->node_new[0];
  const auto& eo = pl.L->elem_old[0];
  const int64_t EC = (int64_t)eo.size();
  std::vector<double> tmp(N);
  double* cols[8] = {b->D.su, b->D.sv, b->D.sw, b->D.sp, b->D.pu, b->D.pv, b->D.pw, b->D.pp};
  for (int c = 0; c < 8; ++c) {
    const double* in = nodes.data() + (size_t)c * N;
    for (int64_t i = 0; i < N; ++i) tmp[nn[i]] = in[i];
    CK(cudaMemcpy(cols[c] + nb, tmp.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  }
  // element columns: padding slots keep their device values
  std::vector<char> col((size_t)EC * 8);
  for (int q = 0; q < ncols; ++q) {
    const int bytes = q < cc.n_sd ? cc.sd_bytes : 8;
    void* dev = ckpt_elem_col(b, cc, q, eb);
    CK(cudaMemcpy(col.data(), dev, (size_t)EC * bytes, cudaMemcpyDeviceToHost));
    for (int64_t k = 0; k < EC; ++k)
      if (eo[k] >= 0) memcpy(&col[(size_t)k * bytes], &ecols[q][(size_t)eo[k] * bytes], bytes);
    CK(cudaMemcpy(dev, col.data(), (size_t)EC * bytes, cudaMemcpyHostToDevice));
  }
  DevProbState st;
  memset(&st, 0, sizeof(st));
  st.iter = h.iter;
  st.status = h.status;
  st.time = h.time;
  st.max_u2 = h.max_u2;
  CK(cudaMemcpy(b->D.pstate + ps, &st, sizeof(st), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b->D.q1p + (int64_t)ps * 8, h.q1p, sizeof(h.q1p), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(const_cast<int32_t*>(b->D.target) + ps, &h.iter, sizeof(int32_t), cudaMemcpyHostToDevice));
  b->iters[ps] = h.iter;
  p->steps_done = h.steps_done;
  return FM_OK;
}

}  // extern "C"

// ---- VMS diagnostics (the reference's log line and res_v / res_p) ----
extern "C" {

int fm_batch_set_wait_limit(fm_batch* b, uint32_t polls) {
  if (!b) return fail(FM_ERR_INVALID, "null batch");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  // captured graphs hold the batch view (and so the limit) by value
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->D.wait_limit = polls;
  return FM_OK;
}

int fm_batch_set_diagnostics(fm_batch* b, int32_t enable) {
  NvtxRange nvtx_range("fm_batch_set_diagnostics");
  if (!b) return fail(FM_ERR_INVALID, "null batch");
  if (b->solver != FM_SOLVER_VMS) return fail(FM_ERR_INVALID, "diagnostics are those of the VMS solver");
  if (b->exchange) return fail(FM_ERR_INVALID, "diagnostics are not kept for partition parts");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  // captured graphs hold the batch view with or without the residual buffer
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  if (!enable) {
    diag_free(b);
    return FM_OK;
  }
  if (b->diag) return FM_OK;
  const size_t ecap = (size_t)std::max<int64_t>(b->D.E, 1);
  cudaError_t e = cudaMalloc((void**)&b->d_diag_res, ecap * 16 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_cres, ecap * 16 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_diag_out, 3 * DIAG_BLOCKS * sizeof(double));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&b->h_diag, 3 * DIAG_BLOCKS * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(b->d_diag_res, 0, ecap * 16 * sizeof(double));
  if (e != cudaSuccess) {
    diag_free(b);
    return fail(e == cudaErrorMemoryAllocation ? FM_ERR_OOM : FM_ERR_CUDA,
                std::string("diagnostics: ") + cudaGetErrorString(e));
  }
  b->D.diag_res = b->d_diag_res;
  b->diag = true;
  for (Placement& pl : b->slots)
    if (pl.p) {
      int r = diag_prepare_problem(pl);
      if (r) {
        diag_free(b);
        return r;
      }
    }
  return FM_OK;
}

int fm_problem_vms_log(fm_problem* p, double* rows, int32_t max_rows, int32_t* n_rows) {
  if (!p || !n_rows) return fail(FM_ERR_INVALID, "null argument");
  const int64_t queued = (int64_t)p->diag_rows.size() / 6;
  if (!rows) {
    *n_rows = (int32_t)std::min<int64_t>(queued, INT32_MAX);
    return FM_OK;
  }
  const int64_t n = std::min<int64_t>(queued, std::max(0, max_rows));
  if (n > 0) {
    memcpy(rows, p->diag_rows.data(), (size_t)n * 6 * sizeof(double));
    p->diag_rows.erase(p->diag_rows.begin(), p->diag_rows.begin() + n * 6);
  }
  *n_rows = (int32_t)n;
  return FM_OK;
}

int fm_problem_vms_residuals(fm_problem* p, double* res_u, double* res_p) {
  if (!p) return fail(FM_ERR_INVALID, "null problem");
  fm_batch* b = p->batch;
  if (!b || !b->diag) return fail(FM_ERR_INVALID, "problem is not in a batch with diagnostics on");
  const Placement& pl = b->slots[p->index];
  if (!pl.dg_el) return fail(FM_ERR_INVALID, "no diagnostics for this problem");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  const int64_t E = p->E;
  std::vector<double> el((size_t)E * 4);
  CK(cudaMemcpy(el.data(), pl.dg_el, el.size() * sizeof(double), cudaMemcpyDeviceToHost));
  for (int64_t e = 0; e < E; ++e) {
    if (res_u)
      for (int c = 0; c < 3; ++c) res_u[e * 3 + c] = el[(size_t)e * 4 + c];
    if (res_p) res_p[e] = el[(size_t)e * 4 + 3];
  }
  return FM_OK;
}

}  // extern "C"
