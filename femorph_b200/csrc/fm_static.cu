// fm_vms_solve_static: a VMS solve that allocates no device memory.
//
// Who needs it: callers that cannot call cudaMalloc.  Examples are a process
// whose device memory is already reserved by another allocator (a
// framework's caching allocator that holds the GPU's memory, where an
// allocation behind its back fails or fragments its pool), and code on a
// latency-bound path, where cudaMalloc and cudaFree synchronise the whole
// device and stall every other stream.  fm_batch_create allocates the
// batch's device arrays; this entry point instead runs the same VMS tile and
// interface kernels over a copy of one problem that it places, together
// with all of the kernels' scratch (interface partial sums, iteration
// counter, subscales), in one file-scope device array of fixed size,
// FM_STATIC_SCRATCH_BYTES.  Every GPU holds that array from the time the
// library's device code is loaded on it (at the latest the first call)
// until the process exits.
//
// The caller passes the inputs (a host fm_problem whose tile layout
// fm_problem_prepare has built) and the outputs (host arrays); each call
// starts from the problem's initial state.  Because every call shares the one
// array, calls must not overlap on the GPU: two calls running at the same
// time, from different host threads or on different streams, race on it.
// What must start at zero (subscales, the pressure history of nodes 0..3,
// the interface pass counter) is cleared by every call; everything else in
// the array is written before it is read.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "fm_device.cuh"
#include "fm_internal.hpp"

namespace fm {
cudaError_t vms_configure(int tn_max, int inc_max);
size_t vms_smem_bytes(int tn_max, int inc_max, int threads, bool mixed);
cudaError_t launch_vms_iteration(const DevBatch& B, int tn_max, int inc_max, int threads, int ctas, int iface_blocks,
                                 bool mixed, bool xpack, cudaStream_t s, cudaEvent_t* ev);
}  // namespace fm

using namespace fm;

static __device__ __align__(256) unsigned char fm_static_scratch[FM_STATIC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of fm_static_scratch on the current device (looked up once
// per device; the host-side name of the array is only a stand-in).
int scratch_address(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[device]) {
    unsigned char* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&ptr, fm_static_scratch);
    if (e != cudaSuccess || !ptr)
      return fail(FM_ERR_CUDA, std::string("cudaGetSymbolAddress(fm_static_scratch): ") + cudaGetErrorString(e));
    e = vms_configure(0, 0);  // kernels' shared-memory limit (no allocation)
    if (e != cudaSuccess) return fail(FM_ERR_CUDA, std::string("kernel attribute: ") + cudaGetErrorString(e));
    g_scratch_addr[device] = ptr;
  }
  *out = g_scratch_addr[device];
  return FM_OK;
}

// Sequential 256-byte-aligned carving of the array.
struct Carve {
  size_t off = 0;
  template <class T>
  size_t take(size_t n) {
    const size_t o = (off + 255) & ~size_t(255);
    off = o + n * sizeof(T);
    return o;
  }
};

struct Offsets {
  size_t node[12], node_bc, recs, tab_off, tab_len, tab_rows, conn, sdus, tiles, tile_nodes, tile_cols, tile_inc,
      tile_off, part, iface_node, iface_beg, iface_cnt, iface_prob, iface_slots, prob, pstate, target, q1p, done,
      in_coords, in_init, in_rec, in_mass, in_node_new, out_u, out_p, total;
};

Offsets plan(const fm_problem* p, const Layout& L) {
  Offsets o;
  Carve c;
  const size_t N = (size_t)p->N, NE = (size_t)L.n_elems, NI = L.iface_node.size();
  for (int k = 0; k < 12; ++k) o.node[k] = c.take<double>(N);
  o.node_bc = c.take<int32_t>(N);
  o.recs = c.take<BCRec>(p->recs.size());
  o.tab_off = c.take<int32_t>(p->tab_off.size());
  o.tab_len = c.take<int32_t>(p->tab_len.size());
  o.tab_rows = c.take<double>(p->tab_rows.size());
  o.conn = c.take<uint16_t>(L.conn_local.size());
  o.sdus = c.take<double>(12 * NE);
  o.tiles = c.take<TileMeta>(L.tiles.size());
  o.tile_nodes = c.take<int32_t>(L.tile_nodes.size());
  o.tile_cols = c.take<int32_t>(L.tile_cols.size());
  o.tile_inc = c.take<uint16_t>(L.tile_inc.size());
  o.tile_off = c.take<uint16_t>(L.tile_off.size());
  o.part = c.take<double>((size_t)L.n_slots * 4);
  o.iface_node = c.take<int32_t>(NI);
  o.iface_beg = c.take<int32_t>(NI + 1);
  o.iface_cnt = c.take<int32_t>(NI);
  o.iface_prob = c.take<int32_t>(NI);
  o.iface_slots = c.take<int32_t>(L.iface_slots.size());
  o.prob = c.take<DevProb>(1);
  o.pstate = c.take<DevProbState>(1);
  o.target = c.take<int32_t>(1);
  o.q1p = c.take<double>(8);
  o.done = c.take<uint32_t>(1);
  o.in_coords = c.take<double>(3 * N);
  o.in_init = c.take<double>(p->init.empty() ? 0 : 4 * N);
  o.in_rec = c.take<int32_t>(N);
  o.in_mass = c.take<double>(N);
  o.in_node_new = c.take<int32_t>(N);
  o.out_u = c.take<double>(3 * N);
  o.out_p = c.take<double>(N);
  o.total = c.off;
  return o;
}

}  // namespace

// Scatters the problem-order inputs into the tile-layout node order and
// applies the BCs at time 0 (the solve() prologue), as fm_batch_create does
// on the host; counts each interface node's partial-sum entries.
__global__ void static_setup_kernel(DevBatch B, const double* coords, const double* init, const int32_t* node_rec,
                                    const double* mass, const int32_t* node_new, int32_t n_nodes) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += stride) {
    const int g = node_new[i];
    double* x = const_cast<double*>(B.x);
    double* y = const_cast<double*>(B.y);
    double* z = const_cast<double*>(B.z);
    x[g] = coords[(int64_t)i * 3 + 0];
    y[g] = coords[(int64_t)i * 3 + 1];
    z[g] = coords[(int64_t)i * 3 + 2];
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    if (init) {
      s[0] = init[(int64_t)i * 4 + 0];
      s[1] = init[(int64_t)i * 4 + 1];
      s[2] = init[(int64_t)i * 4 + 2];
      s[3] = init[(int64_t)i * 4 + 3];
    }
    const int32_t rec = node_rec[i];
    const_cast<int32_t*>(B.node_bc)[g] = rec;
    if (rec >= 0) {
      int32_t status = FM_OK;
      apply_bc(B, rec, 0.0, s, &status);
      if (status != FM_OK) B.pstate[0].status = status;
    }
    B.su[g] = s[0]; B.sv[g] = s[1]; B.sw[g] = s[2]; B.sp[g] = s[3];
    B.pu[g] = s[0]; B.pv[g] = s[1]; B.pw[g] = s[2]; B.pp[g] = s[3];
    const_cast<double*>(B.mass)[g] = mass[i];
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B.n_iface; i += stride)
    const_cast<int32_t*>(B.iface_slot_cnt)[i] = B.iface_slot_beg[i + 1] - B.iface_slot_beg[i];
}

// Gathers velocity and pressure back into the problem's node order.
__global__ void static_gather_kernel(DevBatch B, const int32_t* node_new, int32_t n_nodes, double* u, double* p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += gridDim.x * blockDim.x) {
    const int g = node_new[i];
    u[(int64_t)i * 3 + 0] = B.su[g];
    u[(int64_t)i * 3 + 1] = B.sv[g];
    u[(int64_t)i * 3 + 2] = B.sw[g];
    p[i] = B.sp[g];
  }
}

#define CKS(x)                                                                                        \
  do {                                                                                                \
    cudaError_t _e = (x);                                                                             \
    if (_e != cudaSuccess) return fail(FM_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)); \
  } while (0)

// Puts the caller's current device back on every return path: the entry
// point selects the requested device, and callers that run inside another
// framework's device and stream management must find theirs unchanged.
struct DeviceRestore {
  int prev = -1;
  DeviceRestore() {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  }
  ~DeviceRestore() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

template <class T>
static cudaError_t up(unsigned char* base, size_t off, const T* src, size_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  return cudaMemcpyAsync(base + off, src, n * sizeof(T), cudaMemcpyHostToDevice, s);
}

extern "C" int fm_vms_solve_static(fm_problem* p, int32_t nsteps, int32_t device, double* u, double* pres,
                                   void* stream) {
  NvtxRange nvtx_range("fm_vms_solve_static");
  if (!p || nsteps < 0) return fail(FM_ERR_INVALID, "null problem or negative step count");
  if (p->params.solver != FM_SOLVER_VMS || p->etype != FM_TET4)
    return fail(FM_ERR_INVALID, "fm_vms_solve_static runs the VMS tet4 solver only");
  if (p->params.precision != FM_FP64) return fail(FM_ERR_INVALID, "fm_vms_solve_static runs the FP64 form only");
  if (!p->layout) return fail(FM_ERR_INVALID, "call fm_problem_prepare before fm_vms_solve_static");
  if (p->part >= 0) return fail(FM_ERR_INVALID, "fm_vms_solve_static does not run partition parts");
  const Layout& L = *p->layout;
  const Offsets o = plan(p, L);
  if (o.total > (size_t)FM_STATIC_SCRATCH_BYTES)
    return fail(FM_ERR_INVALID, "problem needs " + std::to_string(o.total) + " bytes of static scratch; the limit is " +
                                    std::to_string((size_t)FM_STATIC_SCRATCH_BYTES) +
                                    " (about 200,000 tetrahedra): use fm_batch_create for larger problems");
  int tn_max = 0;
  for (const TileMeta& tm : L.tiles) tn_max = std::max(tn_max, tm.n_node);
  const int inc_max = (L.max_tile_elems * 4 + 7) / 8 * 8;
  const int threads = 128;
  if (tn_max > FM_MAX_TILE_NODES || vms_smem_bytes(tn_max, inc_max, threads, false) + 1024 > 227 * 1024)
    return fail(FM_ERR_INVALID, "prepared tiles are too large for the VMS kernels");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FM_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= ndev || device >= kMaxDevices) return fail(FM_ERR_INVALID, "bad device ordinal");
  DeviceRestore restore_device;
  CKS(cudaSetDevice(device));
  unsigned char* base = nullptr;
  int r = scratch_address(device, &base);
  if (r) return r;
  cudaStream_t s = (cudaStream_t)stream;

  DevBatch D;
  memset(&D, 0, sizeof(D));
  double* nd[12];
  for (int k = 0; k < 12; ++k) nd[k] = reinterpret_cast<double*>(base + o.node[k]);
  D.x = nd[0]; D.y = nd[1]; D.z = nd[2];
  D.su = nd[3]; D.sv = nd[4]; D.sw = nd[5]; D.sp = nd[6];
  D.pu = nd[7]; D.pv = nd[8]; D.pw = nd[9]; D.pp = nd[10];
  D.mass = nd[11];
  D.node_bc = reinterpret_cast<int32_t*>(base + o.node_bc);
  D.recs = reinterpret_cast<BCRec*>(base + o.recs);
  D.tab_off = reinterpret_cast<int32_t*>(base + o.tab_off);
  D.tab_len = reinterpret_cast<int32_t*>(base + o.tab_len);
  D.tab_rows = reinterpret_cast<double*>(base + o.tab_rows);
  D.conn = reinterpret_cast<uint16_t*>(base + o.conn);
  D.sdus = reinterpret_cast<double*>(base + o.sdus);
  D.sdus32 = nullptr;
  D.E = L.n_elems;
  D.tiles = reinterpret_cast<TileMeta*>(base + o.tiles);
  D.n_tiles = (int32_t)L.tiles.size();
  D.tile_nodes = reinterpret_cast<int32_t*>(base + o.tile_nodes);
  D.tile_cols = reinterpret_cast<int32_t*>(base + o.tile_cols);
  D.tile_inc = reinterpret_cast<uint16_t*>(base + o.tile_inc);
  D.tile_off = reinterpret_cast<uint16_t*>(base + o.tile_off);
  D.part = reinterpret_cast<double2*>(base + o.part);
  D.iface_node = reinterpret_cast<int32_t*>(base + o.iface_node);
  D.iface_slot_beg = reinterpret_cast<int32_t*>(base + o.iface_beg);
  D.iface_slot_cnt = reinterpret_cast<int32_t*>(base + o.iface_cnt);
  D.iface_prob = reinterpret_cast<int32_t*>(base + o.iface_prob);
  D.iface_slots = reinterpret_cast<int32_t*>(base + o.iface_slots);
  D.n_iface = (int32_t)L.iface_node.size();
  D.probs = reinterpret_cast<DevProb*>(base + o.prob);
  D.pstate = reinterpret_cast<DevProbState*>(base + o.pstate);
  D.target = reinterpret_cast<int32_t*>(base + o.target);
  D.q1p = reinterpret_cast<double*>(base + o.q1p);
  D.n_probs = 1;
  D.done = reinterpret_cast<unsigned int*>(base + o.done);
  D.wait_limit = FM_WAIT_LIMIT;

  // problem constants and progress (as fm_batch_create sets them)
  const fm_params& pr = p->params;
  const std::vector<int32_t>& nn = L.node_new[0];
  DevProb d;
  memset(&d, 0, sizeof(d));
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
  d.ndual = std::max(0, pr.tot_dual_steps);
  d.solver = FM_SOLVER_VMS;
  d.precision = FM_FP64;
  d.npe = 4;
  d.glob_fixed = pr.glob_fixed;
  for (int q = 0; q < 4; ++q) d.q1[q] = (q < p->N) ? nn[q] : -1;
  d.node_begin = 0;
  d.n_nodes = p->N;
  d.elem_begin = 0;
  d.n_elems = p->E;
  DevProbState st;
  memset(&st, 0, sizeof(st));
  st.time = 0.0 + pr.time_step;
  const int32_t target = nsteps * (d.ndual + 1);

  // inputs (host -> the array), then the parts that must start at zero
  const size_t N = (size_t)p->N;
  CKS(up(base, o.recs, p->recs.data(), p->recs.size(), s));
  CKS(up(base, o.tab_off, p->tab_off.data(), p->tab_off.size(), s));
  CKS(up(base, o.tab_len, p->tab_len.data(), p->tab_len.size(), s));
  CKS(up(base, o.tab_rows, p->tab_rows.data(), p->tab_rows.size(), s));
  CKS(up(base, o.conn, L.conn_local.data(), L.conn_local.size(), s));
  CKS(up(base, o.tiles, L.tiles.data(), L.tiles.size(), s));
  CKS(up(base, o.tile_nodes, L.tile_nodes.data(), L.tile_nodes.size(), s));
  CKS(up(base, o.tile_cols, L.tile_cols.data(), L.tile_cols.size(), s));
  CKS(up(base, o.tile_inc, L.tile_inc.data(), L.tile_inc.size(), s));
  CKS(up(base, o.tile_off, L.tile_off.data(), L.tile_off.size(), s));
  CKS(up(base, o.iface_node, L.iface_node.data(), L.iface_node.size(), s));
  CKS(up(base, o.iface_beg, L.iface_slot_beg.data(), L.iface_slot_beg.size(), s));
  CKS(up(base, o.iface_prob, L.iface_prob.data(), L.iface_prob.size(), s));
  CKS(up(base, o.iface_slots, L.iface_slots.data(), L.iface_slots.size(), s));
  CKS(up(base, o.prob, &d, 1, s));
  CKS(up(base, o.pstate, &st, 1, s));
  CKS(up(base, o.target, &target, 1, s));
  CKS(up(base, o.in_coords, p->coords.data(), 3 * N, s));
  if (!p->init.empty()) CKS(up(base, o.in_init, p->init.data(), 4 * N, s));
  CKS(up(base, o.in_rec, p->node_rec.data(), N, s));
  CKS(up(base, o.in_mass, p->mass.data(), N, s));
  CKS(up(base, o.in_node_new, nn.data(), N, s));
  CKS(cudaMemsetAsync(base + o.sdus, 0, 12 * (size_t)L.n_elems * sizeof(double), s));
  CKS(cudaMemsetAsync(base + o.q1p, 0, 8 * sizeof(double), s));
  CKS(cudaMemsetAsync(base + o.done, 0, sizeof(uint32_t), s));

  const int blocks = (int)std::min<int64_t>(148 * 8, std::max<int64_t>(1, ((int64_t)N + 255) / 256));
  static_setup_kernel<<<blocks, 256, 0, s>>>(
      D, reinterpret_cast<const double*>(base + o.in_coords),
      p->init.empty() ? nullptr : reinterpret_cast<const double*>(base + o.in_init),
      reinterpret_cast<const int32_t*>(base + o.in_rec), reinterpret_cast<const double*>(base + o.in_mass),
      reinterpret_cast<const int32_t*>(base + o.in_node_new), (int32_t)N);
  CKS(cudaGetLastError());
  const int iface_blocks = (int)std::max<int64_t>(1, std::min<int64_t>((D.n_iface + 255) / 256, 148 * 8));
  for (int32_t it = 0; it < target; ++it)
    CKS(launch_vms_iteration(D, tn_max, inc_max, threads, 0, iface_blocks, false, false, s, nullptr));
  double* du = reinterpret_cast<double*>(base + o.out_u);
  double* dp = reinterpret_cast<double*>(base + o.out_p);
  static_gather_kernel<<<blocks, 256, 0, s>>>(D, reinterpret_cast<const int32_t*>(base + o.in_node_new), (int32_t)N,
                                              du, dp);
  CKS(cudaGetLastError());
  if (u) CKS(cudaMemcpyAsync(u, du, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (pres) CKS(cudaMemcpyAsync(pres, dp, N * sizeof(double), cudaMemcpyDeviceToHost, s));
  DevProbState fin;
  CKS(cudaMemcpyAsync(&fin, D.pstate, sizeof(fin), cudaMemcpyDeviceToHost, s));
  CKS(cudaStreamSynchronize(s));
  if (fin.status != FM_OK) return fail(fin.status, "fm_vms_solve_static: device status " + std::to_string(fin.status));
  return FM_OK;
}
