// Internal host/device data structures of femorph_b200.
#pragma once
#include <cstdint>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/femorph_b200.h"

namespace fm {

// NVTX range over a host phase of the library (preparation, placement,
// stepping, I/O) for the lifetime of the object; without a profiler
// attached the push and pop return at once.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Allocator whose value-initialisation leaves trivial elements unset, so
// large host arrays are first touched (and filled) by the host threads that
// fill them instead of being zeroed by one thread first.
template <class T>
struct uninit_alloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = uninit_alloc<U>;
  };
  uninit_alloc() = default;
  template <class U>
  uninit_alloc(const uninit_alloc<U>&) {}
  template <class U>
  void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
    ::new ((void*)p) U;
  }
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    ::new ((void*)p) U(std::forward<A>(a)...);
  }
};
template <class T>
using hvec = std::vector<T, uninit_alloc<T>>;

// Runs f(begin, end, worker) over [0, n) in contiguous blocks on up to 32
// host threads, at least `grain` items a block (inline for small n).
template <class F>
inline void parallel_blocks(int64_t n, F f, int64_t grain = 4096) {
  const int64_t hc = (int64_t)std::thread::hardware_concurrency();
  const int64_t hw = hc < 1 ? 1 : (hc > 32 ? 32 : hc);
  int64_t nt = n / (grain > 0 ? grain : 1);
  nt = nt < 1 ? 1 : (nt > hw ? hw : nt);
  if (nt <= 1) {
    f((int64_t)0, n, 0);
    return;
  }
  std::vector<std::thread> th;
  for (int64_t t = 0; t < nt; ++t)
    th.emplace_back([&, t] { f(n * t / nt, n * (t + 1) / nt, (int)t); });
  for (auto& x : th) x.join();
}


// Resolved boundary condition of one node.  The reference applies, in this
// order, setNodeVelocity (per NODEVEL node, table-interpolated components
// selected by the direction code), apply_zeroTraction (NODEPRES, VMS only)
// and setDirichletBC (NODEDIRBC, all three components); later rows of the
// same list overwrite earlier ones (femModel.cpp:4581-4643,
// femVMSExplicitFluidSolver.cpp:648-653).
enum : int32_t { BC_VX = 1, BC_VY = 2, BC_VZ = 4, BC_PRES = 8, BC_DIR = 16 };
struct BCRec {
  int32_t tab;    // velocity table index, -1 if none
  int32_t mask;   // BC_* bits
  double p;       // NODEPRES value
  double d[3];    // NODEDIRBC values
};

// Per-problem constants on the device.
struct DevProb {
  double nu, inv_eps, c1, c2, dt, ds, rho, mu, alpha, c_i, exit_cond;
  int32_t ndual, solver, precision, npe;
  int32_t ex_mask;     // SUPG: bit0 euler, bit1 B-bar, bit2..5 K1..K4
  int32_t glob_fixed;  // SUPG FM_FIX_* mask
  int32_t q1[4];       // VMS: batch ids of the problem's nodes 0..3 (-1 absent)
  int32_t xslice;      // partition part: its slice of the exchange buffers (-1: not a part)
  int32_t pad_x;
  int64_t node_begin, n_nodes, elem_begin, n_elems;
};

// Default polls of a tile CTA's bounded wait for one chunk's bulk copies
// (each mbarrier try_wait may itself suspend for a bounded time).
constexpr uint32_t FM_WAIT_LIMIT = 1u << 22;

// Per-problem progress on the device.  iter counts completed dual
// iterations (VMS) or steps (SUPG); a pass only works on problems with
// iter < target[p] (a separate array, set by the host per launch block).
// time is the physical time of the step iter belongs to, accumulated by
// repeated addition like the reference's currentTime.
struct DevProbState {
  int32_t iter;
  int32_t status;   // FM_OK or an FM_ERR_* raised on the device
  int32_t pad0, pad1;
  double time;
  double max_u2;    // max |u|^2 seen in the last node pass (SUPG EXITCOND)
};

// One tile = the elements one CTA owns, their distinct nodes (interior
// nodes first), and the colour ranges of its elements.
struct TileMeta {
  int32_t elem_begin, n_elem;   // batch element range
  int32_t node_begin, n_node;   // range in tile_nodes
  int32_t n_int;                // first n_int local nodes are interior
  int32_t slot_base;            // partial slot of local node n_int
  int32_t col_begin, n_col;     // colour offsets in tile_cols[col_begin .. +n_col]
  int32_t problem;
  int32_t inc_begin;            // node->element incidence entries in tile_inc (multiple of 8)
  int32_t off_begin;            // per-node offsets (n_node+1) into those entries, in tile_off
  int32_t node0;                // batch id of local node 0 when the interior nodes are
                                // consecutive batch ids from it (-1 otherwise); set at placement
};

struct HostProblem;

struct Layout;
}  // namespace fm

struct fm_problem {
  int32_t etype = 4;
  int64_t N = 0, E = 0;
  fm::hvec<double> coords;
  fm::hvec<int32_t> conn;
  fm_params params{};
  std::vector<int32_t> vel_node, vel_dir, dir_node, pres_node;
  std::vector<double> vel_vals, dir_vals, pres_vals;
  std::vector<double> init;  // N*4 or empty
  // Resolved BCs
  std::vector<int32_t> node_rec;   // per node: -1 or record index
  std::vector<fm::BCRec> recs;
  std::vector<int32_t> tab_off, tab_len;
  std::vector<double> tab_rows;    // rows x 4
  // Lumped mass (problem numbering): VMS N, SUPG N*3
  std::vector<double> mass;
  // Prepared tile layout (fm_problem_prepare) and the tile sizes it was built for
  std::shared_ptr<fm::Layout> layout;
  int32_t layout_te = 0, layout_tn = 0;
  // Partition part (fm_problem_partition): its index among n_parts, the
  // global node / element of each local one, and per local node its index
  // in the partition's exchange list (-1: the node is not shared)
  int32_t part = -1, n_parts = 0;
  int64_t x_total = 0;
  std::vector<int32_t> node_global, elem_global, xidx;
  // Batch membership
  fm_batch* batch = nullptr;
  int32_t index = -1;
  int64_t steps_done = 0;
  // VMS diagnostics (fm_batch_set_diagnostics): queued log rows, 6 doubles
  // each, the smallest element length, and the last step whose time was formed
  std::vector<double> diag_rows;
  double diag_min_h = 0.0;
  int64_t diag_step = -1;
  double diag_time = 0.0;
};

namespace fm {
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int resolve_bcs(fm_problem* p);
void compute_mass(fm_problem* p);

// Host arrays of a Poisson solver that its VTK writer needs
// (fm_poisson_write_vtk, fm_io.cpp): the model's coordinates, the fixed
// connectivity, the diffusivity rows, and the exporter's source, Neumann and
// Dirichlet fields.
struct PoissonHostView {
  int64_t N, E;
  int npe, problem;
  const double* coords;
  const int32_t* conn;
  const double* diff;
  const double* src;
  const double* neu;
  const double* dir;
};
const PoissonHostView* poisson_host_view(const fm_poisson* s);

// Host-side layout of a batch (all arrays in batch numbering).
struct Layout {
  int64_t n_nodes = 0, n_elems = 0;
  std::vector<TileMeta> tiles;
  hvec<int32_t> tile_nodes;
  std::vector<int32_t> tile_cols;
  // Per tile, for every local node, the (element-in-tile * npe + corner)
  // entries of its incident elements in element order: the fixed order in
  // which the node-owner threads add element contributions.
  hvec<uint16_t> tile_inc, tile_off;
  int32_t max_tile_elems = 0;
  hvec<uint16_t> conn_local;          // n_elems x npe
  std::vector<int32_t> iface_node, iface_slot_beg, iface_slots, iface_prob;
  std::vector<int32_t> iface_xidx;    // exchange index of each interface node (-1: none); partition parts only
  int64_t n_slots = 0;
  int32_t max_colors = 0;
  // per problem: batch node id of each problem node, problem element of each batch element
  std::vector<std::vector<int32_t>> node_new;   // [prob][old] -> batch id
  std::vector<hvec<int32_t>> elem_old;   // [prob][batch e - elem_begin] -> old element
  std::vector<int64_t> node_begin, elem_begin;
  std::vector<int64_t> elem_count;   // per problem: padded element slots (elem_old has this size, -1 = padding)
};

// Tiles start at multiples of this many element slots.
constexpr int ELEM_ALIGN = 32;
// SUPG hexa8 FP64: stored geometry values per Gauss point (inverse Jacobian
// and det J), 8 points an element.
constexpr int FM_GEO_PER_GP = 10;
// VMS tiles: at most this many nodes (each CTA thread owns up to
// FM_MAX_TILE_NODES / threads of them during accumulation).
#define FM_MAX_TILE_NODES 512

int build_layout(fm_problem* const* probs, int n, int tile_elems, int tile_nodes, Layout& L);
int check_layout(const fm_problem* p, const Layout& L);
void morton_order(const fm_problem* p, hvec<int64_t>& order);
}  // namespace fm
