// Host-side preparation: problem copies, boundary-condition resolution,
// lumped masses and the tiled batch layout.
#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstring>
#include <functional>
#include <numeric>
#include <thread>

#include "fm_internal.hpp"

namespace fm {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
const char* last_error() { return g_last_error.c_str(); }

// NODEVEL direction code -> component mask (femModel.cpp:4593-4629).
static int dir_mask(int32_t d) {
  static const int m[7] = {BC_VX, BC_VY, BC_VZ, BC_VX | BC_VY, BC_VY | BC_VZ, BC_VX | BC_VZ, BC_VX | BC_VY | BC_VZ};
  return (d >= 0 && d <= 6) ? m[d] : -1;
}

// Groups NODEVEL rows into per-node tables the way
// femModel::postProcessNodeVelocities does (femModel.cpp:4549-4576): unique
// sorted node ids (femUtils::MakeCompactList), each node's rows in file
// order, and - reproducing the reference - the direction of the k-th input
// row applied to the k-th unique node.  Then resolves, per node, the final
// effect of setNodeVelocity -> apply_zeroTraction (VMS) -> setDirichletBC.
int resolve_bcs(fm_problem* p) {
  const int64_t N = p->N;
  p->node_rec.assign(N, -1);
  p->recs.clear();
  p->tab_off.clear();
  p->tab_len.clear();
  p->tab_rows.clear();
  const int64_t nv = (int64_t)p->vel_node.size();
  std::vector<int32_t> uniq(p->vel_node);
  std::sort(uniq.begin(), uniq.end());
  uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
  std::vector<std::vector<int64_t>> rows(uniq.size());
  for (int64_t r = 0; r < nv; ++r) {
    int32_t n = p->vel_node[r];
    if (n < 0 || n >= N) return fail(FM_ERR_INVALID, "NODEVEL node out of range");
    size_t k = std::lower_bound(uniq.begin(), uniq.end(), n) - uniq.begin();
    rows[k].push_back(r);
  }
  auto rec_of = [&](int32_t n) -> BCRec& {
    if (p->node_rec[n] < 0) {
      p->node_rec[n] = (int32_t)p->recs.size();
      BCRec r;
      r.tab = -1;
      r.mask = 0;
      r.p = 0.0;
      r.d[0] = r.d[1] = r.d[2] = 0.0;
      p->recs.push_back(r);
    }
    return p->recs[p->node_rec[n]];
  };
  for (size_t k = 0; k < uniq.size(); ++k) {
    int m = dir_mask(p->vel_dir[k]);  // quirk: row k's direction for unique node k
    if (m < 0) return fail(FM_ERR_INVALID, "ERROR: Invalid direction for node velocities.");
    BCRec& r = rec_of(uniq[k]);
    r.tab = (int32_t)p->tab_off.size();
    r.mask |= m;
    p->tab_off.push_back((int32_t)(p->tab_rows.size() / 4));
    p->tab_len.push_back((int32_t)rows[k].size());
    for (int64_t row : rows[k])
      for (int c = 0; c < 4; ++c) p->tab_rows.push_back(p->vel_vals[row * 4 + c]);
  }
  if (p->params.solver == FM_SOLVER_VMS) {
    for (size_t i = 0; i < p->pres_node.size(); ++i) {
      int32_t n = p->pres_node[i];
      if (n < 0 || n >= N) return fail(FM_ERR_INVALID, "NODEPRES node out of range");
      BCRec& r = rec_of(n);
      r.mask |= BC_PRES;
      r.p = p->pres_vals[i];
    }
  }
  for (size_t i = 0; i < p->dir_node.size(); ++i) {
    int32_t n = p->dir_node[i];
    if (n < 0 || n >= N) return fail(FM_ERR_INVALID, "NODEDIRBC node out of range");
    BCRec& r = rec_of(n);
    r.mask |= BC_DIR;
    for (int c = 0; c < 3; ++c) r.d[c] = p->dir_vals[i * 3 + c];
  }
  return FM_OK;
}

// ---- lumped masses (one-time, host, reference operation order) ----

// VMS: initial_assemble (femVMSExplicitFluidSolver.cpp:21-91):
// nd_mass[n] += (detJ/6)/4 over elements in file order.
static void vms_mass(fm_problem* p) {
  // element shares in parallel, then added in element order
  hvec<double> share(p->E);
  const double* X = p->coords.data();
  parallel_blocks(p->E, [&](int64_t eb, int64_t ee, int) {
    for (int64_t e = eb; e < ee; ++e) {
      const int32_t* c = &p->conn[e * 4];
      double x[4][3], j[3][3];
      for (int i = 0; i < 4; ++i)
        for (int k = 0; k < 3; ++k) x[i][k] = X[(int64_t)c[i] * 3 + k];
      for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) j[i][k] = x[k + 1][i] - x[0][i];
      double c00 = j[1][1] * j[2][2] - j[2][1] * j[1][2];
      double c01 = j[2][0] * j[1][2] - j[1][0] * j[2][2];
      double c02 = j[1][0] * j[2][1] - j[2][0] * j[1][1];
      double det = j[0][0] * c00 + j[0][1] * c01 + j[0][2] * c02;
      double V = det / 6.0;
      share[e] = V / 4.0;
    }
  });
  p->mass.assign(p->N, 0.0);
  for (int64_t e = 0; e < p->E; ++e) {
    const int32_t* c = &p->conn[e * 4];
    const double q = share[e];
    for (int i = 0; i < 4; ++i) p->mass[c[i]] += q;
  }
}

// SUPG: form_lumped_mass (femSUPGExplicitFluidSolver.cpp:507-598).  The
// row-sum of the consistent mass is the same for the three components of a
// node, so one value per node is kept.
static void supg_mass(fm_problem* p) {
  const int npe = p->etype;
  const double rho = p->params.props[0];
  double gps[8][3], gpw[8];
  int ngp;
  if (npe == 4) {
    const double a = 0.58541020, b = 0.13819660;
    double t[4][3] = {{a, b, b}, {b, a, b}, {b, b, a}, {b, b, b}};
    ngp = 4;
    for (int g = 0; g < 4; ++g) {
      for (int k = 0; k < 3; ++k) gps[g][k] = t[g][k];
      gpw[g] = (1.0 / 6.0) * (1.0 / 4.0);
    }
  } else {
    double s = 1.0 / std::sqrt(3.0);
    double t[8][3] = {{-s, -s, s}, {s, -s, s}, {s, s, s}, {-s, s, s}, {-s, -s, -s}, {s, -s, -s}, {s, s, -s}, {-s, s, -s}};
    ngp = 8;
    for (int g = 0; g < 8; ++g) {
      for (int k = 0; k < 3; ++k) gps[g][k] = t[g][k];
      gpw[g] = 8.0 * (1.0 / 8.0);
    }
  }
  static const double c1[8] = {-1.0, 1.0, 1.0, -1.0, -1.0, 1.0, 1.0, -1.0};
  static const double c2[8] = {-1.0, -1.0, 1.0, 1.0, -1.0, -1.0, 1.0, 1.0};
  static const double c3[8] = {-1.0, -1.0, -1.0, -1.0, 1.0, 1.0, 1.0, 1.0};
  // element row sums in parallel, then added in element order
  hvec<double> rows((size_t)p->E * npe);
  const double* X = p->coords.data();
  parallel_blocks(p->E, [&](int64_t eb, int64_t ee, int) {
  for (int64_t e = eb; e < ee; ++e) {
    const int32_t* cn = &p->conn[e * npe];
    double xe[8][3];
    for (int a = 0; a < npe; ++a)
      for (int k = 0; k < 3; ++k) xe[a][k] = X[(int64_t)cn[a] * 3 + k];
    double M[8][8];
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) M[a][b] = 0.0;
    for (int g = 0; g < ngp; ++g) {
      const double* q = gps[g];
      double Nf[8], dN[8][3];
      if (npe == 4) {
        Nf[0] = q[0]; Nf[1] = q[1]; Nf[2] = q[2]; Nf[3] = 1.0 - q[0] - q[1] - q[2];
        static const double t[4][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}, {-1.0, -1.0, -1.0}};
        for (int a = 0; a < 4; ++a)
          for (int k = 0; k < 3; ++k) dN[a][k] = t[a][k];
      } else {
        for (int a = 0; a < 8; ++a) {
          Nf[a] = (1.0 / 8.0) * (1.0 + q[0] * c1[a]) * (1.0 + q[1] * c2[a]) * (1.0 + q[2] * c3[a]);
          dN[a][0] = (1.0 / 8.0) * c1[a] * (1.0 + q[1] * c2[a]) * (1.0 + q[2] * c3[a]);
          dN[a][1] = (1.0 / 8.0) * c2[a] * (1.0 + q[0] * c1[a]) * (1.0 + q[2] * c3[a]);
          dN[a][2] = (1.0 / 8.0) * c3[a] * (1.0 + q[0] * c1[a]) * (1.0 + q[1] * c2[a]);
        }
      }
      double J[3][3];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double t = 0.0;
          for (int n = 0; n < npe; ++n) t += dN[n][a] * xe[n][b];
          J[a][b] = t;
        }
      double detJ = J[0][0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                    J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
      for (int a = 0; a < npe; ++a)
        for (int b = 0; b < npe; ++b) M[a][b] += rho * Nf[a] * Nf[b] * detJ * gpw[g];
    }
    for (int a = 0; a < npe; ++a) {
      double t = 0.0;
      for (int b = 0; b < npe; ++b) t += M[a][b];
      rows[(size_t)e * npe + a] = t;
    }
  }
  }, 1024);
  p->mass.assign(p->N, 0.0);
  for (int64_t e = 0; e < p->E; ++e)
    for (int a = 0; a < npe; ++a) p->mass[p->conn[e * npe + a]] += rows[(size_t)e * npe + a];
}

void compute_mass(fm_problem* p) {
  if (p->params.solver == FM_SOLVER_VMS)
    vms_mass(p);
  else
    supg_mass(p);
}

// ---- tiled layout ----

// Sorts element indices by (key, index) - the order a stable sort by key
// gives.  Keys are below 2^63 (3 x 21-bit Morton interleave): the pairs are
// distributed into 65536 buckets by their top 16 bits (per-worker histograms),
// then the buckets are sorted in parallel.  The pair array is a trivial type,
// so it is first touched by the distributing threads, not zeroed first.
static void sort_by_key(const hvec<uint64_t>& key, hvec<int64_t>& order) {
  const int64_t E = (int64_t)key.size();
  constexpr int NB = 1 << 16, SHIFT = 63 - 16;
  const int64_t hw = std::max<int64_t>(1, std::min<int64_t>(32, std::thread::hardware_concurrency()));
  const int64_t nw = std::min<int64_t>(hw, std::max<int64_t>(1, E / 65536));
  std::vector<int64_t> hist((size_t)nw * NB, 0);
  auto run = [&](auto&& f) {
    std::vector<std::thread> th;
    for (int64_t w = 0; w < nw; ++w) th.emplace_back([&, w] { f(w, E * w / nw, E * (w + 1) / nw); });
    for (auto& x : th) x.join();
  };
  run([&](int64_t w, int64_t b, int64_t e) {
    int64_t* h = &hist[(size_t)w * NB];
    for (int64_t i = b; i < e; ++i) h[std::min<uint64_t>(key[i] >> SHIFT, NB - 1)]++;
  });
  // bucket-major, worker-minor offsets
  std::vector<int64_t> start(NB + 1, 0);
  {
    int64_t acc = 0;
    for (int k = 0; k < NB; ++k) {
      start[k] = acc;
      for (int64_t w = 0; w < nw; ++w) {
        const int64_t c = hist[(size_t)w * NB + k];
        hist[(size_t)w * NB + k] = acc;
        acc += c;
      }
    }
    start[NB] = acc;
  }
  struct KV {
    uint64_t k;
    int64_t i;
    bool operator<(const KV& o) const { return k < o.k || (k == o.k && i < o.i); }
  };
  hvec<KV> kv(E);
  run([&](int64_t w, int64_t b, int64_t e) {
    int64_t* h = &hist[(size_t)w * NB];
    for (int64_t i = b; i < e; ++i) kv[h[std::min<uint64_t>(key[i] >> SHIFT, NB - 1)]++] = KV{key[i], i};
  });
  // each worker sorts its buckets and writes their part of the order
  order.resize(E);
  {
    std::vector<std::thread> th;
    for (int64_t w = 0; w < nw; ++w)
      th.emplace_back([&, w] {
        const int k0 = (int)(NB * w / nw), k1 = (int)(NB * (w + 1) / nw);
        for (int k = k0; k < k1; ++k) std::sort(kv.begin() + start[k], kv.begin() + start[k + 1]);
        for (int64_t i = start[k0]; i < start[k1]; ++i) order[i] = kv[i].i;
      });
    for (auto& x : th) x.join();
  }
}

// Set of node ids (open addressing, cleared in O(size)), for the distinct
// nodes of one tile.
struct NodeSet {
  std::vector<int32_t> slot, used;
  uint32_t mask = 0;
  explicit NodeSet(int cap_nodes) {
    uint32_t c = 64;
    while (c < (uint32_t)cap_nodes * 4u) c <<= 1;
    slot.assign(c, -1);
    mask = c - 1;
    used.reserve(cap_nodes + 16);
  }
  bool contains(int32_t v) const {
    for (uint32_t h = ((uint32_t)v * 2654435761u) & mask;; h = (h + 1) & mask) {
      if (slot[h] == v) return true;
      if (slot[h] < 0) return false;
    }
  }
  void insert(int32_t v) {
    for (uint32_t h = ((uint32_t)v * 2654435761u) & mask;; h = (h + 1) & mask) {
      if (slot[h] == v) return;
      if (slot[h] < 0) {
        slot[h] = v;
        used.push_back((int32_t)h);
        return;
      }
    }
  }
  void clear() {
    for (int32_t h : used) slot[h] = -1;
    used.clear();
  }
};

// End of the greedy tile that starts at sorted position s: elements are
// taken while the tile has at most TE of them and at most TN distinct nodes
// (an element's repeated node counts once).  Depends on s only.
static int64_t greedy_next(const int32_t* cs, int npe, int64_t E, int TE, int TN, int64_t s, NodeSet& set) {
  int64_t n_el = 0, n_nodes = 0, oi = s;
  for (; oi < E; ++oi) {
    const int32_t* c = &cs[(size_t)oi * npe];
    int fresh = 0;
    for (int a = 0; a < npe; ++a) {
      bool dup = false;
      for (int b = 0; b < a; ++b) dup |= (c[b] == c[a]);
      if (!dup && !set.contains(c[a])) ++fresh;
    }
    if (n_el > 0 && (n_el + 1 > TE || n_nodes + fresh > TN)) break;
    for (int a = 0; a < npe; ++a) set.insert(c[a]);
    n_nodes += fresh;
    ++n_el;
  }
  set.clear();
  return oi;
}

// Tile starts of the greedy cut over the whole sorted order, computed in
// parallel: each worker follows the chain from a segment start (a multiple
// of TE); the true chain is then joined segment by segment, following a
// worker's chain from the first start the two share (the cut from a start
// does not depend on how the start was reached) and recomputing only
// between the true chain's entry into a segment and that meeting point.
static void greedy_tiles(const int32_t* cs, int npe, int64_t E, int TE, int TN, std::vector<int64_t>& starts) {
  const int64_t hw = std::max<int64_t>(1, std::min<int64_t>(32, std::thread::hardware_concurrency()));
  int64_t P = std::min<int64_t>(hw, std::max<int64_t>(1, E / (64 * (int64_t)TE)));
  std::vector<int64_t> b;
  for (int64_t k = 0; k < P; ++k) {
    const int64_t v = (E * k / P) / TE * TE;
    if (b.empty() || v > b.back()) b.push_back(v);
  }
  P = (int64_t)b.size();
  b.push_back(E);
  std::vector<std::vector<int64_t>> chain(P);
  std::vector<int64_t> exit_at(P);
  {
    std::vector<std::thread> th;
    for (int64_t k = 0; k < P; ++k)
      th.emplace_back([&, k] {
        NodeSet set(TN);
        int64_t cur = b[k];
        while (cur < b[k + 1]) {
          chain[k].push_back(cur);
          cur = greedy_next(cs, npe, E, TE, TN, cur, set);
        }
        exit_at[k] = cur;
      });
    for (auto& x : th) x.join();
  }
  NodeSet set(TN);
  starts.assign(chain[0].begin(), chain[0].end());
  int64_t cur = exit_at[0];
  for (int64_t k = 1; k < P; ++k) {
    const std::vector<int64_t>& ck = chain[k];
    while (cur < b[k + 1]) {
      auto it = std::lower_bound(ck.begin(), ck.end(), cur);
      if (it != ck.end() && *it == cur) {
        starts.insert(starts.end(), it, ck.end());
        cur = exit_at[k];
        break;
      }
      starts.push_back(cur);
      cur = greedy_next(cs, npe, E, TE, TN, cur, set);
    }
  }
}

static inline uint64_t spread3(uint64_t v) {
  v &= 0x1fffff;
  v = (v | v << 32) & 0x1f00000000ffffULL;
  v = (v | v << 16) & 0x1f0000ff0000ffULL;
  v = (v | v << 8) & 0x100f00f00f00f00fULL;
  v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
  v = (v | v << 2) & 0x1249249249249249ULL;
  return v;
}

// Element indices sorted by the Morton code of the element centroid (21
// bits per axis over the mesh's bounding cube), ties in element order.
void morton_order(const fm_problem* p, hvec<int64_t>& order) {
  const int npe = p->etype;
  const int64_t E = p->E, N = p->N;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  {
    // bounding box: per-thread extremes combined (min / max are exact)
    std::vector<std::array<double, 6>> part(64, {1e300, 1e300, 1e300, -1e300, -1e300, -1e300});
    parallel_blocks(N, [&](int64_t ib, int64_t ie, int w) {
      std::array<double, 6>& b = part[w];
      for (int64_t i = ib; i < ie; ++i)
        for (int k = 0; k < 3; ++k) {
          b[k] = std::min(b[k], p->coords[i * 3 + k]);
          b[3 + k] = std::max(b[3 + k], p->coords[i * 3 + k]);
        }
    }, 1 << 14);
    for (const auto& b : part)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], b[k]);
        hi[k] = std::max(hi[k], b[3 + k]);
      }
  }
  double span = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
  if (!(span > 0)) span = 1.0;
  hvec<uint64_t> code(E);
  const double inv_npe = 1.0 / npe;  // exact (4 or 8): c * inv_npe equals c / npe
  parallel_blocks(E, [&](int64_t eb, int64_t ee, int) {
    for (int64_t e = eb; e < ee; ++e) {
      double c[3] = {0, 0, 0};
      for (int a = 0; a < npe; ++a)
        for (int k = 0; k < 3; ++k) c[k] += p->coords[(int64_t)p->conn[e * npe + a] * 3 + k];
      uint64_t q[3];
      for (int k = 0; k < 3; ++k) {
        double t = (c[k] * inv_npe - lo[k]) / span;
        t = std::min(std::max(t, 0.0), 1.0);
        q[k] = (uint64_t)(t * 2097151.0);
      }
      code[e] = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
    }
  });
  sort_by_key(code, order);
}

// Orders one tile's interface nodes for the node-owner accumulation of the
// tile kernels, in which the thread p % FM_OWNER_THREADS adds up the
// contributions of the tile's local node p.  Interior nodes keep positions
// [0, n_int) (their batch ids are consecutive from local node 0); the
// interface nodes, heaviest first (incident elements in the tile plus a fixed
// cost per node), take a free position of the thread with the least work so
// far (ties: the lowest thread).  Without it the threads that own an
// interior node (up to 24 incident elements) also own as many interface
// nodes as the others, and the slowest owner sets the length of every
// chunk's accumulation.  Each node's sum keeps its element order, so the
// results do not depend on this order.
//   w_int / w_ifc: incident elements of the interior / interface nodes (in
//   their current order); ifc: the interface nodes, reordered in place.
constexpr int FM_OWNER_THREADS = 128;
struct BalanceScratch {
  std::vector<int32_t> by_w, count, out;
  std::vector<uint64_t> heap;
};
static void balance_owners(const std::vector<int32_t>& w_int, const std::vector<int32_t>& w_ifc,
                           std::vector<int32_t>& ifc, BalanceScratch& sc) {
  const int n_int = (int)w_int.size(), n_ifc = (int)w_ifc.size(), n_node = n_int + n_ifc;
  constexpr int64_t kNodeCost = 2;  // accumulator load / store and walk set-up, in entry units
  int64_t load[FM_OWNER_THREADS] = {};
  int next[FM_OWNER_THREADS];
  for (int q = 0; q < n_int; ++q) load[q % FM_OWNER_THREADS] += w_int[q] + kNodeCost;
  // min-heap of (load, thread) packed as load * 256 + thread (thread < 256,
  // so the order is that of the pairs) over the threads with a free
  // interface position
  std::vector<uint64_t>& heap = sc.heap;
  heap.clear();
  for (int t = 0; t < FM_OWNER_THREADS; ++t) {
    int q = n_int + ((t - n_int % FM_OWNER_THREADS) + FM_OWNER_THREADS) % FM_OWNER_THREADS;
    next[t] = q;
    if (q < n_node) heap.push_back((uint64_t)load[t] * 256u + (uint64_t)t);
  }
  std::make_heap(heap.begin(), heap.end(), std::greater<uint64_t>());
  // interface nodes heaviest first, equal weights in their current order (a
  // stable counting sort on the weight)
  int32_t wmax = 0;
  for (int32_t w : w_ifc) wmax = std::max(wmax, w);
  std::vector<int32_t>& count = sc.count;
  count.assign((size_t)wmax + 2, 0);
  for (int32_t w : w_ifc) count[wmax - w + 1]++;
  for (int32_t k = 0; k <= wmax; ++k) count[k + 1] += count[k];
  std::vector<int32_t>& by_w = sc.by_w;
  by_w.resize(n_ifc);
  for (int32_t i = 0; i < n_ifc; ++i) by_w[count[wmax - w_ifc[i]]++] = i;
  std::vector<int32_t>& out = sc.out;
  out.resize(n_ifc);
  for (int32_t i : by_w) {
    std::pop_heap(heap.begin(), heap.end(), std::greater<uint64_t>());
    const uint64_t key = heap.back();
    heap.pop_back();
    const int t = (int)(key & 255u);
    out[next[t] - n_int] = ifc[i];
    next[t] += FM_OWNER_THREADS;
    if (next[t] < n_node) {
      heap.push_back(key + (uint64_t)(w_ifc[i] + kNodeCost) * 256u);
      std::push_heap(heap.begin(), heap.end(), std::greater<uint64_t>());
    }
  }
  ifc.swap(out);
}

// Builds the batch layout:
//  1. elements of each problem sorted by the Morton code of their centroid;
//  2. cut greedily into tiles of <= tile_elems elements and <= tile_nodes
//     distinct nodes (tiles never span problems, so a problem's arithmetic
//     does not depend on what else is in the batch);
//  3. nodes touched by one tile are "interior" to it, the others are
//     "interface" nodes; nodes are renumbered tile-major (each tile's
//     interior nodes contiguous), interface nodes after them;
//  4. inside a tile, elements are coloured greedily (no two elements of a
//     colour share a node) and sorted by colour, which fixes the order in
//     which contributions reach every node;
//  5. each (tile, interface node) pair gets a partial-sum slot; the slots of
//     an interface node are listed in tile order.
// Nodes of a partition part that are shared with other parts (p->xidx >= 0)
// are interface nodes even when one tile touches them: their sums are
// completed by the exchange between the parts.
int build_layout(fm_problem* const* probs, int n, int TE, int TN, Layout& L) {
  L = Layout();
  L.node_new.resize(n);
  L.elem_old.resize(n);
  int64_t node_base = 0, elem_base = 0, slot_base = 0;
  for (int pi = 0; pi < n; ++pi) {
    fm_problem* p = probs[pi];
    const int npe = p->etype;
    const int64_t E = p->E, N = p->N;
    L.node_begin.push_back(node_base);
    L.elem_begin.push_back(elem_base);
    // 1. Morton order
    hvec<int64_t> order;
    morton_order(p, order);
    // connectivity in sorted order: the sequential passes below then read
    // contiguous memory
    hvec<int32_t> cs((size_t)E * npe);
    parallel_blocks(E, [&](int64_t b, int64_t e, int) {
      for (int64_t oi = b; oi < e; ++oi)
        for (int a = 0; a < npe; ++a) cs[(size_t)oi * npe + a] = p->conn[order[oi] * npe + a];
    });
    // 2. greedy tiles
    std::vector<int64_t> tile_start;
    greedy_tiles(cs.data(), npe, E, TE, TN, tile_start);
    tile_start.push_back(E);
    const int ntile = (int)tile_start.size() - 1;
    // 3. node tile counts and first tile (shared partition nodes count as
    // touched by two tiles), tiles split over the host threads
    std::vector<int32_t> ntiles(N, 0), first_tile(N, INT32_MAX);
    parallel_blocks(ntile, [&](int64_t tb, int64_t te2, int) {
      NodeSet set(TN);
      for (int64_t t = tb; t < te2; ++t) {
        for (int64_t oi = tile_start[t]; oi < tile_start[t + 1]; ++oi) {
          const int32_t* c = &cs[(size_t)oi * npe];
          for (int a = 0; a < npe; ++a) set.insert(c[a]);
        }
        for (int32_t h : set.used) {
          const int32_t v = set.slot[h];
          __atomic_fetch_add(&ntiles[v], 1, __ATOMIC_RELAXED);
          int32_t cur = __atomic_load_n(&first_tile[v], __ATOMIC_RELAXED);
          while ((int32_t)t < cur &&
                 !__atomic_compare_exchange_n(&first_tile[v], &cur, (int32_t)t, true, __ATOMIC_RELAXED,
                                              __ATOMIC_RELAXED)) {
          }
        }
        set.clear();
      }
    }, 64);
    if (!p->xidx.empty())
      for (int64_t i = 0; i < N; ++i)
        if (p->xidx[i] >= 0 && ntiles[i] == 1) ntiles[i] = 2;
    // node renumbering: interior nodes tile by tile, interface nodes after
    // them, each group in order of first touch along the sorted elements
    // (per-tile first-touch lists in parallel, then prefix offsets)
    const int64_t hwt = std::max<int64_t>(1, std::min<int64_t>(32, std::thread::hardware_concurrency()));
    const int64_t nwk = std::min<int64_t>(hwt, std::max<int64_t>(1, ntile / 4));
    std::vector<std::vector<int32_t>> first_int(ntile), first_ifc(ntile);
    {
      std::vector<std::thread> th;
      for (int64_t w = 0; w < nwk; ++w)
        th.emplace_back([&, w] {
          std::vector<int32_t> stamp2(N, -1);
          for (int t = (int)(ntile * w / nwk); t < (int)(ntile * (w + 1) / nwk); ++t)
            for (int64_t oi = tile_start[t]; oi < tile_start[t + 1]; ++oi) {
              const int32_t* c = &cs[(size_t)oi * npe];
              for (int a = 0; a < npe; ++a) {
                const int32_t v = c[a];
                if (stamp2[v] == t) continue;
                stamp2[v] = t;
                if (ntiles[v] == 1) first_int[t].push_back(v);
                else if (first_tile[v] == t) first_ifc[t].push_back(v);
              }
            }
        });
      for (auto& x : th) x.join();
    }
    std::vector<int32_t>& nn = L.node_new[pi];
    nn.assign(N, -1);
    // numbers in tile order from prefix offsets, written in parallel
    std::vector<int64_t> int_at(ntile + 1, 0), ifc_at(ntile + 1, 0);
    for (int t = 0; t < ntile; ++t) {
      int_at[t + 1] = int_at[t] + (int64_t)first_int[t].size();
      ifc_at[t + 1] = ifc_at[t] + (int64_t)first_ifc[t].size();
    }
    const int64_t iface_begin = int_at[ntile];
    parallel_blocks(ntile, [&](int64_t tb, int64_t te2, int) {
      for (int64_t t = tb; t < te2; ++t) {
        int64_t k = node_base + int_at[t];
        for (int32_t v : first_int[t]) nn[v] = (int32_t)k++;
        k = node_base + iface_begin + ifc_at[t];
        for (int32_t v : first_ifc[t]) nn[v] = (int32_t)k++;
      }
    }, 16);
    std::vector<std::vector<int32_t>>().swap(first_int);
    std::vector<std::vector<int32_t>>().swap(first_ifc);
    int64_t next = iface_begin + ifc_at[ntile];
    for (int64_t i = 0; i < N; ++i)
      if (nn[i] < 0) nn[i] = (int32_t)(node_base + next++);  // isolated nodes
    // 4./5. tiles: local nodes, colouring, local connectivity, incidence
    // lists - built for every tile in parallel (per-worker scratch), then
    // placed in tile order
    struct TileWork {
      std::vector<int32_t> inter, ifc;  // old node ids in local order
      std::vector<int32_t> eo;          // old element of each tile element (colour order)
      std::vector<uint16_t> conn;       // ne x npe tile-local ids
      std::vector<int32_t> colcnt;      // colour offsets (ncol + 1)
      std::vector<uint16_t> off, inc;   // incidence offsets (n_node + 1) and entries (ne * npe)
      int ncol = 0;
      int err = 0;                      // 1: > 128 colours, 2: 16-bit incidence overflow
    };
    std::vector<TileWork> tw(ntile);
    {
      const int64_t hw = std::max<int64_t>(1, std::min<int64_t>(32, std::thread::hardware_concurrency()));
      const int64_t nw = std::min<int64_t>(hw, std::max<int64_t>(1, ntile / 4));
      std::vector<std::thread> th;
      for (int64_t w = 0; w < nw; ++w)
        th.emplace_back([&, w] {
          std::vector<int32_t> local(N, -1);
          std::vector<uint64_t> used;                 // per-worker scratch, reused tile by tile
          std::vector<int32_t> col, idx, cnt, pos, w_int, w_ifc, own;
          BalanceScratch bal;
          for (int t = (int)(ntile * w / nw); t < (int)(ntile * (w + 1) / nw); ++t) {
            TileWork& W = tw[t];
            own.clear();
            for (int64_t oi = tile_start[t]; oi < tile_start[t + 1]; ++oi) {
              const int32_t* c = &cs[(size_t)oi * npe];
              for (int a = 0; a < npe; ++a) {
                const int32_t v = c[a];
                if (local[v] == -2 - t) continue;
                local[v] = -2 - t;
                if (ntiles[v] == 1) W.inter.push_back(v);
                else if (first_tile[v] == t) own.push_back(v);
                else W.ifc.push_back(v);
              }
            }
            // interior nodes in their (contiguous) batch order, then interface
            // nodes by id, reordered to balance the owner threads.  The
            // interior nodes and the interface nodes this tile touches first
            // were numbered in this same first-touch walk, so they arrive in
            // id order; only the interface nodes of earlier tiles (all with
            // smaller ids) are sorted
            std::sort(W.ifc.begin(), W.ifc.end(), [&](int32_t x, int32_t y) { return nn[x] < nn[y]; });
            W.ifc.insert(W.ifc.end(), own.begin(), own.end());
            int32_t li = 0;
            for (int32_t v : W.inter) local[v] = li++;
            for (int32_t v : W.ifc) local[v] = li++;
            const int32_t n_node = li;
            {
              cnt.assign(n_node, 0);
              for (int64_t oi = tile_start[t]; oi < tile_start[t + 1]; ++oi)
                for (int a = 0; a < npe; ++a) cnt[local[cs[(size_t)oi * npe + a]]]++;
              const int n_int = (int)W.inter.size();
              w_int.assign(cnt.begin(), cnt.begin() + n_int);
              w_ifc.assign(cnt.begin() + n_int, cnt.end());
              balance_owners(w_int, w_ifc, W.ifc, bal);
              li = n_int;
              for (int32_t v : W.ifc) local[v] = li++;
            }
            // colouring (greedy, up to 128 colours)
            const int64_t ne = tile_start[t + 1] - tile_start[t];
            used.assign(2 * (size_t)n_node, 0);
            col.resize(ne);
            int ncol = 0;
            for (int64_t i = 0; i < ne; ++i) {
              const int32_t* c = &cs[(size_t)(tile_start[t] + i) * npe];
              uint64_t m0 = 0, m1 = 0;
              for (int a = 0; a < npe; ++a) {
                m0 |= used[2 * local[c[a]]];
                m1 |= used[2 * local[c[a]] + 1];
              }
              int k;
              if (~m0) k = __builtin_ctzll(~m0);
              else if (~m1) k = 64 + __builtin_ctzll(~m1);
              else {
                W.err = 1;
                break;
              }
              col[i] = k;
              ncol = std::max(ncol, k + 1);
              for (int a = 0; a < npe; ++a) used[2 * local[c[a]] + (k >> 6)] |= (1ULL << (k & 63));
            }
            if (W.err) continue;
            // elements sorted by colour: SUPG processes a tile one colour at a
            // time; for VMS it spreads each chunk's contributions over all of
            // the tile's nodes (one or two per node and chunk, which balances
            // the node-owner accumulation; the space-filling order measured
            // slower)
            // (counting sort by colour: stable, as the element order within a
            // colour must stay the sorted order)
            W.ncol = ncol;
            W.colcnt.assign(ncol + 1, 0);
            for (int64_t i = 0; i < ne; ++i) W.colcnt[col[i] + 1]++;
            for (int k = 0; k < ncol; ++k) W.colcnt[k + 1] += W.colcnt[k];
            idx.resize(ne);
            pos.assign(W.colcnt.begin(), W.colcnt.end() - 1);
            for (int64_t i = 0; i < ne; ++i) idx[pos[col[i]]++] = (int32_t)i;
            W.eo.resize(ne);
            W.conn.resize((size_t)ne * npe);
            for (int64_t i = 0; i < ne; ++i) {
              const int64_t oi = tile_start[t] + idx[i];
              W.eo[i] = (int32_t)order[oi];
              const int32_t* c = &cs[(size_t)oi * npe];
              for (int a = 0; a < npe; ++a) W.conn[(size_t)i * npe + a] = (uint16_t)local[c[a]];
            }
            // node -> incident (element, corner) lists in element order
            if (ne * npe > 65535) {
              W.err = 2;
              continue;
            }
            cnt.assign(n_node + 1, 0);
            for (int64_t i = 0; i < ne * npe; ++i) cnt[W.conn[i] + 1]++;
            for (int k2 = 0; k2 < n_node; ++k2) cnt[k2 + 1] += cnt[k2];
            W.off.resize(n_node + 1);
            for (int k2 = 0; k2 <= n_node; ++k2) W.off[k2] = (uint16_t)cnt[k2];
            W.inc.resize((size_t)ne * npe);
            pos.assign(cnt.begin(), cnt.end() - 1);
            for (int64_t i = 0; i < ne; ++i)
              for (int a = 0; a < npe; ++a) W.inc[pos[W.conn[i * npe + a]]++] = (uint16_t)(i * npe + a);
          }
        });
      for (auto& x : th) x.join();
    }
    for (int t = 0; t < ntile; ++t) {
      if (tw[t].err == 1) return fail(FM_ERR_INVALID, "element colouring needs more than 128 colours in one tile");
      if (tw[t].err == 2) return fail(FM_ERR_INVALID, "tile_elems too large for 16-bit incidence entries");
    }
    // placement: every tile starts at a multiple of ELEM_ALIGN element slots
    // (padding slots in between are never processed, so each chunk of a
    // tile's element arrays starts on a 16-byte, in fact 128-byte, boundary)
    // and its incidence entries at a multiple of 8; offsets first, then the
    // blocks are copied in parallel
    std::vector<TileMeta> tms(ntile);
    int64_t e_out = 0, inc_prev = 0;
    {
      int64_t tn_off = (int64_t)L.tile_nodes.size(), col_off = (int64_t)L.tile_cols.size();
      int64_t inc_off = (int64_t)L.tile_inc.size(), off_off = (int64_t)L.tile_off.size(), sb = slot_base;
      inc_prev = inc_off;
      for (int t = 0; t < ntile; ++t) {
        const TileWork& W = tw[t];
        TileMeta& tm = tms[t];
        memset(&tm, 0, sizeof(tm));
        e_out = (e_out + ELEM_ALIGN - 1) / ELEM_ALIGN * ELEM_ALIGN;
        tm.problem = pi;
        tm.elem_begin = (int32_t)(elem_base + e_out);
        tm.n_elem = (int32_t)(tile_start[t + 1] - tile_start[t]);
        tm.node_begin = (int32_t)tn_off;
        tm.n_int = (int32_t)W.inter.size();
        tm.n_node = (int32_t)(W.inter.size() + W.ifc.size());
        tm.slot_base = (int32_t)sb;
        tm.col_begin = (int32_t)col_off;
        tm.n_col = W.ncol;
        inc_off = (inc_off + 7) / 8 * 8;
        tm.inc_begin = (int32_t)inc_off;
        tm.off_begin = (int32_t)off_off;
        e_out += tm.n_elem;
        tn_off += tm.n_node;
        sb += (int64_t)W.ifc.size();
        col_off += (int64_t)W.colcnt.size();
        inc_off += (int64_t)W.inc.size();
        off_off += (int64_t)W.off.size();
        L.max_colors = std::max(L.max_colors, W.ncol);
        L.max_tile_elems = std::max<int32_t>(L.max_tile_elems, tm.n_elem);
      }
      // final sizes at once (the last problem includes the trailing
      // padding: chunk copies round their length up to 16 bytes, and the
      // incidence lists are copied in 16-byte pieces); the new ranges are
      // first written by the per-tile copies below
      const bool last_prob = pi == n - 1;
      L.tile_nodes.resize(tn_off);
      L.tile_cols.resize(col_off);
      L.tile_inc.resize(last_prob ? (inc_off + 7) / 8 * 8 + 8 : inc_off);
      L.tile_off.resize(off_off);
      slot_base = sb;
    }
    e_out = (e_out + ELEM_ALIGN - 1) / ELEM_ALIGN * ELEM_ALIGN;
    auto& eo = L.elem_old[pi];
    eo.resize(e_out);
    const int64_t conn_end = elem_base + e_out + (pi == n - 1 ? ELEM_ALIGN : 0);
    L.conn_local.resize((size_t)conn_end * npe);
    const int64_t inc_end = (int64_t)L.tile_inc.size();
    if (ntile > 0)  // alignment gap after the previous problem's entries
      std::fill(L.tile_inc.begin() + inc_prev, L.tile_inc.begin() + tms[0].inc_begin, 0);
    // each tile fills its ranges and the padding up to the next tile (a few
    // tiles a block: the per-tile copies are large)
    parallel_blocks(ntile, [&](int64_t tb, int64_t te2, int) {
      for (int64_t t = tb; t < te2; ++t) {
        const TileWork& W = tw[t];
        const TileMeta& tm = tms[t];
        int32_t* tn = &L.tile_nodes[tm.node_begin];
        for (int32_t v : W.inter) *tn++ = nn[v];
        for (int32_t v : W.ifc) *tn++ = nn[v];
        std::copy(W.colcnt.begin(), W.colcnt.end(), L.tile_cols.begin() + tm.col_begin);
        std::copy(W.off.begin(), W.off.end(), L.tile_off.begin() + tm.off_begin);
        const int64_t inc_next = t + 1 < ntile ? tms[t + 1].inc_begin : inc_end;
        std::copy(W.inc.begin(), W.inc.end(), L.tile_inc.begin() + tm.inc_begin);
        std::fill(L.tile_inc.begin() + tm.inc_begin + (int64_t)W.inc.size(), L.tile_inc.begin() + inc_next, 0);
        const int64_t el_next = t + 1 < ntile ? tms[t + 1].elem_begin : conn_end;
        std::copy(W.conn.begin(), W.conn.end(), L.conn_local.begin() + (size_t)tm.elem_begin * npe);
        std::fill(L.conn_local.begin() + (size_t)(tm.elem_begin + tm.n_elem) * npe,
                  L.conn_local.begin() + (size_t)el_next * npe, 0);
        const int64_t eo_next = std::min<int64_t>(el_next, elem_base + e_out) - elem_base;
        std::copy(W.eo.begin(), W.eo.end(), eo.begin() + (tm.elem_begin - elem_base));
        std::fill(eo.begin() + (tm.elem_begin - elem_base) + tm.n_elem, eo.begin() + eo_next, -1);
      }
    }, 8);
    if (ntile == 0) {
      std::fill(L.conn_local.begin() + (size_t)elem_base * npe, L.conn_local.end(), 0);
      std::fill(eo.begin(), eo.end(), -1);
    }
    L.tiles.insert(L.tiles.end(), tms.begin(), tms.end());
    // interface nodes: one partial-sum slot per (tile, node), listed per node
    // in tile order (per-worker counts over contiguous tile ranges give each
    // worker its write positions, so the lists fill in parallel)
    {
      const int64_t NI = N - iface_begin;
      const int64_t hw2 = std::max<int64_t>(1, std::min<int64_t>(32, std::thread::hardware_concurrency()));
      const int64_t nw = std::min<int64_t>(hw2, std::max<int64_t>(1, ntile / 64));
      std::vector<std::vector<int32_t>> wc(nw);
      auto node_of = [&](int32_t v) { return (int64_t)nn[v] - node_base - iface_begin; };
      {
        std::vector<std::thread> th;
        for (int64_t w = 0; w < nw; ++w)
          th.emplace_back([&, w] {
            wc[w].assign(NI, 0);
            for (int64_t t = ntile * w / nw; t < ntile * (w + 1) / nw; ++t)
              for (int32_t v : tw[t].ifc) wc[w][node_of(v)]++;
          });
        for (auto& x : th) x.join();
      }
      std::vector<int32_t> cnt(NI + 1, 0);
      parallel_blocks(NI, [&](int64_t jb, int64_t je, int) {
        for (int64_t j = jb; j < je; ++j) {
          int32_t c = 0;
          for (int64_t w = 0; w < nw; ++w) c += wc[w][j];
          cnt[j + 1] = c;
        }
      }, 1 << 14);
      for (int64_t k = 0; k < NI; ++k) cnt[k + 1] += cnt[k];
      // worker w's first position for node j: the node's start plus the
      // counts of the workers before it
      parallel_blocks(NI, [&](int64_t jb, int64_t je, int) {
        for (int64_t j = jb; j < je; ++j) {
          int32_t at = cnt[j];
          for (int64_t w = 0; w < nw; ++w) {
            const int32_t c = wc[w][j];
            wc[w][j] = at;
            at += c;
          }
        }
      }, 1 << 14);
      const int64_t s0 = (int64_t)L.iface_slots.size();
      L.iface_slots.resize(s0 + cnt[NI]);
      {
        std::vector<std::thread> th;
        for (int64_t w = 0; w < nw; ++w)
          th.emplace_back([&, w] {
            for (int64_t t = ntile * w / nw; t < ntile * (w + 1) / nw; ++t) {
              int32_t k = 0;
              for (int32_t v : tw[t].ifc) L.iface_slots[s0 + wc[w][node_of(v)]++] = tms[t].slot_base + k++;
            }
          });
        for (auto& x : th) x.join();
      }
      const size_t i0 = L.iface_node.size();
      L.iface_node.resize(i0 + NI);
      L.iface_slot_beg.resize(i0 + NI);
      L.iface_prob.resize(i0 + NI);
      L.iface_xidx.resize(i0 + NI);
      parallel_blocks(NI, [&](int64_t jb, int64_t je, int) {
        for (int64_t k = jb; k < je; ++k) {
          L.iface_node[i0 + k] = (int32_t)(node_base + iface_begin + k);
          L.iface_slot_beg[i0 + k] = (int32_t)(s0 + cnt[k]);
          L.iface_prob[i0 + k] = pi;
          L.iface_xidx[i0 + k] = -1;
        }
      }, 1 << 14);
      if (!p->xidx.empty())
        for (int64_t i = 0; i < N; ++i) {
          const int64_t j = nn[i] - node_base - iface_begin;
          if (j >= 0) L.iface_xidx[i0 + j] = p->xidx[i];
        }
    }
    node_base += N;
    e_out = (e_out + ELEM_ALIGN - 1) / ELEM_ALIGN * ELEM_ALIGN;
    eo.resize(e_out, -1);
    L.elem_count.push_back(e_out);
    elem_base += e_out;
  }
  elem_base += ELEM_ALIGN;  // trailing padding (sized with the last problem)
  L.iface_slot_beg.push_back((int32_t)L.iface_slots.size());
  L.n_nodes = node_base;
  L.n_elems = elem_base;
  L.n_slots = slot_base;
  if (node_base >= INT32_MAX || elem_base >= INT32_MAX || slot_base >= INT32_MAX)
    return fail(FM_ERR_INVALID, "batch too large for 32-bit indices");
  return FM_OK;
}

}  // namespace fm

namespace fm {

// Checks the invariants the tile kernels rely on in one problem's layout
// (one problem, built by build_layout): local connectivity inside the tile's
// node list; distinct nodes in a tile, interior ones touched by this tile
// only; elements of one colour sharing no node (the hexa8 colour rounds add
// without ordering); every (element, corner) once in its node's incidence
// list, in element order; each interface node's partial slots, one per
// touching tile, in tile order; every element and node of the problem once.
int check_layout(const fm_problem* p, const Layout& L) {
  auto bad = [](const std::string& m) { return fail(FM_ERR_INVALID, "layout check: " + m); };
  const int npe = p->etype;
  const int64_t N = p->N, E = p->E;
  const std::vector<int32_t>& nn = L.node_new[0];
  if ((int64_t)nn.size() != N) return bad("node map size");
  std::vector<int32_t> seen_node(N, 0), tiles_of(N, 0);
  {
    std::vector<char> used((size_t)N, 0);
    for (int64_t v = 0; v < N; ++v) {
      if (nn[v] < 0 || nn[v] >= N || used[nn[v]]) return bad("node renumbering is not a permutation");
      used[nn[v]] = 1;
    }
  }
  std::vector<int32_t> old_of(N);
  for (int64_t v = 0; v < N; ++v) old_of[nn[v]] = (int32_t)v;
  std::vector<char> elem_seen((size_t)E, 0);
  std::vector<int32_t> stamp(N, -1), colour_stamp;
  // slot -> (tile, interface node batch id)
  std::vector<int32_t> slot_node((size_t)L.n_slots, -1), slot_tile((size_t)L.n_slots, -1);
  for (size_t t = 0; t < L.tiles.size(); ++t) {
    const TileMeta& tm = L.tiles[t];
    const int32_t ne = tm.n_elem, nl = tm.n_node;
    if (tm.n_int < 0 || tm.n_int > nl) return bad("tile " + std::to_string(t) + ": interior count");
    const int32_t* tn = &L.tile_nodes[tm.node_begin];
    for (int32_t l = 0; l < nl; ++l) {
      const int32_t g = tn[l];
      if (g < 0 || g >= N) return bad("tile " + std::to_string(t) + ": node id out of range");
      if (stamp[g] == (int32_t)t) return bad("tile " + std::to_string(t) + ": node listed twice");
      stamp[g] = (int32_t)t;
      tiles_of[g]++;
      if (l < tm.n_int) seen_node[g]++;
      else {
        const int64_t s = (int64_t)tm.slot_base + (l - tm.n_int);
        if (s < 0 || s >= L.n_slots || slot_node[s] >= 0) return bad("tile " + std::to_string(t) + ": slot");
        slot_node[s] = g;
        slot_tile[s] = (int32_t)t;
      }
    }
    // local connectivity (bit 15 of the first id flags an FP64-Jacobian
    // element in the mixed form)
    const uint16_t* cl = &L.conn_local[(size_t)tm.elem_begin * npe];
    for (int32_t i = 0; i < ne; ++i) {
      const int64_t oe = L.elem_old[0][tm.elem_begin + i];
      if (oe < 0 || oe >= E || elem_seen[oe]) return bad("tile " + std::to_string(t) + ": element map");
      elem_seen[oe] = 1;
      for (int a = 0; a < npe; ++a) {
        const int32_t ln = a == 0 ? (cl[i * npe] & 0x7fff) : cl[i * npe + a];
        if (ln >= nl) return bad("tile " + std::to_string(t) + ": local node id out of range");
        if (old_of[tn[ln]] != p->conn[oe * npe + a]) return bad("tile " + std::to_string(t) + ": connectivity");
      }
    }
    // colours
    const int32_t* co = &L.tile_cols[tm.col_begin];
    if (co[0] != 0 || co[tm.n_col] != ne) return bad("tile " + std::to_string(t) + ": colour offsets");
    colour_stamp.assign(nl, -1);
    for (int32_t c = 0; c < tm.n_col; ++c)
      for (int32_t i = co[c]; i < co[c + 1]; ++i)
        for (int a = 0; a < npe; ++a) {
          const int32_t ln = a == 0 ? (cl[i * npe] & 0x7fff) : cl[i * npe + a];
          if (colour_stamp[ln] == c) return bad("tile " + std::to_string(t) + ": two elements of a colour share a node");
          colour_stamp[ln] = c;
        }
    // incidence lists
    const uint16_t* off = &L.tile_off[tm.off_begin];
    const uint16_t* inc = &L.tile_inc[tm.inc_begin];
    if (off[0] != 0 || off[nl] != ne * npe) return bad("tile " + std::to_string(t) + ": incidence offsets");
    for (int32_t l = 0; l < nl; ++l)
      for (int32_t k = off[l]; k < off[l + 1]; ++k) {
        const int32_t el = inc[k] / npe, a = inc[k] % npe;
        if (el >= ne) return bad("tile " + std::to_string(t) + ": incidence element");
        const int32_t ln = a == 0 ? (cl[el * npe] & 0x7fff) : cl[el * npe + a];
        if (ln != l) return bad("tile " + std::to_string(t) + ": incidence entry of another node");
        if (k > off[l] && inc[k - 1] / npe >= el) return bad("tile " + std::to_string(t) + ": incidence order");
      }
  }
  for (int64_t e = 0; e < E; ++e)
    if (!elem_seen[e]) return bad("element " + std::to_string(e) + " in no tile");
  for (int64_t g = 0; g < N; ++g) {
    if (seen_node[g] > 1) return bad("node interior to two tiles");
    if (seen_node[g] == 1 && tiles_of[g] != 1) return bad("interior node touched by another tile");
  }
  // interface lists: every node some tile touches but none owns is listed
  // once (no interior node is); node i's slots name the node, one a touching
  // tile, in tile order, and the slot map of the tiles is a permutation
  const int64_t NI = (int64_t)L.iface_node.size();
  if ((int64_t)L.iface_slot_beg.size() != NI + 1) return bad("interface list size");
  std::vector<char> listed((size_t)N, 0);
  for (int64_t i = 0; i < NI; ++i) {
    const int32_t g = L.iface_node[i];
    if (g < 0 || g >= N || listed[g] || seen_node[g]) return bad("interface node list");
    listed[g] = 1;
  }
  for (int64_t g = 0; g < N; ++g)
    if (tiles_of[g] > 0 && !seen_node[g] && !listed[g]) return bad("touched node neither interior nor interface");
  // partition parts: a node shared with another part is never interior, and
  // its interface entry carries its exchange index (unique in the part, below
  // the partition's total); other entries carry -1
  if (p->part >= 0) {
    if ((int64_t)p->xidx.size() != N || (int64_t)L.iface_xidx.size() != NI) return bad("exchange index size");
    std::vector<char> xused((size_t)std::max<int64_t>(p->x_total, 0), 0);
    for (int64_t v = 0; v < N; ++v) {
      const int32_t x = p->xidx[v];
      if (x < 0) continue;
      if (x >= p->x_total || xused[x]) return bad("exchange index out of range or repeated");
      xused[x] = 1;
      if (seen_node[nn[v]]) return bad("shared node interior to a tile");
      if (tiles_of[nn[v]] > 0 && !listed[nn[v]]) return bad("shared node without an interface entry");
    }
    for (int64_t i = 0; i < NI; ++i)
      if (L.iface_xidx[i] != p->xidx[old_of[L.iface_node[i]]]) return bad("interface entry's exchange index");
  }
  for (int64_t i = 0; i < NI; ++i) {
    const int32_t g = L.iface_node[i];
    const int32_t k0 = L.iface_slot_beg[i], k1 = L.iface_slot_beg[i + 1];
    if (k1 - k0 != tiles_of[g] && tiles_of[g] > 0) return bad("interface node slot count");
    for (int32_t k = k0; k < k1; ++k) {
      const int32_t s = L.iface_slots[k];
      if (s < 0 || s >= L.n_slots || slot_node[s] != g) return bad("interface slot of another node");
      if (k > k0 && slot_tile[L.iface_slots[k - 1]] >= slot_tile[s]) return bad("interface slots not in tile order");
    }
  }
  return FM_OK;
}

}  // namespace fm
