// Partitioned single mesh: one problem split into parts, one part per GPU.
//
// Every part is an ordinary problem over the elements it owns and the nodes
// they touch.  Nodes touched by more than one part, and for VMS the
// problem's nodes 0..3 (every element reads their pressures, the reference's
// femVMSExplicitFluidSolver.cpp:489), form the partition's exchange list,
// numbered in global node order and identical on every part.  Each dual
// iteration (VMS) or step (SUPG) a part sums its elements' contributions to
// its exchange nodes into its slice of a packed buffer (4 doubles a node);
// the parts' buffers are summed (NCCL all-reduce across processes, or a
// plain sum when all parts share one batch); every part then updates its own
// copy of each exchange node from the same sum, so the copies stay equal.
// Lumped masses and boundary conditions are those of the whole mesh,
// restricted to the part's nodes (the NODEVEL row/direction pairing of the
// reference depends on the whole list, so BCs are resolved before the
// split).
#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "fm_internal.hpp"

using namespace fm;

static int default_parts(const fm_problem* full, int32_t n_parts, std::vector<int32_t>& part) {
  hvec<int64_t> order;
  morton_order(full, order);
  const int64_t E = full->E;
  part.assign(E, 0);
  for (int64_t i = 0; i < E; ++i) part[order[i]] = (int32_t)((i * n_parts) / E);
  return FM_OK;
}

extern "C" {

// Elements split into n_parts bands of equal size along the Morton order of
// their centroids (compact, cube-like parts of a structured mesh).
FM_API int fm_partition_elements(const fm_problem* full, int32_t n_parts, int32_t* elem_part) {
  if (!full || !elem_part) return fail(FM_ERR_INVALID, "null argument");
  if (n_parts < 1 || n_parts > full->E) return fail(FM_ERR_INVALID, "n_parts must be in [1, n_elems]");
  if (full->part >= 0) return fail(FM_ERR_INVALID, "a partition part cannot be partitioned again");
  std::vector<int32_t> part;
  default_parts(full, n_parts, part);
  std::copy(part.begin(), part.end(), elem_part);
  return FM_OK;
}

FM_API int fm_problem_partition(const fm_problem* full, const int32_t* elem_part, int32_t n_parts, int32_t part,
                                fm_problem** out) {
  NvtxRange nvtx_range("fm_problem_partition");
  if (!full || !out) return fail(FM_ERR_INVALID, "null argument");
  *out = nullptr;
  if (full->part >= 0) return fail(FM_ERR_INVALID, "a partition part cannot be partitioned again");
  if (n_parts < 1 || n_parts > full->E) return fail(FM_ERR_INVALID, "n_parts must be in [1, n_elems]");
  if (part < 0 || part >= n_parts) return fail(FM_ERR_INVALID, "part out of range");
  const int npe = full->etype;
  const int64_t N = full->N, E = full->E;
  std::vector<int32_t> dflt;
  if (!elem_part) {
    default_parts(full, n_parts, dflt);
    elem_part = dflt.data();
  }
  for (int64_t e = 0; e < E; ++e)
    if (elem_part[e] < 0 || elem_part[e] >= n_parts) return fail(FM_ERR_INVALID, "elem_part value out of range");
  const bool vms = full->params.solver == FM_SOLVER_VMS;
  // lowest and highest part touching each node
  std::vector<int32_t> lo(N, INT32_MAX), hi(N, -1);
  std::vector<char> mine(N, 0);
  int64_t ne = 0;
  for (int64_t e = 0; e < E; ++e) {
    const int32_t q = elem_part[e];
    ne += (q == part);
    for (int a = 0; a < npe; ++a) {
      const int32_t n = full->conn[e * npe + a];
      lo[n] = std::min(lo[n], q);
      hi[n] = std::max(hi[n], q);
      if (q == part) mine[n] = 1;
    }
  }
  if (ne == 0) return fail(FM_ERR_INVALID, "partition part has no elements");
  // exchange list (global order)
  std::vector<int32_t> xpos(N, -1);
  int64_t nx = 0;
  for (int64_t n = 0; n < N; ++n)
    if ((hi[n] >= 0 && lo[n] != hi[n]) || (vms && n < 4)) xpos[n] = (int32_t)nx++;
  if (vms)
    for (int64_t n = 0; n < std::min<int64_t>(N, 4); ++n) mine[n] = 1;
  fm_problem* p = new fm_problem();
  p->etype = npe;
  p->params = full->params;
  p->part = part;
  p->n_parts = n_parts;
  p->x_total = nx;
  // local nodes in global order (so for VMS local nodes 0..3 are global 0..3)
  std::vector<int32_t> loc(N, -1);
  for (int64_t n = 0; n < N; ++n)
    if (mine[n]) {
      loc[n] = (int32_t)p->node_global.size();
      p->node_global.push_back((int32_t)n);
    }
  const int64_t NL = (int64_t)p->node_global.size();
  p->N = NL;
  p->E = ne;
  p->coords.resize(NL * 3);
  p->mass.resize(NL);
  p->node_rec.resize(NL);
  p->xidx.resize(NL);
  if (!full->init.empty()) p->init.resize(NL * 4);
  for (int64_t i = 0; i < NL; ++i) {
    const int32_t g = p->node_global[i];
    for (int k = 0; k < 3; ++k) p->coords[i * 3 + k] = full->coords[(int64_t)g * 3 + k];
    p->mass[i] = full->mass[g];
    p->node_rec[i] = full->node_rec[g];
    p->xidx[i] = xpos[g];
    if (!full->init.empty())
      for (int k = 0; k < 4; ++k) p->init[i * 4 + k] = full->init[(int64_t)g * 4 + k];
  }
  // the BC rows of the part's nodes, in local ids (the BCs themselves are
  // the resolved records above; the rows serve the output writers' dirBC
  // markers)
  for (size_t r = 0; r < full->vel_node.size(); ++r)
    if (loc[full->vel_node[r]] >= 0) {
      p->vel_node.push_back(loc[full->vel_node[r]]);
      p->vel_dir.push_back(r < full->vel_dir.size() ? full->vel_dir[r] : 0);
      for (int k = 0; k < 4; ++k) p->vel_vals.push_back(full->vel_vals[r * 4 + k]);
    }
  for (size_t r = 0; r < full->pres_node.size(); ++r)
    if (loc[full->pres_node[r]] >= 0) {
      p->pres_node.push_back(loc[full->pres_node[r]]);
      p->pres_vals.push_back(full->pres_vals[r]);
    }
  for (size_t r = 0; r < full->dir_node.size(); ++r)
    if (loc[full->dir_node[r]] >= 0) {
      p->dir_node.push_back(loc[full->dir_node[r]]);
      for (int k = 0; k < 3; ++k) p->dir_vals.push_back(full->dir_vals[r * 3 + k]);
    }
  p->recs = full->recs;
  p->tab_off = full->tab_off;
  p->tab_len = full->tab_len;
  p->tab_rows = full->tab_rows;
  p->elem_global.reserve(ne);
  p->conn.reserve(ne * npe);
  for (int64_t e = 0; e < E; ++e)
    if (elem_part[e] == part) {
      p->elem_global.push_back((int32_t)e);
      for (int a = 0; a < npe; ++a) p->conn.push_back(loc[full->conn[e * npe + a]]);
    }
  *out = p;
  return FM_OK;
}

FM_API int fm_problem_part_info(const fm_problem* p, int32_t* part, int32_t* n_parts, int64_t* x_total) {
  if (!p) return fail(FM_ERR_INVALID, "null problem");
  if (part) *part = p->part;
  if (n_parts) *n_parts = p->n_parts;
  if (x_total) *x_total = p->x_total;
  return FM_OK;
}

FM_API int fm_problem_part_map(const fm_problem* p, int32_t* node_global, int32_t* elem_global, int32_t* xidx) {
  if (!p) return fail(FM_ERR_INVALID, "null problem");
  if (p->part < 0) return fail(FM_ERR_INVALID, "problem is not a partition part");
  if (node_global) std::copy(p->node_global.begin(), p->node_global.end(), node_global);
  if (elem_global) std::copy(p->elem_global.begin(), p->elem_global.end(), elem_global);
  if (xidx) std::copy(p->xidx.begin(), p->xidx.end(), xidx);
  return FM_OK;
}

}  // extern "C"
