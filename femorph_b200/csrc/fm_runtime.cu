// Device runtime and C ABI of femorph_b200.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "fm_device.cuh"
#include "fm_internal.hpp"

namespace fm {
const char* last_error();
size_t vms_smem_bytes(int tn_max, int inc_max, int threads, bool mixed);
cudaError_t vms_configure(int tn_max, int inc_max);
cudaError_t launch_vms_iteration(const DevBatch& B, int tn_max, int inc_max, int threads, int iface_blocks, bool mixed,
                                 cudaStream_t s, cudaEvent_t* ev);

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
size_t supg_smem_bytes(int tn_max, int npe);
cudaError_t supg_configure(size_t smem, int npe);
cudaError_t launch_supg_step(const DevBatch& B, int tn_max, int threads, int iface_blocks, int npe, cudaStream_t s,
                             cudaEvent_t* ev);
cudaError_t launch_supg_pressure(const DevBatch& B, int tn_max, int npe, double* pres, cudaStream_t s);
}  // namespace fm

using namespace fm;

struct fm_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<fm_problem*> probs;
  Layout L;
  DevBatch D;
  std::vector<void*> allocs;
  int tn_max = 0, inc_max = 0, threads = 128, iface_blocks = 1, graph_steps = 0;
  int solver = 0, npe = 4, precision = 0;
  std::vector<int32_t> iters;   // host copy of each problem's completed iterations
  int32_t* h_targets = nullptr;    // pinned staging of the target array
  int32_t* d_targets = nullptr;
  cudaEvent_t ev_tgt = nullptr;    // targets copied (staging reusable)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int64_t last_launches = 0;
  bool timed = false;
  cudaGraphExec_t graph = nullptr;
  int graph_iters = 0;
  double* d_scratch = nullptr;  // element-sized scratch for output passes
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

template <class T>
static int upload(fm_batch* b, T** dst, const std::vector<T>& src) {
  int r = dalloc(b, (void**)dst, src.size() * sizeof(T));
  if (r) return r;
  if (!src.empty()) CK(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
  return FM_OK;
}

static void release(fm_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (void* p : b->allocs) cudaFree(p);
  b->allocs.clear();
  if (b->h_targets) cudaFreeHost(b->h_targets);
  if (b->ev_tgt) cudaEventDestroy(b->ev_tgt);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
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
int fm_version(void) { return 100; }

int fm_problem_create(const fm_mesh* m, const fm_bc* bc, const fm_params* prm, const double* init, fm_problem** out) {
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
  p->coords.assign(m->coords, m->coords + m->n_nodes * 3);
  p->conn.assign(m->conn, m->conn + m->n_elems * m->elem_type);
  for (int32_t c : p->conn)
    if (c < 0 || c >= p->N) {
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

static void default_tuning(int solver, int npe, fm_tuning& t) {
  if (t.threads != 128 && t.threads != 256) t.threads = 128;
  if (t.tile_elems <= 0) t.tile_elems = (npe == 8) ? 384 : 1024;
  if (t.tile_nodes <= 0) t.tile_nodes = (npe == 8) ? 640 : 512;
  if (t.tile_nodes > 4096) t.tile_nodes = 4096;
  if (solver == FM_SOLVER_VMS && t.tile_nodes > FM_MAX_TILE_NODES) t.tile_nodes = FM_MAX_TILE_NODES;
  if (t.graph_steps < 0) t.graph_steps = 0;
  (void)solver;
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
  // nodes: coords 24 + state 32 + pre 32 + mass 8 + bc 4; elements: conn + 12 or 24 doubles;
  // tiles/interface: bounded by ~24 B per element.
  int64_t per_e = (int64_t)npe * 2 + (probs[0]->params.solver == FM_SOLVER_VMS ? 96 : 192 + 16) + 24;
  *bytes = N * 100 + E * per_e + (64 << 20);
  return FM_OK;
}

int fm_batch_create(fm_problem* const* probs, int32_t n, const fm_tuning* tuning, int32_t device, fm_batch** out) {
  if (!probs || n <= 0 || !out) return fail(FM_ERR_INVALID, "null argument");
  *out = nullptr;
  const int solver = probs[0]->params.solver, npe = probs[0]->etype, prec = probs[0]->params.precision;
  for (int i = 0; i < n; ++i) {
    if (!probs[i]) return fail(FM_ERR_INVALID, "null problem");
    if (probs[i]->batch) return fail(FM_ERR_INVALID, "problem already belongs to a batch");
    if (probs[i]->params.solver != solver || probs[i]->etype != npe || probs[i]->params.precision != prec)
      return fail(FM_ERR_INVALID, "all problems of a batch must share solver, element type and precision");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FM_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(FM_ERR_INVALID, "bad device ordinal");
  CK(cudaSetDevice(device));
  fm_tuning t;
  memset(&t, 0, sizeof(t));
  if (tuning) t = *tuning;
  default_tuning(solver, npe, t);
  fm_batch* b = new fm_batch();
  b->device = device;
  b->solver = solver;
  b->npe = npe;
  b->precision = prec;
  b->threads = t.threads;
  b->graph_steps = t.graph_steps;
  b->probs.assign(probs, probs + n);
  int r = build_layout(probs, n, t.tile_elems, t.tile_nodes, b->L);
  if (r) {
    delete b;
    return r;
  }
  Layout& L = b->L;
  for (auto& tm : L.tiles) b->tn_max = std::max(b->tn_max, tm.n_node);
  b->inc_max = (L.max_tile_elems * npe + 7) / 8 * 8;
  size_t smem = solver == FM_SOLVER_VMS ? vms_smem_bytes(b->tn_max, b->inc_max, b->threads, prec == FM_MIXED)
                                        : supg_smem_bytes(b->tn_max, npe);
  if (smem > 227 * 1024) {
    delete b;
    return fail(FM_ERR_INVALID, "tile too large for shared memory; lower tile_nodes");
  }
  cudaError_t ce = solver == FM_SOLVER_VMS ? vms_configure(b->tn_max, b->inc_max) : supg_configure(smem, npe);
  if (ce != cudaSuccess) {
    delete b;
    return fail(FM_ERR_CUDA, std::string("kernel attribute: ") + cudaGetErrorString(ce));
  }
  const int64_t NN = L.n_nodes, NE = L.n_elems;
  // ---- host arrays in batch numbering ----
  std::vector<double> hx(NN), hy(NN), hz(NN), hu(NN), hv(NN), hw(NN), hp(NN), hm(NN);
  std::vector<int32_t> hbc(NN, -1);
  std::vector<BCRec> recs;
  std::vector<int32_t> toff, tlen;
  std::vector<double> trows;
  std::vector<DevProb> dprob(n);
  std::vector<DevProbState> dstate(n);
  for (int pi = 0; pi < n; ++pi) {
    fm_problem* p = probs[pi];
    const std::vector<int32_t>& nn = L.node_new[pi];
    const int32_t rbase = (int32_t)recs.size(), tbase = (int32_t)toff.size(), rowbase = (int32_t)(trows.size() / 4);
    for (const BCRec& rr : p->recs) {
      BCRec q = rr;
      if (q.tab >= 0) q.tab += tbase;
      recs.push_back(q);
    }
    for (size_t k = 0; k < p->tab_off.size(); ++k) {
      toff.push_back(p->tab_off[k] + rowbase);
      tlen.push_back(p->tab_len[k]);
    }
    trows.insert(trows.end(), p->tab_rows.begin(), p->tab_rows.end());
    // initial state: init then BCs at time 0 (solve() prologue)
    std::vector<double> s0(p->N * 4, 0.0);
    if (!p->init.empty()) s0 = p->init;
    for (int64_t i = 0; i < p->N; ++i) {
      const int64_t g = nn[i];
      hx[g] = p->coords[i * 3 + 0];
      hy[g] = p->coords[i * 3 + 1];
      hz[g] = p->coords[i * 3 + 2];
      double s[4] = {s0[i * 4 + 0], s0[i * 4 + 1], s0[i * 4 + 2], s0[i * 4 + 3]};
      if (solver == FM_SOLVER_SUPG) s[3] = 0.0;
      if (p->node_rec[i] >= 0) {
        const BCRec& rr = p->recs[p->node_rec[i]];
        hbc[g] = rbase + p->node_rec[i];
        if (rr.tab >= 0) {
          // time 0 through the same table rule the device uses
          const double* tab = p->tab_rows.data() + (int64_t)p->tab_off[rr.tab] * 4;
          int nrow = p->tab_len[rr.tab];
          double v[3];
          bool ok = true;
          if (0.0 >= tab[(nrow - 1) * 4 + 3]) {
            for (int c = 0; c < 3; ++c) v[c] = tab[(nrow - 1) * 4 + c];
          } else {
            int cnt = 1;
            bool found = false;
            while (!found && cnt < nrow) {
              found = (0.0 >= tab[(cnt - 1) * 4 + 3]) && (0.0 < tab[cnt * 4 + 3]);
              if (!found) cnt++;
            }
            ok = found;
            if (found) {
              double t1 = tab[(cnt - 1) * 4 + 3], t2 = tab[cnt * 4 + 3];
              for (int c = 0; c < 3; ++c)
                v[c] = tab[(cnt - 1) * 4 + c] + ((tab[cnt * 4 + c] - tab[(cnt - 1) * 4 + c]) / (t2 - t1)) * (0.0 - t1);
            }
          }
          if (!ok) {
            delete b;
            return fail(FM_ERR_TABLE, "Could not find time in femUtils::interpTableData.");
          }
          if (rr.mask & BC_VX) s[0] = v[0];
          if (rr.mask & BC_VY) s[1] = v[1];
          if (rr.mask & BC_VZ) s[2] = v[2];
        }
        if (rr.mask & BC_PRES) s[3] = rr.p;
        if (rr.mask & BC_DIR) {
          s[0] = rr.d[0];
          s[1] = rr.d[1];
          s[2] = rr.d[2];
        }
      }
      hu[g] = s[0];
      hv[g] = s[1];
      hw[g] = s[2];
      hp[g] = s[3];
      hm[g] = p->mass[i];
    }
    DevProb& d = dprob[pi];
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
    d.ndual = solver == FM_SOLVER_VMS ? std::max(0, pr.tot_dual_steps) : 0;
    d.solver = solver;
    d.precision = prec;
    d.npe = npe;
    d.ex_mask = 0;
    for (int k = 0; k < 6; ++k)
      if (pr.ex_opts[k]) d.ex_mask |= (1 << k);
    d.glob_fixed = pr.glob_fixed;
    for (int k = 0; k < 4; ++k) d.q1[k] = (k < p->N) ? nn[k] : -1;
    d.node_begin = L.node_begin[pi];
    d.n_nodes = p->N;
    d.elem_begin = L.elem_begin[pi];
    d.n_elems = p->E;
    DevProbState& s = dstate[pi];
    memset(&s, 0, sizeof(s));
    s.iter = 0;
    s.status = FM_OK;
    s.time = 0.0 + pr.time_step;
  }
  // q1 pressures at "iteration -1": pre-BC initial = post-BC initial except pinned nodes;
  // never read before iteration 1 writes them.
  std::vector<double> hq1(n * 8, 0.0);
  DevBatch& D = b->D;
  memset(&D, 0, sizeof(D));
#define UP(dst, src)                              \
  do {                                            \
    r = upload(b, &dst, src);                     \
    if (r) {                                      \
      release(b);                                 \
      delete b;                                   \
      return r;                                   \
    }                                             \
  } while (0)
  double *x, *y, *z, *su, *sv, *sw, *sp, *pu, *pv, *pw, *pp, *ms;
  UP(x, hx); UP(y, hy); UP(z, hz);
  UP(su, hu); UP(sv, hv); UP(sw, hw); UP(sp, hp);
  UP(pu, hu); UP(pv, hv); UP(pw, hw); UP(pp, hp);
  UP(ms, hm);
  D.x = x; D.y = y; D.z = z; D.su = su; D.sv = sv; D.sw = sw; D.sp = sp;
  D.pu = pu; D.pv = pv; D.pw = pw; D.pp = pp; D.mass = ms;
  int32_t* nbc;
  UP(nbc, hbc);
  D.node_bc = nbc;
  BCRec* drecs;
  UP(drecs, recs);
  D.recs = drecs;
  int32_t *dtoff, *dtlen;
  UP(dtoff, toff);
  UP(dtlen, tlen);
  D.tab_off = dtoff;
  D.tab_len = dtlen;
  double* dtrows;
  UP(dtrows, trows);
  D.tab_rows = dtrows;
  uint16_t* dconn;
  UP(dconn, L.conn_local);
  D.conn = dconn;
  D.E = NE;
  // Per-element history: VMS subscales (12 per element, FP64 or FP32 in the
  // mixed form); SUPG the previous step's element forces for AB2 (3*npe).
  bool any_ab2 = false;
  for (int pi = 0; pi < n; ++pi) any_ab2 |= (probs[pi]->params.ex_opts[0] == 0);
  if (solver == FM_SOLVER_VMS && prec == FM_MIXED) {
    r = dalloc(b, (void**)&D.sdus32, (size_t)NE * 12 * sizeof(float));
    if (r) { release(b); delete b; return r; }
    CK(cudaMemset(D.sdus32, 0, (size_t)NE * 12 * sizeof(float)));
    // elements whose Jacobian inverse stays in FP64 (aspect ratio above the
    // limit): flagged in bit 15 of their first tile-local node id
    for (int pi = 0; pi < n; ++pi) {
      fm_problem* p = probs[pi];
      for (int64_t k = 0; k < L.elem_count[pi]; ++k) {
        const int32_t oe = L.elem_old[pi][k];
        if (oe >= 0 && tet_aspect_ratio(p->coords.data(), &p->conn[(int64_t)oe * 4]) > FM_MIXED_ASPECT_LIMIT)
          L.conn_local[(size_t)(L.elem_begin[pi] + k) * 4] |= 0x8000;
      }
    }
    CK(cudaMemcpy(dconn, L.conn_local.data(), L.conn_local.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
  } else if (solver == FM_SOLVER_VMS || any_ab2) {
    const int nhist = solver == FM_SOLVER_VMS ? 12 : 3 * npe;
    r = dalloc(b, (void**)&D.sdus, (size_t)NE * nhist * sizeof(double));
    if (r) { release(b); delete b; return r; }
    CK(cudaMemset(D.sdus, 0, (size_t)NE * nhist * sizeof(double)));
  }
  if (solver == FM_SOLVER_SUPG) {
    r = dalloc(b, (void**)&D.el_lam, (size_t)NE * sizeof(double));
    if (!r) r = dalloc(b, (void**)&D.el_reg, (size_t)NE * sizeof(double));
    if (!r) r = dalloc(b, (void**)&b->d_scratch, (size_t)NE * sizeof(double));
    if (r) { release(b); delete b; return r; }
    CK(cudaMemset(D.el_lam, 0, (size_t)NE * sizeof(double)));
    CK(cudaMemset(D.el_reg, 0, (size_t)NE * sizeof(double)));
  }
  TileMeta* dtiles;
  UP(dtiles, L.tiles);
  D.tiles = dtiles;
  D.n_tiles = (int32_t)L.tiles.size();
  int32_t *dtn, *dtc;
  UP(dtn, L.tile_nodes);
  UP(dtc, L.tile_cols);
  D.tile_nodes = dtn;
  D.tile_cols = dtc;
  uint16_t *dinc, *doff;
  UP(dinc, L.tile_inc);
  UP(doff, L.tile_off);
  D.tile_inc = dinc;
  D.tile_off = doff;
  for (double** pp2 : {&D.part0, &D.part1, &D.part2, &D.part3}) {
    r = dalloc(b, (void**)pp2, (size_t)std::max<int64_t>(L.n_slots, 1) * sizeof(double));
    if (r) { release(b); delete b; return r; }
  }
  int32_t *din, *dsb, *dsl, *dip;
  UP(din, L.iface_node);
  UP(dsb, L.iface_slot_beg);
  UP(dsl, L.iface_slots);
  UP(dip, L.iface_prob);
  D.iface_node = din;
  D.iface_slot_beg = dsb;
  D.iface_slots = dsl;
  D.iface_prob = dip;
  D.n_iface = (int32_t)L.iface_node.size();
  DevProb* dp;
  UP(dp, dprob);
  D.probs = dp;
  DevProbState* ds;
  UP(ds, dstate);
  D.pstate = ds;
  double* dq1;
  UP(dq1, hq1);
  D.q1p = dq1;
  D.n_probs = n;
  std::vector<int32_t> zt(n, 0);
  int32_t* dtg;
  UP(dtg, zt);
  D.target = dtg;
  b->d_targets = dtg;
  std::vector<uint32_t> zero1(1, 0);
  uint32_t* ddone;
  UP(ddone, zero1);
  D.done = ddone;
#undef UP
  b->iface_blocks = (int)std::max<int64_t>(1, std::min<int64_t>((D.n_iface + 255) / 256, 148 * 8));
  b->iters.assign(n, 0);
  CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&b->ev0));
  CK(cudaEventCreate(&b->ev1));
  CK(cudaEventCreateWithFlags(&b->ev_tgt, cudaEventDisableTiming));
  CK(cudaMallocHost((void**)&b->h_targets, sizeof(int32_t) * n));
  for (int i = 0; i < n; ++i) {
    probs[i]->batch = b;
    probs[i]->index = i;
    probs[i]->steps_done = 0;
  }
  *out = b;
  return FM_OK;
}

int fm_batch_destroy(fm_batch* b) {
  if (!b) return FM_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (fm_problem* p : b->probs) {
    p->batch = nullptr;
    p->index = -1;
  }
  release(b);
  delete b;
  return FM_OK;
}

// One iteration (dual iteration for VMS, step for SUPG): tile kernel +
// interface kernel.
static cudaError_t launch_one(fm_batch* b, cudaStream_t s, cudaEvent_t* ev) {
  if (b->solver == FM_SOLVER_VMS)
    return launch_vms_iteration(b->D, b->tn_max, b->inc_max, b->threads, b->iface_blocks, b->precision == FM_MIXED, s,
                                ev);
  return launch_supg_step(b->D, b->tn_max, b->threads, b->iface_blocks, b->npe, s, ev);
}

// Sets per-problem targets (iterations) and launches enough iterations.
// With prof != nullptr every kernel is bracketed by CUDA events and the
// per-kernel device times are summed into prof[0] (element/tile kernel) and
// prof[1] (interface kernel), in milliseconds.
static int run_iterations(fm_batch* b, const std::vector<int32_t>& add_iters, cudaStream_t s, double* prof = nullptr) {
  const int n = (int)b->probs.size();
  int32_t maxit = 0;
  for (int i = 0; i < n; ++i) maxit = std::max(maxit, add_iters[i]);
  if (maxit == 0) return FM_OK;
  // new targets (the host tracks every problem's iteration count exactly)
  CK(cudaEventSynchronize(b->ev_tgt));  // staging buffer free again
  for (int i = 0; i < n; ++i) b->h_targets[i] = b->iters[i] + add_iters[i];
  CK(cudaMemcpyAsync(b->d_targets, b->h_targets, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
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
  // (the per-problem targets live in device memory, so the same graph serves
  // every block and every ragged step pattern)
  if (!prof && b->graph_steps > 0 && maxit >= b->graph_steps) {
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
      launches += 2 * (int64_t)b->graph_iters;
    }
  }
  for (; it < maxit; ++it) {
    cudaEvent_t* ev = prof ? &evs[(size_t)it * 3] : nullptr;
    cudaError_t e = launch_one(b, s, ev);
    if (e != cudaSuccess) return fail(FM_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    launches += 2;
  }
  CK(cudaEventRecord(b->ev1, s));
  if (prof) {
    CK(cudaEventSynchronize(b->ev1));
    prof[0] = prof[1] = 0.0;
    for (int it = 0; it < maxit; ++it) {
      float a = 0.f, c = 0.f;
      CK(cudaEventElapsedTime(&a, evs[it * 3], evs[it * 3 + 1]));
      CK(cudaEventElapsedTime(&c, evs[it * 3 + 1], evs[it * 3 + 2]));
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

int fm_batch_step_ragged(fm_batch* b, const int32_t* nsteps, void* stream) {
  if (!b || !nsteps) return fail(FM_ERR_INVALID, "null argument");
  CK(cudaSetDevice(b->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : b->stream;
  const int n = (int)b->probs.size();
  std::vector<int32_t> add(n);
  for (int i = 0; i < n; ++i) {
    if (nsteps[i] < 0) return fail(FM_ERR_INVALID, "negative step count");
    const int per = b->solver == FM_SOLVER_VMS ? b->probs[i]->params.tot_dual_steps + 1 : 1;
    add[i] = nsteps[i] * std::max(1, per);
  }
  int r = run_iterations(b, add, s);
  if (r) return r;
  for (int i = 0; i < n; ++i) b->probs[i]->steps_done += nsteps[i];
  return FM_OK;
}

int fm_batch_profile(fm_batch* b, int32_t nsteps, double* kernel_ms, int64_t* launches) {
  if (!b || nsteps < 0) return fail(FM_ERR_INVALID, "bad argument");
  CK(cudaSetDevice(b->device));
  const int n = (int)b->probs.size();
  std::vector<int32_t> add(n);
  int64_t per_kernel = 0;
  for (int i = 0; i < n; ++i) {
    const int per = b->solver == FM_SOLVER_VMS ? b->probs[i]->params.tot_dual_steps + 1 : 1;
    add[i] = nsteps * std::max(1, per);
    per_kernel = std::max<int64_t>(per_kernel, add[i]);
  }
  double prof[2] = {0.0, 0.0};
  int r = run_iterations(b, add, b->stream, prof);
  if (r) return r;
  for (int i = 0; i < n; ++i) b->probs[i]->steps_done += nsteps;
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

int fm_batch_step(fm_batch* b, int32_t nsteps, void* stream) {
  if (!b) return fail(FM_ERR_INVALID, "null batch");
  std::vector<int32_t> v(b->probs.size(), nsteps);
  return fm_batch_step_ragged(b, v.data(), stream);
}

int fm_batch_sync(fm_batch* b) {
  if (!b) return fail(FM_ERR_INVALID, "null batch");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  CK(cudaDeviceSynchronize());
  const int n = (int)b->probs.size();
  std::vector<DevProbState> st(n);
  CK(cudaMemcpy(st.data(), b->D.pstate, sizeof(DevProbState) * n, cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; ++i)
    if (st[i].status != FM_OK) return fail(st[i].status, fm_strerror(st[i].status));
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
  if (nt) *nt = (int64_t)b->L.tiles.size();
  if (ni) *ni = (int64_t)b->L.iface_node.size();
  if (mc) *mc = b->L.max_colors;
  if (ns) *ns = b->L.n_slots;
  return FM_OK;
}

int fm_problem_get_state(fm_problem* p, double* u, double* pres, double* elem3, double* sdus) {
  if (!p) return fail(FM_ERR_INVALID, "null problem");
  fm_batch* b = p->batch;
  if (!b) return fail(FM_ERR_INVALID, "problem is not in a batch");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  const int pi = p->index;
  const int64_t nb = b->L.node_begin[pi], eb = b->L.elem_begin[pi];
  const int64_t N = p->N, E = p->E, EC = b->L.elem_count[pi];
  const std::vector<int32_t>& nn = b->L.node_new[pi];
  const std::vector<int32_t>& eo = b->L.elem_old[pi];
  std::vector<double> tmp(N);
  double* cols[4] = {b->D.su, b->D.sv, b->D.sw, b->D.sp};
  if (u) {
    for (int c = 0; c < 3; ++c) {
      CK(cudaMemcpy(tmp.data(), cols[c] + nb, sizeof(double) * N, cudaMemcpyDeviceToHost));
      for (int64_t i = 0; i < N; ++i) u[i * 3 + c] = tmp[nn[i] - nb];
    }
    if (b->solver == FM_SOLVER_SUPG && p->params.glob_fixed)
      for (int64_t i = 0; i < N; ++i)
        for (int c = 0; c < 3; ++c)
          if (p->params.glob_fixed & (1 << c)) u[i * 3 + c] = 0.0;
  }
  if (b->solver == FM_SOLVER_VMS) {
    if (pres) {
      CK(cudaMemcpy(tmp.data(), cols[3] + nb, sizeof(double) * N, cudaMemcpyDeviceToHost));
      for (int64_t i = 0; i < N; ++i) pres[i] = tmp[nn[i] - nb];
    }
    if (elem3 || sdus) {
      std::vector<double> h((size_t)E * 12), col(EC);
      std::vector<float> colf(b->D.sdus32 ? EC : 0);
      for (int q = 0; q < 12; ++q) {
        if (b->D.sdus32) {
          CK(cudaMemcpy(colf.data(), b->D.sdus32 + (int64_t)q * b->L.n_elems + eb, sizeof(float) * EC,
                        cudaMemcpyDeviceToHost));
          for (int64_t k = 0; k < EC; ++k) col[k] = colf[k];
        } else {
          CK(cudaMemcpy(col.data(), b->D.sdus + (int64_t)q * b->L.n_elems + eb, sizeof(double) * EC,
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
