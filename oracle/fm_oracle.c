/* Oracle B: plain-C CPU restatement of feMorph's explicit flow step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker used by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg; the product
 * (femorph_b200/csrc) never links or calls it.
 *
 * It follows the reference statement by statement, keeping its loop and
 * operand order so that it agrees with the compiled reference (oracle A) to
 * the last bits on x86-64 without FMA contraction:
 *   VMS  : src/femVMSExplicitFluidSolver.cpp:4-13 (constants), 21-91
 *          (initial_assemble), 93-399 (assemble_RHS), 406-588
 *          (assemble_projRes_explicit), 593-646 (update_subscales_explicit),
 *          648-653 (apply_zeroTraction), 726-752 (update_solution), 754-772
 *          (update_dual_solution), 842-1334 (solve).
 *   SUPG : src/femSUPGExplicitFluidSolver.cpp:138-331 (L/U/S/B/D/H matrices),
 *          336-377 (eval_stabilization), 382-441 (eval_bulk_modulus), 446-501
 *          (compute_pressure), 507-598 (form_lumped_mass), 660-707
 *          (eval_avg_shapeDeriv), 794-1735 (solve).
 *   Elements : src/femElement.cpp:104-127, 192-232, 272-354;
 *          src/femTetra4.cpp:295-330; src/femHexa8.cpp:13-42;
 *          src/femIntegrationRule.cpp:11-337; src/femUtils.cpp:716-770
 *          (invert3x3Matrix), 818-871 (interpVelocity, interpTableData).
 *   BCs  : src/femModel.cpp:4549-4576 (postProcessNodeVelocities, including
 *          its quirk: the direction of the k-th *row* is used for the k-th
 *          unique node), 4581-4643 (setNodeVelocity, setDirichletBC).
 * Diagnostics that do not feed the state (norms, CFL, logs) are left out,
 * except the VMS centroid subgrid average that the reference writes out.
 *
 * Host threads.  The element loops run in parallel over element ranges; the
 * reference's nodal scatters (rhs[node] += lRes in element order, the SUPG
 * solN and l_M sums) are computed per node, each walking its incident
 * (element, corner) entries in increasing element order, so every nodal sum
 * is formed from the same terms in the same order as the reference's serial
 * loop and the results do not depend on the thread count (bit for bit).
 * FMO_THREADS (environment) or fmo_set_threads() sets the thread count;
 * default: the CPUs this process may run on.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <sched.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define FMO_OK 0
#define FMO_ERR_INVALID 1
#define FMO_ERR_TABLE 2

typedef struct {
  int64_t N, E;
  int npe; /* 4 (tet4) or 8 (hexa8) */
  const double* x;
  const int32_t* conn;
  int solver; /* 0 VMS, 1 SUPG */
  double props[5];
  double dt, ds;
  int ndual;
  int ex_opts[6];
  int glob_fixed; /* bit0 X, bit1 Y, bit2 Z */
  /* velocity tables after postProcessNodeVelocities */
  int nvel;
  int32_t* vel_node;
  int64_t* vel_off;
  int64_t* vel_len;
  double* vel_tab; /* rows of (vx,vy,vz,t) */
  int32_t* vel_dir;
  int ndir;
  int32_t* dir_node;
  double* dir_vals;
  int npres;
  int32_t* pres_node;
  double* pres_vals;
  double cur_time;
  int64_t step;
  int err;
  /* VMS */
  double *sol_n, *sol_prev, *sol_tau, *rhs, *sdus, *sgps, *volumes, *DNs, *char_length, *nd_mass, *elmTaus, *projRHS;
  double *el_u_sdus; /* centroid subgrid velocity (E x 3) of the last dual pass */
  /* SUPG */
  double *sol_p, *solN, *l_M, *k_p, *k_pp, *el_lam, *el_regime, *pres_n;
  /* node -> incident (element * npe + corner) entries, increasing element order */
  int64_t* inc_off;
  int64_t* inc_ent;
  double* lres; /* VMS: [E][16] element residuals of the current pass; SUPG: [E][24] mass row sums */
  const double* pres_src; /* SUPG: the state compute_pressure reads */
} fmo_ctx;

/* ------------------------------------------------------------------ */
/* Host threads                                                        */
/* ------------------------------------------------------------------ */
#define FMO_MAX_THREADS 256
static int g_threads = 0;

void fmo_set_threads(int n) { g_threads = n < 1 ? 1 : (n > FMO_MAX_THREADS ? FMO_MAX_THREADS : n); }

int fmo_get_threads(void) {
  if (g_threads > 0) return g_threads;
  const char* s = getenv("FMO_THREADS");
  int n = s ? atoi(s) : 0;
  if (n <= 0) {
    cpu_set_t set;
    n = sched_getaffinity(0, sizeof(set), &set) == 0 ? CPU_COUNT(&set) : (int)sysconf(_SC_NPROCESSORS_ONLN);
  }
  fmo_set_threads(n);
  return g_threads;
}

typedef void (*fmo_range_fn)(fmo_ctx* c, int64_t b, int64_t e);
typedef struct {
  fmo_range_fn fn;
  fmo_ctx* c;
  int64_t b, e;
} fmo_job;

static void* fmo_job_run(void* p) {
  fmo_job* j = (fmo_job*)p;
  j->fn(j->c, j->b, j->e);
  return NULL;
}

/* fn(c, b, e) over [0, n) split into contiguous ranges, one per thread. */
static void par_for(fmo_ctx* c, int64_t n, fmo_range_fn fn) {
  int T = fmo_get_threads();
  if ((int64_t)T > n / 64) T = (int)(n / 64);
  if (T <= 1) {
    fn(c, 0, n);
    return;
  }
  pthread_t th[FMO_MAX_THREADS];
  fmo_job job[FMO_MAX_THREADS];
  int started[FMO_MAX_THREADS];
  for (int t = 0; t < T; ++t) {
    job[t].fn = fn;
    job[t].c = c;
    job[t].b = n * t / T;
    job[t].e = n * (t + 1) / T;
  }
  for (int t = 1; t < T; ++t) started[t] = pthread_create(&th[t], NULL, fmo_job_run, &job[t]) == 0;
  fmo_job_run(&job[0]);
  for (int t = 1; t < T; ++t) {
    if (started[t])
      pthread_join(th[t], NULL);
    else
      fmo_job_run(&job[t]); /* no thread: run the range here */
  }
}

/* Node incidence lists in element order (counting sort of conn). */
static void build_incidence(fmo_ctx* c) {
  int64_t N = c->N, E = c->E;
  int npe = c->npe;
  c->inc_off = (int64_t*)calloc(N + 1, sizeof(int64_t));
  c->inc_ent = (int64_t*)malloc(sizeof(int64_t) * (E * npe + 1));
  for (int64_t q = 0; q < E * npe; ++q) c->inc_off[c->conn[q] + 1]++;
  for (int64_t n = 0; n < N; ++n) c->inc_off[n + 1] += c->inc_off[n];
  int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (N + 1));
  memcpy(fill, c->inc_off, sizeof(int64_t) * (N + 1));
  for (int64_t q = 0; q < E * npe; ++q) c->inc_ent[fill[c->conn[q]]++] = q;
  free(fill);
}

/* ------------------------------------------------------------------ */
/* Boundary conditions                                                 */
/* ------------------------------------------------------------------ */
static int cmp_i32(const void* a, const void* b) {
  int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

/* femUtils.cpp:830-871 */
static int interp_table(double time, const double* tab, int64_t n, double out[3]) {
  if (time >= tab[(n - 1) * 4 + 3]) {
    for (int c = 0; c < 3; ++c) out[c] = tab[(n - 1) * 4 + c];
    return 0;
  }
  int found = 0;
  int64_t count = 1;
  while (!found && count < n) {
    found = (time >= tab[(count - 1) * 4 + 3]) && (time < tab[count * 4 + 3]);
    if (!found) count++;
  }
  if (!found) return FMO_ERR_TABLE;
  double t1 = tab[(count - 1) * 4 + 3], t2 = tab[count * 4 + 3];
  for (int c = 0; c < 3; ++c) {
    double v1 = tab[(count - 1) * 4 + c], v2 = tab[count * 4 + c];
    out[c] = v1 + ((v2 - v1) / (t2 - t1)) * (time - t1); /* femUtils.cpp:818-828 */
  }
  return 0;
}

/* femModel.cpp:4581-4633; sol has ncol columns */
static void set_node_velocity(fmo_ctx* c, double t, double* sol, int ncol) {
  for (int k = 0; k < c->nvel; ++k) {
    int32_t n = c->vel_node[k];
    double v[3];
    int e = interp_table(t, c->vel_tab + c->vel_off[k] * 4, c->vel_len[k], v);
    if (e) { c->err = e; return; }
    double* s = sol + (int64_t)n * ncol;
    switch (c->vel_dir[k]) {
      case 0: s[0] = v[0]; break;
      case 1: s[1] = v[1]; break;
      case 2: s[2] = v[2]; break;
      case 3: s[0] = v[0]; s[1] = v[1]; break;
      case 4: s[1] = v[1]; s[2] = v[2]; break;
      case 5: s[0] = v[0]; s[2] = v[2]; break;
      case 6: s[0] = v[0]; s[1] = v[1]; s[2] = v[2]; break;
      default: c->err = FMO_ERR_INVALID; return;
    }
  }
}

/* femModel.cpp:4635-4643 */
static void set_dirichlet(fmo_ctx* c, double* sol, int ncol) {
  for (int k = 0; k < c->ndir; ++k) {
    double* s = sol + (int64_t)c->dir_node[k] * ncol;
    s[0] = c->dir_vals[k * 3 + 0];
    s[1] = c->dir_vals[k * 3 + 1];
    s[2] = c->dir_vals[k * 3 + 2];
  }
}

/* femVMSExplicitFluidSolver.cpp:648-653 */
static void apply_zero_traction(fmo_ctx* c, double* sol) {
  for (int k = 0; k < c->npres; ++k) sol[(int64_t)c->pres_node[k] * 4 + 3] = c->pres_vals[k];
}

/* femModel.cpp:4549-4576 (postProcessNodeVelocities + MakeCompactList) */
static int build_vel_tables(fmo_ctx* c, int nrows, const int32_t* node, const double* vals, const int32_t* dir) {
  c->nvel = 0;
  if (nrows == 0) return 0;
  int32_t* sorted = (int32_t*)malloc(sizeof(int32_t) * nrows);
  memcpy(sorted, node, sizeof(int32_t) * nrows);
  qsort(sorted, nrows, sizeof(int32_t), cmp_i32);
  int nu = 0;
  for (int i = 0; i < nrows; ++i)
    if (i == nrows - 1 || sorted[i] != sorted[i + 1]) sorted[nu++] = sorted[i];
  c->nvel = nu;
  c->vel_node = sorted;
  c->vel_off = (int64_t*)calloc(nu, sizeof(int64_t));
  c->vel_len = (int64_t*)calloc(nu, sizeof(int64_t));
  c->vel_dir = (int32_t*)calloc(nu, sizeof(int32_t));
  c->vel_tab = (double*)malloc(sizeof(double) * 4 * nrows);
  for (int i = 0; i < nrows; ++i) {
    int lo = 0, hi = nu - 1;
    while (lo < hi) { int m = (lo + hi) / 2; if (sorted[m] < node[i]) lo = m + 1; else hi = m; }
    c->vel_len[lo]++;
  }
  int64_t acc = 0;
  for (int k = 0; k < nu; ++k) { c->vel_off[k] = acc; acc += c->vel_len[k]; c->vel_len[k] = 0; }
  for (int i = 0; i < nrows; ++i) {
    int lo = 0, hi = nu - 1;
    while (lo < hi) { int m = (lo + hi) / 2; if (sorted[m] < node[i]) lo = m + 1; else hi = m; }
    int64_t r = c->vel_off[lo] + c->vel_len[lo]++;
    memcpy(c->vel_tab + r * 4, vals + (int64_t)i * 4, 4 * sizeof(double));
  }
  /* Quirk: velNodesDir is filled per input row, read per unique node. */
  for (int k = 0; k < nu; ++k) c->vel_dir[k] = dir[k];
  return 0;
}

/* ------------------------------------------------------------------ */
/* VMS (tet4)                                                          */
/* ------------------------------------------------------------------ */
static const double V_w[4] = {0.25, 0.25, 0.25, 0.25};
static const double V_lN[4][4] = {{0.58541020, 0.13819660, 0.13819660, 0.13819660},
                                  {0.13819660, 0.58541020, 0.13819660, 0.13819660},
                                  {0.13819660, 0.13819660, 0.58541020, 0.13819660},
                                  {0.13819660, 0.13819660, 0.13819660, 0.58541020}};
static const double V_lDN[3][4] = {{-1.0, 1.0, 0.0, 0.0}, {-1.0, 0.0, 1.0, 0.0}, {-1.0, 0.0, 0.0, 1.0}};

/* femVMSExplicitFluidSolver.cpp:21-91 */
static void vms_initial_assemble(fmo_ctx* c, int64_t e) {
  int64_t E = c->E;
  int64_t ids[4];
  double xc[4][3], jac[3][3], cof[3][3], inv[3][3];
  for (int i = 0; i < 4; ++i) {
    ids[i] = c->conn[e * 4 + i];
    for (int j = 0; j < 3; ++j) xc[i][j] = c->x[ids[i] * 3 + j];
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) jac[i][j] = xc[j + 1][i] - xc[0][i];
  cof[0][0] = jac[1][1] * jac[2][2] - jac[2][1] * jac[1][2];
  cof[0][1] = jac[2][0] * jac[1][2] - jac[1][0] * jac[2][2];
  cof[0][2] = jac[1][0] * jac[2][1] - jac[2][0] * jac[1][1];
  cof[1][0] = jac[2][1] * jac[0][2] - jac[0][1] * jac[2][2];
  cof[1][1] = jac[0][0] * jac[2][2] - jac[2][0] * jac[0][2];
  cof[1][2] = jac[2][0] * jac[0][1] - jac[0][0] * jac[2][1];
  cof[2][0] = jac[0][1] * jac[1][2] - jac[1][1] * jac[0][2];
  cof[2][1] = jac[1][0] * jac[0][2] - jac[0][0] * jac[1][2];
  cof[2][2] = jac[0][0] * jac[1][1] - jac[1][0] * jac[0][1];
  double detJ = jac[0][0] * cof[0][0] + jac[0][1] * cof[0][1] + jac[0][2] * cof[0][2];
  double iDetJ = 1.0 / detJ;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) inv[i][j] = cof[j][i] * iDetJ;
  c->volumes[e] = detJ / 6.0;
  c->char_length[e] = pow(6.0 * c->volumes[e], 1.0 / 3.0);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 4; ++j)
      c->DNs[(i * 4 + j) * E + e] = V_lDN[0][j] * inv[0][i] + V_lDN[1][j] * inv[1][i] + V_lDN[2][j] * inv[2][i];
  /* nd_mass[ids[i]] += volumes[e] / 4.0 is summed per node in element order
     (vms_mass_nodes) */
}

static void vms_initial_range(fmo_ctx* c, int64_t b, int64_t e) {
  for (int64_t k = b; k < e; ++k) vms_initial_assemble(c, k);
}

/* femVMSExplicitFluidSolver.cpp:89 (nd_mass scatter) per node */
static void vms_mass_nodes(fmo_ctx* c, int64_t b, int64_t e) {
  for (int64_t n = b; n < e; ++n) {
    double acc = 0.0;
    for (int64_t j = c->inc_off[n]; j < c->inc_off[n + 1]; ++j) acc += c->volumes[c->inc_ent[j] >> 2] / 4.0;
    c->nd_mass[n] = acc;
  }
}

/* femVMSExplicitFluidSolver.cpp:93-399 (sol_n := sol_tau, sol_prev := sol_n) */
static void vms_assemble_rhs(fmo_ctx* c, int64_t e, const double* soln, const double* solprev, double sdu_out[4][3]) {
  int64_t E = c->E;
  double dt = c->dt;
  int64_t ids[4];
  double DN[3][4], f[4][3], hdu[4][3], u_prev[4][3], hp[4], sdu[4][3], sgp[4], grad[3][3];
  double u_gp_curr[3], u_gp_prev[3], hah[4][3], fh[3], ahGradHu[3], lRes[4][4];
  double nu = c->props[1] / c->props[0];
  double invEpsilon = c->props[2];
  double trGradHdu = 0.0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) lRes[i][j] = 0.0;
  for (int i = 0; i < 4; ++i) {
    ids[i] = c->conn[e * 4 + i];
    for (int j = 0; j < 3; ++j) {
      f[i][j] = 0.0; /* femNode::force is never set by the reader */
      hdu[i][j] = soln[ids[i] * 4 + j];
      u_prev[i][j] = solprev[ids[i] * 4 + j];
      sdu[i][j] = c->sdus[(i * 3 + j) * E + e];
    }
    hp[i] = soln[ids[i] * 4 + 3];
    sgp[i] = c->sgps[i * E + e];
  }
  double Ve = c->volumes[e];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 4; ++j) DN[i][j] = c->DNs[(i * 4 + j) * E + e];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j)
      grad[i][j] = DN[j][0] * hdu[0][i] + DN[j][1] * hdu[1][i] + DN[j][2] * hdu[2][i] + DN[j][3] * hdu[3][i];
    trGradHdu += grad[i][i];
  }
  for (int g = 0; g < 4; ++g) {
    double wGp = V_w[g] * Ve;
    double sgp_gp = sgp[g];
    for (int i = 0; i < 3; ++i) {
      hah[g][i] = 0.0;
      fh[i] = 0.0;
      u_gp_curr[i] = 0.0;
      u_gp_prev[i] = 0.0;
      for (int j = 0; j < 4; ++j) {
        hah[g][i] += hdu[j][i] * V_lN[g][j];
        u_gp_curr[i] += hdu[j][i] * V_lN[g][j];
        u_gp_prev[i] += u_prev[j][i] * V_lN[g][j];
        fh[i] += f[j][i] * V_lN[g][j];
      }
      hah[g][i] += sdu[g][i];
    }
    double hph = 0.0;
    for (int i = 0; i < 4; ++i) hph += hp[i] * V_lN[g][i];
    for (int i = 0; i < 3; ++i) {
      ahGradHu[i] = 0.0;
      for (int j = 0; j < 3; ++j) ahGradHu[i] += grad[i][j] * hah[g][j];
    }
    for (int a = 0; a < 4; ++a) {
      double ahDN = 0.0, sduhDN = 0.0;
      for (int i = 0; i < 3; ++i) {
        ahDN += hah[g][i] * DN[i][a];
        sduhDN += sdu[g][i] * DN[i][a];
      }
      for (int i = 0; i < 3; ++i) {
        lRes[a][i] += wGp * ((u_gp_curr[i] - u_gp_prev[i]) / dt) * V_lN[g][a];
        for (int j = 0; j < 3; ++j) lRes[a][i] += wGp * nu * (grad[i][j]) * DN[j][a];
        lRes[a][i] += wGp * ahGradHu[i] * V_lN[g][a];
        lRes[a][i] += -wGp * hph * DN[i][a];
        lRes[a][i] += -wGp * sdu[g][i] * ahDN;
        lRes[a][i] += -wGp * sgp_gp * DN[i][a];
        lRes[a][i] += -wGp * fh[i] * V_lN[g][a];
      }
      lRes[a][3] += wGp * trGradHdu * V_lN[g][a] * invEpsilon;
      lRes[a][3] += -wGp * sduhDN * invEpsilon;
    }
  }
  /* rhs[ids[a]*4+i] += lRes[a][i] (src lines 393-396): kept per element
     and summed per node in element order (vms_rhs_nodes) */
  for (int a = 0; a < 4; ++a)
    for (int i = 0; i < 4; ++i) c->lres[e * 16 + a * 4 + i] = lRes[a][i];
  for (int a = 0; a < 4; ++a)
    for (int i = 0; i < 3; ++i) sdu_out[a][i] = sdu[a][i];
}

static void vms_rhs_range(fmo_ctx* c, int64_t b, int64_t e) {
  for (int64_t k = b; k < e; ++k) {
    double sdu[4][3];
    vms_assemble_rhs(c, k, c->sol_tau, c->sol_n, sdu);
    for (int j = 0; j < 3; ++j) c->el_u_sdus[k * 3 + j] = 0.0;
    for (int a = 0; a < 4; ++a)
      for (int j = 0; j < 3; ++j) c->el_u_sdus[k * 3 + j] += sdu[a][j] * 0.25;
  }
}

/* The nodal scatter of assemble_RHS per node, then update_dual_solution
   (src lines 754-772) on the node. */
static void vms_rhs_nodes(fmo_ctx* c, int64_t b, int64_t e) {
  for (int64_t n = b; n < e; ++n) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t j = c->inc_off[n]; j < c->inc_off[n + 1]; ++j) {
      const double* r = c->lres + (c->inc_ent[j] >> 2) * 16 + (c->inc_ent[j] & 3) * 4;
      for (int i = 0; i < 4; ++i) acc[i] += r[i];
    }
    for (int i = 0; i < 4; ++i) {
      c->rhs[n * 4 + i] = acc[i];
      c->sol_tau[n * 4 + i] = c->sol_n[n * 4 + i] - c->ds * acc[i] / c->nd_mass[n];
    }
  }
}

/* femVMSExplicitFluidSolver.cpp:406-588 (proj_res_at_nodes = false) */
static void vms_assemble_proj(fmo_ctx* c, int64_t e, const double* soln) {
  int64_t E = c->E;
  int64_t ids[4];
  double DN[3][4], sdu[4][3], hdu[4][3], du[4][3], p[4], grad[3][3], gradP[3];
  double hah[3], ahGradDu[3], projL[4][4], proj_den[4][4];
  double maxA = 0.0;
  double nu = c->props[1] / c->props[0];
  double invEps = c->props[2], c1 = c->props[3], c2 = c->props[4];
  double dt = c->dt;
  double insDiameter = c->char_length[e];
  double divu = 0.0;
  for (int i = 0; i < 4; ++i) {
    ids[i] = c->conn[e * 4 + i];
    for (int j = 0; j < 3; ++j) {
      du[i][j] = soln[ids[i] * 4 + j];
      hdu[i][j] = du[i][j];
      sdu[i][j] = c->sdus[(i * 3 + j) * E + e];
      projL[i][j] = 0.0;
      proj_den[i][j] = 0.0;
    }
    p[i] = soln[(int64_t)i * 4 + 3]; /* quirk: global nodes 0..3, src line 489 */
  }
  double Ve = c->volumes[e];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 4; ++j) DN[i][j] = c->DNs[(i * 4 + j) * E + e];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j)
      grad[i][j] = DN[j][0] * du[0][i] + DN[j][1] * du[1][i] + DN[j][2] * du[2][i] + DN[j][3] * du[3][i];
    gradP[i] = DN[i][0] * p[0] + DN[i][1] * p[1] + DN[i][2] * p[2] + DN[i][3] * p[3];
  }
  /* projL[a][3]/proj_den[a][3] are set through the += below from their
     uninitialised values in the reference only for the i<3 columns; the
     pressure column starts at the values left by the loop above (column 3
     is never zeroed there).  The reference's local arrays hold whatever the
     stack had; its pressure projection is unused (include_sg_p = false), so
     the column is zeroed here. */
  for (int a = 0; a < 4; ++a) { projL[a][3] = 0.0; proj_den[a][3] = 0.0; }
  for (int g = 0; g < 4; ++g) {
    double wGp = V_w[g] * Ve;
    for (int i = 0; i < 3; ++i)
      hah[i] = hdu[0][i] * V_lN[g][0] + hdu[1][i] * V_lN[g][1] + hdu[2][i] * V_lN[g][2] + hdu[3][i] * V_lN[g][3] + sdu[g][i];
    maxA = fmax(maxA, sqrt(hah[0] * hah[0] + hah[1] * hah[1] + hah[2] * hah[2]));
    divu = 0.0;
    for (int i = 0; i < 3; ++i) {
      ahGradDu[i] = grad[i][0] * hah[0] + grad[i][1] * hah[1] + grad[i][2] * hah[2];
      divu += grad[i][i];
    }
    for (int i = 0; i < 3; ++i) c->sdus[(g * 3 + i) * E + e] = sdu[g][i] / dt - ahGradDu[i] - gradP[i];
    c->sgps[g * E + e] += c->sgps[g * E + e] / dt - invEps * divu;
    for (int a = 0; a < 4; ++a) {
      for (int i = 0; i < 3; ++i) {
        projL[a][i] += wGp * (ahGradDu[i] + gradP[i]) * V_lN[g][a];
        proj_den[a][i] += wGp * V_lN[g][a];
      }
      projL[a][3] += wGp * (invEps * divu) * V_lN[g][a];
      proj_den[a][3] += wGp * V_lN[g][a];
    }
  }
  /* projRHS is zeroed before each pass (src line 1047) and receives one
     term an entry: 0.0 + x */
  for (int a = 0; a < 4; ++a)
    for (int i = 0; i < 4; ++i) c->projRHS[(a * 4 + i) * E + e] = 0.0 + projL[a][i] / proj_den[a][i];
  double tau_u = 1.0 / (c1 * nu / (insDiameter * insDiameter) + c2 * maxA / insDiameter);
  double tau_p = (insDiameter * insDiameter) / (c1 * tau_u);
  c->elmTaus[0 * E + e] = 1.0 / (1.0 / dt + 1.0 / tau_u);
  c->elmTaus[1 * E + e] = 1.0 / (1.0 / dt + 1.0 / tau_p);
}

/* femVMSExplicitFluidSolver.cpp:593-646 (include_sg_p = false) */
static void vms_update_subscales(fmo_ctx* c, int64_t e) {
  int64_t E = c->E;
  double projL[4][4];
  double tau1 = c->elmTaus[e];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) projL[i][j] = c->projRHS[(i * 4 + j) * E + e];
  for (int g = 0; g < 4; ++g) {
    for (int i = 0; i < 3; ++i) {
      double projIGp = projL[0][i] * V_lN[g][0] + projL[1][i] * V_lN[g][1] + projL[2][i] * V_lN[g][2] + projL[3][i] * V_lN[g][3];
      c->sdus[(g * 3 + i) * E + e] = (c->sdus[(g * 3 + i) * E + e] + projIGp) * tau1;
    }
    c->sgps[g * E + e] = 0.0;
  }
}

static void vms_proj_range(fmo_ctx* c, int64_t b, int64_t e) {
  for (int64_t k = b; k < e; ++k) vms_assemble_proj(c, k, c->sol_tau);
}

static void vms_subscale_range(fmo_ctx* c, int64_t b, int64_t e) {
  for (int64_t k = b; k < e; ++k) vms_update_subscales(c, k);
}

/* One time step of femVMSExplicitFluidSolver::solve (src lines 1025-1234). */
static void vms_step(fmo_ctx* c) {
  int64_t N = c->N, E = c->E;
  c->cur_time += c->dt;
  int loopTau = 0, conv = 0;
  while (!conv) {
    loopTau++;
    par_for(c, E, vms_rhs_range);
    /* nodal sums + update_dual_solution, src lines 754-772 */
    par_for(c, N, vms_rhs_nodes);
    memcpy(c->sol_n, c->sol_tau, sizeof(double) * N * 4);
    /* the pressures of nodes 0..3 that every element reads (quirk Q1) are
       final here: the element passes below do not write the state */
    par_for(c, E, vms_proj_range);
    par_for(c, E, vms_subscale_range);
    set_node_velocity(c, c->cur_time, c->sol_tau, 4);
    apply_zero_traction(c, c->sol_tau);
    set_dirichlet(c, c->sol_tau, 4);
    conv = (loopTau > c->ndual);
  }
  /* update_solution, src lines 726-752 */
  memcpy(c->sol_prev, c->sol_n, sizeof(double) * N * 4);
  memcpy(c->sol_n, c->sol_tau, sizeof(double) * N * 4);
  c->step++;
}

/* ------------------------------------------------------------------ */
/* Element library (tet4 / hexa8) for SUPG                             */
/* ------------------------------------------------------------------ */
static const double H_c1[8] = {-1.0, 1.0, 1.0, -1.0, -1.0, 1.0, 1.0, -1.0};
static const double H_c2[8] = {-1.0, -1.0, 1.0, 1.0, -1.0, -1.0, 1.0, 1.0};
static const double H_c3[8] = {-1.0, -1.0, -1.0, -1.0, 1.0, 1.0, 1.0, 1.0};

/* femIntegrationRule.cpp: irSecondOrder coordinates and weights */
static void gauss_rule(int npe, int* ngp, double gps[8][3], double gpw[8]) {
  if (npe == 4) {
    const double a = 0.58541020, b = 0.13819660;
    double t[4][3] = {{a, b, b}, {b, a, b}, {b, b, a}, {b, b, b}};
    *ngp = 4;
    for (int g = 0; g < 4; ++g) {
      for (int k = 0; k < 3; ++k) gps[g][k] = t[g][k];
      gpw[g] = (1.0 / 6.0) * (1.0 / 4.0);
    }
  } else {
    double s = 1.0 / sqrt(3.0);
    double t[8][3] = {{-s, -s, s}, {s, -s, s}, {s, s, s}, {-s, s, s}, {-s, -s, -s}, {s, -s, -s}, {s, s, -s}, {-s, s, -s}};
    *ngp = 8;
    for (int g = 0; g < 8; ++g) {
      for (int k = 0; k < 3; ++k) gps[g][k] = t[g][k];
      gpw[g] = 8.0 * (1.0 / 8.0);
    }
  }
}

/* femTetra4.cpp:295-301, femHexa8.cpp:13-26 */
static void shape_fn(int npe, const double* q, double N[8]) {
  if (npe == 4) {
    N[0] = q[0]; N[1] = q[1]; N[2] = q[2]; N[3] = 1.0 - q[0] - q[1] - q[2];
  } else {
    for (int a = 0; a < 8; ++a)
      N[a] = (1.0 / 8.0) * (1.0 + q[0] * H_c1[a]) * (1.0 + q[1] * H_c2[a]) * (1.0 + q[2] * H_c3[a]);
  }
}

/* femTetra4.cpp:304-330, femHexa8.cpp:28-42 */
static void local_deriv(int npe, const double* q, double dN[8][3]) {
  if (npe == 4) {
    static const double t[4][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}, {-1.0, -1.0, -1.0}};
    for (int a = 0; a < 4; ++a)
      for (int k = 0; k < 3; ++k) dN[a][k] = t[a][k];
  } else {
    for (int a = 0; a < 8; ++a) {
      dN[a][0] = (1.0 / 8.0) * H_c1[a] * (1.0 + q[1] * H_c2[a]) * (1.0 + q[2] * H_c3[a]);
      dN[a][1] = (1.0 / 8.0) * H_c2[a] * (1.0 + q[0] * H_c1[a]) * (1.0 + q[2] * H_c3[a]);
      dN[a][2] = (1.0 / 8.0) * H_c3[a] * (1.0 + q[0] * H_c1[a]) * (1.0 + q[1] * H_c2[a]);
    }
  }
}

/* femUtils.cpp:716-770 */
static void invert3x3(const double m[3][3], double inv[3][3], double* det) {
  double m00 = m[0][0], m01 = m[0][1], m02 = m[0][2];
  double m10 = m[1][0], m11 = m[1][1], m12 = m[1][2];
  double m20 = m[2][0], m21 = m[2][1], m22 = m[2][2];
  *det = m00 * (m11 * m22 - m21 * m12) - m01 * (m10 * m22 - m12 * m20) + m02 * (m10 * m21 - m11 * m20);
  double invdet = 1 / *det;
  inv[0][0] = (m11 * m22 - m21 * m12) * invdet;
  inv[0][1] = (m02 * m21 - m01 * m22) * invdet;
  inv[0][2] = (m01 * m12 - m02 * m11) * invdet;
  inv[1][0] = (m12 * m20 - m10 * m22) * invdet;
  inv[1][1] = (m00 * m22 - m02 * m20) * invdet;
  inv[1][2] = (m10 * m02 - m00 * m12) * invdet;
  inv[2][0] = (m10 * m21 - m20 * m11) * invdet;
  inv[2][1] = (m20 * m01 - m00 * m21) * invdet;
  inv[2][2] = (m00 * m11 - m10 * m01) * invdet;
}

/* femElement.cpp:104-127 + 272-354 (+192-232 for G) */
static void global_deriv(int npe, const double xe[8][3], const double* q, double* detJ, double gd[8][3], double G[3][3]) {
  double dN[8][3], J[3][3], inv[3][3];
  local_deriv(npe, q, dN);
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double t = 0.0;
      for (int n = 0; n < npe; ++n) t += dN[n][a] * xe[n][b];
      J[a][b] = t;
    }
  invert3x3(J, inv, detJ);
  for (int n = 0; n < npe; ++n)
    for (int b = 0; b < 3; ++b) {
      gd[n][b] = 0.0;
      for (int c = 0; c < 3; ++c) gd[n][b] += inv[b][c] * dN[n][c];
    }
  if (G)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        G[a][b] = 0.0;
        for (int c = 0; c < 3; ++c) G[a][b] += inv[c][a] * inv[c][b];
      }
}

/* ------------------------------------------------------------------ */
/* Poisson (femPoissonSolver::solve, femSolver.cpp:409-654): element   */
/* matrices and sources of its Gauss loops, and the wall distance.     */
/* ------------------------------------------------------------------ */
static void poisson_coords(int npe, const double* x, const int32_t* conn, int64_t e, double xe[8][3]) {
  for (int a = 0; a < npe; ++a)
    for (int k = 0; k < 3; ++k) xe[a][k] = x[(int64_t)conn[e * npe + a] * 3 + k];
}

/* femModel::FixedElementConnectivities (femModel.cpp:3554-3569), which the
 * Poisson driver runs after reading the model (main.cpp:491): an element
 * whose smallest Jacobian determinant over the irSecondOrder points
 * (femElement::checkMinDetJ, femElement.cpp:63-81) is <= 0 gets one swap,
 * tet4 nodes 0 and 1 (femTetra4.cpp:160-170), hexa8 nodes 2 / 3 and 6 / 7
 * (femHexa8.cpp:93-103).  conn is modified in place; returns the count. */
int64_t fmo_poisson_fix(int npe, int64_t E, const double* x, int32_t* conn) {
  int ngp;
  double gps[8][3], gpw[8];
  int64_t fixed = 0;
  gauss_rule(npe, &ngp, gps, gpw);
  for (int64_t e = 0; e < E; ++e) {
    double xe[8][3], gd[8][3], detJ, mn = 1e308;
    poisson_coords(npe, x, conn, e, xe);
    for (int g = 0; g < ngp; ++g) {
      global_deriv(npe, xe, gps[g], &detJ, gd, NULL);
      if (detJ < mn) mn = detJ;
    }
    if (mn <= 0.0) {
      int32_t* c = conn + e * npe;
      int32_t t;
      if (npe == 4) {
        t = c[1]; c[1] = c[0]; c[0] = t;
      } else {
        t = c[2]; c[2] = c[3]; c[3] = t;
        t = c[6]; c[6] = c[7]; c[7] = t;
      }
      ++fixed;
    }
  }
  return fixed;
}

/* femElement::formPoissonMatrix (femElement.cpp:903-944), irSecondOrder
 * rule, for elements [0, E): Ke[e][a][b] (npe x npe each). */
void fmo_poisson_elements(int npe, int64_t E, const double* x, const int32_t* conn, const double* diff, double* Ke) {
  int ngp;
  double gps[8][3], gpw[8];
  gauss_rule(npe, &ngp, gps, gpw);
  for (int64_t e = 0; e < E; ++e) {
    double xe[8][3], gd[8][3], detJ;
    double* K = Ke + e * npe * npe;
    poisson_coords(npe, x, conn, e, xe);
    for (int a = 0; a < npe * npe; ++a) K[a] = 0.0;
    for (int g = 0; g < ngp; ++g) {
      global_deriv(npe, xe, gps[g], &detJ, gd, NULL);
      for (int a = 0; a < npe; ++a)
        for (int b = 0; b < npe; ++b) {
          double st = 0.0;
          for (int d = 0; d < 3; ++d) st += diff[e * 3 + d] * gd[a][d] * gd[b][d];
          K[a * npe + b] += st * detJ * gpw[g];
        }
    }
  }
}

/* femElement::formPoissonSource (femElement.cpp:949-981): f[a] of element e
 * with source value `value` (detJ as femElement::evalJacobian,
 * femElement.cpp:149-186). */
void fmo_poisson_source(int npe, const double* x, const int32_t* conn, int64_t e, double value, double* f) {
  int ngp;
  double gps[8][3], gpw[8], xe[8][3], gd[8][3], N[8], detJ;
  gauss_rule(npe, &ngp, gps, gpw);
  poisson_coords(npe, x, conn, e, xe);
  for (int a = 0; a < npe; ++a) f[a] = 0.0;
  for (int g = 0; g < ngp; ++g) {
    shape_fn(npe, gps[g], N);
    global_deriv(npe, xe, gps[g], &detJ, gd, NULL);
    for (int a = 0; a < npe; ++a) f[a] += N[a] * value * detJ * gpw[g];
  }
}

/* fmo_poisson_source for every ELSOURCE row k (element elems[k], value
 * values[k]): out[k][a]. */
void fmo_poisson_sources(int npe, const double* x, const int32_t* conn, int64_t n, const int32_t* elems,
                         const double* values, double* out) {
  for (int64_t k = 0; k < n; ++k) fmo_poisson_source(npe, x, conn, elems[k], values[k], out + k * npe);
}

/* evalDistanceFromPoissonSolution (femSolver.cpp:366-403): per element the
 * solution and its gradient at local coordinates (0, 0, 0). */
void fmo_poisson_distance(int npe, int64_t E, const double* x, const int32_t* conn, const double* sol, double* dist) {
  const double q0[3] = {0.0, 0.0, 0.0};
  for (int64_t e = 0; e < E; ++e) {
    double xe[8][3], gd[8][3], N[8], detJ, phi = 0.0, g[3] = {0.0, 0.0, 0.0};
    poisson_coords(npe, x, conn, e, xe);
    shape_fn(npe, q0, N);
    global_deriv(npe, xe, q0, &detJ, gd, NULL);
    for (int a = 0; a < npe; ++a) {
      const double u = sol[conn[e * npe + a]];
      phi += N[a] * u;
      g[0] += gd[a][0] * u;
      g[1] += gd[a][1] * u;
      g[2] += gd[a][2] * u;
    }
    dist[e] = -sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]) + sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2] + 2.0 * phi);
  }
}

static void elem_coords(fmo_ctx* c, int64_t e, double xe[8][3]) {
  for (int a = 0; a < c->npe; ++a)
    for (int k = 0; k < 3; ++k) xe[a][k] = c->x[(int64_t)c->conn[e * c->npe + a] * 3 + k];
}

/* ------------------------------------------------------------------ */
/* SUPG                                                                */
/* ------------------------------------------------------------------ */
/* femSUPGExplicitFluidSolver.cpp:507-598 */
static void supg_lumped_mass_range(fmo_ctx* c, int64_t eb, int64_t ee) {
  double rho = c->props[0];
  int npe = c->npe, nd = npe * 3;
  int ngp;
  double gps[8][3], gpw[8];
  gauss_rule(npe, &ngp, gps, gpw);
  double BM[24][24];
  for (int64_t e = eb; e < ee; ++e) {
    double xe[8][3];
    elem_coords(c, e, xe);
    for (int a = 0; a < nd; ++a)
      for (int b = 0; b < nd; ++b) BM[a][b] = 0.0;
    for (int g = 0; g < ngp; ++g) {
      double N[8], gd[8][3], detJ, L[3][24];
      shape_fn(npe, gps[g], N);
      global_deriv(npe, xe, gps[g], &detJ, gd, NULL);
      for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 24; ++k) L[r][k] = 0.0;
      for (int a = 0; a < npe; ++a) { L[0][a * 3] = N[a]; L[1][a * 3 + 1] = N[a]; L[2][a * 3 + 2] = N[a]; }
      for (int a = 0; a < nd; ++a)
        for (int b = 0; b < nd; ++b) {
          double t = 0.0;
          for (int r = 0; r < 3; ++r) t += rho * L[r][a] * L[r][b] * detJ * gpw[g];
          BM[a][b] += t;
        }
    }
    /* l_M[conn[e][a/3]*3 + a%3] += row sum a: kept per element and summed
       per node in element order (supg_mass_nodes) */
    for (int a = 0; a < nd; ++a) {
      double t = 0.0;
      for (int b = 0; b < nd; ++b) t += BM[a][b];
      c->lres[e * 24 + a] = t;
    }
  }
}

static void supg_mass_nodes(fmo_ctx* c, int64_t b, int64_t e) {
  int npe = c->npe;
  for (int64_t n = b; n < e; ++n) {
    double acc[3] = {0.0, 0.0, 0.0};
    for (int64_t j = c->inc_off[n]; j < c->inc_off[n + 1]; ++j) {
      int64_t q = c->inc_ent[j];
      const double* r = c->lres + (q / npe) * 24 + (q % npe) * 3;
      for (int d = 0; d < 3; ++d) acc[d] += r[d];
    }
    for (int d = 0; d < 3; ++d) c->l_M[n * 3 + d] = acc[d];
  }
}

static void supg_lumped_mass(fmo_ctx* c) {
  par_for(c, c->E, supg_lumped_mass_range);
  par_for(c, c->N, supg_mass_nodes);
}

/* femSUPGExplicitFluidSolver.cpp:446-501 */
static void supg_pressure_range(fmo_ctx* c, int64_t eb, int64_t ee) {
  const double* sol = c->pres_src;
  int npe = c->npe;
  int ngp;
  double gps[8][3], gpw[8];
  gauss_rule(npe, &ngp, gps, gpw);
  for (int64_t e = eb; e < ee; ++e) {
    double xe[8][3], es[24];
    elem_coords(c, e, xe);
    for (int a = 0; a < npe; ++a)
      for (int k = 0; k < 3; ++k) es[a * 3 + k] = sol[(int64_t)c->conn[e * npe + a] * 3 + k];
    double num = 0.0, den = 0.0;
    for (int g = 0; g < ngp; ++g) {
      double gd[8][3], detJ;
      global_deriv(npe, xe, gps[g], &detJ, gd, NULL);
      double div = 0.0;
      for (int k = 0; k < npe * 3; ++k) div += gd[k / 3][k % 3] * es[k];
      num += div * detJ * gpw[g];
      den += detJ * gpw[g];
    }
    c->pres_n[e] = -c->el_lam[e] * (num / den);
  }
}

static void supg_compute_pressure(fmo_ctx* c, const double* sol) {
  c->pres_src = sol;
  par_for(c, c->E, supg_pressure_range);
}

/* femSUPGExplicitFluidSolver.cpp:660-707 (hexa8 only; tet4 reads out of
   bounds in the reference, so B-bar is rejected for tet4 by the caller). */
static void supg_avg_shape_deriv(fmo_ctx* c, const double xe[8][3], double avg[8][3]) {
  int ngp;
  double gps[8][3], gpw[8], den[8][3];
  gauss_rule(c->npe, &ngp, gps, gpw);
  for (int a = 0; a < 8; ++a)
    for (int b = 0; b < 3; ++b) { avg[a][b] = 0.0; den[a][b] = 0.0; }
  for (int g = 0; g < ngp; ++g) {
    double gd[8][3], detJ;
    global_deriv(c->npe, xe, gps[g], &detJ, gd, NULL);
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 3; ++b) {
        avg[a][b] += gd[a][b] * detJ * gpw[g];
        den[a][b] += detJ * gpw[g];
      }
  }
  for (int a = 0; a < 8; ++a)
    for (int b = 0; b < 3; ++b) avg[a][b] = avg[a][b] / den[a][b];
}

/* The element loop of femSUPGExplicitFluidSolver::solve (src lines
   1095-1472) over elements [eb, ee): k_p, el_lam, el_regime. */
static void supg_element_range(fmo_ctx* c, int64_t eb, int64_t ee) {
  int64_t E = c->E;
  int npe = c->npe, nd = npe * 3;
  double rho = c->props[0], mu = c->props[1], alpha = c->props[2], cI = c->props[3];
  int use_B_hat = c->ex_opts[1];
  int iK1 = c->ex_opts[2], iK2 = c->ex_opts[3], iK3 = c->ex_opts[4], iK4 = c->ex_opts[5];
  double dt = c->dt;
  int ngp;
  double gps[8][3], gpw[8];
  gauss_rule(npe, &ngp, gps, gpw);
  double K1[24][24], K2[24][24], K3[24][24], K4[24][24], K[24][24];
  for (int64_t e = eb; e < ee; ++e) {
    double xe[8][3], es[24], sd0[8][3];
    elem_coords(c, e, xe);
    for (int a = 0; a < npe; ++a)
      for (int k = 0; k < 3; ++k) es[a * 3 + k] = c->sol_p[(int64_t)c->conn[e * npe + a] * 3 + k];
    for (int a = 0; a < nd; ++a)
      for (int b = 0; b < nd; ++b) { K1[a][b] = 0.0; K2[a][b] = 0.0; K3[a][b] = 0.0; K4[a][b] = 0.0; }
    if (use_B_hat) supg_avg_shape_deriv(c, xe, sd0);
    double el_volume = 0.0;
    c->el_lam[e] = 0.0;
    c->el_regime[e] = 0.0;
    for (int g = 0; g < ngp; ++g) {
      double Nf[8], gd[8][3], G[3][3], detJ, u[3] = {0.0, 0.0, 0.0};
      shape_fn(npe, gps[g], Nf);
      for (int a = 0; a < npe; ++a) {
        u[0] += Nf[a] * es[a * 3 + 0];
        u[1] += Nf[a] * es[a * 3 + 1];
        u[2] += Nf[a] * es[a * 3 + 2];
      }
      global_deriv(npe, xe, gps[g], &detJ, gd, G);
      el_volume += detJ * gpw[g];
      /* eval_stabilization, src lines 336-377 */
      double trG = G[0][0] + G[1][1] + G[2][2];
      double t2 = 0.0;
      for (int a = 0; a < 3; ++a) {
        double tmp = 0.0;
        for (int b = 0; b < 3; ++b) tmp += G[a][b] * u[b];
        t2 += u[a] * tmp;
      }
      double t3 = 0.0;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) t3 += G[a][b] * G[a][b];
      t3 = t3 * (mu / rho) * (mu / rho) * cI;
      double tau = 1.0 / sqrt(t2 + t3);
      double nuC = 1.0 / (trG * tau);
      /* eval_bulk_modulus, src lines 382-441 */
      double iG[3][3], dG, iGu[3];
      invert3x3(G, iG, &dG);
      double lim1 = (mu / rho);
      for (int a = 0; a < 3; ++a) {
        iGu[a] = 0.0;
        for (int b = 0; b < 3; ++b) iGu[a] += iG[a][b] * u[b];
      }
      double lim2 = 0.0;
      for (int a = 0; a < 3; ++a) lim2 += iGu[a] * u[a];
      lim2 = sqrt(lim2);
      double lam = alpha * ((lim1 < lim2) ? lim2 : lim1); /* std::max(limit_1, limit_2) */
      double regime = (lim1 > lim2) ? 1 : 2;
      c->el_lam[e] += lam * detJ * gpw[g];
      c->el_regime[e] += regime;
      /* L, U, S, US, B, D, DB, H (src lines 138-331, 1247-1303) */
      double L[3][24], US[3][24], B[6][24], D[6][6], DB[6][24], H[24];
      for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 24; ++k) { L[r][k] = 0.0; US[r][k] = 0.0; }
      for (int a = 0; a < npe; ++a) { L[0][a * 3] = Nf[a]; L[1][a * 3 + 1] = Nf[a]; L[2][a * 3 + 2] = Nf[a]; }
      {
        double U[3][9], S[9][24];
        for (int r = 0; r < 3; ++r)
          for (int k = 0; k < 9; ++k) U[r][k] = 0.0;
        U[0][0] = u[0]; U[0][1] = u[1]; U[0][2] = u[2];
        U[1][3] = u[0]; U[1][4] = u[1]; U[1][5] = u[2];
        U[2][6] = u[0]; U[2][7] = u[1]; U[2][8] = u[2];
        for (int r = 0; r < 9; ++r)
          for (int k = 0; k < 24; ++k) S[r][k] = 0.0;
        for (int a = 0; a < npe; ++a)
          for (int d = 0; d < 3; ++d) {
            S[0 + d][a * 3 + 0] = gd[a][d];
            S[3 + d][a * 3 + 1] = gd[a][d];
            S[6 + d][a * 3 + 2] = gd[a][d];
          }
        for (int r = 0; r < 3; ++r)
          for (int k = 0; k < nd; ++k) {
            double t = 0.0;
            for (int m = 0; m < 9; ++m) t += U[r][m] * S[m][k];
            US[r][k] = t;
          }
      }
      for (int r = 0; r < 6; ++r)
        for (int k = 0; k < 24; ++k) B[r][k] = 0.0;
      for (int a = 0; a < npe; ++a) {
        if (use_B_hat) {
          double B1 = (1.0 / 3.0) * (sd0[a][0] - gd[a][0]);
          double B2 = gd[a][0] - B1;
          double B3 = (1.0 / 3.0) * (sd0[a][1] - gd[a][1]);
          double B4 = gd[a][1] - B3;
          double B5 = (1.0 / 3.0) * (sd0[a][2] - gd[a][2]);
          double B6 = gd[a][2] - B5;
          B[0][a * 3 + 0] = B2; B[0][a * 3 + 1] = B3; B[0][a * 3 + 2] = B5;
          B[1][a * 3 + 0] = B1; B[1][a * 3 + 1] = B4; B[1][a * 3 + 2] = B5;
          B[2][a * 3 + 0] = B1; B[2][a * 3 + 1] = B3; B[2][a * 3 + 2] = B6;
        } else {
          B[0][a * 3 + 0] = gd[a][0];
          B[1][a * 3 + 1] = gd[a][1];
          B[2][a * 3 + 2] = gd[a][2];
        }
        B[3][a * 3 + 0] = gd[a][1]; B[3][a * 3 + 1] = gd[a][0];
        B[4][a * 3 + 1] = gd[a][2]; B[4][a * 3 + 2] = gd[a][1];
        B[5][a * 3 + 0] = gd[a][2]; B[5][a * 3 + 2] = gd[a][0];
      }
      for (int r = 0; r < 6; ++r)
        for (int k = 0; k < 6; ++k) D[r][k] = 0.0;
      D[0][0] = lam + 2 * mu; D[0][1] = lam; D[0][2] = lam;
      D[1][0] = lam; D[1][1] = lam + 2 * mu; D[1][2] = lam;
      D[2][0] = lam; D[2][1] = lam; D[2][2] = lam + 2 * mu;
      D[3][3] = mu; D[4][4] = mu; D[5][5] = mu;
      for (int r = 0; r < 6; ++r)
        for (int k = 0; k < nd; ++k) {
          double t = 0.0;
          for (int m = 0; m < 6; ++m) t += D[r][m] * B[m][k];
          DB[r][k] = t;
        }
      for (int k = 0; k < 24; ++k) H[k] = 0.0;
      for (int a = 0; a < npe; ++a) { H[a * 3] = gd[a][0]; H[a * 3 + 1] = gd[a][1]; H[a * 3 + 2] = gd[a][2]; }
      for (int a = 0; a < nd; ++a)
        for (int b = 0; b < nd; ++b) {
          double t = 0.0;
          for (int r = 0; r < 3; ++r) t += rho * L[r][a] * US[r][b] * detJ * gpw[g];
          K1[a][b] += t;
          t = 0.0;
          for (int r = 0; r < 6; ++r) t += B[r][a] * DB[r][b] * detJ * gpw[g];
          K2[a][b] += t;
          t = 0.0;
          for (int r = 0; r < 3; ++r) t += rho * tau * US[r][a] * US[r][b] * detJ * gpw[g];
          K3[a][b] += t;
          K4[a][b] += rho * nuC * H[a] * H[b] * detJ * gpw[g];
        }
    }
    for (int a = 0; a < nd; ++a)
      for (int b = 0; b < nd; ++b) {
        K[a][b] = 0.0;
        if (iK1) K[a][b] += K1[a][b];
        if (iK2) K[a][b] += K2[a][b];
        if (iK3) K[a][b] += K3[a][b];
        if (iK4) K[a][b] += K4[a][b];
      }
    c->el_lam[e] = (c->el_lam[e] / el_volume);
    c->el_regime[e] = c->el_regime[e] / ngp;
    for (int a = 0; a < nd; ++a) {
      double* kp = c->k_p + (int64_t)a * E + e;
      *kp = 0.0;
      for (int b = 0; b < nd; ++b) *kp += -dt * K[a][b] * es[b];
    }
  }
}

/* The scatter of k_p into solN (src lines 1475-1498: Euler, or AB2 after the
   first step), per node in element order, then the update u^{n+1} = u^n +
   solN / l_M (src lines 1510-1514). */
static void supg_update_nodes(fmo_ctx* c, int64_t b, int64_t e) {
  int64_t E = c->E;
  int npe = c->npe;
  int euler = c->ex_opts[0] || c->step == 1;
  for (int64_t n = b; n < e; ++n) {
    double acc[3] = {0.0, 0.0, 0.0};
    for (int64_t j = c->inc_off[n]; j < c->inc_off[n + 1]; ++j) {
      int64_t q = c->inc_ent[j], el = q / npe;
      int a = (int)(q % npe);
      for (int d = 0; d < 3; ++d) {
        double kp = c->k_p[(int64_t)(a * 3 + d) * E + el];
        if (euler)
          acc[d] += kp;
        else
          acc[d] += (3.0 / 2.0) * kp - (1.0 / 2.0) * c->k_pp[(int64_t)(a * 3 + d) * E + el];
      }
    }
    for (int d = 0; d < 3; ++d) c->solN[n * 3 + d] = c->sol_p[n * 3 + d] + (1.0 / c->l_M[n * 3 + d]) * acc[d];
  }
}

/* One time step of femSUPGExplicitFluidSolver::solve (src lines 1034-1591). */
static void supg_step(fmo_ctx* c) {
  int64_t N = c->N, E = c->E;
  c->step++;
  c->cur_time += c->dt;
  par_for(c, E, supg_element_range);
  par_for(c, N, supg_update_nodes);
  set_node_velocity(c, c->cur_time, c->solN, 3);
  set_dirichlet(c, c->solN, 3);
  supg_compute_pressure(c, c->solN);
  if (c->glob_fixed)
    for (int64_t i = 0; i < N; ++i)
      for (int d = 0; d < 3; ++d)
        if (c->glob_fixed & (1 << d)) c->solN[i * 3 + d] = 0.0;
  memcpy(c->sol_p, c->solN, sizeof(double) * N * 3);
  memcpy(c->k_pp, c->k_p, sizeof(double) * E * 24);
}

/* ------------------------------------------------------------------ */
/* Public interface                                                    */
/* ------------------------------------------------------------------ */
/* Creates a solve and applies the initial BCs exactly as the reference's
   solve() prologue does (VMS: src lines 855-952; SUPG: lines 826-1010).
   init: N x 4 (u, v, w, p) initial values before BCs, or NULL for zeros. */
void* fmo_create(int64_t N, int64_t E, int npe, const double* x, const int32_t* conn, int solver, const double* props,
                 double dt, double ds, int ndual, const int32_t* ex_opts, int glob_fixed, int nvel_rows,
                 const int32_t* vel_node, const double* vel_vals, const int32_t* vel_dir, int ndir, const int32_t* dir_node,
                 const double* dir_vals, int npres, const int32_t* pres_node, const double* pres_vals, const double* init) {
  fmo_ctx* c = (fmo_ctx*)calloc(1, sizeof(fmo_ctx));
  c->N = N; c->E = E; c->npe = npe; c->x = x; c->conn = conn; c->solver = solver;
  for (int i = 0; i < 5; ++i) c->props[i] = props[i];
  c->dt = dt; c->ds = ds; c->ndual = ndual;
  for (int i = 0; i < 6; ++i) c->ex_opts[i] = ex_opts ? ex_opts[i] : 0;
  c->glob_fixed = glob_fixed;
  build_vel_tables(c, nvel_rows, vel_node, vel_vals, vel_dir);
  c->ndir = ndir; c->dir_node = (int32_t*)malloc(sizeof(int32_t) * (ndir + 1)); c->dir_vals = (double*)malloc(sizeof(double) * (3 * ndir + 1));
  memcpy(c->dir_node, dir_node, sizeof(int32_t) * ndir); memcpy(c->dir_vals, dir_vals, sizeof(double) * 3 * ndir);
  c->npres = npres; c->pres_node = (int32_t*)malloc(sizeof(int32_t) * (npres + 1)); c->pres_vals = (double*)malloc(sizeof(double) * (npres + 1));
  memcpy(c->pres_node, pres_node, sizeof(int32_t) * npres); memcpy(c->pres_vals, pres_vals, sizeof(double) * npres);
  if (solver == 0) {
    c->sol_n = (double*)calloc(N * 4, sizeof(double));
    c->sol_prev = (double*)calloc(N * 4, sizeof(double));
    c->sol_tau = (double*)calloc(N * 4, sizeof(double));
    c->rhs = (double*)calloc(N * 4, sizeof(double));
    c->sdus = (double*)calloc(E * 12, sizeof(double));
    c->sgps = (double*)calloc(E * 4, sizeof(double));
    c->volumes = (double*)calloc(E, sizeof(double));
    c->DNs = (double*)calloc(E * 12, sizeof(double));
    c->char_length = (double*)calloc(E, sizeof(double));
    c->nd_mass = (double*)calloc(N, sizeof(double));
    c->elmTaus = (double*)calloc(E * 2, sizeof(double));
    c->projRHS = (double*)calloc(E * 16, sizeof(double));
    c->el_u_sdus = (double*)calloc(E * 3, sizeof(double));
    c->lres = (double*)malloc(sizeof(double) * (E * 16 + 1));
    build_incidence(c);
    if (init) memcpy(c->sol_tau, init, sizeof(double) * N * 4);
    set_node_velocity(c, 0.0, c->sol_tau, 4);
    apply_zero_traction(c, c->sol_tau);
    set_dirichlet(c, c->sol_tau, 4);
    memcpy(c->sol_prev, c->sol_tau, sizeof(double) * N * 4);
    memcpy(c->sol_n, c->sol_tau, sizeof(double) * N * 4);
    par_for(c, E, vms_initial_range);
    par_for(c, N, vms_mass_nodes);
  } else {
    c->sol_p = (double*)calloc(N * 3, sizeof(double));
    c->solN = (double*)calloc(N * 3, sizeof(double));
    c->l_M = (double*)calloc(N * 3, sizeof(double));
    c->k_p = (double*)calloc(E * 24, sizeof(double));
    c->k_pp = (double*)calloc(E * 24, sizeof(double));
    c->el_lam = (double*)calloc(E, sizeof(double));
    c->el_regime = (double*)calloc(E, sizeof(double));
    c->pres_n = (double*)calloc(E, sizeof(double));
    c->lres = (double*)malloc(sizeof(double) * (E * 24 + 1));
    build_incidence(c);
    if (init)
      for (int64_t i = 0; i < N; ++i)
        for (int d = 0; d < 3; ++d) c->sol_p[i * 3 + d] = init[i * 4 + d];
    set_node_velocity(c, 0.0, c->sol_p, 3);
    set_dirichlet(c, c->sol_p, 3);
    supg_compute_pressure(c, c->sol_p);
    supg_lumped_mass(c);
  }
  return c;
}

int fmo_step(void* h, int nsteps) {
  fmo_ctx* c = (fmo_ctx*)h;
  for (int s = 0; s < nsteps && !c->err; ++s) {
    if (c->solver == 0) vms_step(c); else supg_step(c);
  }
  return c->err;
}

/* state: N x 4 (VMS: sol_n after the step = u, v, w, p; SUPG: u, v, w, 0).
   elem: VMS -> E x 3 centroid subgrid velocity read in the last pass;
         SUPG -> E x 3 (pressure, lambda, regime). */
int fmo_get(void* h, double* state, double* elem, double* sdus, double* time_out) {
  fmo_ctx* c = (fmo_ctx*)h;
  int64_t N = c->N, E = c->E;
  if (c->solver == 0) {
    if (state) memcpy(state, c->sol_n, sizeof(double) * N * 4);
    if (elem) memcpy(elem, c->el_u_sdus, sizeof(double) * E * 3);
    if (sdus) memcpy(sdus, c->sdus, sizeof(double) * E * 12);
  } else {
    if (state)
      for (int64_t i = 0; i < N; ++i) {
        for (int d = 0; d < 3; ++d) state[i * 4 + d] = c->sol_p[i * 3 + d];
        state[i * 4 + 3] = 0.0;
      }
    if (elem)
      for (int64_t e = 0; e < E; ++e) {
        elem[e * 3 + 0] = c->pres_n[e];
        elem[e * 3 + 1] = c->el_lam[e];
        elem[e * 3 + 2] = c->el_regime[e];
      }
    if (sdus) memcpy(sdus, c->l_M, sizeof(double) * N * 3);
  }
  if (time_out) *time_out = c->cur_time;
  return c->err;
}

/* VMS: the state before the last BC application (sol_prev after
   update_solution), N x 4. */
int fmo_get_prebc(void* h, double* state) {
  fmo_ctx* c = (fmo_ctx*)h;
  if (c->solver != 0) return FMO_ERR_INVALID;
  memcpy(state, c->sol_prev, sizeof(double) * c->N * 4);
  return 0;
}

void fmo_destroy(void* h) {
  fmo_ctx* c = (fmo_ctx*)h;
  if (!c) return;
  void* ptrs[] = {c->vel_node, c->vel_off, c->vel_len, c->vel_tab, c->vel_dir, c->dir_node, c->dir_vals, c->pres_node,
                  c->pres_vals, c->sol_n, c->sol_prev, c->sol_tau, c->rhs, c->sdus, c->sgps, c->volumes, c->DNs,
                  c->char_length, c->nd_mass, c->elmTaus, c->projRHS, c->el_u_sdus, c->sol_p, c->solN, c->l_M,
                  c->k_p, c->k_pp, c->el_lam, c->el_regime, c->pres_n, c->inc_off, c->inc_ent, c->lres};
  for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); ++i) free(ptrs[i]);
  free(c);
}
