// femSolver adapters: feMorph's explicit flow solvers on a B200.
#include "femExplicitFluidSolverGPU.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <string>
#include <vector>

#include "femException.h"
#include "femResult.h"
#include "femUtils.h"
#include "femorph_b200.h"

namespace {

struct ModelArrays {
  int32_t etype = 0;
  std::vector<double> coords, vel_vals, dir_vals, pres_vals;
  std::vector<int32_t> conn, vel_node, vel_dir, dir_node, pres_node;
};

void fm_check(int rc) {
  if (rc != FM_OK) throw femException((std::string("femorph_b200: ") + fm_strerror(rc) + ": " + fm_last_error_message() + "\n").c_str());
}

// femModel -> plain arrays.  NODEVEL rows are re-emitted grouped by node in
// each node's table order (velNodesTimeVals, femModel.cpp:4549-4576); the
// per-row direction list velNodesDir is passed as is, so the library applies
// the same direction to the k-th unique node as the reference does.
void gather(femModel* m, ModelArrays& a) {
  const size_t N = m->nodeList.size(), E = m->elementList.size();
  a.coords.resize(N * 3);
  for (size_t i = 0; i < N; ++i)
    for (int k = 0; k < 3; ++k) a.coords[i * 3 + k] = m->nodeList[i]->coords[k];
  for (size_t e = 0; e < E; ++e) {
    const std::vector<int>& c = m->elementList[e]->elementConnections;
    if (a.etype == 0) a.etype = (int32_t)c.size();
    if ((int32_t)c.size() != a.etype || (a.etype != 4 && a.etype != 8))
      throw femException("femorph_b200: explicit flow needs a mesh of only TET4 or only HEXA8 elements.\n");
    for (int v : c) a.conn.push_back(v);
  }
  for (size_t k = 0; k < m->velNodesID.size(); ++k)
    for (const femDoubleVec& row : m->velNodesTimeVals[k]) {
      a.vel_node.push_back(m->velNodesID[k]);
      for (int c = 0; c < 4; ++c) a.vel_vals.push_back(row[c]);
    }
  for (int d : m->velNodesDir) a.vel_dir.push_back(d);
  a.vel_dir.resize(a.vel_node.size(), 6);
  for (size_t k = 0; k < m->diricheletBCNode.size(); ++k) {
    a.dir_node.push_back(m->diricheletBCNode[k]);
    const femDoubleVec& v = m->diricheletBCValues[k];
    for (int c = 0; c < 3; ++c) a.dir_vals.push_back(c < (int)v.size() ? v[c] : 0.0);
  }
  for (size_t k = 0; k < m->presNodesID.size(); ++k) {
    a.pres_node.push_back(m->presNodesID[k]);
    a.pres_vals.push_back(m->presNodesValue[k]);
  }
}

void fill(const ModelArrays& a, femModel* m, fm_mesh& mesh, fm_bc& bc) {
  mesh.elem_type = a.etype;
  mesh.n_nodes = (int64_t)m->nodeList.size();
  mesh.n_elems = (int64_t)m->elementList.size();
  mesh.coords = a.coords.data();
  mesh.conn = a.conn.data();
  bc.n_vel_rows = (int64_t)a.vel_node.size();
  bc.vel_node = a.vel_node.data();
  bc.vel_vals = a.vel_vals.data();
  bc.vel_dir = a.vel_dir.data();
  bc.n_dir = (int64_t)a.dir_node.size();
  bc.dir_node = a.dir_node.data();
  bc.dir_vals = a.dir_vals.data();
  bc.n_pres = (int64_t)a.pres_node.size();
  bc.pres_node = a.pres_node.data();
  bc.pres_vals = a.pres_vals.data();
}

// The reference's save counter (femVMSExplicitFluidSolver.cpp:1237,1332;
// femSUPGExplicitFluidSolver.cpp:1648,1733) saves steps s+1, 2s+1, ... and,
// for s = 0, step 1 only.
bool is_save_step(long step, long s) { return s == 0 ? step == 1 : (step >= s + 1 && (step - 1) % s == 0); }

femResult* make_result(const char* label, femResultType type, int nc, const double* v, size_t n, size_t stride) {
  femResult* r = new femResult();
  r->label = label;
  r->type = type;
  r->numComponents = nc;
  for (size_t i = 0; i < n; ++i) {
    femDoubleVec row;
    for (int c = 0; c < nc; ++c) row.push_back(v ? v[i * stride + c] : 0.0);
    r->values.push_back(row);
  }
  return r;
}

struct Session {
  fm_problem* p = nullptr;
  fm_batch* b = nullptr;
  ~Session() {
    if (b) fm_batch_destroy(b);
    if (p) fm_problem_destroy(p);
  }
};

}  // namespace

femVMSExplicitFluidSolverGPU::femVMSExplicitFluidSolverGPU(int device, bool mixed, bool log)
    : device_(device), mixed_(mixed), log_(log) {}

namespace {
// Prints the queued diagnostics rows as the reference's log lines
// (src/femVMSExplicitFluidSolver.cpp:1215).  Its time loop counts steps from
// 1 (:1025), so the header it guards with loopTime == 0 (:1211-1214) is
// never printed, and neither is it here.
void print_vms_log(fm_problem* p) {
  int32_t n = 0;
  fm_check(fm_problem_vms_log(p, nullptr, 0, &n));
  std::vector<double> rows((size_t)n * 6);
  if (n > 0) fm_check(fm_problem_vms_log(p, rows.data(), n, &n));
  for (int32_t i = 0; i < n; ++i) {
    const double* r = &rows[(size_t)i * 6];
    printf("%4d.%-4d %20.8f %20.3e %20.3e %10.3f\n", (int)r[0] + 1, (int)r[1], r[2], r[3], r[4], r[5]);
  }
}
}  // namespace

// femVMSExplicitFluidSolver::solve (src/femVMSExplicitFluidSolver.cpp:842-1334).
void femVMSExplicitFluidSolverGPU::solve(femModel* model) {
  ModelArrays a;
  gather(model, a);
  if (a.etype != 4) throw femException("femorph_b200: the VMS solver is tet4-only.\n");
  fm_mesh mesh;
  fm_bc bc;
  fill(a, model, mesh, bc);
  fm_params prm = {};
  prm.solver = FM_SOLVER_VMS;
  prm.precision = mixed_ ? FM_MIXED : FM_FP64;
  for (int i = 0; i < 5 && i < (int)model->vmsProps.size(); ++i) prm.props[i] = model->vmsProps[i];
  prm.time_step = model->timeStep;
  prm.total_steps = model->totalSteps;
  prm.save_every = model->saveEvery;
  prm.dual_step = model->dual_step;
  prm.tot_dual_steps = model->tot_dual_steps;
  Session s;
  fm_check(fm_problem_create(&mesh, &bc, &prm, nullptr, &s.p));
  fm_check(fm_batch_create(&s.p, 1, nullptr, device_, &s.b));
  if (log_) fm_check(fm_batch_set_diagnostics(s.b, 1));
  const size_t N = (size_t)mesh.n_nodes, E = (size_t)mesh.n_elems;
  std::vector<double> u(N * 3), pr(N), sg(E * 3), ru(log_ ? E * 3 : 0), rp(log_ ? E : 0);
  fm_check(fm_problem_get_state(s.p, u.data(), pr.data(), nullptr, nullptr));
  model->resultList.push_back(make_result("velocity", frNode, 3, u.data(), N, 3));
  model->resultList.push_back(make_result("pressure", frNode, 1, pr.data(), N, 1));
  model->ExportToVTKLegacy(std::string("out_Step_" + femUtils::intToStr(0) + ".vtk"), false);
  const long steps = (long)model->totalSteps - 1;
  long done = 0;
  while (done < steps) {
    long next = done + 1;
    while (next < steps && !is_save_step(next, model->saveEvery)) ++next;
    fm_check(fm_batch_step(s.b, (int32_t)(next - done), nullptr));
    fm_check(fm_batch_sync(s.b));
    if (log_) print_vms_log(s.p);
    done = next;
    if (is_save_step(done, model->saveEvery)) {
      fm_check(fm_problem_get_state(s.p, u.data(), pr.data(), sg.data(), nullptr));
      if (log_) fm_check(fm_problem_vms_residuals(s.p, ru.data(), rp.data()));
      model->resultList.clear();
      model->resultList.push_back(make_result("velocity", frNode, 3, u.data(), N, 3));
      model->resultList.push_back(make_result("pressure", frNode, 1, pr.data(), N, 1));
      // res_v / res_p: centroid averages of the partially assembled residual
      // of the last dual iteration (zero without the diagnostics)
      model->resultList.push_back(make_result("res_v", frElement, 3, log_ ? ru.data() : nullptr, E, 3));
      model->resultList.push_back(make_result("res_p", frElement, 1, log_ ? rp.data() : nullptr, E, 1));
      model->resultList.push_back(make_result("subgrid_u", frElement, 3, sg.data(), E, 3));
      model->resultList.push_back(make_result("subgrid_p", frElement, 1, nullptr, E, 1));
      model->ExportToVTKLegacy(std::string("out_Step_" + femUtils::intToStr(done) + ".vtk"), false);
    }
  }
}

femSUPGExplicitFluidSolverGPU::femSUPGExplicitFluidSolverGPU(int device, bool mixed) : device_(device), mixed_(mixed) {}

// femSUPGExplicitFluidSolver::solve (src/femSUPGExplicitFluidSolver.cpp:794-1735).
void femSUPGExplicitFluidSolverGPU::solve(femModel* model) {
  if (model->exOpts.size() < 6) throw femException("femorph_b200: EXOPTS is required by the SUPG solver.\n");
  ModelArrays a;
  gather(model, a);
  fm_mesh mesh;
  fm_bc bc;
  fill(a, model, mesh, bc);
  fm_params prm = {};
  prm.solver = FM_SOLVER_SUPG;
  prm.precision = mixed_ ? FM_MIXED : FM_FP64;
  for (int i = 0; i < 5 && i < (int)model->vmsProps.size(); ++i) prm.props[i] = model->vmsProps[i];
  prm.time_step = model->timeStep;
  prm.total_steps = model->totalSteps;
  prm.save_every = model->saveEvery;
  for (int i = 0; i < 6; ++i) prm.ex_opts[i] = model->exOpts[i] != 0.0;
  const std::string& g = model->glob_fixed_dofs;
  if (g == "NONE") prm.glob_fixed = FM_FIX_NONE;
  else if (g == "X") prm.glob_fixed = FM_FIX_X;
  else if (g == "Y") prm.glob_fixed = FM_FIX_Y;
  else if (g == "Z") prm.glob_fixed = FM_FIX_Z;
  else if (g == "XY") prm.glob_fixed = FM_FIX_X | FM_FIX_Y;
  else if (g == "YZ") prm.glob_fixed = FM_FIX_Y | FM_FIX_Z;
  else if (g == "XZ") prm.glob_fixed = FM_FIX_X | FM_FIX_Z;
  else {
    printf("ERROR: Invalid global fixed DOFs string.\n");
    exit(-1);
  }
  prm.exit_condition = model->exit_condition;
  Session s;
  fm_check(fm_problem_create(&mesh, &bc, &prm, nullptr, &s.p));
  fm_check(fm_batch_create(&s.p, 1, nullptr, device_, &s.b));
  const size_t N = (size_t)mesh.n_nodes, E = (size_t)mesh.n_elems;
  std::vector<double> u(N * 3), pe(E), lr(E * 2);
  fm_check(fm_problem_get_state(s.p, u.data(), pe.data(), nullptr, nullptr));
  model->resultList.push_back(make_result("velocity", frNode, 3, u.data(), N, 3));
  model->resultList.push_back(make_result("pressure", frElement, 1, pe.data(), E, 1));
  model->ExportToVTKLegacy(std::string(model->sol_file_prefix + "_" + femUtils::intToStr(0) + ".vtk"), false);
  FILE* lf = fopen(model->log_file.c_str(), "w");
  if (lf) fclose(lf);
  const long steps = (long)model->totalSteps - 1;
  double t = 0.0;
  double l_cfl_max = 0.0;  // the reference never resets it between steps (src line 996)
  for (long step = 1; step <= steps; ++step) {
    t += model->timeStep;
    // Gauss-point log quantities of the state this step starts from, as the
    // reference's element loop accumulates them (src lines 1066-1459), and
    // the velocity extrema after the step (get_solution_extrema, src lines
    // 604-655): both reduced on the device
    double st[11], ex[7];
    fm_check(fm_problem_supg_log_stats(s.p, st));
    fm_check(fm_batch_step(s.b, 1, nullptr));
    int rc = fm_batch_sync(s.b);
    if (rc != FM_OK && rc != FM_ERR_DIVERGED) fm_check(rc);
    fm_check(fm_problem_velocity_extrema(s.p, ex));
    if (st[6] > l_cfl_max) l_cfl_max = st[6];
    FILE* f = fopen(model->log_file.c_str(), "a");
    if (f) {
      if (step == 1 || step % 10 == 0)
        fprintf(f, "%5s %10s %10s %10s %10s %10s %10s %10s %10s %10s %10s %10s %10s %10s %10s %10s %10s %10s %10s\n",
                "IT", "Time", "min X", "max X", "min Y", "max Y", "min Z", "max Z", "min tau", "max tau", "min lambda",
                "max lambda", "CFL v", "CFL a", "CFL l", "E_min", "E_max", "nu_min", "nu_max");
      fprintf(f,
              "%5ld %10.3e %10.3e %10.3e %10.3e %10.3e %10.3e %10.3e %10.3e %10.3e %10.3e %10.3e %10.3f %10.3f %10.3f "
              "%10.3e %10.3e %10.3e %10.3e\n",
              step, t, ex[0], ex[1], ex[2], ex[3], ex[4], ex[5], st[0], st[1], st[2], st[3], st[4], st[5], l_cfl_max,
              st[7], st[8], st[9], st[10]);
      fclose(f);
    }
    if (rc == FM_ERR_DIVERGED || ex[6] > model->exit_condition) {
      FILE* f2 = fopen(model->log_file.c_str(), "a");
      if (f2) {
        fprintf(f2, "ERROR: Maximum velocity module larger than admissible threshold.\n");
        fprintf(f2, "SOLUTION TERMINATED.\n");
        fclose(f2);
      }
      printf("ERROR: Maximum velocity module larger than admissible threshold.\n");
      printf("SOLUTION TERMINATED.\n");
      exit(-1);
    }
    if (is_save_step(step, model->saveEvery)) {
      fm_check(fm_problem_get_state(s.p, u.data(), pe.data(), lr.data(), nullptr));
      std::vector<double> lam(E), reg(E);
      for (size_t e = 0; e < E; ++e) {
        lam[e] = lr[e * 2];
        reg[e] = lr[e * 2 + 1];
      }
      model->resultList.clear();
      model->resultList.push_back(make_result("velocity", frNode, 3, u.data(), N, 3));
      model->resultList.push_back(make_result("pressure", frElement, 1, pe.data(), E, 1));
      model->resultList.push_back(make_result("lambda", frElement, 1, lam.data(), E, 1));
      model->resultList.push_back(make_result("regime", frElement, 1, reg.data(), E, 1));
      model->ExportToVTKLegacy(std::string(model->sol_file_prefix + "_" + femUtils::intToStr(step) + ".vtk"), false);
    }
  }
}
