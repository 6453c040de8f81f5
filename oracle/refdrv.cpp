// Oracle A driver (test infrastructure only, never part of the product).
//
// Links the unmodified feMorph reference objects and runs its explicit
// solvers exactly as src/main.cpp:788-806 (solveExplicitNS) does:
// femModel::ReadFromFEMTextFile, then femVMSExplicitFluidSolver::solve or
// femSUPGExplicitFluidSolver::solve.  Two femModel members are intercepted
// with GNU ld --wrap (symbols passed in FM_EXPORT_SYM / FM_SETVEL_SYM):
//
//  * femModel::ExportToVTKLegacy (src/femModel.cpp:1294-1530) - the only state
//    the reference emits is 6-digit ASCII VTK, too lossy for 1e-12 parity, so
//    the hook dumps model->resultList as raw FP64 (and forwards to the real
//    writer when --vtk is given).
//  * femModel::setNodeVelocity (src/femModel.cpp:4581-4633) - on its first
//    call (time 0, before the solvers copy the initial state, see
//    src/femVMSExplicitFluidSolver.cpp:883-898 and
//    src/femSUPGExplicitFluidSolver.cpp:891-893) the hook loads a seeded
//    initial state from --ic, because the reference has no initial-condition
//    input for these solvers.  Every call is timestamped for --timing.
//
// Usage: fm_refdrv model.dat vms|supg [--ic f64file ncomp] [--dump dir]
//                  [--vtk] [--timing file]
//        fm_refdrv model.dat poisson-elements --dump dir [--sol f64file]
//        fm_gpudrv model.dat poisson-gpu --dump dir   (drop-in check build)
// The second form reads a Poisson model (src/main.cpp:476-490:
// ReadFromFEMTextFile, FixedElementConnectivities) and writes the reference's
// own element arithmetic of femPoissonSolver::solve: the element matrix of
// femElement::formPoissonMatrix for every element (src/femSolver.cpp:
// 446-459), then the element vector of femElement::formPoissonSource for
// every ELSOURCE row (src/femSolver.cpp:478-494), irSecondOrder rule, as raw
// FP64 in dir/poisson_elements.f64, followed, with --sol, by the wall
// distance evalDistanceFromPoissonSolution (src/femSolver.cpp:367-403)
// computes from that nodal solution.  (The reference solves the system only
// through Trilinos, src/femSolver.cpp:590-600.)
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <unistd.h>

#include "femIntegrationRule.h"
#include "femModel.h"
#include "femVector.h"
#include "femSUPGExplicitFluidSolver.h"
#include "femVMSExplicitFluidSolver.h"
#ifdef FM_WITH_GPU_ADAPTER
// Drop-in check: the same driver with femorph_b200's femSolver adapters
// ("vms-gpu", "supg-gpu"), i.e. the reference's reader and VTK exporter
// around the B200 solver.
#include "femExplicitFluidSolverGPU.h"
#include "femPoissonSolverGPU.h"
#endif

void real_export(femModel*, std::string, bool) __asm__("__real_" FM_EXPORT_SYM);
void real_setvel(femModel*, double, femDoubleMat&) __asm__("__real_" FM_SETVEL_SYM);
void wrap_export(femModel*, std::string, bool) __asm__("__wrap_" FM_EXPORT_SYM);
void wrap_setvel(femModel*, double, femDoubleMat&) __asm__("__wrap_" FM_SETVEL_SYM);

// defined at file scope in src/femSolver.cpp:367-403 (no header declares it)
void evalDistanceFromPoissonSolution(femVector* femSolution, femModel* model, femDoubleVec& cellDistance);

static std::vector<double> g_ic;
static std::vector<double> g_sol;
static int g_ic_ncomp = 0;
static bool g_ic_done = false;
static bool g_dump = false;
static bool g_vtk = false;
static std::string g_dump_dir;
static FILE* g_timing = nullptr;
static double g_last_time = 0.0;
static long g_export_calls = 0;
static std::chrono::steady_clock::time_point g_t0;

void wrap_setvel(femModel* m, double t, femDoubleMat& sol) {
  if (!g_ic_done) {
    g_ic_done = true;
    if (!g_ic.empty()) {
      size_t n = sol.size();
      if (g_ic.size() != n * (size_t)g_ic_ncomp) {
        fprintf(stderr, "fm_refdrv: --ic has %zu values, expected %zu\n", g_ic.size(), n * (size_t)g_ic_ncomp);
        exit(3);
      }
      for (size_t i = 0; i < n; ++i) {
        size_t nc = sol[i].size() < (size_t)g_ic_ncomp ? sol[i].size() : (size_t)g_ic_ncomp;
        for (size_t c = 0; c < nc; ++c) sol[i][c] = g_ic[i * g_ic_ncomp + c];
      }
    }
  }
  g_last_time = t;
  if (g_timing) {
    double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - g_t0).count();
    fprintf(g_timing, "%.9f %.17e\n", s, t);
    fflush(g_timing);
  }
  real_setvel(m, t, sol);
}

void wrap_export(femModel* m, std::string name, bool msg) {
  ++g_export_calls;
  if (g_dump) {
    std::string path = g_dump_dir + "/" + name + ".f64";
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) { perror(path.c_str()); exit(4); }
    const char magic[8] = {'F', 'M', 'D', 'U', 'M', 'P', '1', 0};
    fwrite(magic, 1, 8, f);
    int nres = (int)m->resultList.size();
    fwrite(&g_last_time, sizeof(double), 1, f);
    fwrite(&nres, sizeof(int), 1, f);
    for (int r = 0; r < nres; ++r) {
      femResult* res = m->resultList[r];
      char label[32];
      memset(label, 0, sizeof(label));
      strncpy(label, res->label.c_str(), sizeof(label) - 1);
      int type = (res->type == frNode) ? 0 : 1;
      int nc = res->numComponents;
      long long nv = (long long)res->values.size();
      fwrite(label, 1, 32, f);
      fwrite(&type, sizeof(int), 1, f);
      fwrite(&nc, sizeof(int), 1, f);
      fwrite(&nv, sizeof(long long), 1, f);
      std::vector<double> buf((size_t)nv * nc);
      for (long long i = 0; i < nv; ++i)
        for (int c = 0; c < nc; ++c) buf[(size_t)i * nc + c] = res->values[i][c];
      fwrite(buf.data(), sizeof(double), buf.size(), f);
    }
    fclose(f);
  }
  if (g_vtk) real_export(m, name, msg);
}

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s model.dat vms|supg|parse [--ic file ncomp] [--dump dir] [--vtk] [--timing file]\n", argv[0]);
    return 2;
  }
  std::string model_path = argv[1], solver = argv[2];
  std::string timing_path;
  for (int i = 3; i < argc; ++i) {
    if (!strcmp(argv[i], "--ic") && i + 2 < argc) {
      FILE* f = fopen(argv[i + 1], "rb");
      if (!f) { perror(argv[i + 1]); return 2; }
      fseek(f, 0, SEEK_END);
      long sz = ftell(f);
      fseek(f, 0, SEEK_SET);
      g_ic.resize(sz / sizeof(double));
      if (fread(g_ic.data(), sizeof(double), g_ic.size(), f) != g_ic.size()) { fclose(f); return 2; }
      fclose(f);
      g_ic_ncomp = atoi(argv[i + 2]);
      i += 2;
    } else if (!strcmp(argv[i], "--dump") && i + 1 < argc) {
      g_dump = true;
      g_dump_dir = argv[++i];
    } else if (!strcmp(argv[i], "--sol") && i + 1 < argc) {
      FILE* f = fopen(argv[i + 1], "rb");
      if (!f) { perror(argv[i + 1]); return 2; }
      fseek(f, 0, SEEK_END);
      long sz = ftell(f);
      fseek(f, 0, SEEK_SET);
      g_sol.resize(sz / sizeof(double));
      if (fread(g_sol.data(), sizeof(double), g_sol.size(), f) != g_sol.size()) { fclose(f); return 2; }
      fclose(f);
      ++i;
    } else if (!strcmp(argv[i], "--vtk")) {
      g_vtk = true;
    } else if (!strcmp(argv[i], "--timing") && i + 1 < argc) {
      timing_path = argv[++i];
    } else {
      fprintf(stderr, "unknown argument %s\n", argv[i]);
      return 2;
    }
  }
  g_t0 = std::chrono::steady_clock::now();
  if (!timing_path.empty()) g_timing = fopen(timing_path.c_str(), "w");
  try {
    femModel* model = new femModel();
    model->ReadFromFEMTextFile(model_path);
    if (g_timing) {
      double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - g_t0).count();
      fprintf(g_timing, "# parsed %.9f\n", s);
    }
    if (solver == "parse") return 0;  // the reader alone (its time under --timing)
    if (solver == "poisson-elements") {
      if (!g_dump) {
        fprintf(stderr, "poisson-elements needs --dump dir\n");
        return 2;
      }
      model->FixedElementConnectivities();
      femIntegrationRule* rule = new femIntegrationRule(irSecondOrder);
      std::string path = g_dump_dir + "/poisson_elements.f64";
      FILE* f = fopen(path.c_str(), "wb");
      if (!f) { perror(path.c_str()); return 4; }
      femDoubleMat elMat(kMaxConnections, femDoubleVec(kMaxConnections, 0.0));
      for (size_t e = 0; e < model->elementList.size(); ++e) {
        femElement* el = model->elementList[e];
        el->formPoissonMatrix(model->nodeList, rule, (femDoubleVec)model->elDiffusivity[e], elMat);
        const size_t npe = el->elementConnections.size();
        for (size_t a = 0; a < npe; ++a) fwrite(elMat[a].data(), sizeof(double), npe, f);
      }
      femDoubleVec elSrc(kMaxConnections, 0.0);
      for (size_t k = 0; k < model->sourceElement.size(); ++k) {
        femElement* el = model->elementList[model->sourceElement[k]];
        el->formPoissonSource(model->nodeList, rule, model->sourceValues[k], elSrc);
        fwrite(elSrc.data(), sizeof(double), el->elementConnections.size(), f);
      }
      // with --sol: the reference's wall distance of that nodal solution
      if (!g_sol.empty()) {
        femDenseVector sol((int)g_sol.size());
        for (size_t i = 0; i < g_sol.size(); ++i) sol.setComponent((int)i, g_sol[i]);
        femDoubleVec dist;
        evalDistanceFromPoissonSolution(&sol, model, dist);
        fwrite(dist.data(), sizeof(double), dist.size(), f);
      }
      fclose(f);
      return 0;
    }
#ifdef FM_WITH_GPU_ADAPTER
    if (solver == "poisson-gpu") {
      // src/main.cpp:476-511 with the B200 adapter in place of femPoissonSolver;
      // the results go through the export hook (--dump)
      model->FixedElementConnectivities();
      femPoissonSolverGPU* s = new femPoissonSolverGPU(0, 1e-14, 100000);
      femPoissonSolverOptions* o = new femPoissonSolverOptions();
      s->solve(o, model);
      model->ExportToVTKLegacy("poisson", false);
      return 0;
    }
#endif
    if (solver == "vms") {
      femVMSExplicitFluidSolver* s = new femVMSExplicitFluidSolver();
      s->solve(model);
    } else if (solver == "supg") {
      femSUPGExplicitFluidSolver* s = new femSUPGExplicitFluidSolver();
      s->solve(model);
#ifdef FM_WITH_GPU_ADAPTER
    } else if (solver == "vms-gpu" || solver == "vms-gpu-mixed") {
      femVMSExplicitFluidSolverGPU* s = new femVMSExplicitFluidSolverGPU(0, solver == "vms-gpu-mixed");
      s->solve(model);
    } else if (solver == "supg-gpu") {
      femSUPGExplicitFluidSolverGPU* s = new femSUPGExplicitFluidSolverGPU(0, false);
      s->solve(model);
#endif
    } else {
      fprintf(stderr, "unknown solver %s\n", solver.c_str());
      return 2;
    }
  } catch (femException& e) {
    fprintf(stderr, "%s\nProgram Terminated.\n", e.what());
    return 1;
  }
  if (g_timing) fclose(g_timing);
  return 0;
}
