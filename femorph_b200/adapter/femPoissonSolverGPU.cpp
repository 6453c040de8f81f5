// femSolver adapter: feMorph's Poisson solver (femPoissonSolver::solve,
// src/femSolver.cpp:409-654) on a B200.
#include "femPoissonSolverGPU.h"

#include <cstdio>
#include <string>
#include <vector>

#include "femException.h"
#include "femResult.h"
#include "femUtils.h"
#include "femorph_b200.h"

namespace {

void fm_check(int rc) {
  if (rc != FM_OK)
    throw femException((std::string("femorph_b200: ") + fm_strerror(rc) + ": " + fm_last_error_message() + "\n").c_str());
}

struct PoissonHandle {
  fm_poisson* s = nullptr;
  ~PoissonHandle() { fm_poisson_destroy(s); }
};

}  // namespace

femPoissonSolverGPU::femPoissonSolverGPU(int device, double rel_tol, int max_iter)
    : device_(device), rel_tol_(rel_tol), max_iter_(max_iter) {}

void femPoissonSolverGPU::solve(femOption* options, femModel* model) {
  (void)options;  // femPoissonSolverOptions carries no settings (src/femOption.h)
  const size_t N = model->nodeList.size(), E = model->elementList.size();
  std::vector<double> coords(N * 3), diff(E * 3, 0.0), src_val(model->sourceValues.begin(), model->sourceValues.end()),
      neu_val(model->neumannBCValues.begin(), model->neumannBCValues.end()), dir_val;
  std::vector<int32_t> conn, src_el(model->sourceElement.begin(), model->sourceElement.end()), neu_off(1, 0), neu_nodes,
      dir_node(model->diricheletBCNode.begin(), model->diricheletBCNode.end());
  for (size_t i = 0; i < N; ++i)
    for (int k = 0; k < 3; ++k) coords[i * 3 + k] = model->nodeList[i]->coords[k];
  int32_t etype = 0;
  for (size_t e = 0; e < E; ++e) {
    const std::vector<int>& c = model->elementList[e]->elementConnections;
    if (etype == 0) etype = (int32_t)c.size();
    if ((int32_t)c.size() != etype || (etype != 4 && etype != 8))
      throw femException("femorph_b200: the Poisson solver needs a mesh of only TET4 or only HEXA8 elements.\n");
    for (int v : c) conn.push_back(v);
  }
  // elDiffusivity rows are used element by element (src/femSolver.cpp:456)
  if (model->elDiffusivity.size() < E) throw femException("femorph_b200: fewer ELDIFF rows than elements.\n");
  for (size_t e = 0; e < E; ++e)
    for (int k = 0; k < 3; ++k) diff[e * 3 + k] = model->elDiffusivity[e][k];
  for (const femIntVec& f : model->neumannBCFaceNodes) {
    for (int v : f) neu_nodes.push_back(v);
    neu_off.push_back((int32_t)neu_nodes.size());
  }
  for (const femDoubleVec& v : model->diricheletBCValues) dir_val.push_back(v.empty() ? 0.0 : v[0]);
  fm_poisson_desc d;
  d.elem_type = etype;
  d.problem = model->problemType == ptPPE ? FM_POISSON_PPE
              : model->problemType == ptPoissonDistance ? FM_POISSON_DISTANCE
                                                        : FM_POISSON_CLASSIC;
  d.n_nodes = (int64_t)N;
  d.n_elems = (int64_t)E;
  d.coords = coords.data();
  d.conn = conn.data();
  d.diffusivity = diff.data();
  d.n_sources = (int64_t)src_el.size();
  d.source_elem = src_el.data();
  d.source_value = src_val.data();
  d.n_neumann = (int64_t)neu_val.size();
  d.neumann_off = neu_off.data();
  d.neumann_nodes = neu_nodes.data();
  d.neumann_value = neu_val.data();
  d.n_dirichlet = (int64_t)dir_node.size();
  d.dir_node = dir_node.data();
  d.dir_value = dir_val.data();
  PoissonHandle h;
  fm_check(fm_poisson_create(&d, device_, &h.s));
  int32_t iters = 0;
  double rel_res = 0.0, ms = 0.0;
  fm_check(fm_poisson_solve(h.s, rel_tol_, max_iter_, &iters, &rel_res, &ms));
  printf("Solving Linear System... CG: %d iterations, relative residual %e\n", iters, rel_res);
  std::vector<double> x(N), dist;
  if (d.problem == FM_POISSON_DISTANCE) dist.resize(E);
  fm_check(fm_poisson_get_solution(h.s, x.data(), dist.empty() ? nullptr : dist.data()));
  if (d.problem == FM_POISSON_DISTANCE) {
    femResult* cellRes = new femResult();
    cellRes->label = std::string("cellDistance");
    cellRes->type = frElement;
    cellRes->numComponents = 1;
    for (double v : dist) cellRes->values.push_back(femDoubleVec(1, v));
    model->resultList.push_back(cellRes);
    femUtils::writeVectorToFile(std::string("cellDistance.txt"), dist);
  }
  femResult* res = new femResult();
  res->label = std::string("PoissonResult");
  res->type = frNode;
  res->numComponents = 1;
  for (double v : x) res->values.push_back(femDoubleVec(1, v));
  model->resultList.push_back(res);
}
