// Drop-in femSolver class for feMorph's Poisson solver on a B200 through
// libfemorph_b200 (include/femorph_b200.h, fm_poisson_*).
//
// It keeps the reference's plugin interface, femPoissonSolver
// (src/femSolver.h:56-61): a femSolver subclass overriding
// `virtual void solve(femOption* options, femModel* model)`, constructed
// directly by the caller (src/main.cpp:502-508).  It reads the same femModel
// fields (nodeList, elementList, elDiffusivity, sourceElement / sourceValues,
// neumannBCFaceNodes / neumannBCValues, diricheletBCNode / Values,
// problemType), appends the same results to model->resultList
// ("PoissonResult" per node, minus its average for PPE; "cellDistance" per
// element for DISTANCE, also written to cellDistance.txt) and reports errors
// as femException.  The caller runs model->FixedElementConnectivities first,
// as src/main.cpp:491 does (the library applies the same fix, which leaves
// fixed elements as they are).
//
// Build: compile this file inside the feMorph source tree (it includes
// femSolver.h / femModel.h) and link libfemorph_b200.so.
#ifndef FEMPOISSONSOLVERGPU_H
#define FEMPOISSONSOLVERGPU_H

#include "femModel.h"
#include "femOption.h"
#include "femSolver.h"

class femPoissonSolverGPU : public femSolver {
 public:
  // rel_tol: CG stops at ||r|| <= rel_tol ||b||
  femPoissonSolverGPU(int device = 0, double rel_tol = 1e-12, int max_iter = 100000);
  virtual void solve(femOption* options, femModel* model);

 private:
  int device_;
  double rel_tol_;
  int max_iter_;
};

#endif
