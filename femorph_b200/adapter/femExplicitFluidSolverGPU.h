// Drop-in femSolver classes for feMorph that run the explicit flow step on a
// B200 through libfemorph_b200 (include/femorph_b200.h).
//
// They keep the reference's plugin interface: a femSolver subclass with
// `virtual void solve(femModel* model)` (src/femVMSExplicitFluidSolver.h:9-14,
// src/femSUPGExplicitFluidSolver.h:9-14), constructed directly by the caller
// (src/main.cpp:797-801).  They read the same femModel fields, write
// model->resultList and call model->ExportToVTKLegacy on the reference's save
// schedule, and report errors as femException (or, for the SUPG exit
// condition, the reference's message and exit(-1)).
//
// Build: compile this file inside the feMorph source tree (it includes
// femSolver.h / femModel.h) and link libfemorph_b200.so.
#ifndef FEMEXPLICITFLUIDSOLVERGPU_H
#define FEMEXPLICITFLUIDSOLVERGPU_H

#include "femModel.h"
#include "femSolver.h"

class femVMSExplicitFluidSolverGPU : public femSolver {
 public:
  // log: print the reference's per-dual-iteration line and write its res_v /
  // res_p fields (device diagnostics, which slow the solve); off: neither.
  femVMSExplicitFluidSolverGPU(int device = 0, bool mixed = false, bool log = true);
  virtual void solve(femModel* model);

 private:
  int device_;
  bool mixed_;
  bool log_;
};

class femSUPGExplicitFluidSolverGPU : public femSolver {
 public:
  femSUPGExplicitFluidSolverGPU(int device = 0, bool mixed = false);
  virtual void solve(femModel* model);

 private:
  int device_;
  bool mixed_;
};

#endif
