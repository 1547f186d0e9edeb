// PGJ.h -- projected Gauss-Jacobi (src/PGJ.cuh): System(5).  Defaults
// tolerance 1e-4, maxIterations 1000000, omega 0.3, lambda 2/3
// (src/PGJ.cu:6-16).  The iterations run inside the GPU time step; solve()
// runs the step's solve alone (dv_apgd_solve).
#pragma once

#include "Solver.h"

class PGJ : public Solver {
  friend class System;

 public:
  double omega;
  double lambda;
  explicit PGJ(System* sys) : Solver(sys), omega(0.3), lambda(2.0 / 3.0) {
    tolerance = 1e-4;
    maxIterations = 1000000;
    iterations = 0;
  }
  int setup();
  int solve();
};
