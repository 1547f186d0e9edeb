// PGS.h -- projected Gauss-Seidel (src/PGS.cuh): System(6).  Defaults
// tolerance 1e-4, maxIterations 1000000, omega 0.3, lambda 2/3
// (src/PGS.cu:6-16).  The iterations run inside the GPU time step; the sweep
// over contacts is sequential by definition (each update reads the velocities
// the previous ones wrote), one GPU thread per scene.  FP64 only.  solve()
// runs the step's solve alone (dv_apgd_solve) and, as the reference's, leaves
// its working velocities in System::v.
#pragma once

#include "Solver.h"

class PGS : public Solver {
  friend class System;

 public:
  double omega;
  double lambda;
  explicit PGS(System* sys) : Solver(sys), omega(0.3), lambda(2.0 / 3.0) {
    tolerance = 1e-4;
    maxIterations = 1000000;
    iterations = 0;
  }
  int setup();
  int solve();
};
