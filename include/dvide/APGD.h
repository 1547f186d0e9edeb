// APGD.h -- accelerated projected gradient descent (src/APGD.cuh:18-68):
// defaults tolerance 1e-4, maxIterations 100000, warm start and
// anti-relaxation off (src/APGD.cu:6-16); setAntiRelaxation(true) runs the
// reference's anti-relaxation block (APGD.cu:335-345).  The iterations run inside the
// GPU time step; solve() runs the step's solve alone on the current state and
// the last collision detection's contacts (no update; dv_apgd_solve).
#pragma once

#include "Solver.h"

class APGD : public Solver {
  friend class System;

 private:
  int warmStartMode;  // 0 off, 1 positional (the reference's), 2 matched by contact pair
  bool useAntiRelaxation;

 public:
  explicit APGD(System* sys) : Solver(sys), warmStartMode(0), useAntiRelaxation(false) {
    tolerance = 1e-4;
    maxIterations = 100000;
    iterations = 0;
  }
  // APGD.cuh:62: positional warm start on or off
  void setWarmStarting(bool w) { warmStartMode = w ? 1 : 0; }
  // extension: 2 starts each contact from the impulse its (A, B) pair had at
  // the last solve (a new pair from zero); 0 and 1 as above
  void setWarmStarting(int mode) { warmStartMode = mode; }
  void setAntiRelaxation(bool a) { useAntiRelaxation = a; }
  bool getWarmStarting() const { return warmStartMode != 0; }
  int getWarmStartMode() const { return warmStartMode; }
  int setup();
  int solve();
};
