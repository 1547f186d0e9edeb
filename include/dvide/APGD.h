// APGD.h -- accelerated projected gradient descent (src/APGD.cuh:18-68):
// defaults tolerance 1e-4, maxIterations 100000, warm start and
// anti-relaxation off (src/APGD.cu:6-16).  The iterations run inside the
// GPU time step; solve() reports the last step's solve.
#pragma once

#include "Solver.h"

class APGD : public Solver {
  friend class System;

 private:
  bool useWarmStarting;
  bool useAntiRelaxation;

 public:
  explicit APGD(System* sys) : Solver(sys), useWarmStarting(false), useAntiRelaxation(false) {
    tolerance = 1e-4;
    maxIterations = 100000;
    iterations = 0;
  }
  void setWarmStarting(bool w) { useWarmStarting = w; }
  void setAntiRelaxation(bool a) { useAntiRelaxation = a; }
  bool getWarmStarting() const { return useWarmStarting; }
  int setup();
  int solve();
};
