// Solver.h -- the reference's abstract solver (src/Solver.cuh:17-45):
// tolerance, maxIterations, iterations, verbose, setup(), solve().
#pragma once

class System;

class Solver {
  friend class System;

 protected:
  System* system;

 public:
  double tolerance;
  int maxIterations;
  int iterations;
  bool verbose;

  Solver() : system(0), tolerance(0), maxIterations(1000000), iterations(0), verbose(false) {}
  explicit Solver(System* sys)
      : system(sys), tolerance(0), maxIterations(1000000), iterations(0), verbose(false) {}
  virtual int setup() = 0;
  virtual int solve() = 0;
  virtual ~Solver() {}
};
