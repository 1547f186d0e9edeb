// settle.cpp -- a driver written against the reference's C++ API
// (System, Body, APGD; compare models/test_compaction.cu:184-431): 1,000
// spheres (r = 0.05 m, rho = 2600) on a 10x10x10 lattice in an open box of
// five fixed boxes, mu = 0.25, h = 1e-3, APGD with warm start.
// Usage: settle <steps> <solverType> <tolerance> [maxIterations] [warmStartMode]
//               [pinnedSpheres] [antiRelaxation]
// Prints one line per step: time, contacts, iterations, weight carried by
// the fixed boxes, and the four CCP violations.  With pinnedSpheres = n > 0
// the x and y DOFs of the first n spheres are held by bilateral constraints
// (System::addBilateralConstraintDOF, as the reference drivers pin DOFs) and
// the largest drift of those DOFs is printed at the end.  The bodies as built
// (settle_initial.txt) and the final positions and velocities
// (settle_final_full.txt) are written at full precision, so that the run can
// be replayed and compared elsewhere.  antiRelaxation = 1 turns on APGD's
// anti-relaxation (APGD::setAntiRelaxation).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include "dvide/System.h"

static unsigned long long rng = 88172645463325252ull;
static double getRandomNumber(double lo, double hi) {
  rng ^= rng << 13;
  rng ^= rng >> 7;
  rng ^= rng << 17;
  return lo + (hi - lo) * ((rng >> 11) * (1.0 / 9007199254740992.0));
}

int main(int argc, char** argv) {
  int steps = argc > 1 ? atoi(argv[1]) : 100;
  int solverType = argc > 2 ? atoi(argv[2]) : 1;
  double tolerance = argc > 3 ? atof(argv[3]) : 1e-4;
  int maxIterations = argc > 4 ? atoi(argv[4]) : 1000;
  int warmStartMode = argc > 5 ? atoi(argv[5]) : 1;
  int pinned = argc > 6 ? atoi(argv[6]) : 0;
  int antiRelaxation = argc > 7 ? atoi(argv[7]) : 0;

  System* sys = new System(solverType);
  sys->setTimeStep(1e-3);
  sys->gravity = make_double3(0, 0, -9.81);
  sys->solver->tolerance = tolerance;
  sys->solver->maxIterations = maxIterations;
  sys->collisionDetector->setBinsPerAxis(make_uint3(10, 10, 10));
  if (solverType == 1) {
    dynamic_cast<APGD*>(sys->solver)->setWarmStarting(warmStartMode);
    if (antiRelaxation) dynamic_cast<APGD*>(sys->solver)->setAntiRelaxation(true);
  }

  const double t = 0.05, inner = 0.6, H = 0.75;
  double3 c[5] = {make_double3(0, 0, -t), make_double3(-inner - t, 0, H), make_double3(inner + t, 0, H),
                  make_double3(0, -inner - t, H), make_double3(0, inner + t, H)};
  double3 g[5] = {make_double3(inner + 2 * t, inner + 2 * t, t), make_double3(t, inner + 2 * t, H),
                  make_double3(t, inner + 2 * t, H), make_double3(inner, t, H),
                  make_double3(inner, t, H)};
  for (int i = 0; i < 5; ++i) {
    Body* b = new Body(c[i]);
    b->setBodyFixed(true);
    b->setGeometry(g[i]);
    sys->add(b);
  }
  const double r = 0.05, rho = 2600.0, sp = 0.11;
  double totalWeight = 0;
  for (int i = 0; i < 10; ++i)
    for (int j = 0; j < 10; ++j)
      for (int k = 0; k < 10; ++k) {
        Body* b = new Body(make_double3(-0.495 + sp * i + getRandomNumber(-0.005, 0.005),
                                        -0.495 + sp * j + getRandomNumber(-0.005, 0.005),
                                        0.06 + sp * k + getRandomNumber(-0.005, 0.005)));
        b->setGeometry(make_double3(r, 0, 0));
        b->setMass(rho * 4.0 / 3.0 * M_PI * r * r * r);
        totalWeight += b->getMass() * 9.81;
        sys->add(b);
      }
  std::vector<double> pin0;
  for (int i = 0; i < pinned; ++i) {
    Body* b = sys->bodies[5 + i];
    sys->addBilateralConstraintDOF(3 * (5 + i), -1);
    sys->addBilateralConstraintDOF(3 * (5 + i) + 1, -1);
    pin0.push_back(b->getPosition().x);
    pin0.push_back(b->getPosition().y);
  }
  FILE* fi = fopen("settle_initial.txt", "w");
  for (Body* b : sys->bodies) {
    const double3 p = b->getPosition(), v = b->getVelocity(), g = b->getGeometry();
    fprintf(fi, "%.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %d\n", p.x, p.y, p.z,
            v.x, v.y, v.z, b->getMass(), g.x, g.y, g.z, b->isFixed() ? 1 : 0);
  }
  fclose(fi);
  int rc = sys->initializeSystem();
  if (rc != 0) {
    fprintf(stderr, "initializeSystem failed: %s\n", dv_status_string(rc));
    return 1;
  }
  printf("System initialized! bodies %zu, expected weight %.6f\n", sys->bodies.size(), totalWeight);
  for (int s = 0; s < steps; ++s) {
    rc = sys->DoTimeStep();
    if (rc != 0) {
      fprintf(stderr, "DoTimeStep failed at step %d: %s\n", s, dv_status_string(rc));
      return 2;
    }
    double4 v = sys->getCCPViolation();
    sys->f_contact_h = sys->f_contact_d;
    double weight = 0;
    for (int i = 0; i < 5; ++i) weight -= sys->f_contact_h[3 * i + 2];
    printf("%f, %u, %d, %.6f, %g, %g, %g, %g, %f\n", sys->time, sys->collisionDetector->numCollisions,
           sys->solver->iterations, weight, v.x, v.y, v.z, v.w, sys->elapsedTime);
  }
  if (pinned > 0) {
    std::vector<double> p = sys->p_d;
    double drift = 0;
    for (int i = 0; i < pinned; ++i)
      for (int k = 0; k < 2; ++k) drift = fmax(drift, fabs(p[3 * (5 + i) + k] - pin0[2 * i + k]));
    printf("pinned drift: %g\n", drift);
  }
  // the contact list through the reference's field names (handles)
  std::vector<uint> ida = sys->collisionDetector->collisionIdentifierA_d;
  std::vector<double3> loc = sys->collisionDetector->collisionLocations_d;
  sys->gamma_h = sys->gamma_d;
  bool handles_ok = ida.size() == sys->collisionDetector->numCollisions &&
                    loc.size() == sys->collisionDetector->collisionLocations_d.size() &&
                    sys->gamma_h.size() == sys->gamma_d.size();
  for (size_t i = 0; i < ida.size() && i < 16; ++i)
    handles_ok = handles_ok && ida[i] == sys->collisionDetector->collisionIdentifierA_d[i] &&
                 ida[i] < sys->collisionDetector->collisionIdentifierB_d[i];
  printf("contact handles: %s\n", handles_ok ? "ok" : "mismatch");
  sys->exportSystem("settle_final.csv");
  {
    std::vector<double> p = sys->p_d, v = sys->v_d;
    FILE* ff = fopen("settle_final_full.txt", "w");
    for (size_t i = 0; i < sys->bodies.size(); ++i)
      fprintf(ff, "%.17g %.17g %.17g %.17g %.17g %.17g\n", p[3 * i], p[3 * i + 1], p[3 * i + 2],
              v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    fclose(ff);
  }
  sys->exportMatrices(".");
  delete sys;
  return 0;
}
