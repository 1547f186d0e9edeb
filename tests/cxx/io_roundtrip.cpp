// io_roundtrip.cpp -- System::exportSystem -> System::importSystem -> steps,
// through the C++ layer of include/dvide/System.h (a test program: the
// tests compile and run it, then read what it wrote).
//
// Usage: io_roundtrip <dir> <steps>
// A scene whose numbers all have at most six significant digits (so that the
// six-digit CSV holds them exactly) is built in System A and exported; System
// B imports the file.  Both are checked bit for bit (bodies, masses), stepped
// side by side and compared bit for bit after every step.  Then A's files are
// written for the format checks, each beside a full-precision dump of the
// values it holds:
//   a_end.csv / a_end_full.txt      System::exportSystem and p, v, geometry, fixed
//   cd_end.csv / cd_end_full.txt    CollisionDetector::exportSystem and A, B, nP
//   forces.csv / forces_full.txt    outputContactForcePerCollision(file) and the
//                                   per-contact forces calculateContactForcePerCollision left
//   masses.txt                      radius and imported mass of every body of B
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "dvide/System.h"

static System* make_system() {
  System* s = new System(1);
  s->setTimeStep(1e-3);
  s->gravity = make_double3(0, 0, -9.81);
  s->solver->tolerance = 1e-6;
  s->solver->maxIterations = 500;
  dynamic_cast<APGD*>(s->solver)->setWarmStarting(true);
  return s;
}

static bool same(const std::vector<double>& a, const std::vector<double>& b) {
  return a.size() == b.size() && (a.empty() || memcmp(a.data(), b.data(), 8 * a.size()) == 0);
}

int main(int argc, char** argv) {
  if (argc < 3) return 64;
  const std::string dir = argv[1];
  const int steps = atoi(argv[2]);
  System* A = make_system();
  // an open box: floor and four walls (fixed)
  const double bc[5][3] = {{0, 0, -0.05}, {-0.205, 0, 0.25}, {0.205, 0, 0.25}, {0, -0.205, 0.25},
                           {0, 0.205, 0.25}};
  const double bh[5][3] = {{0.25, 0.25, 0.05}, {0.05, 0.25, 0.25}, {0.05, 0.25, 0.25},
                           {0.155, 0.05, 0.25}, {0.155, 0.05, 0.25}};
  for (int i = 0; i < 5; ++i) {
    Body* b = new Body(make_double3(bc[i][0], bc[i][1], bc[i][2]));
    b->setBodyFixed(true);
    b->setGeometry(make_double3(bh[i][0], bh[i][1], bh[i][2]));
    b->setMass(1.0);
    A->add(b);
  }
  // 3 x 3 x 4 spheres of radius 0.05 on a lattice of six-digit coordinates
  // literals only: a computed sum such as -0.1015 + 0.0022 is not the double
  // nearest to its six-digit decimal, and would not survive the file
  const double xs[3] = {-0.1015, 0.0003, 0.1012};
  const double ys[4][3] = {{-0.1015, 0.0003, 0.1012}, {-0.1004, 0.0014, 0.1023},
                           {-0.0993, 0.0025, 0.1034}, {-0.0982, 0.0036, 0.1045}};
  const double zs[4] = {0.0502, 0.1511, 0.2524, 0.3533};
  const double vx[3] = {0.25, -0.125, 0.0};
  const double r = 0.05;
  for (int k = 0; k < 4; ++k)
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) {
        Body* b = new Body(make_double3(xs[i], ys[k][j], zs[k]));
        b->setGeometry(make_double3(r, 0, 0));
        b->setVelocity(make_double3(vx[(i + k) % 3], vx[(j + 2 * k) % 3], -0.0625 * (k % 2)));
        b->setMass(2600 * 4.0 * 3.14159 * pow(r, 3.0) / 3.0);
        A->add(b);
      }
  if (A->initializeSystem() != 0) return 2;
  if (A->exportSystem(dir + "/a0.csv") != 0) return 2;

  System* B = make_system();
  if (B->importSystem(dir + "/a0.csv") != 0) return 2;
  if (B->initializeSystem() != 0) return 2;
  if (B->bodies.size() != A->bodies.size()) return 3;
  for (size_t i = 0; i < A->bodies.size(); ++i) {
    Body* a = A->bodies[i];
    Body* b = B->bodies[i];
    const double ma = a->getMass(), mb = b->getMass();
    const double3 ga = a->getGeometry(), gb = b->getGeometry();
    if (memcmp(&ma, &mb, 8) || a->isFixed() != b->isFixed() || memcmp(&ga, &gb, sizeof(double3))) {
      printf("body %zu differs after import\n", i);
      return 3;
    }
  }
  if (!same(A->p_d, B->p_d) || !same(A->v_d, B->v_d)) {
    printf("state differs after import\n");
    return 3;
  }
  int contacts = 0;
  for (int s = 0; s < steps; ++s) {
    if (A->DoTimeStep() != 0 || B->DoTimeStep() != 0) return 2;
    if (A->collisionDetector->numCollisions != B->collisionDetector->numCollisions ||
        A->solver->iterations != B->solver->iterations || !same(A->p_d, B->p_d) ||
        !same(A->v_d, B->v_d) || !same(A->gamma_d, B->gamma_d)) {
      printf("step %d differs\n", s);
      return 3;
    }
    contacts += A->collisionDetector->numCollisions;
  }
  printf("roundtrip identical over %d steps, %d contacts\n", steps, contacts);

  if (A->exportSystem(dir + "/a_end.csv") != 0) return 2;
  std::vector<double> p = A->p_d, v = A->v_d;
  FILE* f = fopen((dir + "/a_end_full.txt").c_str(), "w");
  for (size_t i = 0; i < A->bodies.size(); ++i) {
    const double3 g = A->bodies[i]->getGeometry();
    fprintf(f, "%d %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n",
            A->bodies[i]->isFixed() ? 1 : 0, p[3 * i], p[3 * i + 1], p[3 * i + 2], v[3 * i],
            v[3 * i + 1], v[3 * i + 2], g.x, g.y, g.z);
  }
  fclose(f);

  if (A->collisionDetector->exportSystem(dir + "/cd_end.csv") != 0) return 2;
  std::vector<uint> ida = A->collisionDetector->collisionIdentifierA_d;
  std::vector<uint> idb = A->collisionDetector->collisionIdentifierB_d;
  std::vector<double4> nP = A->collisionDetector->getNormalsAndPenetrations();
  f = fopen((dir + "/cd_end_full.txt").c_str(), "w");
  for (size_t i = 0; i < ida.size(); ++i)
    fprintf(f, "%u %u %.17g %.17g %.17g %.17g\n", ida[i], idb[i], nP[i].x, nP[i].y, nP[i].z,
            nP[i].w);
  fclose(f);

  if (A->outputContactForcePerCollision(dir + "/forces.csv") != 0) return 2;
  if (A->calculateContactForcePerCollision() != 0) return 2;
  f = fopen((dir + "/forces_full.txt").c_str(), "w");
  for (size_t i = 0; i < A->normalForcePerCollision_h.size(); ++i) {
    const double3 n = A->normalForcePerCollision_h[i], t = A->frictionForcePerCollision_h[i];
    fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g\n", n.x, n.y, n.z, t.x, t.y, t.z);
  }
  fclose(f);

  f = fopen((dir + "/masses.txt").c_str(), "w");
  for (size_t i = 0; i < B->bodies.size(); ++i)
    fprintf(f, "%.17g %.17g\n", B->bodies[i]->getGeometry().x, B->bodies[i]->getMass());
  fclose(f);
  delete A;
  delete B;
  return 0;
}
