// shear_moves.cpp -- the reference shear driver's way of moving bodies
// (models/test_shear.cu:378-406), through the C++ layer of
// include/dvide/System.h (a test program: the tests compile and run it, then
// replay the same sequence in the oracle).
//
// Usage: shear_moves <dir> <steps>
// An open box (floor and four fixed walls) holds 3 x 3 x 4 spheres.  Every
// step, as the driver does:
//   p0 = p_d; DoTimeStep(); v_h = v_d;
//   the +x wall's v set to (-0.2, 0, 0) (it pushes in), one sphere's x and z
//   velocity set to 0;
//   p_d = p0; v_d = v_h; p = h v + p (the driver's cusp::blas::axpy, here on
//   the host: p_h = p_d, the loop, p_d = p_h).
// Writes shear_initial.txt (p, v, mass, geometry, fixed of every body, full
// precision) before the first step, prints "step,contacts,iterations" per
// step, and writes shear_final.txt (p, v).  Also checks the upload's errors:
// wrong sizes, f_contact_d, and gamma_d written back unchanged.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "dvide/System.h"

static bool same(const std::vector<double>& a, const std::vector<double>& b) {
  return a.size() == b.size() && (a.empty() || memcmp(a.data(), b.data(), 8 * a.size()) == 0);
}

int main(int argc, char** argv) {
  if (argc < 3) return 64;
  const std::string dir = argv[1];
  const int steps = atoi(argv[2]);
  System* sys = new System(1);
  sys->setTimeStep(1e-3);
  sys->gravity = make_double3(0, 0, -9.81);
  sys->solver->tolerance = 1e-6;
  sys->solver->maxIterations = 500;
  dynamic_cast<APGD*>(sys->solver)->setWarmStarting(true);

  // an upload before initializeSystem is refused
  bool early = false;
  try {
    sys->p_d = std::vector<double>(3, 0.0);
  } catch (const std::logic_error&) {
    early = true;
  }

  const double bc[5][3] = {{0, 0, -0.05}, {-0.205, 0, 0.25}, {0.205, 0, 0.25}, {0, -0.205, 0.25},
                           {0, 0.205, 0.25}};
  const double bh[5][3] = {{0.25, 0.25, 0.05}, {0.05, 0.25, 0.25}, {0.05, 0.25, 0.25},
                           {0.155, 0.05, 0.25}, {0.155, 0.05, 0.25}};
  for (int i = 0; i < 5; ++i) {
    Body* b = new Body(make_double3(bc[i][0], bc[i][1], bc[i][2]));
    b->setBodyFixed(true);
    b->setGeometry(make_double3(bh[i][0], bh[i][1], bh[i][2]));
    b->setMass(1.0);
    sys->add(b);
  }
  const double r = 0.05;
  for (int k = 0; k < 4; ++k)
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) {
        Body* b = new Body(make_double3(-0.1 + 0.1 * i + 0.002 * k, -0.1 + 0.1 * j + 0.001 * k,
                                        0.051 + 0.101 * k));
        b->setGeometry(make_double3(r, 0, 0));
        b->setMass(2600 * 4.0 * 3.14159 * pow(r, 3.0) / 3.0);
        sys->add(b);
      }
  if (sys->initializeSystem() != 0) return 2;
  const int nb = (int)sys->bodies.size();
  const int wall = 2;     // the +x wall
  const int held = 5 + 30;  // a sphere of the top layer, held in x and z

  {
    std::vector<double> p = sys->p_d, v = sys->v_d;
    FILE* f = fopen((dir + "/shear_initial.txt").c_str(), "w");
    for (int i = 0; i < nb; ++i) {
      const double3 g = sys->bodies[i]->getGeometry();
      fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %d\n", p[3 * i],
              p[3 * i + 1], p[3 * i + 2], v[3 * i], v[3 * i + 1], v[3 * i + 2],
              sys->bodies[i]->getMass(), g.x, g.y, g.z, sys->bodies[i]->isFixed() ? 1 : 0);
    }
    fclose(f);
  }

  bool sized = false, output = false;
  try {
    sys->v_d = std::vector<double>(3 * nb - 1, 0.0);
  } catch (const std::invalid_argument&) {
    sized = true;
  }
  try {
    sys->f_contact_d = std::vector<double>(3 * nb, 0.0);
  } catch (const std::logic_error&) {
    output = true;
  }
  printf("upload checks: early %d sized %d output %d\n", early, sized, output);

  bool gamma_kept = true;
  for (int s = 0; s < steps; ++s) {
    std::vector<double> p0_h = sys->p_d;
    if (sys->DoTimeStep() != 0) return 2;
    printf("%d,%d,%d\n", s, sys->collisionDetector->numCollisions, sys->solver->iterations);
    sys->v_h = sys->v_d;
    sys->v_h[3 * wall] = -0.2;
    sys->v_h[3 * wall + 1] = 0;
    sys->v_h[3 * wall + 2] = 0;
    sys->v_h[3 * held] = 0;
    sys->v_h[3 * held + 2] = 0;
    sys->p_d = p0_h;
    sys->v_d = sys->v_h;
    sys->p_h = sys->p_d;
    for (int k = 0; k < 3 * nb; ++k) sys->p_h[k] = sys->h * sys->v_h[k] + sys->p_h[k];
    sys->p_d = sys->p_h;
    if (s == steps / 2) {
      // gamma_d written back as it is: the next step must not notice
      std::vector<double> g = sys->gamma_d;
      sys->gamma_d = g;
      gamma_kept = same(static_cast<std::vector<double>>(sys->gamma_d), g);
    }
  }
  printf("gamma kept: %d\n", gamma_kept);
  std::vector<double> p = sys->p_d, v = sys->v_d;
  FILE* f = fopen((dir + "/shear_final.txt").c_str(), "w");
  for (int i = 0; i < nb; ++i)
    fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g\n", p[3 * i], p[3 * i + 1], p[3 * i + 2],
            v[3 * i], v[3 * i + 1], v[3 * i + 2]);
  fclose(f);
  delete sys;
  return 0;
}
