// ref_helper_probe.cpp -- prints length(), normalize() and cross() of the
// reference's own vector helpers (src/helper_math_double.h, compiled from the
// reference tree, host build) on seeded inputs, one JSON record per line.
// Used only to pin the oracle's float-sqrt semantics (tests/golden/).
#include <stdint.h>
#include <stdio.h>

#include "helper_math_double.h"

static uint64_t rng_state = 0x9E3779B97F4A7C15ull;
static double urand() {  // splitmix64 -> [0, 1)
  uint64_t z = (rng_state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

static void emit(double3 a, double3 b) {
  double3 n = normalize(a);
  double3 c = cross(a, b);
  printf("{\"a\": [%.17g, %.17g, %.17g], \"b\": [%.17g, %.17g, %.17g], \"length\": %.17g, "
         "\"normalize\": [%.17g, %.17g, %.17g], \"cross\": [%.17g, %.17g, %.17g]}\n",
         a.x, a.y, a.z, b.x, b.y, b.z, length(a), n.x, n.y, n.z, c.x, c.y, c.z);
}

int main() {
  for (int i = 0; i < 200; ++i) {
    double s = (i % 4 == 0) ? 1e-3 : (i % 4 == 1) ? 1.0 : (i % 4 == 2) ? 0.0123 : 37.5;
    double3 a = make_double3(s * (2 * urand() - 1), s * (2 * urand() - 1), s * (2 * urand() - 1));
    double3 b = make_double3(2 * urand() - 1, 2 * urand() - 1, 2 * urand() - 1);
    emit(a, b);
  }
  emit(make_double3(0.1, 0.0, 0.0), make_double3(0, 1, 0));
  emit(make_double3(0.0, -0.0999, 0.0), make_double3(1, 0, 0));
  emit(make_double3(3e-4, 4e-4, 0.0), make_double3(0, 0, 1));
  return 0;
}
