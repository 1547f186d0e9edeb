// CollisionDetector.h -- the reference's public collision interface
// (src/CollisionDetector.cuh:88-103).  Contact arrays are read back from the
// device through accessor methods.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

#include "PhysicsItem.h"

class System;

class CollisionDetector {
  friend class System;

 private:
  System* system;
  double envelope;
  uint3 binsPerAxis;

 public:
  uint numCollisions;
  uint numPossibleCollisions;

  explicit CollisionDetector(System* sys)
      : system(sys), envelope(0.001), binsPerAxis(make_uint3(20, 20, 20)), numCollisions(0),
        numPossibleCollisions(0) {}
  // The uniform grid is sized from the scene; the bin count is kept for
  // source compatibility (the candidate set does not depend on it).
  void setBinsPerAxis(uint3 b) { binsPerAxis = b; }
  int setEnvelope(double e);
  double getEnvelope() const { return envelope; }
  int detectCollisions();
  std::vector<uint32_t> getCollisionIdentifierA();
  std::vector<uint32_t> getCollisionIdentifierB();
  std::vector<double4> getNormalsAndPenetrations();
  int exportSystem(std::string filename);
};
