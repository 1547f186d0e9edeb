// CollisionDetector.h -- the reference's public collision interface
// (src/CollisionDetector.cuh:88-103).  Contact arrays are read back from the
// device through accessor methods.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

#include "PhysicsItem.h"

class System;
class CollisionDetector;

// The reference's thrust::device_vector fields of the contact list
// (CollisionDetector.cuh:88-91) as handles that read the device when
// converted, sized or indexed: `std::vector<uint> a = cd->collisionIdentifierA_d;`.
class ContactIdArray {
 public:
  ContactIdArray(CollisionDetector* cd, bool b_side) : cd_(cd), b_(b_side) {}
  operator std::vector<uint>() const;
  size_t size() const;
  uint operator[](size_t i) const;

 private:
  CollisionDetector* cd_;
  bool b_;
};

class ContactLocationArray {
 public:
  explicit ContactLocationArray(CollisionDetector* cd) : cd_(cd) {}
  operator std::vector<double3>() const;
  size_t size() const;
  double3 operator[](size_t i) const;

 private:
  CollisionDetector* cd_;
};

class CollisionDetector {
  friend class System;

 private:
  System* system;
  double envelope;
  uint3 binsPerAxis;

 public:
  uint numCollisions;
  uint numPossibleCollisions;
  ContactIdArray collisionIdentifierA_d;
  ContactIdArray collisionIdentifierB_d;
  ContactLocationArray collisionLocations_d;

  explicit CollisionDetector(System* sys)
      : system(sys), envelope(0.001), binsPerAxis(make_uint3(20, 20, 20)), numCollisions(0),
        numPossibleCollisions(0), collisionIdentifierA_d(this, false),
        collisionIdentifierB_d(this, true), collisionLocations_d(this) {}
  CollisionDetector(const CollisionDetector&) = delete;
  CollisionDetector& operator=(const CollisionDetector&) = delete;
  // The uniform grid is sized from the scene; the bin count is kept for
  // source compatibility (the candidate set does not depend on it).
  void setBinsPerAxis(uint3 b) { binsPerAxis = b; }
  int setEnvelope(double e);
  double getEnvelope() const { return envelope; }
  // The reference's three stages (CollisionDetector.cu:547-665).  The B200
  // pipeline forms the AABBs inside its collision pass, so the first is
  // accepted and does nothing; either broadphase entry runs the whole
  // detection (the candidate set does not depend on the method).
  int generateAxisAlignedBoundingBoxes() { return 0; }
  int detectPossibleCollisions_spatialSubdivision() { return detectCollisions(); }
  int detectPossibleCollisions_nSquared() { return detectCollisions(); }
  int detectCollisions();
  std::vector<double3> getCollisionLocations();
  std::vector<uint32_t> getCollisionIdentifierA();
  std::vector<uint32_t> getCollisionIdentifierB();
  std::vector<double4> getNormalsAndPenetrations();
  int exportSystem(std::string filename);
};
