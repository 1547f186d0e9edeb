// PhysicsItem.h -- same members as the reference's src/PhysicsItem.cuh:13-33.
#pragma once

#include <vector_functions.h>
#include <vector_types.h>

typedef unsigned int uint;

class PhysicsItem {
  friend class System;

 protected:
  uint identifier;
  uint index;
  int numDOF;
  int collisionFamily;

 public:
  PhysicsItem() : identifier(0), index(0), numDOF(0), collisionFamily(-1) {}
  uint getIndex() { return index; }
  void setIndex(uint i) { index = i; }
  uint getIdentifier() { return identifier; }
  void setIdentifier(uint i) { identifier = i; }
  int getCollisionFamily() { return collisionFamily; }
  void setCollisionFamily(int f) { collisionFamily = f; }
};
