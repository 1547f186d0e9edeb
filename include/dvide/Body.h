// Body.h -- rigid point mass with a sphere or box contact geometry, the
// interface of the reference's src/Body.cuh:14-100 (3 translational DOF,
// mass 1.0 by default, geometry (r,0,0) = sphere, (hx,hy,hz) = box).
#pragma once

#include "PhysicsItem.h"

class Body : public PhysicsItem {
  friend class System;

 private:
  double3 pos;
  double3 vel;
  double3 acc;
  double mass;
  bool fixed;
  double3 contactGeometry;

  void init(double3 p) {
    numDOF = 3;
    identifier = 0;
    index = 0;
    collisionFamily = -1;
    pos = p;
    vel = make_double3(0, 0, 0);
    acc = make_double3(0, 0, 0);
    mass = 1.0;
    fixed = false;
    contactGeometry = make_double3(1.0, 0, 0);
  }

 public:
  Body() { init(make_double3(0, 0, 0)); }
  explicit Body(double3 position) { init(position); }
  bool isFixed() { return fixed; }
  double3 getPosition() { return pos; }
  double3 getVelocity() { return vel; }
  double getMass() { return mass; }
  void setMass(double m) { mass = m; }
  void setBodyFixed(bool f) { fixed = f; }
  double3 getGeometry() { return contactGeometry; }
  void setGeometry(double3 g) { contactGeometry = g; }
  void setVelocity(double3 v) { vel = v; }
};
