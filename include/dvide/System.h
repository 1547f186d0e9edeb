// System.h -- the reference's System (src/System.cuh:279-326) for rigid
// spheres and boxes, backed by the B200 contact step of include/dvide.h.
// Device vectors of the reference (p_d, v_d, f_contact_d, gamma_d) are
// DeviceArray handles: assigning one to a std::vector downloads it, so
// driver lines such as `sys->f_contact_h = sys->f_contact_d;` keep working.
#pragma once

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../dvide.h"
#include "APGD.h"
#include "PGJ.h"
#include "PGS.h"
#include "Body.h"
#include "CollisionDetector.h"
#include "Solver.h"

class System;

class DeviceArray {
 public:
  enum Which { kPos, kVel, kContactForce, kGamma };
  DeviceArray(System* s, Which w) : sys(s), which(w) {}
  operator std::vector<double>() const;
  size_t size() const;
  // Uploads, as the reference's drivers write System::p_d, v_d and gamma_d
  // from host vectors between steps (models/test_shear.cu:404-405): p_d and
  // v_d take 3 values per body; gamma_d takes 3 per contact, the warm start of
  // the next solve, on a System without bilateral rows.  Throws
  // std::logic_error before initializeSystem, for f_contact_d (the output of
  // the last step) and for gamma_d with bilateral rows;
  // std::invalid_argument on a size that does not fit; std::runtime_error
  // when the C ABI reports an error.
  DeviceArray& operator=(const std::vector<double>& x);
  // another System's array (or this one's): its values, not its handle
  DeviceArray& operator=(const DeviceArray& o) {
    return *this = static_cast<std::vector<double>>(o);
  }
  // any other container of doubles (a thrust::host_vector, say)
  template <class C, class = decltype(std::declval<const C&>().begin())>
  DeviceArray& operator=(const C& c) {
    return *this = std::vector<double>(c.begin(), c.end());
  }

 private:
  System* sys;
  Which which;
};

class System {
  friend class APGD;
  friend class PGJ;
  friend class PGS;
  friend class CollisionDetector;
  friend class DeviceArray;

 private:
  dv_scene* scene;
  double frictionCoefficient;
  double tol;
  int solverType;
  int sync_params();
  int solveNow();  // Solver::solve() of this System's solver (dv_apgd_solve)
  struct BilateralDOF {
    int dofA, dofB;
    double velocity, startTime;
  };
  std::vector<BilateralDOF> bilaterals;  // handed to the scene at initializeSystem

 public:
  System();
  explicit System(int solverType);
  ~System();

  std::vector<Body*> bodies;
  Solver* solver;
  CollisionDetector* collisionDetector;
  double3 gravity;
  double h;
  double time;
  int timeIndex;
  double elapsedTime;
  double totalGPUMemoryUsed;
  double objectiveCCP;
  DeviceArray p_d, v_d, f_contact_d, gamma_d;
  std::vector<double> p_h, v_h, f_contact_h, gamma_h;
  // per-contact forces of the last step (System::normalForcePerCollision_d /
  // frictionForcePerCollision_d, filled by calculateContactForcePerCollision)
  std::vector<double3> normalForcePerCollision_h, frictionForcePerCollision_h;

  double getCurrentTime() const { return time; }
  double getTimeStep() const { return h; }
  double getTolerance() const { return tol; }
  int getTimeIndex() const { return timeIndex; }
  void setTimeStep(double step_size) { h = step_size; }
  void setFrictionCoefficient(double mu) { frictionCoefficient = mu; }
  int add(Body* body);
  // System.cu:510-532: +1 at DOF DOFA (3 body + axis), -1 at DOF DOFB, or DOFA
  // alone held at its position when DOFB < 0; moving at `velocity` from
  // `startTime` on.  Added before initializeSystem, as in the reference.
  int addBilateralConstraintDOF(int DOFA, int DOFB);
  int addBilateralConstraintDOF(int DOFA, int DOFB, double velocity, double startTime);
  int initializeSystem();
  int DoTimeStep();
  // applied forces are not part of the reference dynamics (System.cu:1510)
  int applyForce(Body* body, double3 force);
  int clearAppliedForces() { return 0; }
  double4 getCCPViolation();
  double getPotentialEnergy();
  double getKineticEnergy();
  double getStrainEnergy() { return 0.0; }
  double getTotalEnergy() { return getPotentialEnergy() + getKineticEnergy(); }
  int exportSystem(std::string filename);
  int importSystem(std::string filename);
  int calculateContactForcePerCollision();
  int outputContactForcePerCollision();
  int outputContactForcePerCollision(std::string filename);
  // D, Minv, r, b, k of the last step as Matrix Market files in `directory`
  int exportMatrices(std::string directory);
  std::vector<double> getPositions();
  std::vector<double> getVelocities();
  std::vector<double> getContactForces();
  dv_scene* native() { return scene; }
};
