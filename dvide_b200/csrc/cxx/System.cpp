// System.cpp -- the reference's System / APGD / CollisionDetector classes for
// rigid spheres and boxes (src/System.cu:14-133, 148-602, 1605-1930;
// src/CollisionDetector.cu:503-545, 665-711) implemented on the C ABI of
// include/dvide.h.  Each method keeps the reference's name, argument meaning
// and "return 0 on success" convention; failures return the dv status code.
#include "../../../include/dvide/System.h"

#include <cuda_runtime.h>
#include <stdio.h>

#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {
std::vector<double> download3(dv_scene* s, int which, int nb) {
  std::vector<double> out(3 * (size_t)nb, 0.0);
  if (!s || nb == 0) return out;
  if (which == 0) dv_get_state(s, out.data(), nullptr);
  else if (which == 1) dv_get_state(s, nullptr, out.data());
  else dv_get_contact_force(s, out.data());
  return out;
}
}  // namespace

DeviceArray::operator std::vector<double>() const {
  if (which == kGamma) {
    int32_t n = 0;
    dv_get_gamma(sys->scene, nullptr, 0, &n);
    // after a solve the reference's vector holds the bilateral rows first
    // (APGD.cu:166); before the first step it is 3 nb zeros (System.cu:185)
    int32_t nb = 0;
    if (sys->timeIndex > 0) dv_get_bilateral_gamma(sys->scene, nullptr, 0, &nb);
    std::vector<double> g((size_t)nb + 3 * (size_t)n);
    if (nb) dv_get_bilateral_gamma(sys->scene, g.data(), nb, &nb);
    if (n) dv_get_gamma(sys->scene, g.data() + nb, n, &n);
    return g;
  }
  int w = which == kPos ? 0 : which == kVel ? 1 : 2;
  return download3(sys->scene, w, (int)sys->bodies.size());
}

DeviceArray& DeviceArray::operator=(const std::vector<double>& x) {
  if (!sys->scene) throw std::logic_error("System device arrays are written after initializeSystem");
  const size_t nb = sys->bodies.size();
  int rc = 0;
  if (which == kPos || which == kVel) {
    if (x.size() != 3 * nb)
      throw std::invalid_argument("System::p_d / v_d take 3 values per body (" +
                                  std::to_string(3 * nb) + "), not " + std::to_string(x.size()));
    rc = dv_set_state(sys->scene, which == kPos ? x.data() : nullptr,
                      which == kVel ? x.data() : nullptr);
  } else if (which == kGamma) {
    if (!sys->bilaterals.empty())
      throw std::logic_error("System::gamma_d of a System with bilateral rows is not writable");
    if (x.size() % 3)
      throw std::invalid_argument("System::gamma_d takes 3 values per contact, not " +
                                  std::to_string(x.size()));
    rc = dv_set_gamma(sys->scene, x.data(), (int32_t)(x.size() / 3));
  } else {
    throw std::logic_error("System::f_contact_d is the output of the last step");
  }
  if (rc != 0) throw std::runtime_error(std::string("dv_set_state / dv_set_gamma: ") + dv_last_error());
  return *this;
}

size_t DeviceArray::size() const {
  if (which == kGamma) {
    int32_t n = 0, nb = 0;
    dv_get_gamma(sys->scene, nullptr, 0, &n);
    if (sys->timeIndex > 0) dv_get_bilateral_gamma(sys->scene, nullptr, 0, &nb);
    return (size_t)nb + 3 * (size_t)n;
  }
  return 3 * sys->bodies.size();
}

System::System()
    : scene(nullptr), frictionCoefficient(0.25), tol(1e-8), solverType(1),
      p_d(this, DeviceArray::kPos), v_d(this, DeviceArray::kVel),
      f_contact_d(this, DeviceArray::kContactForce), gamma_d(this, DeviceArray::kGamma) {
  gravity = make_double3(0, -9.81, 0);
  h = 1e-3;
  time = 0;
  timeIndex = 0;
  elapsedTime = 0;
  totalGPUMemoryUsed = 0;
  objectiveCCP = 0;
  collisionDetector = new CollisionDetector(this);
  solver = new APGD(this);
}

System::System(int type) : System() {
  // System.cu:77-101: 1 = APGD (also the default), 5 = PGJ, 6 = PGS; the
  // interior-point and active-set solvers are not part of this build.
  solverType = type;
  if (type == 5) {
    delete solver;
    solver = new PGJ(this);
  } else if (type == 6) {
    delete solver;
    solver = new PGS(this);
  }
}

System::~System() {
  if (scene) dv_scene_destroy(scene);
  delete collisionDetector;
  delete solver;
}

int System::add(Body* body) {
  bodies.push_back(body);
  return (int)bodies.size();
}

int System::applyForce(Body*, double3) { return 0; }

int System::sync_params() {
  dv_params P;
  dv_params_default(&P);
  P.h = h;
  P.mu = frictionCoefficient;
  P.gravity[0] = gravity.x;
  P.gravity[1] = gravity.y;
  P.gravity[2] = gravity.z;
  P.envelope = collisionDetector->envelope;
  P.tolerance = solver->tolerance;
  P.max_iterations = solver->maxIterations;
  APGD* apgd = dynamic_cast<APGD*>(solver);
  P.warm_start = apgd ? apgd->warmStartMode : 0;
  P.solver = solverType == 5 ? DV_SOLVER_PGJ : solverType == 6 ? DV_SOLVER_PGS : DV_SOLVER_APGD;
  P.verbose = solver->verbose ? 1 : 0;
  P.anti_relaxation = apgd && apgd->useAntiRelaxation ? 1 : 0;
  if (!scene) return DV_ERR_ARG;
  return dv_set_params(scene, &P);
}

int System::addBilateralConstraintDOF(int DOFA, int DOFB) {
  return addBilateralConstraintDOF(DOFA, DOFB, 0.0, 0.0);
}

int System::addBilateralConstraintDOF(int DOFA, int DOFB, double velocity, double startTime) {
  bilaterals.push_back(BilateralDOF{DOFA, DOFB, velocity, startTime});
  return 0;
}

int System::initializeSystem() {
  if (solverType < 1 || solverType > 7) solverType = 1;
  if (solverType != 1 && solverType != 5 && solverType != 6) return DV_ERR_UNSUPPORTED;
  APGD* apgd = dynamic_cast<APGD*>(solver);
  std::vector<dv_body_desc> desc(bodies.size());
  for (size_t j = 0; j < bodies.size(); ++j) {
    Body* b = bodies[j];
    b->setIdentifier((uint)j);   // System.cu:346-347
    b->setIndex((uint)(3 * j));
    dv_body_desc& d = desc[j];
    d.pos[0] = b->pos.x; d.pos[1] = b->pos.y; d.pos[2] = b->pos.z;
    d.vel[0] = b->vel.x; d.vel[1] = b->vel.y; d.vel[2] = b->vel.z;
    d.mass = b->mass;
    d.geom[0] = b->contactGeometry.x; d.geom[1] = b->contactGeometry.y;
    d.geom[2] = b->contactGeometry.z;
    d.fixed = b->fixed ? 1 : 0;
    d.family = b->collisionFamily;
  }
  dv_params P;
  dv_params_default(&P);
  P.h = h;
  P.mu = frictionCoefficient;
  P.gravity[0] = gravity.x;
  P.gravity[1] = gravity.y;
  P.gravity[2] = gravity.z;
  P.envelope = collisionDetector->envelope;
  P.tolerance = solver->tolerance;
  P.max_iterations = solver->maxIterations;
  P.warm_start = apgd ? apgd->warmStartMode : 0;
  P.solver = solverType == 5 ? DV_SOLVER_PGJ : solverType == 6 ? DV_SOLVER_PGS : DV_SOLVER_APGD;
  P.anti_relaxation = apgd && apgd->useAntiRelaxation ? 1 : 0;
  if (scene) dv_scene_destroy(scene);
  scene = nullptr;
  int rc = dv_scene_create(desc.data(), (int32_t)desc.size(), &P, &scene);
  if (rc != DV_OK) return rc;
  // System::processConstraints (System.cu:303-315): the rows reach the
  // device here, p0 of a single-DOF row from the positions now
  for (const BilateralDOF& c : bilaterals) {
    rc = dv_add_bilateral_dof(scene, c.dofA, c.dofB, c.velocity, c.startTime);
    if (rc != DV_OK) return rc;
  }
  return solver->setup();
}

int System::DoTimeStep() {
  int rc = sync_params();
  if (rc != DV_OK) return rc;
  rc = dv_step(scene, 1);
  dv_step_stats st;
  dv_get_step_stats(scene, &st);
  elapsedTime = st.elapsed_ms;
  objectiveCCP = st.objective;
  collisionDetector->numCollisions = (uint)st.num_contacts;
  collisionDetector->numPossibleCollisions = (uint)st.num_possible;
  solver->iterations = st.iterations;
  time = st.time;
  timeIndex = st.time_index;
  size_t avail = 0, total = 0;
  if (cudaMemGetInfo(&avail, &total) == cudaSuccess)
    totalGPUMemoryUsed = (double)(total - avail) / 1000000.0;
  return rc;
}

double4 System::getCCPViolation() {
  double o[4] = {0, 0, 0, 0};
  if (scene) dv_ccp_violation(scene, o);
  return make_double4(o[0], o[1], o[2], o[3]);
}

double System::getKineticEnergy() {
  double k = 0, p = 0;
  if (scene) dv_energies(scene, &k, &p);
  return k;
}

double System::getPotentialEnergy() {
  double k = 0, p = 0;
  if (scene) dv_energies(scene, &k, &p);
  return p;
}

std::vector<double> System::getPositions() { return p_d; }
std::vector<double> System::getVelocities() { return v_d; }
std::vector<double> System::getContactForces() { return f_contact_d; }

// The rigid-body rows of the System CSV file: System.cu:1699-1737 writes
// them and :1856-1910 reads them back.  Header: the body count followed by
// the (here always zero) counts of beams, plates and 2-D bodies.  One row per
// body: index, fixed flag, position, the unit orientation quaternion
// (1, 0, 0, 0), velocity, then the shape code with its geometry -- 0 and the
// radius for a sphere, 2 and the three half-extents for a box.  Every field
// is followed by ", "; numbers use the stream's default formatting (six
// significant digits), as the reference's files do.
namespace {

struct BodyRow {
  int index = 0, fixed = 0, shape = 0;
  double p[3] = {0, 0, 0}, v[3] = {0, 0, 0}, geom[3] = {0, 0, 0};
};

void write_body_row(std::ostream& os, const BodyRow& r) {
  os << r.index << ", " << r.fixed << ", " << r.p[0] << ", " << r.p[1] << ", " << r.p[2]
     << ", 1, 0, 0, 0, " << r.v[0] << ", " << r.v[1] << ", " << r.v[2] << ", " << r.shape << ", ";
  const int ng = r.shape == 0 ? 1 : 3;
  for (int k = 0; k < ng; ++k) os << r.geom[k] << ", ";
  os << "\n";
}

// The comma-separated fields of one line as numbers (empty fields skipped).
std::vector<double> csv_numbers(const std::string& line) {
  std::vector<double> out;
  size_t i = 0;
  while (i < line.size()) {
    size_t j = line.find(',', i);
    if (j == std::string::npos) j = line.size();
    const std::string f = line.substr(i, j - i);
    const char* c = f.c_str();
    char* e = nullptr;
    const double x = strtod(c, &e);
    if (e != c) out.push_back(x);
    i = j + 1;
  }
  return out;
}

bool parse_body_row(const std::string& line, BodyRow* r) {
  const std::vector<double> f = csv_numbers(line);
  // index, fixed, p (3), quaternion (4), v (3), shape, geometry (1 or 3)
  if (f.size() < 14) return false;
  r->index = (int)f[0];
  r->fixed = (int)f[1];
  for (int k = 0; k < 3; ++k) {
    r->p[k] = f[2 + k];
    r->v[k] = f[9 + k];
  }
  r->shape = (int)f[12];
  const size_t ng = r->shape == 0 ? 1 : 3;
  if (f.size() < 13 + ng) return false;
  for (int k = 0; k < 3; ++k) r->geom[k] = (size_t)k < ng ? f[13 + k] : 0.0;
  return true;
}

}  // namespace

int System::exportSystem(std::string filename) {
  std::ofstream fs(filename.c_str());
  if (!fs) return DV_ERR_ARG;
  p_h = p_d;
  v_h = v_d;
  f_contact_h = f_contact_d;
  fs << bodies.size() << ", " << 0 << ", " << 0 << ", " << 0 << ", " << std::endl;
  for (size_t i = 0; i < bodies.size(); ++i) {
    BodyRow r;
    r.index = (int)i;
    r.fixed = bodies[i]->isFixed() ? 1 : 0;
    const double3 g = bodies[i]->contactGeometry;
    r.shape = g.y == 0 ? 0 : 2;
    r.geom[0] = g.x;
    r.geom[1] = g.y;
    r.geom[2] = g.z;
    for (int k = 0; k < 3; ++k) {
      r.p[k] = p_h[3 * i + k];
      r.v[k] = v_h[3 * i + k];
    }
    write_body_row(fs, r);
  }
  return 0;
}

// Adds the file's bodies.  A sphere gets the mass the reference's importer
// gives every sphere (density 2600 and its value of pi,
// 2600 * 4 * 3.14159 * r^3 / 3 with r^3 = pow(r, 3)); a box gets mass 1.
int System::importSystem(std::string filename) {
  std::ifstream in(filename.c_str());
  if (!in) return DV_ERR_ARG;
  std::string line;
  if (!std::getline(in, line)) return DV_ERR_ARG;
  const std::vector<double> head = csv_numbers(line);
  if (head.empty()) return DV_ERR_ARG;
  const int count = (int)head[0];
  for (int i = 0; i < count; ++i) {
    BodyRow r;
    if (!std::getline(in, line) || !parse_body_row(line, &r)) return DV_ERR_ARG;
    Body* b = new Body(make_double3(r.p[0], r.p[1], r.p[2]));
    b->setBodyFixed(r.fixed != 0);
    b->setGeometry(make_double3(r.geom[0], r.geom[1], r.geom[2]));
    b->setVelocity(make_double3(r.v[0], r.v[1], r.v[2]));
    b->setMass(r.shape == 0 ? 2600 * 4.0 * 3.14159 * std::pow(r.geom[0], 3.0) / 3.0 : 1.0);
    add(b);
  }
  return 0;
}

// System.cu:1259-1295: the normal and friction force of every contact of the
// last step, gamma_n n / h and (gamma_u u + gamma_v v) / h, into
// normalForcePerCollision_h and frictionForcePerCollision_h.
int System::calculateContactForcePerCollision() {
  normalForcePerCollision_h.clear();
  frictionForcePerCollision_h.clear();
  if (!scene) return DV_ERR_ARG;
  int32_t nc = 0, np = 0;
  int rc = dv_get_num_contacts(scene, &nc, &np);
  if (rc != DV_OK) return rc;
  std::vector<double> fn(3 * (size_t)nc), ff(3 * (size_t)nc);
  if (nc && (rc = dv_contact_forces_per_collision(scene, fn.data(), ff.data())) != DV_OK) return rc;
  normalForcePerCollision_h.resize(nc);
  frictionForcePerCollision_h.resize(nc);
  for (int i = 0; i < nc; ++i) {
    normalForcePerCollision_h[i] = make_double3(fn[3 * i], fn[3 * i + 1], fn[3 * i + 2]);
    frictionForcePerCollision_h[i] = make_double3(ff[3 * i], ff[3 * i + 1], ff[3 * i + 2]);
  }
  return 0;
}

// System.cu:1672-1697
int System::outputContactForcePerCollision(std::string filename) {
  std::ofstream fs(filename.c_str());
  if (!fs || !scene) return DV_ERR_ARG;
  int rc = calculateContactForcePerCollision();
  if (rc != 0) return rc;
  const int nc = (int)normalForcePerCollision_h.size();
  std::vector<uint32_t> a(nc), b(nc);
  std::vector<double> loc(3 * (size_t)nc);
  if (nc) dv_get_contacts(scene, a.data(), b.data(), nullptr, loc.data());
  fs << nc << ", " << bodies.size() << ", " << 0 << ", " << 0 << ", " << 0 << ", " << std::endl;
  for (int i = 0; i < nc; ++i) {
    const double3 fn = normalForcePerCollision_h[i], ff = frictionForcePerCollision_h[i];
    fs << i << ", " << a[i] << ", " << b[i] << ", " << loc[3 * i] << ", " << loc[3 * i + 1] << ", "
       << loc[3 * i + 2] << ", " << fn.x << ", " << fn.y << ", " << fn.z << ", " << ff.x << ", "
       << ff.y << ", " << ff.z << ", \n";
  }
  return 0;
}

// System.cu:1297-1319: the contact forces of the last step on stdout.
int System::outputContactForcePerCollision() {
  if (!scene) return DV_ERR_ARG;
  int rc = calculateContactForcePerCollision();
  if (rc != 0) return rc;
  const int nc = (int)normalForcePerCollision_h.size();
  std::vector<uint32_t> a(nc), b(nc);
  std::vector<double> loc(3 * (size_t)nc);
  if (nc) dv_get_contacts(scene, a.data(), b.data(), nullptr, loc.data());
  for (int i = 0; i < nc; ++i) {
    const double3 fn = normalForcePerCollision_h[i], ff = frictionForcePerCollision_h[i];
    printf("Collision #%d: Body %u to %u\n", i, a[i], b[i]);
    printf("  Collision location: (%f, %f, %f)\n", loc[3 * i], loc[3 * i + 1], loc[3 * i + 2]);
    printf("  Collision normal:   (%f, %f, %f)\n", fn.x, fn.y, fn.z);
    printf("  Collision friction: (%f, %f, %f)\n\n", ff.x, ff.y, ff.z);
  }
  return 0;
}

namespace {

struct MMEntry {
  int i, j;
  double v;
};

// Matrix Market files as cusp::io::write_matrix_market_file writes them
// (coordinate for sparse matrices, array for vectors; 1-based indices);
// values with 17 significant digits.
int write_mm_coo(const std::string& path, int rows, int cols, const std::vector<MMEntry>& e) {
  FILE* f = fopen(path.c_str(), "w");
  if (!f) return DV_ERR_ARG;
  fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n\t%d\t%d\t%zu\n", rows, cols,
          e.size());
  for (const MMEntry& x : e) fprintf(f, "%d %d %.17g\n", x.i + 1, x.j + 1, x.v);
  fclose(f);
  return 0;
}

int write_mm_array(const std::string& path, const std::vector<double>& v) {
  FILE* f = fopen(path.c_str(), "w");
  if (!f) return DV_ERR_ARG;
  fprintf(f, "%%%%MatrixMarket matrix array real general\n\t%zu\t1\n", v.size());
  for (double x : v) fprintf(f, "%.17g\n", x);
  fclose(f);
  return 0;
}

}  // namespace

// System.cu:1912-1934: D, Minv, r, b and k of the last step in
// <directory>/{D,Minv,r,b,k}.mtx.  D's rows: the bilateral rows (+1 at DOF A,
// -1 at DOF B), then per contact the n, u and v rows with +F at body A's
// three columns and -F at body B's (System.cu:622-638, 676-1257).
int System::exportMatrices(std::string directory) {
  if (!scene) return DV_ERR_ARG;
  int32_t nc = 0, np = 0;
  int rc = dv_get_num_contacts(scene, &nc, &np);
  if (rc != DV_OK) return rc;
  const int nb = (int)bodies.size(), nbil = (int)bilaterals.size();
  const int rows = 3 * nc + nbil, cols = 3 * nb;
  std::vector<uint32_t> ia(nc), ib(nc);
  std::vector<double> F(9 * (size_t)nc);
  if (nc) {
    if ((rc = dv_get_contacts(scene, ia.data(), ib.data(), nullptr, nullptr)) != DV_OK) return rc;
    if ((rc = dv_get_frames(scene, F.data())) != DV_OK) return rc;
  }
  std::vector<MMEntry> D;
  D.reserve((size_t)nbil * 2 + 18 * (size_t)nc);
  for (int i = 0; i < nbil; ++i) {
    D.push_back(MMEntry{i, bilaterals[i].dofA, 1.0});
    if (bilaterals[i].dofB >= 0) D.push_back(MMEntry{i, bilaterals[i].dofB, -1.0});
  }
  for (int c = 0; c < nc; ++c)
    for (int k = 0; k < 3; ++k) {
      const int row = nbil + 3 * c + k;
      const double* f = &F[9 * (size_t)c + 3 * k];
      for (int j = 0; j < 3; ++j) D.push_back(MMEntry{row, 3 * (int)ia[c] + j, f[j]});
      for (int j = 0; j < 3; ++j) D.push_back(MMEntry{row, 3 * (int)ib[c] + j, -f[j]});
    }
  if ((rc = write_mm_coo(directory + "/D.mtx", rows, cols, D)) != 0) return rc;
  std::vector<MMEntry> M;
  for (int i = 0; i < nb; ++i) {
    const double mi = bodies[i]->isFixed() ? 0.0 : 1.0 / bodies[i]->getMass();
    for (int k = 0; k < 3; ++k) M.push_back(MMEntry{3 * i + k, 3 * i + k, mi});
  }
  if ((rc = write_mm_coo(directory + "/Minv.mtx", cols, cols, M)) != 0) return rc;
  std::vector<double> r(rows), b(rows), k(cols);
  if ((rc = dv_get_step_vectors(scene, r.data(), b.data(), k.data())) != DV_OK) return rc;
  if ((rc = write_mm_array(directory + "/r.mtx", r)) != 0) return rc;
  if ((rc = write_mm_array(directory + "/b.mtx", b)) != 0) return rc;
  return write_mm_array(directory + "/k.mtx", k);
}

int APGD::setup() { return 0; }

// Solver::solve() (APGD.cu:164-361, PGJ.cu:152-224, PGS.cu:367-459): the
// step's solve on the current state and the last collision detection's
// contacts, without the update (dv_apgd_solve); System::objectiveCCP and
// iterations as the reference sets them.
int System::solveNow() {
  if (!scene) return DV_ERR_ARG;
  int rc = sync_params();
  if (rc != DV_OK) return rc;
  rc = dv_apgd_solve(scene);
  dv_step_stats st;
  dv_get_step_stats(scene, &st);
  objectiveCCP = st.objective;
  solver->iterations = st.iterations;
  return rc;
}

int APGD::solve() { return system ? system->solveNow() : DV_ERR_ARG; }
int PGJ::setup() { return 0; }
int PGJ::solve() { return system ? system->solveNow() : DV_ERR_ARG; }
int PGS::setup() { return 0; }
int PGS::solve() { return system ? system->solveNow() : DV_ERR_ARG; }

int CollisionDetector::setEnvelope(double e) {
  envelope = e;
  return 0;
}

int CollisionDetector::detectCollisions() {
  if (!system->scene) return DV_ERR_ARG;
  int rc = dv_collide(system->scene);
  int32_t nc = 0, np = 0;
  dv_get_num_contacts(system->scene, &nc, &np);
  numCollisions = (uint)nc;
  numPossibleCollisions = (uint)np;
  return rc;
}

std::vector<uint32_t> CollisionDetector::getCollisionIdentifierA() {
  std::vector<uint32_t> a(numCollisions);
  if (numCollisions) dv_get_contacts(system->scene, a.data(), nullptr, nullptr, nullptr);
  return a;
}

std::vector<uint32_t> CollisionDetector::getCollisionIdentifierB() {
  std::vector<uint32_t> b(numCollisions);
  if (numCollisions) dv_get_contacts(system->scene, nullptr, b.data(), nullptr, nullptr);
  return b;
}

std::vector<double3> CollisionDetector::getCollisionLocations() {
  std::vector<double> raw(3 * (size_t)numCollisions);
  if (numCollisions) dv_get_contacts(system->scene, nullptr, nullptr, nullptr, raw.data());
  std::vector<double3> out(numCollisions);
  for (uint i = 0; i < numCollisions; ++i)
    out[i] = make_double3(raw[3 * i], raw[3 * i + 1], raw[3 * i + 2]);
  return out;
}

ContactIdArray::operator std::vector<uint>() const {
  std::vector<uint32_t> v = b_ ? cd_->getCollisionIdentifierB() : cd_->getCollisionIdentifierA();
  return std::vector<uint>(v.begin(), v.end());
}
size_t ContactIdArray::size() const { return cd_->numCollisions; }
uint ContactIdArray::operator[](size_t i) const {
  return static_cast<std::vector<uint>>(*this).at(i);
}

ContactLocationArray::operator std::vector<double3>() const { return cd_->getCollisionLocations(); }
size_t ContactLocationArray::size() const { return cd_->numCollisions; }
double3 ContactLocationArray::operator[](size_t i) const {
  return cd_->getCollisionLocations().at(i);
}

std::vector<double4> CollisionDetector::getNormalsAndPenetrations() {
  std::vector<double> raw(4 * (size_t)numCollisions);
  if (numCollisions) dv_get_contacts(system->scene, nullptr, nullptr, raw.data(), nullptr);
  std::vector<double4> out(numCollisions);
  for (uint i = 0; i < numCollisions; ++i)
    out[i] = make_double4(raw[4 * i], raw[4 * i + 1], raw[4 * i + 2], raw[4 * i + 3]);
  return out;
}

// CollisionDetector.cu:665-711
int CollisionDetector::exportSystem(std::string filename) {
  std::ofstream fs(filename.c_str());
  if (!fs || !system->scene) return DV_ERR_ARG;
  std::vector<uint32_t> A = getCollisionIdentifierA(), B = getCollisionIdentifierB();
  std::vector<double4> nP = getNormalsAndPenetrations();
  std::vector<double> p = system->p_d, v = system->v_d;
  for (uint i = 0; i < numCollisions; ++i) {
    double3 ga = system->bodies[A[i]]->getGeometry(), gb = system->bodies[B[i]]->getGeometry();
    fs << i << ", " << A[i] << ", " << B[i] << ", " << nP[i].x << ", " << nP[i].y << ", "
       << nP[i].z << ", " << nP[i].w << ", " << p[3 * A[i]] << ", " << p[3 * A[i] + 1] << ", "
       << p[3 * A[i] + 2] << ", " << v[3 * A[i]] << ", " << v[3 * A[i] + 1] << ", "
       << v[3 * A[i] + 2] << ", " << ga.x << ", " << ga.y << ", " << ga.z << ", " << p[3 * B[i]]
       << ", " << p[3 * B[i] + 1] << ", " << p[3 * B[i] + 2] << ", " << v[3 * B[i]] << ", "
       << v[3 * B[i] + 1] << ", " << v[3 * B[i] + 2] << ", " << gb.x << ", " << gb.y << ", "
       << gb.z << ", " << "\n";
  }
  return 0;
}
