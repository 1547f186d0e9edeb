/*
 * dv_oracle.cpp -- CPU restatement of DVIDE's rigid-body frictional-contact
 * time step (sphere + fixed/dynamic box bodies, APGD solver).
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg, never by the product library.
 *
 * PARITY UNPINNED against the reference binary: melanz/DVIDE cannot be built
 * here (CUSP headers absent) and ships no golden vectors.  This file follows
 * the reference source, cited by file:line (paths relative to the DVIDE tree):
 *   state layout ........ src/System.cu:342-424 (p, v, f = m g, Minv = 1/m, 0 if fixed)
 *   time step ........... src/System.cu:544-583 (DoTimeStep)
 *   applied impulse ..... src/System.cu:1411-1417, 1502-1514 (k = M v + h f)
 *   Jacobian frame ...... src/System.cu:753-762, body branches :905-1203
 *   Schur vector ........ src/System.cu:1516-1524, 1561-1580 (r = D Minv k + b)
 *   CCP violation ....... src/System.cu:1590-1643
 *   AABBs / bins ........ src/CollisionDetector.cu:10-110, 547-631
 *   narrowphase ......... src/CollisionDetector.cu:187-501
 *   APGD ................ src/APGD.cu:6-361
 *   vector helpers ...... src/helper_math_double.h:58-61, 555-605, 689-697
 *                         (length = float sqrtf, normalize = float 1/sqrtf)
 * Third-party arithmetic: CUSP (version unpinned, CMakeLists.txt:28) supplies
 * COO SpMV and BLAS-1 in the reference; each call is restated from its
 * definition (multiply: y = A x; axpby: z = a x + b y; axpy: y = a x + y;
 * axpbypcz: w = a x + b y + c z; nrm2 = sqrt(sum x^2); nrmmax = max |x|).
 *
 * Floating-point conventions shared bit-for-bit with the CUDA kernels:
 *  - built with -ffp-contract=off: no fused multiply-add anywhere;
 *  - pow(x, 2.0) is evaluated as x*x;
 *  - reductions (dot, nrm2) use one fixed tiled order, ordered_sum() below,
 *    which the GPU reproduces exactly (reduce_mode 0).  reduce_mode 1 sums
 *    sequentially like CUSP's host backend; spmv_mode 1 applies D and D^T in
 *    literal COO entry order.  Tests use modes 1/1 to show that the choice of
 *    summation order moves results far less than the 1e-10 parity bar.
 *  - the matrix-free product groups D^T x per contact, q_c = F_c x_c with
 *    q_k = (n_k x0 + u_k x1) + v_k x2, then sums +-q_c over a body's contacts
 *    in ascending contact order; D w is n.(w_A - w_B) = (n_x d_x + n_y d_y) + n_z d_z.
 */
#include "dv_oracle.h"

#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

// The bin sort of the collision pass runs on Thrust's OpenMP backend where
// the CUDA toolkit's headers are on the include path (the reference sorts
// with Thrust: CollisionDetector.cu:583-590), else with std::sort; the sorted
// order is the same either way.
#if defined(_OPENMP) && defined(__has_include)
#if __has_include(<thrust/sort.h>)
#define DV_ORACLE_THRUST_OMP 1
#include <thrust/sort.h>
#include <thrust/system/omp/execution_policy.h>
#endif
#endif

namespace {

struct V3 {
  double x, y, z;
};

inline V3 mk(double x, double y, double z) { return V3{x, y, z}; }
inline V3 add(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 sub(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 scale(V3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
inline V3 neg(V3 a) { return mk(-a.x, -a.y, -a.z); }

/* helper_math_double.h:559-562 */
inline double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* helper_math_double.h:576-579 with the host sqrtf (float) */
inline double length3(V3 a) { return (double)sqrtf((float)dot3(a, a)); }
/* helper_math_double.h:594-597 with the host rsqrtf = 1.0f / sqrtf(x) (:58-61) */
inline V3 normalize3(V3 a) {
  double inv = (double)(1.0f / sqrtf((float)dot3(a, a)));
  return scale(a, inv);
}
/* The opt-in FP64 forms (not the reference's semantics): double sqrt, then
 * 1 / length and a scale, as normalize3 does in float. */
inline double length3x(V3 a, bool exact) { return exact ? std::sqrt(dot3(a, a)) : length3(a); }
inline V3 normalize3x(V3 a, bool exact) {
  if (!exact) return normalize3(a);
  double inv = 1.0 / std::sqrt(dot3(a, a));
  return scale(a, inv);
}
/* helper_math_double.h:692-695 */
inline V3 cross3(V3 a, V3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

/* ---------------------------------------------------------------------
 * Ordered reduction shared with the GPU.
 * Items are grouped in tiles of 512.  In tile t, slot j (0..255) sums
 * items 512t + j + 256m for m = 0..1, starting from 0.0; the 256 slots are
 * folded as 8 warps of 32 by halving strides 16,8,4,2,1 (slot l += slot
 * l+off), then the 8 warp results by strides 4,2,1.  The tile partials are
 * folded the same way: slot j sums tiles j, j+256, ... then the 256-tree.
 * ------------------------------------------------------------------- */
double tree256(double* s) {
  double W[8];
  for (int w = 0; w < 8; ++w) {
    double* a = s + 32 * w;
    for (int off = 16; off >= 1; off >>= 1)
      for (int l = 0; l < off; ++l) a[l] = a[l] + a[l + off];
    W[w] = a[0];
  }
  for (int off = 4; off >= 1; off >>= 1)
    for (int l = 0; l < off; ++l) W[l] = W[l] + W[l + off];
  return W[0];
}

/* Partials of the tiles of n items, appended to P. */
void tile_partials(const double* v, int64_t n, std::vector<double>& P) {
  if (n <= 0) return;
  const int64_t T = (n + 511) / 512, base = (int64_t)P.size();
  P.resize(base + T);
#pragma omp parallel for schedule(static)
  for (int64_t t = 0; t < T; ++t) {
    double s[256];
    for (int j = 0; j < 256; ++j) {
      double acc = 0.0;
      for (int m = 0; m < 2; ++m) {
        int64_t i = 512 * t + j + 256 * m;
        if (i < n) acc = acc + v[i];
      }
      s[j] = acc;
    }
    P[base + t] = tree256(s);
  }
}

double fold_partials(const std::vector<double>& P) {
  const int64_t T = (int64_t)P.size();
  double a[256];
  for (int j = 0; j < 256; ++j) {
    double acc = 0.0;
    for (int64_t t = j; t < T; t += 256) acc = acc + P[t];
    a[j] = acc;
  }
  return tree256(a);
}

double ordered_sum(const double* v, int64_t n) {
  if (n <= 0) return 0.0;
  std::vector<double> P;
  tile_partials(v, n, P);
  return fold_partials(P);
}

/* Two item lists whose tiles are folded as one list: the contacts' tiles,
 * then the tiles of the bilateral rows (a scene's tile range on the GPU). */
double ordered_sum2(const double* v, int64_t n, const double* w, int64_t m) {
  if (n <= 0 && m <= 0) return 0.0;
  std::vector<double> P;
  tile_partials(v, n, P);
  tile_partials(w, m, P);
  return fold_partials(P);
}

/* APGD.cu:47-78, friction-cone projection of one contact impulse. */
inline void project3(double* g, double mu) {
  double gn = g[0];
  double gt = sqrt(g[1] * g[1] + g[2] * g[2]);
  double o0, o1, o2;
  if (mu == 0) {
    o0 = gn; o1 = 0; o2 = 0;
    if (gn < 0) { o0 = 0; o1 = 0; o2 = 0; }
  } else if (gt < mu * gn) {
    return;
  } else if ((gt < -(1.0 / mu) * gn) || (fabs(gn) < 10e-15)) {
    o0 = 0; o1 = 0; o2 = 0;
  } else {
    double gnp = (gt * mu + gn) / (mu * mu + 1.0);
    double gtp = gnp * mu;
    double ratio = gtp / gt;
    o0 = gnp; o1 = ratio * g[1]; o2 = ratio * g[2];
  }
  g[0] = o0; g[1] = o1; g[2] = o2;
}

/* System.cu:753-762, tangent frame from the stored normal. */
inline void frame_from_normal(V3 n, V3* u, V3* v, bool exact = false) {
  V3 uu;
  if (n.z != 0) {
    uu = normalize3x(mk(1, 0, -n.x / n.z), exact);
  } else if (n.x != 0) {
    uu = normalize3x(mk(-n.z / n.x, 0, 1), exact);
  } else {
    uu = normalize3x(mk(1, -n.x / n.y, 0), exact);
  }
  *u = uu;
  *v = normalize3x(cross3(n, uu), exact);
}

struct Scene {
  or_params P;
  int nb = 0;
  std::vector<double> p, v, minv, f, k, fcont, geom;
  std::vector<int> fixed, family;
  /* contacts (sorted by (A, B)) */
  int nc = 0, npossible = 0;
  std::vector<uint32_t> A, B;
  std::vector<double> nP, loc, F, r, bst;
  std::vector<double> gamma;  // warm-start buffer, 3 * capacity
  int gsize = 0;              // contacts currently held (System.cu:185 starts at nb)
  /* warm_start 2: the (A, B) pairs the held gamma belongs to (sorted) */
  std::vector<uint32_t> wA, wB;
  /* body incidence, ascending contact order, sign +1 = body A */
  std::vector<int> incStart, incC;
  std::vector<signed char> incS;
  /* bilateral DOF constraints (System.cu:510-532, 622-638, 1526-1544): one
   * scalar row each, +1 at DOF A and -1 at DOF B (B < 0: DOF A alone).  The
   * reference puts these rows ahead of the contacts; every solve vector here
   * holds the contacts' 3 nc entries, then the nbil bilateral entries. */
  int nbil = 0;
  std::vector<int> bilA, bilB;
  std::vector<double> bilVel, bilT0, bilP0;  // infoConstraintBilateralDOF (x, y, z)
  std::vector<double> gammaB;                // bilateral impulses of the last solve (0 before)
  std::vector<double> bB;                    // b of the bilateral rows at the last step
  /* per body, its bilateral entries in ascending row order (A before B):
   * (row << 3) | (axis << 1) | (1 for the -1 entry of DOF B) */
  std::vector<int> bincStart, binc;
  or_stats st;
  double time = 0;
  int timeIndex = 0;
};

/* ------------------------------ reductions ------------------------------ */
/* x . y over a solve vector (contacts, then bilateral rows): one item per
 * contact and one per bilateral row, the contacts' tiles first. */
double dotv(const Scene& S, const double* x, const double* y, int nc) {
  const int nbil = S.nbil;
  const double* xb = x + 3 * (int64_t)nc;
  const double* yb = y + 3 * (int64_t)nc;
  if (S.P.reduce_mode == 1) {
    /* the flat order of the reference's vectors: bilateral rows first */
    double s = 0.0;
    for (int i = 0; i < nbil; ++i) s = s + xb[i] * yb[i];
    for (int64_t i = 0; i < 3 * (int64_t)nc; ++i) s = s + x[i] * y[i];
    return s;
  }
  std::vector<double> it(nc), itb(nbil);
#pragma omp parallel for schedule(static)
  for (int c = 0; c < nc; ++c) {
    const double* a = x + 3 * c;
    const double* b = y + 3 * c;
    it[c] = (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
  }
  for (int i = 0; i < nbil; ++i) itb[i] = xb[i] * yb[i];
  return ordered_sum2(it.data(), nc, itb.data(), nbil);
}

double nrm2v(const Scene& S, const double* x, int nc) { return sqrt(dotv(S, x, x, nc)); }

double nrmmaxv(const Scene& S, const double* x, int nc, int* nan_flag) {
  double m = 0.0;
  for (int64_t i = 0; i < 3 * (int64_t)nc + S.nbil; ++i) {
    double a = fabs(x[i]);
    if (a != a) *nan_flag = 1;
    if (a > m) m = a;
  }
  return m;
}

/* ------------------------------ collision ------------------------------- */
struct AabbSet {
  std::vector<V3> mn, mx;  // shifted by the global origin (CollisionDetector.cu:574)
};

inline bool is_sphere(const Scene& S, int i) { return S.geom[3 * i + 1] == 0; }

/* CollisionDetector.cu:24-79 (rigid-body branch) and :555-576. */
void build_aabbs(const Scene& S, AabbSet& a) {
  int nb = S.nb;
  a.mn.resize(nb);
  a.mx.resize(nb);
  double env = S.P.envelope;
  for (int i = 0; i < nb; ++i) {
    V3 g = mk(S.geom[3 * i], S.geom[3 * i + 1], S.geom[3 * i + 2]);
    if (g.y == 0) g = mk(g.x, g.x, g.x);
    g = add(g, mk(env, env, env));
    V3 pos = mk(S.p[3 * i], S.p[3 * i + 1], S.p[3 * i + 2]);
    a.mn[i] = sub(pos, g);
    a.mx[i] = add(pos, g);
  }
  if (nb == 0) return;
  V3 lo = a.mn[0], hi = a.mn[0];
  for (int pass = 0; pass < 2; ++pass) {
    const std::vector<V3>& pts = pass ? a.mx : a.mn;
    for (int i = 0; i < nb; ++i) {
      lo = mk(fmin(lo.x, pts[i].x), fmin(lo.y, pts[i].y), fmin(lo.z, pts[i].z));
      hi = mk(fmax(hi.x, pts[i].x), fmax(hi.y, pts[i].y), fmax(hi.z, pts[i].z));
    }
  }
  V3 origin = sub(lo, mk(0.01, 0.01, 0.01));
  for (int i = 0; i < nb; ++i) {
    a.mn[i] = sub(a.mn[i], origin);
    a.mx[i] = sub(a.mx[i], origin);
  }
}

/* CollisionDetector.cu:112-178: overlap on shifted boxes, identity and family filters. */
inline bool candidate(const Scene& S, const AabbSet& a, int i, int j) {
  const V3 &Amn = a.mn[i], &Amx = a.mx[i], &Bmn = a.mn[j], &Bmx = a.mx[j];
  bool in = (Amn.x <= Bmx.x && Bmn.x <= Amx.x) && (Amn.y <= Bmx.y && Bmn.y <= Amx.y) &&
            (Amn.z <= Bmx.z && Bmn.z <= Amx.z);
  if (i == j) in = false;
  int fa = S.family[i], fb = S.family[j];
  if (fa == fb && fa != -1) in = false;
  return in;
}

struct ContactOut {
  uint32_t b;
  V3 nstored;  // -normal (B -> A)
  double gap;  // -penetration
  V3 loc;
};

/* CollisionDetector.cu:187-331 (count) and :333-501 (store), rigid bodies. */
bool narrowphase(const Scene& S, int ia, int ib, double env, ContactOut* out) {
  V3 posA = mk(S.p[3 * ia], S.p[3 * ia + 1], S.p[3 * ia + 2]);
  V3 posB = mk(S.p[3 * ib], S.p[3 * ib + 1], S.p[3 * ib + 2]);
  V3 gA = mk(S.geom[3 * ia], S.geom[3 * ia + 1], S.geom[3 * ia + 2]);
  V3 gB = mk(S.geom[3 * ib], S.geom[3 * ib + 1], S.geom[3 * ib + 2]);
  const bool exact = S.P.fp64_narrowphase != 0;
  double pen;
  V3 normal, location;
  if (gA.y == 0 && gB.y == 0) {
    V3 d = sub(posB, posA);
    pen = (gA.x + gB.x) - length3x(d, exact);
    if (!(pen >= -env)) return false;
    normal = normalize3x(d, exact);
    location = add(posA, scale(normal, gA.x));
  } else if ((gA.y != 0 && gB.y == 0) || (gA.y == 0 && gB.y != 0)) {
    double dmin = 0;
    double r = gB.x;
    V3 center = posB;
    V3 bmin = sub(posA, gA);
    V3 bmax = add(posA, gA);
    bool sphereA = (gA.y == 0 && gB.y != 0);
    if (sphereA) {
      r = gA.x;
      center = posA;
      bmin = sub(posB, gB);
      bmax = add(posB, gB);
    }
    V3 nrm = mk(0, 0, 0);
    double t;
    if (center.x < bmin.x) { t = center.x - bmin.x; dmin += t * t; nrm.x = nrm.x + t; }
    else if (center.x > bmax.x) { t = center.x - bmax.x; dmin += t * t; nrm.x = nrm.x + t; }
    if (center.y < bmin.y) { t = center.y - bmin.y; dmin += t * t; nrm.y = nrm.y + t; }
    else if (center.y > bmax.y) { t = center.y - bmax.y; dmin += t * t; nrm.y = nrm.y + t; }
    if (center.z < bmin.z) { t = center.z - bmin.z; dmin += t * t; nrm.z = nrm.z + t; }
    else if (center.z > bmax.z) { t = center.z - bmax.z; dmin += t * t; nrm.z = nrm.z + t; }
    pen = r - sqrt(dmin);
    if (!(pen >= -env)) return false;
    normal = normalize3x(nrm, exact);
    location = sub(center, scale(normal, r));
    if (sphereA) normal = neg(normal);
  } else {
    return false;  // box-box is never a contact
  }
  out->b = (uint32_t)ib;
  out->nstored = neg(normal);
  out->gap = -pen;
  out->loc = location;
  return true;
}

void collide(Scene& S) {
  int nb = S.nb;
  AabbSet a;
  build_aabbs(S, a);
  double env = S.P.envelope;

  /* Spheres go in a uniform grid keyed on their shifted AABB min corner with
   * cell size above the largest sphere box; boxes are tested against all
   * bodies.  The candidate set is exactly the AABB-overlap set of
   * CollisionDetector.cu:112-178, which does not depend on the binning. */
  std::vector<int> small, large;
  double W = 0;
  for (int i = 0; i < nb; ++i) {
    if (is_sphere(S, i)) {
      small.push_back(i);
      W = std::max(W, a.mx[i].x - a.mn[i].x);
      W = std::max(W, a.mx[i].y - a.mn[i].y);
      W = std::max(W, a.mx[i].z - a.mn[i].z);
    } else {
      large.push_back(i);
    }
  }
  double w = W * (1.0 + 1e-7) + 1e-300;
  std::vector<int64_t> ckey(nb, -1);
  std::vector<int> cx(nb), cy(nb), cz(nb);
  int mxc[3] = {0, 0, 0};
  for (int i : small) {
    cx[i] = (int)floor(a.mn[i].x / w);
    cy[i] = (int)floor(a.mn[i].y / w);
    cz[i] = (int)floor(a.mn[i].z / w);
    mxc[0] = std::max(mxc[0], cx[i]);
    mxc[1] = std::max(mxc[1], cy[i]);
    mxc[2] = std::max(mxc[2], cz[i]);
  }
  int64_t D0 = mxc[0] + 1, D1 = mxc[1] + 1;
  std::vector<std::pair<int64_t, int>> cells;
  cells.reserve(small.size());
  for (int i : small) {
    ckey[i] = cx[i] + D0 * (cy[i] + D1 * (int64_t)cz[i]);
    cells.push_back(std::make_pair(ckey[i], i));
  }
#ifdef DV_ORACLE_THRUST_OMP
  {
    // (cell, body) order: a stable sort by cell of bodies in ascending id
    std::vector<int64_t> keys(cells.size());
    std::vector<int> ids(cells.size());
    for (size_t k = 0; k < cells.size(); ++k) {
      keys[k] = cells[k].first;
      ids[k] = cells[k].second;
    }
    thrust::stable_sort_by_key(thrust::omp::par, keys.data(), keys.data() + keys.size(), ids.data());
    for (size_t k = 0; k < cells.size(); ++k) cells[k] = std::make_pair(keys[k], ids[k]);
  }
#else
  std::sort(cells.begin(), cells.end());
#endif

  std::vector<std::vector<ContactOut>> per(nb);
  std::vector<int> ncand(nb, 0);
#pragma omp parallel for schedule(dynamic, 64)
  for (int ia = 0; ia < nb; ++ia) {
    std::vector<int> cand;
    if (is_sphere(S, ia)) {
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int x = cx[ia] + dx, y = cy[ia] + dy, z = cz[ia] + dz;
            if (x < 0 || y < 0 || z < 0 || x >= D0 || y >= D1) continue;
            int64_t key = x + D0 * (y + D1 * (int64_t)z);
            auto it = std::lower_bound(cells.begin(), cells.end(), std::make_pair(key, -1));
            for (; it != cells.end() && it->first == key; ++it) {
              int jb = it->second;
              if (jb > ia && candidate(S, a, ia, jb)) cand.push_back(jb);
            }
          }
      for (int jb : large)
        if (jb > ia && candidate(S, a, ia, jb)) cand.push_back(jb);
    } else {
      for (int jb = ia + 1; jb < nb; ++jb)
        if (candidate(S, a, ia, jb)) cand.push_back(jb);
    }
    std::sort(cand.begin(), cand.end());
    ncand[ia] = (int)cand.size();
    for (int jb : cand) {
      ContactOut o;
      if (narrowphase(S, ia, jb, env, &o)) per[ia].push_back(o);
    }
  }
  int64_t np = 0, nc = 0;
  for (int i = 0; i < nb; ++i) {
    np += ncand[i];
    nc += (int64_t)per[i].size();
  }
  S.npossible = (int)np;
  S.nc = (int)nc;
  S.A.resize(nc);
  S.B.resize(nc);
  S.nP.resize(4 * nc);
  S.loc.resize(3 * nc);
  int64_t c = 0;
  for (int ia = 0; ia < nb; ++ia)
    for (const ContactOut& o : per[ia]) {
      S.A[c] = (uint32_t)ia;
      S.B[c] = o.b;
      S.nP[4 * c + 0] = o.nstored.x;
      S.nP[4 * c + 1] = o.nstored.y;
      S.nP[4 * c + 2] = o.nstored.z;
      S.nP[4 * c + 3] = o.gap;
      S.loc[3 * c + 0] = o.loc.x;
      S.loc[3 * c + 1] = o.loc.y;
      S.loc[3 * c + 2] = o.loc.z;
      ++c;
    }
  S.st.num_contacts = S.nc;
  S.st.num_possible = S.npossible;
}

/* System.cu:676-1257 (rigid-body branches): frames, b = gap / h (:1516-1524). */
void build_frames(Scene& S) {
  int nc = S.nc;
  S.F.resize(9 * (size_t)nc);
  S.bst.resize(3 * (size_t)nc);
#pragma omp parallel for schedule(static)
  for (int c = 0; c < nc; ++c) {
    V3 n = mk(S.nP[4 * c], S.nP[4 * c + 1], S.nP[4 * c + 2]);
    V3 u, v;
    frame_from_normal(n, &u, &v, S.P.fp64_narrowphase != 0);
    double* F = &S.F[9 * (size_t)c];
    F[0] = n.x; F[1] = n.y; F[2] = n.z;
    F[3] = u.x; F[4] = u.y; F[5] = u.z;
    F[6] = v.x; F[7] = v.y; F[8] = v.z;
    S.bst[3 * c + 0] = S.nP[4 * c + 3] / S.P.h;
    S.bst[3 * c + 1] = 0;
    S.bst[3 * c + 2] = 0;
  }
  /* incidence in ascending contact order (the row order of sort_by_row(D^T),
   * System.cu:1388-1409) */
  int nb = S.nb;
  std::vector<int> cnt(nb + 1, 0);
  for (int c = 0; c < nc; ++c) {
    cnt[S.A[c] + 1]++;
    cnt[S.B[c] + 1]++;
  }
  for (int i = 0; i < nb; ++i) cnt[i + 1] += cnt[i];
  S.incStart = cnt;
  S.incC.assign(2 * (size_t)nc, 0);
  S.incS.assign(2 * (size_t)nc, 0);
  std::vector<int> pos(cnt.begin(), cnt.end() - 1);
  for (int c = 0; c < nc; ++c) {
    int b = S.B[c], a = S.A[c];
    S.incC[pos[b]] = c; S.incS[pos[b]] = -1; pos[b]++;
    S.incC[pos[a]] = c; S.incS[pos[a]] = +1; pos[a]++;
  }
}

/* The bilateral rows' part of (D^T x)_b, added after the contacts' part:
 * +x_i at DOF A, -x_i at DOF B of row i (System.cu:622-638), ascending rows. */
inline void add_bilateral_DT(const Scene& S, const double* x, int b, double* acc) {
  if (!S.nbil) return;
  const double* xb = x + 3 * (int64_t)S.nc;
  for (int e = S.bincStart[b]; e < S.bincStart[b + 1]; ++e) {
    const int code = S.binc[e];
    const int row = code >> 3, k = (code >> 1) & 3;
    if (code & 1) acc[k] = acc[k] - xb[row];
    else acc[k] = acc[k] + xb[row];
  }
}

/* The bilateral rows of D w: w[A] - w[B], or w[A]. */
inline void bilateral_D(const Scene& S, const double* w, double* out) {
  for (int i = 0; i < S.nbil; ++i)
    out[i] = S.bilB[i] >= 0 ? w[S.bilA[i]] - w[S.bilB[i]] : w[S.bilA[i]];
}

/* D^T x (one value per body DOF). */
void apply_DT(const Scene& S, const double* x, double* out) {
  int nb = S.nb;
  if (S.P.spmv_mode == 1) {
#pragma omp parallel for schedule(static)
    for (int b = 0; b < nb; ++b) {
      for (int k = 0; k < 3; ++k) {
        double y = 0.0;
        for (int e = S.incStart[b]; e < S.incStart[b + 1]; ++e) {
          int c = S.incC[e];
          double s = S.incS[e];
          const double* F = &S.F[9 * (size_t)c];
          y = y + (s * F[k]) * x[3 * c];
          y = y + (s * F[3 + k]) * x[3 * c + 1];
          y = y + (s * F[6 + k]) * x[3 * c + 2];
        }
        out[3 * b + k] = y;
      }
      add_bilateral_DT(S, x, b, &out[3 * b]);
    }
    return;
  }
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; ++b) {
    double acc[3] = {0.0, 0.0, 0.0};
    for (int e = S.incStart[b]; e < S.incStart[b + 1]; ++e) {
      int c = S.incC[e];
      const double* F = &S.F[9 * (size_t)c];
      const double* xc = x + 3 * c;
      for (int k = 0; k < 3; ++k) {
        double q = (F[k] * xc[0] + F[3 + k] * xc[1]) + F[6 + k] * xc[2];
        if (S.incS[e] > 0) acc[k] = acc[k] + q;
        else acc[k] = acc[k] - q;
      }
    }
    add_bilateral_DT(S, x, b, acc);
    out[3 * b] = acc[0];
    out[3 * b + 1] = acc[1];
    out[3 * b + 2] = acc[2];
  }
}

/* D w (one value per contact row). */
void apply_D(const Scene& S, const double* w, double* out) {
  int nc = S.nc;
  if (S.P.spmv_mode == 1) {
#pragma omp parallel for schedule(static)
    for (int c = 0; c < nc; ++c) {
      const double* F = &S.F[9 * (size_t)c];
      const double* wa = w + 3 * (size_t)S.A[c];
      const double* wb = w + 3 * (size_t)S.B[c];
      for (int row = 0; row < 3; ++row) {
        const double* f = F + 3 * row;
        double y = 0.0;
        y = y + f[0] * wa[0];
        y = y + f[1] * wa[1];
        y = y + f[2] * wa[2];
        y = y + (-f[0]) * wb[0];
        y = y + (-f[1]) * wb[1];
        y = y + (-f[2]) * wb[2];
        out[3 * c + row] = y;
      }
    }
    bilateral_D(S, w, out + 3 * (int64_t)nc);
    return;
  }
#pragma omp parallel for schedule(static)
  for (int c = 0; c < nc; ++c) {
    const double* F = &S.F[9 * (size_t)c];
    const double* wa = w + 3 * (size_t)S.A[c];
    const double* wb = w + 3 * (size_t)S.B[c];
    double d0 = wa[0] - wb[0], d1 = wa[1] - wb[1], d2 = wa[2] - wb[2];
    for (int row = 0; row < 3; ++row) {
      const double* f = F + 3 * row;
      out[3 * c + row] = (f[0] * d0 + f[1] * d1) + f[2] * d2;
    }
  }
  bilateral_D(S, w, out + 3 * (int64_t)nc);
}

/* APGD.cu:81-87: gammaTmp = D (Minv (D^T x)). */
void schur(const Scene& S, const double* x, double* out, std::vector<double>& bodytmp) {
  bodytmp.resize(3 * (size_t)S.nb);
  apply_DT(S, x, bodytmp.data());
  for (size_t i = 0; i < bodytmp.size(); ++i) bodytmp[i] = S.minv[i] * bodytmp[i];
  apply_D(S, bodytmp.data(), out);
}

/* APGD.cu:90-102 with N src already available.  gdiff = 1 / (nc + nbil)^2
 * (:92); without contacts the reference skips the projection and both axpby
 * (:96-100), and the residual is max |N src + r|. */
double residual_from(const Scene& S, const double* src, const double* Nsrc, std::vector<double>& T,
                     int* nan_flag) {
  const int nc = S.nc;
  const int64_t n = 3 * (int64_t)nc + S.nbil;
  const double m = (double)(nc + S.nbil);
  double gdiff = 1.0 / (m * m);
  for (int64_t i = 0; i < n; ++i) T[i] = S.r[i] + Nsrc[i];
  if (nc) {
    for (int64_t i = 0; i < n; ++i) T[i] = src[i] + (-gdiff) * T[i];
    for (int c = 0; c < nc; ++c) project3(&T[3 * c], S.P.mu);
    double a = 1.0 / gdiff, b = -1.0 / gdiff;
    for (int64_t i = 0; i < n; ++i) T[i] = a * src[i] + b * T[i];
  }
  return nrmmaxv(S, T.data(), nc, nan_flag);
}

/* APGD.cu:90-102 */
double get_residual(const Scene& S, const double* src, std::vector<double>& T,
                    std::vector<double>& bt, int* nan_flag) {
  std::vector<double> N(3 * (size_t)S.nc + S.nbil);
  schur(S, src, N.data(), bt);
  return residual_from(S, src, N.data(), T, nan_flag);
}

/* warm_start 2 (an opt-in improvement over the reference, not parity
 * mode): every contact starts from the impulse the same (A, B) pair had at the
 * last solve, a new pair from zero. */
void match_gamma(Scene& S) {
  const int nc = S.nc;
  const int64_t n3 = 3 * (int64_t)nc;
  std::vector<double> g(n3, 0.0);
  const size_t m = S.wA.size();
  for (int c = 0; c < nc; ++c) {
    size_t lo = 0, hi = m;
    const uint32_t a = S.A[c], b = S.B[c];
    while (lo < hi) {  // first held pair >= (a, b)
      const size_t mid = (lo + hi) / 2;
      if (S.wA[mid] < a || (S.wA[mid] == a && S.wB[mid] < b)) lo = mid + 1;
      else hi = mid;
    }
    if (lo < m && S.wA[lo] == a && S.wB[lo] == b && (int64_t)lo < S.gsize)
      for (int k = 0; k < 3; ++k) g[3 * c + k] = S.gamma[3 * lo + k];
  }
  if ((int64_t)S.gamma.size() < n3) S.gamma.resize(n3, 0.0);
  for (int64_t i = 0; i < n3; ++i) S.gamma[i] = g[i];
  S.gsize = nc;
}

// the pairs the solved gamma belongs to
void keep_pairs(Scene& S) {
  S.wA = S.A;
  S.wB = S.B;
  S.wA.resize(S.nc);
  S.wB.resize(S.nc);
}

void resize_gamma(Scene& S) {
  int nc = S.nc;
  int64_t n3 = 3 * (int64_t)nc;
  if (S.P.warm_start == 2) {
    match_gamma(S);
    return;
  }
  /* thrust resize keeps the prefix and zero-fills growth (APGD.cu:166). */
  if ((int64_t)S.gamma.size() < n3) S.gamma.resize(n3, 0.0);
  if (S.gsize < nc)
    for (int64_t i = 3 * (int64_t)S.gsize; i < n3; ++i) S.gamma[i] = 0.0;
  S.gsize = nc;
  if (!S.P.warm_start && S.nbil == 0) {
    for (int c = 0; c < nc; ++c) {
      S.gamma[3 * c] = 1.0;
      S.gamma[3 * c + 1] = 0.0;
      S.gamma[3 * c + 2] = 0.0;
    }
  } else if (!S.P.warm_start) {
    /* initializeImpulseVector_APGD (APGD.cu:114-120, called at :200) writes
     * (1, 0, 0) to flat entries 0 .. 3 nc - 1 of the vector whose first nbil
     * entries are the bilateral rows (no offset): flat entry j < 3 nc takes
     * 1 if j is a multiple of 3, else 0; entries from 3 nc on keep what the
     * resize kept (the last solve's value at that position, or 0). */
    const int64_t lim = 3 * (int64_t)nc;
    for (int i = 0; i < S.nbil; ++i)
      if (i < lim) S.gammaB[i] = (i % 3 == 0) ? 1.0 : 0.0;
    for (int64_t j = 0; j < n3; ++j) {
      const int64_t f = S.nbil + j;
      if (f < lim) S.gamma[j] = (f % 3 == 0) ? 1.0 : 0.0;
    }
  }
}

/* APGD.cu:335-345, the anti-relaxation block at the end of an iteration that
 * did not converge, with gamma the new iterate: r -= ar; v = Minv (k + D^T
 * gamma); ar_c = (sqrt(s_u^2 + s_v^2) mu, 0, 0) with s = (D v)_c
 * (updateAntiRelaxationVector, :104-112); r += ar.  Contacts only (the
 * reference indexes ar without the bilateral rows' offset). */
void anti_relax(Scene& S, const double* gamma, std::vector<double>& ar) {
  const int nc = S.nc, nb = S.nb;
  const int64_t n3 = 3 * (int64_t)nc;
  for (int64_t i = 0; i < n3; ++i) S.r[i] = (-1.0 * ar[i]) + S.r[i];
  std::vector<double> fc(3 * (size_t)nb), v(3 * (size_t)nb), dv(n3);
  apply_DT(S, gamma, fc.data());
  for (int i = 0; i < 3 * nb; ++i) {
    const double tmp = S.k[i] + fc[i];
    v[i] = S.minv[i] * tmp;
  }
  apply_D(S, v.data(), dv.data());
  for (int c = 0; c < nc; ++c) {
    const double su = dv[3 * c + 1], sv = dv[3 * c + 2];
    ar[3 * c] = sqrt(su * su + sv * sv) * S.P.mu;
    ar[3 * c + 1] = 0.0;
    ar[3 * c + 2] = 0.0;
  }
  for (int64_t i = 0; i < n3; ++i) S.r[i] = (1.0 * ar[i]) + S.r[i];
}

/* The solve's starting vector: the contacts' held impulses, then the
 * bilateral rows'. */
std::vector<double> solve_vector(const Scene& S) {
  const int64_t n3 = 3 * (int64_t)S.nc;
  std::vector<double> x(n3 + S.nbil);
  for (int64_t i = 0; i < n3; ++i) x[i] = S.gamma[i];
  for (int i = 0; i < S.nbil; ++i) x[n3 + i] = S.gammaB[i];
  return x;
}

/* gamma = gamma_hat (APGD.cu:358), split back into contacts and rows. */
void store_solution(Scene& S, const std::vector<double>& x) {
  const int64_t n3 = 3 * (int64_t)S.nc;
  for (int64_t i = 0; i < n3; ++i) S.gamma[i] = x[i];
  for (int i = 0; i < S.nbil; ++i) S.gammaB[i] = x[n3 + i];
}

/* APGD.cu:164-361 in the order the GPU evaluates it.  The reference computes
 * N y with a Schur product (APGD.cu:229, 239); y_k = (1+b) g_k - b g_{k-1}
 * (APGD.cu:273, or g_k after a restart, :315), so here N y_k is formed from the
 * stored products of the two iterates, (1+b) N g_k - b N g_{k-1}: one Schur
 * product per iteration (N gamma_new, reused by the objective and the
 * residual) plus one per backtrack.  The first iteration's N y_0 is a product. */
void apgd_solve_fused(Scene& S) {
  int nc = S.nc;
  int64_t n3 = 3 * (int64_t)nc + S.nbil;  // contacts, then bilateral rows
  resize_gamma(S);
  std::vector<double> Gc = solve_vector(S), Gp(n3, 0.0), NGc(n3), NGp(n3, 0.0), ar(n3, 0.0);
  std::vector<double> gNew(n3), NgNew(n3), g(n3), y(n3), Ny(n3), T(n3), best(n3, 1.0), bt;
  double theta = 1.0, thetaNew = theta, Beta = 0.0, obj1 = 0.0, obj2 = 0.0;
  double residual = 10e30;
  int nan_flag = 0, status = 0, backtracks = 0;
  bool have_best = false;
  double L, t;
  for (int64_t i = 0; i < n3; ++i) T[i] = Gc[i] + (-1.0);
  L = nrm2v(S, T.data(), nc);
  schur(S, T.data(), T.data(), bt);
  L = nrm2v(S, T.data(), nc) / L;
  t = 1.0 / L;
  const double mu = S.P.mu;
  bool y_restart = true;  // y_0 = gamma_0
  double yb = 0.0;
  int k;
  for (k = 0; k < S.P.max_iterations; ++k) {
    if (k == 0) {
      for (int64_t i = 0; i < n3; ++i) y[i] = Gc[i];
      schur(S, y.data(), NGc.data(), bt);
      for (int64_t i = 0; i < n3; ++i) Ny[i] = NGc[i];
    } else if (y_restart) {
      for (int64_t i = 0; i < n3; ++i) { y[i] = Gc[i]; Ny[i] = NGc[i]; }
    } else {
      double a = 1.0 + yb, b = -yb;
      for (int64_t i = 0; i < n3; ++i) {
        y[i] = a * Gc[i] + b * Gp[i];
        Ny[i] = a * NGc[i] + b * NGp[i];
      }
    }
    for (int64_t i = 0; i < n3; ++i) g[i] = Ny[i] + S.r[i];
    double obj2_base = 0.5 * dotv(S, y.data(), Ny.data(), nc) + dotv(S, y.data(), S.r.data(), nc);
    bool first = true;
    for (;;) {
      if (!first) {
        if (backtracks >= S.P.max_backtracks) { status = 3; break; }
        ++backtracks;
        L = 2.0 * L;
        t = 1.0 / L;
      }
      first = false;
      for (int64_t i = 0; i < n3; ++i) gNew[i] = y[i] + (-t) * g[i];
      for (int c = 0; c < nc; ++c) project3(&gNew[3 * c], mu);
      schur(S, gNew.data(), NgNew.data(), bt);
      obj1 = 0.5 * dotv(S, gNew.data(), NgNew.data(), nc) + dotv(S, gNew.data(), S.r.data(), nc);
      for (int64_t i = 0; i < n3; ++i) T[i] = gNew[i] + (-1.0) * y[i];
      double nr = nrm2v(S, T.data(), nc);
      obj2 = obj2_base + (dotv(S, g.data(), T.data(), nc) + 0.5 * L * (nr * nr));
      if (!(obj1 >= obj2)) break;
    }
    if (status) break;
    thetaNew = (-(theta * theta) + theta * sqrt(theta * theta + 4.0)) / 2.0;
    Beta = theta * (1.0 - theta) / (theta * theta + thetaNew);
    double res = residual_from(S, gNew.data(), NgNew.data(), T, &nan_flag);
    if (res < residual) {
      residual = res;
      best = gNew;
      have_best = true;
    }
    if (residual < S.P.tolerance) break;
    for (int64_t i = 0; i < n3; ++i) T[i] = gNew[i] + (-1.0) * Gc[i];
    bool restart = dotv(S, g.data(), T.data(), nc) > 0;
    if (restart) thetaNew = 1.0;
    L = 0.9 * L;
    t = 1.0 / L;
    theta = thetaNew;
    Gp.swap(Gc);
    NGp.swap(NGc);
    Gc = gNew;
    NGc = NgNew;
    y_restart = restart;
    yb = Beta;
    if (S.P.anti_relaxation) anti_relax(S, Gc.data(), ar);
  }
  (void)have_best;
  schur(S, best.data(), T.data(), bt);
  double objective = 0.5 * dotv(S, best.data(), T.data(), nc) + dotv(S, best.data(), S.r.data(), nc);
  store_solution(S, best);
  S.st.iterations = k;
  S.st.backtracks = backtracks;
  S.st.residual = residual;
  S.st.objective = objective;
  if (nan_flag) status = status ? status : 2;
  S.st.status = status;
}

/* APGD.cu:164-361, literally: four Schur products per iteration. */
void apgd_solve(Scene& S) {
  int nc = S.nc;
  int64_t n3 = 3 * (int64_t)nc + S.nbil;  // contacts, then bilateral rows
  resize_gamma(S);
  std::vector<double> gam = solve_vector(S);
  double* gamma = gam.data();
  std::vector<double> gHat(n3, 1.0), gNew(n3), g(n3), y(n3), yNew(n3), T(n3), ar(n3, 0.0), bt;
  for (int64_t i = 0; i < n3; ++i) y[i] = gamma[i];

  double theta = 1.0, thetaNew = theta, Beta = 0.0, obj1 = 0.0, obj2 = 0.0;
  double residual = 10e30;
  int nan_flag = 0, status = 0, backtracks = 0;
  double t;
  double L;
  for (int64_t i = 0; i < n3; ++i) T[i] = gamma[i] + (-1.0) * gHat[i];
  L = nrm2v(S, T.data(), nc);
  schur(S, T.data(), T.data(), bt);
  L = nrm2v(S, T.data(), nc) / L;
  t = 1.0 / L;
  int k;
  const double mu = S.P.mu;
  for (k = 0; k < S.P.max_iterations; ++k) {
    schur(S, y.data(), T.data(), bt);
    for (int64_t i = 0; i < n3; ++i) g[i] = T[i] + S.r[i];
    for (int64_t i = 0; i < n3; ++i) gNew[i] = y[i] + (-t) * g[i];
    for (int c = 0; c < nc; ++c) project3(&gNew[3 * c], mu);
    schur(S, gNew.data(), T.data(), bt);
    obj1 = 0.5 * dotv(S, gNew.data(), T.data(), nc) + dotv(S, gNew.data(), S.r.data(), nc);
    schur(S, y.data(), T.data(), bt);
    obj2 = 0.5 * dotv(S, y.data(), T.data(), nc) + dotv(S, y.data(), S.r.data(), nc);
    for (int64_t i = 0; i < n3; ++i) T[i] = gNew[i] + (-1.0) * y[i];
    {
      double nr = nrm2v(S, T.data(), nc);
      obj2 += dotv(S, g.data(), T.data(), nc) + 0.5 * L * (nr * nr);
    }
    while (obj1 >= obj2) {
      if (backtracks >= S.P.max_backtracks) { status = 3; break; }
      ++backtracks;
      L = 2.0 * L;
      t = 1.0 / L;
      for (int64_t i = 0; i < n3; ++i) gNew[i] = y[i] + (-t) * g[i];
      for (int c = 0; c < nc; ++c) project3(&gNew[3 * c], mu);
      schur(S, gNew.data(), T.data(), bt);
      obj1 = 0.5 * dotv(S, gNew.data(), T.data(), nc) + dotv(S, gNew.data(), S.r.data(), nc);
      schur(S, y.data(), T.data(), bt);
      obj2 = 0.5 * dotv(S, y.data(), T.data(), nc) + dotv(S, y.data(), S.r.data(), nc);
      for (int64_t i = 0; i < n3; ++i) T[i] = gNew[i] + (-1.0) * y[i];
      double nr = nrm2v(S, T.data(), nc);
      obj2 += dotv(S, g.data(), T.data(), nc) + 0.5 * L * (nr * nr);
    }
    if (status) break;
    thetaNew = (-(theta * theta) + theta * sqrt(theta * theta + 4.0)) / 2.0;
    Beta = theta * (1.0 - theta) / (theta * theta + thetaNew);
    for (int64_t i = 0; i < n3; ++i) yNew[i] = (1.0 + Beta) * gNew[i] + (-Beta) * gamma[i];
    double res = get_residual(S, gNew.data(), T, bt, &nan_flag);
    if (res < residual) {
      residual = res;
      for (int64_t i = 0; i < n3; ++i) gHat[i] = gNew[i];
    }
    if (residual < S.P.tolerance) break;
    for (int64_t i = 0; i < n3; ++i) T[i] = gNew[i] + (-1.0) * gamma[i];
    if (dotv(S, g.data(), T.data(), nc) > 0) {
      for (int64_t i = 0; i < n3; ++i) yNew[i] = gNew[i];
      thetaNew = 1.0;
    }
    L = 0.9 * L;
    t = 1.0 / L;
    theta = thetaNew;
    for (int64_t i = 0; i < n3; ++i) gamma[i] = gNew[i];
    for (int64_t i = 0; i < n3; ++i) y[i] = yNew[i];
    if (S.P.anti_relaxation) anti_relax(S, gamma, ar);
  }
  /* APGD.cu:353-354 */
  schur(S, gHat.data(), T.data(), bt);
  double objective = 0.5 * dotv(S, gHat.data(), T.data(), nc) + dotv(S, gHat.data(), S.r.data(), nc);
  store_solution(S, gHat);
  S.st.iterations = k;
  S.st.backtracks = backtracks;
  S.st.residual = residual;
  S.st.objective = objective;
  if (nan_flag || obj1 != obj1) status = status ? status : 2;
  S.st.status = status;
}

/* PGJ.cu:152-224 (System(5)): projected Gauss-Jacobi with relaxation
 * omega = 0.3, lambda = 2/3 (PGJ.cu:14-15).  gamma starts at (1, 0, 0) per
 * contact (:170, no warm start); B_c = 3 / ((minv_A + minv_B) |F_c|^2) with the
 * nine frame entries squared and summed n, u, v in order (buildB, :73-89);
 * each iteration
 *   gamma_hat = P(gamma - omega B (N gamma + r)),
 *   gamma = lambda gamma_hat + (1 - lambda) gamma                  (:176-186)
 * and the residual of the new gamma is max(feasibleX, feasibleY, res3)
 * (:188-211): feasibleX = max -min(0, mu gamma_n - |gamma_t|), feasibleY =
 * max -min(0, g_n / mu - |g_t|) with g = N gamma + r (a NaN term counts 0),
 * res3 = max |g_c . gamma_c|.  The reference computes N gamma of the new
 * iterate twice for the residual and again at the next iteration; it is one
 * product here, reused. */
double pgj_feasible(const double* x, double mu_scale, int nc) {
  double m = -10e30;
  for (int c = 0; c < nc; ++c) {
    const double* g = x + 3 * c;
    double xn = mu_scale * g[0] - sqrt(g[1] * g[1] + g[2] * g[2]);
    if (xn != xn) xn = 0.0;
    m = fmax(m, -fmin(0.0, xn));
  }
  return m;
}

void pgj_solve(Scene& S) {
  const int nc = S.nc;
  const int64_t n3 = 3 * (int64_t)nc;
  const double omega = 0.3, lambda = 2.0 / 3.0, mu = S.P.mu;
  std::vector<double> g(n3), Ng(n3), gh(n3), T(n3), Bc(nc), bt;
  for (int c = 0; c < nc; ++c) {
    g[3 * c] = 1.0;
    g[3 * c + 1] = 0.0;
    g[3 * c + 2] = 0.0;
    const double* F = &S.F[9 * (size_t)c];
    double sum = F[0] * F[0];
    for (int k = 1; k < 9; ++k) sum = sum + F[k] * F[k];
    const double ma = S.minv[3 * (size_t)S.A[c]], mb = S.minv[3 * (size_t)S.B[c]];
    Bc[c] = 3.0 / ((ma + mb) * sum);
  }
  schur(S, g.data(), Ng.data(), bt);
  double residual = 0.0;
  int k;
  for (k = 0; k < S.P.max_iterations; ++k) {
    for (int64_t i = 0; i < n3; ++i) gh[i] = Ng[i] + S.r[i];
    for (int64_t i = 0; i < n3; ++i) T[i] = Bc[i / 3] * gh[i];
    for (int64_t i = 0; i < n3; ++i) gh[i] = g[i] + (-omega) * T[i];
    for (int c = 0; c < nc; ++c) project3(&gh[3 * c], mu);
    const double oml = 1.0 - lambda;
    for (int64_t i = 0; i < n3; ++i) g[i] = lambda * gh[i] + oml * g[i];
    const double fx = pgj_feasible(g.data(), mu, nc);
    schur(S, g.data(), Ng.data(), bt);
    for (int64_t i = 0; i < n3; ++i) T[i] = Ng[i] + S.r[i];
    double res3 = 0.0;
    for (int c = 0; c < nc; ++c) {
      const double d = (T[3 * c] * g[3 * c] + T[3 * c + 1] * g[3 * c + 1]) + T[3 * c + 2] * g[3 * c + 2];
      res3 = fmax(res3, fabs(d));
    }
    const double fy = pgj_feasible(T.data(), 1.0 / mu, nc);
    residual = fmax(fmax(fx, fy), res3);
    if (residual < S.P.tolerance) break;
  }
  if ((int64_t)S.gamma.size() < n3) S.gamma.resize(n3, 0.0);
  for (int64_t i = 0; i < n3; ++i) S.gamma[i] = g[i];
  S.gsize = nc;
  S.st.iterations = k;
  S.st.backtracks = 0;
  S.st.residual = residual;
  S.st.objective = 0.0;
  S.st.status = 0;
}

void build_k(Scene& S) {
  int n = 3 * S.nb;
  double h = S.P.h;
  for (int i = 0; i < n; ++i) {
    double m = S.minv[i];
    if (m) m = 1.0 / m;
    double kk = m * S.v[i];
    S.k[i] = h * S.f[i] + kk;
  }
}

/* PGS.cu:367-459 (solve), :143-224 (updateImpulseVector_CPU, the sweep),
 * :272-304 (buildB_PGS), :335-365 (getFeasibleX/Y_PGS), :327-333
 * (getResidual_PGS).  gamma starts at (1, 0, 0), v = Minv D^T gamma + Minv k,
 * then per iteration a Gauss-Seidel sweep over the contacts in order and the
 * residual max(feasibleX(gamma), feasibleY(N gamma + r), max |(N gamma + r) . gamma|). */
void pgs_solve(Scene& S) {
  const int nc = S.nc, nb = S.nb;
  const int64_t n3 = 3 * (int64_t)nc;
  const double omega = 0.3, lambda = 2.0 / 3.0, mu = S.P.mu;
  std::vector<double> g(n3), T(n3), Bc(nc), bt, fc(3 * (size_t)nb), v(3 * (size_t)nb);
  for (int c = 0; c < nc; ++c) {
    g[3 * c] = 1.0;
    g[3 * c + 1] = 0.0;
    g[3 * c + 2] = 0.0;
    const double* F = &S.F[9 * (size_t)c];
    double sum = F[0] * F[0];
    for (int k = 1; k < 9; ++k) sum = sum + F[k] * F[k];
    const double ma = S.minv[3 * (size_t)S.A[c]], mb = S.minv[3 * (size_t)S.B[c]];
    Bc[c] = 3.0 / ((ma + mb) * sum);
  }
  /* :376-379: f_contact = D^T gamma; v = Minv f_contact; tmp = Minv k; v = tmp + v */
  apply_DT(S, g.data(), fc.data());
  for (size_t i = 0; i < v.size(); ++i) {
    const double a1 = S.minv[i] * fc[i], a2 = S.minv[i] * S.k[i];
    v[i] = a2 + a1;
  }
  double residual = 0.0;
  int k;
  for (k = 0; k < S.P.max_iterations; ++k) {
    for (int c = 0; c < nc; ++c) {
      const double* F = &S.F[9 * (size_t)c];
      const uint32_t ia = S.A[c], ib = S.B[c];
      double* va = &v[3 * (size_t)ia];
      double* vb = &v[3 * (size_t)ib];
      const double mia = S.minv[3 * (size_t)ia], mib = S.minv[3 * (size_t)ib];
      const double bn = S.bst[3 * c];
      const double o0 = g[3 * c], o1 = g[3 * c + 1], o2 = g[3 * c + 2];
      const double ob = omega * Bc[c];
      const double ax = va[0], ay = va[1], az = va[2], bx = vb[0], by = vb[1], bz = vb[2];
      double h[3];
      h[0] = o0 - ob * (F[0] * ax + F[1] * ay + F[2] * az - F[0] * bx - F[1] * by - F[2] * bz + bn);
      h[1] = o1 - ob * (F[3] * ax + F[4] * ay + F[5] * az - F[3] * bx - F[4] * by - F[5] * bz);
      h[2] = o2 - ob * (F[6] * ax + F[7] * ay + F[8] * az - F[6] * bx - F[7] * by - F[8] * bz);
      project3(h, mu);
      const double lb = 1.0 - lambda;
      g[3 * c] = lambda * h[0] + lb * o0;
      g[3 * c + 1] = lambda * h[1] + lb * o1;
      g[3 * c + 2] = lambda * h[2] + lb * o2;
      const double d0 = lambda * (h[0] - o0), d1 = lambda * (h[1] - o1), d2 = lambda * (h[2] - o2);
      const double ex = F[0] * d0 + F[3] * d1 + F[6] * d2;
      const double ey = F[1] * d0 + F[4] * d1 + F[7] * d2;
      const double ez = F[2] * d0 + F[5] * d1 + F[8] * d2;
      va[0] = ax + mia * ex;
      va[1] = ay + mia * ey;
      va[2] = az + mia * ez;
      vb[0] = bx - mib * ex;
      vb[1] = by - mib * ey;
      vb[2] = bz - mib * ez;
    }
    const double fx = pgj_feasible(g.data(), mu, nc);
    schur(S, g.data(), T.data(), bt);
    for (int64_t i = 0; i < n3; ++i) T[i] = S.r[i] + T[i];
    double res3 = 0.0;
    for (int c = 0; c < nc; ++c) {
      const double d = (T[3 * c] * g[3 * c] + T[3 * c + 1] * g[3 * c + 1]) + T[3 * c + 2] * g[3 * c + 2];
      res3 = fmax(res3, fabs(d));
    }
    const double fy = pgj_feasible(T.data(), 1.0 / mu, nc);
    residual = fmax(fmax(fx, fy), res3);
    if (residual < S.P.tolerance) break;
  }
  if ((int64_t)S.gamma.size() < n3) S.gamma.resize(n3, 0.0);
  for (int64_t i = 0; i < n3; ++i) S.gamma[i] = g[i];
  S.gsize = nc;
  /* the sweep works on System::v (PGS.cu:376-379, 143-224): it keeps the last
   * sweep's velocities (the step's update then overwrites them) */
  S.v = v;
  S.st.iterations = k;
  S.st.backtracks = 0;
  S.st.residual = residual;
  S.st.objective = 0.0;
  S.st.status = 0;
}

void build_r(Scene& S) {
  int nb = S.nb, nc = S.nc;
  std::vector<double> tmp(3 * (size_t)nb);
  for (int i = 0; i < 3 * nb; ++i) tmp[i] = S.minv[i] * S.k[i];
  S.r.assign(3 * (size_t)nc + S.nbil, 0.0);
  apply_D(S, tmp.data(), S.r.data());
  for (int64_t i = 0; i < 3 * (int64_t)nc; ++i) S.r[i] = S.bst[i] + S.r[i];
  /* buildStabilizationBilateral (System.cu:1526-1544): b = violation / h at
   * the step's start time, the prescribed velocity 0 before its start time */
  double* rb = S.r.data() + 3 * (int64_t)nc;
  for (int i = 0; i < S.nbil; ++i) {
    const double ts = S.bilT0[i];
    double velocity = S.bilVel[i];
    if (S.time < ts) velocity = 0;
    double violation;
    if (S.bilB[i] < 0) violation = S.p[S.bilA[i]] - S.bilP0[i] - velocity * (S.time - ts);
    else violation = S.p[S.bilA[i]] - S.p[S.bilB[i]] - velocity * (S.time - ts);
    S.bB[i] = violation / S.P.h;
    rb[i] = S.bB[i] + rb[i];
  }
}

/* Solver::solve() alone (APGD.cu:164-361 and the System calls before it,
 * System.cu:559-566): k, the frames, r and the solve on the current state and
 * the contacts of the last collision detection; no update, no clock. */
int solve_only(Scene& S) {
  S.st.status = 0;
  S.st.iterations = 0;
  S.st.backtracks = 0;
  S.st.residual = 0;
  S.st.objective = 0;
  if (S.nbil && S.P.solver != 1) {
    S.st.status = 4;
    return S.st.status;
  }
  build_k(S);
  if (S.nc || S.nbil) {
    build_frames(S);
    build_r(S);
    if (S.P.solver == 5) pgj_solve(S);
    else if (S.P.solver == 6) pgs_solve(S);
    else if (S.P.apgd_mode == 1) apgd_solve(S);
    else apgd_solve_fused(S);
    keep_pairs(S);
  }
  S.st.gamma_size = S.gsize;
  return S.st.status;
}

int do_step(Scene& S) {
  S.st.status = 0;
  S.st.iterations = 0;
  S.st.backtracks = 0;
  S.st.residual = 0;
  S.st.objective = 0;
  collide(S);
  build_k(S);
  int n = 3 * S.nb;
  double h = S.P.h;
  if ((S.nbil && S.P.solver != 1) || (S.nbil && S.P.anti_relaxation)) {
    S.st.status = 4;  /* PGJ / PGS take no bilateral rows (PGJ.cu, PGS.cu size 3 nc) */
    return S.st.status;
  }
  /* System.cu:560: the solve runs with contacts or bilateral rows */
  if (S.nc || S.nbil) {
    build_frames(S);
    build_r(S);
    if (S.P.solver == 5) pgj_solve(S);
    else if (S.P.solver == 6) pgs_solve(S);
    else if (S.P.apgd_mode == 1) apgd_solve(S);
    else apgd_solve_fused(S);
    keep_pairs(S);
    std::vector<double> fc(n);
    apply_DT(S, solve_vector(S).data(), fc.data());
    for (int i = 0; i < n; ++i) {
      double tmp = S.k[i] + fc[i];
      S.v[i] = S.minv[i] * tmp;
      S.fcont[i] = (1.0 / h) * fc[i];
    }
  } else {
    S.F.clear();
    S.r.clear();
    S.bst.clear();
    S.incStart.assign(S.nb + 1, 0);
    for (int i = 0; i < n; ++i) {
      S.v[i] = S.minv[i] * S.k[i];
      S.fcont[i] = 0.0;
    }
  }
  for (int i = 0; i < n; ++i) S.p[i] = h * S.v[i] + S.p[i];
  S.time += h;
  S.timeIndex++;
  S.st.gamma_size = S.gsize;
  return S.st.status;
}

}  // namespace

extern "C" {

void* or_create(int nb, const double* pos, const double* vel, const double* mass,
                const double* geom, const int* fixed, const int* family,
                const or_params* prm) {
  Scene* S = new Scene();
  S->P = *prm;
  S->nb = nb;
  S->p.assign(pos, pos + 3 * (size_t)nb);
  S->v.assign(vel, vel + 3 * (size_t)nb);
  S->geom.assign(geom, geom + 3 * (size_t)nb);
  S->fixed.assign(fixed, fixed + nb);
  S->family.assign(family, family + nb);
  S->minv.resize(3 * (size_t)nb);
  S->f.resize(3 * (size_t)nb);
  S->k.assign(3 * (size_t)nb, 0.0);
  S->fcont.assign(3 * (size_t)nb, 0.0);
  for (int i = 0; i < nb; ++i) {
    for (int d = 0; d < 3; ++d) {
      /* System.cu:368-376, 409-417 */
      S->f[3 * i + d] = fixed[i] ? 0.0 : mass[i] * prm->gravity[d];
      S->minv[3 * i + d] = fixed[i] ? 0.0 : 1.0 / mass[i];
    }
  }
  /* gamma_d = a_h: 3 nb zeros (System.cu:185) */
  S->gamma.assign(3 * (size_t)nb, 0.0);
  S->gsize = nb;
  memset(&S->st, 0, sizeof(S->st));
#ifdef _OPENMP
  if (prm->threads > 0) omp_set_num_threads(prm->threads);
#endif
  return S;
}

void or_destroy(void* s) { delete (Scene*)s; }

int or_set_params(void* s, const or_params* prm) {
  Scene* S = (Scene*)s;
  S->P = *prm;
#ifdef _OPENMP
  if (prm->threads > 0) omp_set_num_threads(prm->threads);
#endif
  return 0;
}

int or_step(void* s, int nsteps) {
  Scene* S = (Scene*)s;
  int st = 0;
  for (int i = 0; i < nsteps; ++i) {
    st = do_step(*S);
    if (st) break;
  }
  return st;
}

int or_solve(void* s) { return solve_only(*(Scene*)s); }

int or_collide(void* s) {
  Scene* S = (Scene*)s;
  collide(*S);
  if (S->nc) build_frames(*S);
  return 0;
}

int or_get_stats(void* s, or_stats* out) {
  Scene* S = (Scene*)s;
  *out = S->st;
  out->num_contacts = S->nc;
  out->num_possible = S->npossible;
  out->gamma_size = S->gsize;
  return 0;
}

int or_get_state(void* s, double* p, double* v) {
  Scene* S = (Scene*)s;
  if (p) memcpy(p, S->p.data(), sizeof(double) * 3 * S->nb);
  if (v) memcpy(v, S->v.data(), sizeof(double) * 3 * S->nb);
  return 0;
}

int or_set_state(void* s, const double* p, const double* v) {
  Scene* S = (Scene*)s;
  if (p) memcpy(S->p.data(), p, sizeof(double) * 3 * S->nb);
  if (v) memcpy(S->v.data(), v, sizeof(double) * 3 * S->nb);
  return 0;
}

int or_get_fcontact(void* s, double* f) {
  Scene* S = (Scene*)s;
  memcpy(f, S->fcont.data(), sizeof(double) * 3 * S->nb);
  return 0;
}

int or_get_gamma(void* s, double* gamma, int cap) {
  Scene* S = (Scene*)s;
  int n = std::min(cap, S->gsize);
  if (gamma && n > 0) memcpy(gamma, S->gamma.data(), sizeof(double) * 3 * (size_t)n);
  return S->gsize;
}

int or_set_gamma(void* s, const double* gamma, int ncont) {
  Scene* S = (Scene*)s;
  if ((int64_t)S->gamma.size() < 3 * (int64_t)ncont) S->gamma.resize(3 * (size_t)ncont, 0.0);
  if (ncont > 0) memcpy(S->gamma.data(), gamma, sizeof(double) * 3 * (size_t)ncont);
  S->gsize = ncont;
  S->wA.clear();  // a positional warm start carries no pairs
  S->wB.clear();
  return 0;
}

int or_get_contacts(void* s, uint32_t* a, uint32_t* b, double* nP, double* loc) {
  Scene* S = (Scene*)s;
  int nc = S->nc;
  if (a) memcpy(a, S->A.data(), sizeof(uint32_t) * nc);
  if (b) memcpy(b, S->B.data(), sizeof(uint32_t) * nc);
  if (nP) memcpy(nP, S->nP.data(), sizeof(double) * 4 * (size_t)nc);
  if (loc) memcpy(loc, S->loc.data(), sizeof(double) * 3 * (size_t)nc);
  return nc;
}

int or_get_frames(void* s, double* F) {
  Scene* S = (Scene*)s;
  if ((int64_t)S->F.size() != 9 * (int64_t)S->nc) return -1;
  memcpy(F, S->F.data(), sizeof(double) * S->F.size());
  return S->nc;
}

/* System::r_d, b_d, k_d of the last step (System.cu:1502-1580), the
 * reference's layout: r and b with the bilateral rows first. */
int or_get_step_vectors(void* s, double* r, double* b, double* k) {
  Scene* S = (Scene*)s;
  const int nc = S->nc, nbil = S->nbil;
  const int64_t n3 = 3 * (int64_t)nc;
  if ((int64_t)S->r.size() < n3 + nbil || (int64_t)S->bst.size() < n3) return -1;
  for (int i = 0; i < nbil; ++i) {
    if (r) r[i] = S->r[n3 + i];
    if (b) b[i] = S->bB[i];
  }
  for (int64_t i = 0; i < n3; ++i) {
    if (r) r[nbil + i] = S->r[i];
    if (b) b[nbil + i] = S->bst[i];
  }
  if (k) memcpy(k, S->k.data(), sizeof(double) * 3 * (size_t)S->nb);
  return (int)(n3 + nbil);
}

int or_get_r(void* s, double* r) {
  Scene* S = (Scene*)s;
  if ((int64_t)S->r.size() < 3 * (int64_t)S->nc) return -1;
  memcpy(r, S->r.data(), sizeof(double) * 3 * (size_t)S->nc);
  return S->nc;
}

/* System.cu:1590-1643 */
int or_ccp_violation(void* s, double* out4) {
  Scene* S = (Scene*)s;
  out4[0] = out4[1] = out4[2] = out4[3] = 0.0;
  int nc = S->nc;
  if (!nc) return 0;
  /* With bilateral rows the reference reads entry 3 c (and 3 c + 1, 3 c + 2)
   * of vectors whose first nbil entries are the bilateral rows, with no
   * offset (getNormalComponent, calculateConeViolation: System.cu:1590-1603);
   * gm and tg below are those flat vectors.  tg = D v + b over every row (the
   * reference's temporary holds 3 nc entries, :1613; the entries read are the
   * same). */
  const int nbil = S->nbil;
  const int64_t n3 = 3 * (int64_t)nc;
  std::vector<double> gm(n3 + nbil), tg(n3 + nbil), dv(n3 + nbil);
  apply_D(*S, S->v.data(), dv.data());
  for (int i = 0; i < nbil; ++i) {
    gm[i] = S->gammaB[i];
    tg[i] = S->bB[i] + dv[n3 + i];
  }
  for (int64_t i = 0; i < n3; ++i) {
    gm[nbil + i] = S->gamma[i];
    tg[nbil + i] = S->bst[i] + dv[i];
  }
  double x = gm[0];
  for (int c = 1; c < nc; ++c) x = std::min(x, gm[3 * c]);
  if (x > 0) x = 0;
  double y = tg[0];
  for (int c = 1; c < nc; ++c) y = std::min(y, tg[3 * c]);
  if (y > 0) y = 0;
  std::vector<double> it(nc);
  for (int c = 0; c < nc; ++c) it[c] = gm[3 * c] * tg[3 * c];
  double z;
  if (S->P.reduce_mode == 1) {
    z = 0.0;
    for (int c = 0; c < nc; ++c) z = z + it[c];
  } else {
    z = ordered_sum(it.data(), nc);
  }
  for (int c = 0; c < nc; ++c) {
    double gt = sqrt(gm[3 * c + 1] * gm[3 * c + 1] + gm[3 * c + 2] * gm[3 * c + 2]);
    double cv = S->P.mu * gm[3 * c] - gt;
    if (cv > 0) cv = 0;
    it[c] = cv * cv;
  }
  double w2;
  if (S->P.reduce_mode == 1) {
    w2 = 0.0;
    for (int c = 0; c < nc; ++c) w2 = w2 + it[c];
  } else {
    w2 = ordered_sum(it.data(), nc);
  }
  out4[0] = x;
  out4[1] = y;
  out4[2] = z;
  out4[3] = sqrt(w2);
  return 0;
}

/* System.cu:1645-1658 */
double or_kinetic_energy(void* s) {
  Scene* S = (Scene*)s;
  std::vector<double> it(S->nb);
  for (int b = 0; b < S->nb; ++b) {
    double a[3];
    for (int d = 0; d < 3; ++d) {
      double m = S->minv[3 * b + d];
      if (m) m = 1.0 / m;
      a[d] = S->v[3 * b + d] * (m * S->v[3 * b + d]);
    }
    it[b] = (a[0] + a[1]) + a[2];
  }
  return 0.5 * ordered_sum(it.data(), S->nb);
}

double or_potential_energy(void* s) {
  Scene* S = (Scene*)s;
  std::vector<double> it(S->nb);
  for (int b = 0; b < S->nb; ++b)
    it[b] = (S->f[3 * b] * S->p[3 * b] + S->f[3 * b + 1] * S->p[3 * b + 1]) + S->f[3 * b + 2] * S->p[3 * b + 2];
  return -ordered_sum(it.data(), S->nb);
}

/* System::addBilateralConstraintDOF (System.cu:510-532) and processConstraints
 * (:303-315): p0 = the DOF's position now, for a single-DOF row. */
int or_add_bilateral(void* s, int dofA, int dofB, double velocity, double start_time) {
  Scene* S = (Scene*)s;
  const int n = 3 * S->nb;
  if (dofA < 0 || dofA >= n || dofB >= n) return -1;
  if (dofB < 0) dofB = -1;
  const int row = S->nbil++;
  S->bilA.push_back(dofA);
  S->bilB.push_back(dofB);
  S->bilVel.push_back(velocity);
  S->bilT0.push_back(start_time);
  S->bilP0.push_back(dofB < 0 ? S->p[dofA] : 0.0);
  S->gammaB.push_back(0.0);
  S->bB.push_back(0.0);
  /* per-body entries, ascending rows, A before B */
  std::vector<std::vector<int>> per(S->nb);
  for (int i = 0; i <= row; ++i) {
    per[S->bilA[i] / 3].push_back((i << 3) | ((S->bilA[i] % 3) << 1));
    if (S->bilB[i] >= 0) per[S->bilB[i] / 3].push_back((i << 3) | ((S->bilB[i] % 3) << 1) | 1);
  }
  S->bincStart.assign(S->nb + 1, 0);
  S->binc.clear();
  for (int b = 0; b < S->nb; ++b) {
    S->bincStart[b] = (int)S->binc.size();
    S->binc.insert(S->binc.end(), per[b].begin(), per[b].end());
  }
  S->bincStart[S->nb] = (int)S->binc.size();
  return 0;
}

/* The bilateral rows' impulses of the last solve (System::gamma's first
 * nbil entries); returns nbil. */
int or_get_bilateral_gamma(void* s, double* out) {
  Scene* S = (Scene*)s;
  if (out && S->nbil) memcpy(out, S->gammaB.data(), sizeof(double) * S->nbil);
  return S->nbil;
}

void or_project(double* x3, double mu) { project3(x3, mu); }

void or_frame(const double* n3, double* u3, double* v3) {
  V3 u, v;
  frame_from_normal(mk(n3[0], n3[1], n3[2]), &u, &v);
  u3[0] = u.x; u3[1] = u.y; u3[2] = u.z;
  v3[0] = v.x; v3[1] = v.y; v3[2] = v.z;
}

double or_length3(const double* v3) { return length3(mk(v3[0], v3[1], v3[2])); }

void or_normalize3(const double* v3, double* out3) {
  V3 r = normalize3(mk(v3[0], v3[1], v3[2]));
  out3[0] = r.x; out3[1] = r.y; out3[2] = r.z;
}

double or_ordered_sum(const double* v, int64_t n) { return ordered_sum(v, n); }

void or_schur(int nb, int nc, const uint32_t* a, const uint32_t* b, const double* F,
              const double* minv, const double* x, double* out, int spmv_mode) {
  Scene S;
  S.nb = nb;
  S.nc = nc;
  S.P.spmv_mode = spmv_mode;
  S.A.assign(a, a + nc);
  S.B.assign(b, b + nc);
  S.F.assign(F, F + 9 * (size_t)nc);
  S.minv.assign(minv, minv + 3 * (size_t)nb);
  S.nP.assign(4 * (size_t)nc, 0.0);
  for (int c = 0; c < nc; ++c)
    for (int d = 0; d < 3; ++d) S.nP[4 * c + d] = F[9 * (size_t)c + d];
  S.P.h = 1.0;
  /* incidence only */
  std::vector<int> cnt(nb + 1, 0);
  for (int c = 0; c < nc; ++c) { cnt[a[c] + 1]++; cnt[b[c] + 1]++; }
  for (int i = 0; i < nb; ++i) cnt[i + 1] += cnt[i];
  S.incStart = cnt;
  S.incC.assign(2 * (size_t)nc, 0);
  S.incS.assign(2 * (size_t)nc, 0);
  std::vector<int> pos(cnt.begin(), cnt.end() - 1);
  for (int c = 0; c < nc; ++c) {
    S.incC[pos[b[c]]] = c; S.incS[pos[b[c]]] = -1; pos[b[c]]++;
    S.incC[pos[a[c]]] = c; S.incS[pos[a[c]]] = +1; pos[a[c]]++;
  }
  std::vector<double> bt;
  schur(S, x, out, bt);
}

}  // extern "C"
