/*
 * dv_oracle.h -- C ABI of the CPU oracle for the DVIDE rigid-body contact step.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links or calls
 * this code; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load liboracle.so, and only as the checker / the timed CPU baseline.
 *
 * Parity status: UNPINNED against the reference binary.  The reference
 * (melanz/DVIDE) cannot be built here (it needs the CUSP headers, which are
 * absent) and ships no golden vectors or tests.  The oracle restates the
 * reference source line by line (citations in dv_oracle.cpp) and is pinned on
 * (a) the reference's own float-sqrt vector helpers, compiled from
 * src/helper_math_double.h by oracle/ref_helper_probe.cpp, and (b) analytic
 * known-answer tests taken from the reference drivers (ball at rest on the
 * ground, static equilibrium of a settled pile).
 */
#ifndef DV_ORACLE_H_
#define DV_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_params {
  double h;               /* time step (System::h, System.cu:66) */
  double mu;              /* friction coefficient (System.cu:65) */
  double gravity[3];      /* System::gravity (System.cu:64) */
  double envelope;        /* CollisionDetector envelope (CollisionDetector.cu:512) */
  double tolerance;       /* APGD tolerance (APGD.cu:10) */
  int max_iterations;     /* APGD maxIterations (APGD.cu:11) */
  int warm_start;         /* APGD::setWarmStarting (APGD.cuh:62) */
  int reduce_mode;        /* 0 = tiled order shared with the GPU, 1 = sequential (host CUSP) */
  int spmv_mode;          /* 0 = grouped matrix-free product, 1 = literal COO entry order */
  int max_backtracks;     /* cap on Lipschitz doublings per iteration (unbounded in the reference) */
  int threads;            /* OpenMP threads, 0 = runtime default */
  int apgd_mode;          /* 0 = fused sequence shared with the GPU, 1 = literal reference sequence */
  int solver;             /* System(solverType): 1 = APGD (APGD.cu), 5 = PGJ (PGJ.cu) */
  int anti_relaxation;    /* APGD::setAntiRelaxation (APGD.cuh:63, APGD.cu:335-345) */
  int fp64_narrowphase;   /* extension: 1 = FP64 sqrt in length/normalize of the narrowphase and
                             the tangent frame (the reference uses float, helper_math_double.h) */
} or_params;

typedef struct or_stats {
  int num_contacts;       /* CollisionDetector::numCollisions */
  int num_possible;       /* CollisionDetector::numPossibleCollisions */
  int iterations;         /* Solver::iterations */
  int backtracks;         /* total Lipschitz doublings in the last solve */
  double residual;        /* best residual of the last solve */
  double objective;       /* System::objectiveCCP */
  int status;             /* 0 ok, 2 = NaN, 3 = backtracking cap hit, 4 = bilateral rows with PGJ/PGS */
  int gamma_size;         /* warm-start buffer length in contacts */
} or_stats;

void* or_create(int nb, const double* pos, const double* vel, const double* mass,
                const double* geom, const int* fixed, const int* family,
                const or_params* prm);
void or_destroy(void* s);
int or_set_params(void* s, const or_params* prm);

int or_step(void* s, int nsteps);          /* System::DoTimeStep */
int or_collide(void* s);                   /* AABB + broadphase + narrowphase only */
int or_solve(void* s);                     /* Solver::solve() alone: no update, no clock */
int or_get_stats(void* s, or_stats* out);
int or_get_state(void* s, double* p, double* v);
int or_set_state(void* s, const double* p, const double* v);
int or_get_fcontact(void* s, double* f);
int or_get_gamma(void* s, double* gamma, int cap);  /* returns gamma_size (contacts) */
int or_set_gamma(void* s, const double* gamma, int ncont);
int or_get_contacts(void* s, uint32_t* a, uint32_t* b, double* nP, double* loc);
int or_get_frames(void* s, double* F);     /* 9 per contact: n, u, v */
int or_get_r(void* s, double* r);          /* 3 per contact (Schur vector of the last step) */
/* r, b (bilateral rows first, then 3 per contact) and k (3 per body) of the last step */
int or_get_step_vectors(void* s, double* r, double* b, double* k);
int or_ccp_violation(void* s, double* out4);
/* System::addBilateralConstraintDOF (before the first step); 0 or -1 */
int or_add_bilateral(void* s, int dofA, int dofB, double velocity, double start_time);
int or_get_bilateral_gamma(void* s, double* out);  /* returns the row count */
double or_kinetic_energy(void* s);
double or_potential_energy(void* s);

/* Unit restatements for known-answer tests. */
void or_project(double* x3, double mu);
void or_frame(const double* n3, double* u3, double* v3);
double or_length3(const double* v3);
void or_normalize3(const double* v3, double* out3);
double or_ordered_sum(const double* v, int64_t n);
/* N x for an explicit contact set: F (9 per contact), ids, minv per body. */
void or_schur(int nb, int nc, const uint32_t* a, const uint32_t* b, const double* F,
              const double* minv, const double* x, double* out, int spmv_mode);

#ifdef __cplusplus
}
#endif
#endif
