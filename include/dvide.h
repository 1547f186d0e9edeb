/*
 * dvide.h -- C ABI of the B200-native DVIDE rigid-body contact step.
 *
 * One scene = one DVIDE System holding rigid spheres and boxes (3 DOF each,
 * src/Body.cuh:14-100).  A time step is the reference's System::DoTimeStep
 * (src/System.cu:544-602): collision detection, APGD cone-complementarity
 * solve, half-implicit velocity/position update.  All state lives on the GPU;
 * every call returns a status (0 = DV_OK).  Plain pointers and sizes only.
 *
 * The reference has no C ABI; each entry point names the C++ member of the
 * reference it stands in for.
 */
#ifndef DVIDE_H_
#define DVIDE_H_

#include <stddef.h>
#include <stdint.h>

#if defined(_WIN32)
#define DV_API __declspec(dllexport)
#else
#define DV_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (the reference returns 0 from every method and checks no CUDA
 * errors; src/System.cu, src/APGD.cu). */
enum {
  DV_OK = 0,
  DV_ERR_ARG = 1,        /* invalid argument */
  DV_ERR_CUDA = 2,       /* a CUDA runtime call failed */
  DV_ERR_NAN = 3,        /* non-finite value in the solve (e.g. sphere centre inside a box) */
  DV_ERR_NOCONV = 4,     /* Lipschitz backtracking exceeded max_backtracks */
  DV_ERR_OOM = 5,        /* device allocation failed or over the memory budget */
  DV_ERR_TIMEOUT = 6,    /* a persistent kernel's bounded wait expired */
  DV_ERR_UNSUPPORTED = 7,
  DV_ERR_ABORTED = 8     /* cancelled through dv_*_abort */
};

enum { DV_PREC_FP64 = 0, DV_PREC_MIXED = 1 };
/* System(int solverType) numbering (System.cu:77-101): 1 APGD, 5 PGJ, 6 PGS
   (PGS: FP64 only). */
enum { DV_SOLVER_APGD = 1, DV_SOLVER_PGJ = 5, DV_SOLVER_PGS = 6 };

/* One rigid body, as System::initializeSystem flattens it (System.cu:344-424). */
typedef struct dv_body_desc {
  double pos[3];
  double vel[3];
  double mass;       /* Body::mass, default 1.0 (Body.cuh:39) */
  double geom[3];    /* (r, 0, 0) sphere, (hx, hy, hz) box half-extents (Body.cuh:18-60) */
  int32_t fixed;     /* Body::fixed */
  int32_t family;    /* PhysicsItem::collisionFamily, -1 collides with all */
} dv_body_desc;

typedef struct dv_params {
  double h;              /* System::h (System.cu:66), default 1e-3 */
  double mu;             /* System::frictionCoefficient (System.cu:65), default 0.25 */
  double gravity[3];     /* System::gravity (System.cu:64), default (0, -9.81, 0) */
  double envelope;       /* CollisionDetector::envelope (CollisionDetector.cu:512), default 1e-3 */
  double tolerance;      /* Solver::tolerance (APGD.cu:10), default 1e-4 */
  int32_t max_iterations;/* Solver::maxIterations (APGD.cu:11), default 100000 */
  int32_t warm_start;    /* APGD::setWarmStarting (APGD.cuh:62), default 0 */
  int32_t solver;        /* System(int solverType) (System.cu:84-107); 1 = APGD */
  int32_t precision;     /* DV_PREC_FP64 (drop-in) or DV_PREC_MIXED */
  int32_t max_backtracks;/* cap on Lipschitz doublings per solve (reference: unbounded) */
  int32_t verbose;       /* print the per-step line of System.cu:592 */
  int32_t fp64_narrowphase; /* extension, default 0: 1 computes length/normalize of the
                               narrowphase and the tangent frame with FP64 square roots
                               (the reference's are float, helper_math_double.h:576-597);
                               not the reference's results, so never with parity checks */
  int32_t anti_relaxation;  /* APGD::setAntiRelaxation (APGD.cuh:63, APGD.cu:335-345), default 0;
                               FP64 APGD scenes of their own (not in batches or servers),
                               without bilateral rows and without dv_apgd_solve */
  int32_t refine_iterations; /* extension, default 0 (off); used by DV_PREC_MIXED APGD and
                               ignored by FP64 scenes, PGJ and PGS: at most this many FP64
                               APGD iterations after the FP32 ones, started from the FP32
                               best iterate, for every solve whose FP32 phase ended above
                               the tolerance (iteration cap, or no new best residual for 50
                               accepted iterations) */
} dv_params;

/* Per-step report (System.cu:586-599 and APGD.cu:351-357). */
typedef struct dv_step_stats {
  int32_t num_contacts;      /* CollisionDetector::numCollisions */
  int32_t num_possible;      /* CollisionDetector::numPossibleCollisions */
  int32_t iterations;        /* Solver::iterations */
  int32_t backtracks;        /* Lipschitz doublings in the solve */
  double residual;           /* best APGD residual */
  double objective;          /* System::objectiveCCP */
  double elapsed_ms;         /* System::elapsedTime (device time of the step) */
  double time;               /* System::time */
  int32_t time_index;        /* System::timeIndex */
  int32_t status;
  double collide_ms;         /* device time of collision detection */
  double solve_ms;           /* device time of the persistent solve kernel */
  int32_t sweeps;            /* APGD iterations executed (iterations + 1 when converged) */
  int32_t refine_iterations; /* of `iterations`, those of the FP64 refinement (mixed precision) */
} dv_step_stats;

typedef struct dv_scene dv_scene;

/* Fills *p with the reference defaults listed above. */
DV_API int dv_params_default(dv_params* p);

/* System(int solverType) + add(Body*) for each body + initializeSystem()
 * (System.cu:62-133, 148-152, 342-508).  Copies the bodies to the device. */
DV_API int dv_scene_create(const dv_body_desc* bodies, int32_t nb, const dv_params* params,
                           dv_scene** out);
DV_API int dv_scene_destroy(dv_scene* s);

/* Runs the scene's kernels on a caller-provided cudaStream_t (NULL = the
 * scene's own stream). */
DV_API int dv_scene_set_stream(dv_scene* s, void* cuda_stream);
DV_API int dv_set_params(dv_scene* s, const dv_params* params);

/* System::DoTimeStep (System.cu:544-602), nsteps times.  DV_ERR_ARG (with
 * dv_last_error's text) when a sphere has more than 8192 contact partners of
 * larger id, or more than 65536 spheres have over 128 in one step; that step
 * leaves the state as it was. */
DV_API int dv_step(dv_scene* s, int32_t nsteps);

/* CollisionDetector::generateAxisAlignedBoundingBoxes +
 * detectPossibleCollisions_spatialSubdivision + detectCollisions
 * (CollisionDetector.cu:547-665): detection only, no solve or update. */
DV_API int dv_collide(dv_scene* s);

/* The scene solver's solve() (APGD::solve, APGD.cu:164-361; PGJ, PGS
 * likewise): k = M v + h f, the Schur vector and the solve on the current
 * state and the contacts of the last collision detection (dv_collide, or the
 * last step's), gamma into the warm start, and the statistics of
 * dv_get_step_stats; v, p, the contact forces and the clock are left as they
 * are (PGS leaves its working velocities in v, as the reference's PGS::solve
 * does with System::v).  dv_collide + dv_apgd_solve + the update is dv_step. */
DV_API int dv_apgd_solve(dv_scene* s);

/* Body state, 3 doubles per body as System::p_d / v_d (System.cu:355-366). */
DV_API int dv_get_state(dv_scene* s, double* p, double* v);
DV_API int dv_set_state(dv_scene* s, const double* p, const double* v);
/* System::f_contact_d after a step (System.cu:570-573), 3 per body. */
DV_API int dv_get_contact_force(dv_scene* s, double* f);

DV_API int dv_get_num_contacts(dv_scene* s, int32_t* nc, int32_t* npossible);
/* collisionIdentifierA_d / B_d, normalsAndPenetrations_d (double4: stored
 * normal B->A and gap) and collisionLocations_d (CollisionDetector.cuh:88-92,
 * CollisionDetector.cu:493-498); any pointer may be NULL. */
DV_API int dv_get_contacts(dv_scene* s, uint32_t* a, uint32_t* b, double* nP, double* loc);
/* System::gamma_d, 3 per contact (warm-start buffer after the solve).
 * Returns its length in contacts through *n. */
DV_API int dv_get_gamma(dv_scene* s, double* gamma, int32_t cap, int32_t* n);
/* Overwrites the warm-start buffer (length n contacts). */
DV_API int dv_set_gamma(dv_scene* s, const double* gamma, int32_t n);
/* System::addBilateralConstraintDOF(DOFA, DOFB, velocity, startTime)
 * (System.cu:510-532; the two-argument form is velocity 0, start time 0): a
 * scalar constraint row, +1 at DOF dof_a and -1 at DOF dof_b, where DOF
 * 3 i + k is axis k of body i; dof_b < 0 holds DOF dof_a alone at its
 * position at this call.  Its stabilisation b = (violation minus velocity
 * times the time since start_time) / h (System.cu:1526-1544).  Only before the
 * scene's first step (the reference copies the rows to the device once, at
 * initializeSystem); APGD in FP64 only: DV_ERR_UNSUPPORTED for PGJ, PGS and
 * the mixed precision, here and in dv_set_params. */
DV_API int dv_add_bilateral_dof(dv_scene* s, int32_t dof_a, int32_t dof_b, double velocity,
                                double start_time);
/* The bilateral rows' impulses of the last solve (the first entries of the
 * reference's System::gamma_d), in the order the rows were added; their count
 * through *n. */
DV_API int dv_get_bilateral_gamma(dv_scene* s, double* gamma, int32_t cap, int32_t* n);
/* Contact frames n, u, v (9 per contact) and Schur vector r (3 per contact)
 * of the last step: System.cu:753-762, 1561-1580. */
DV_API int dv_get_frames(dv_scene* s, double* F);
DV_API int dv_get_schur_vector(dv_scene* s, double* r);
/* The last step's vectors as the reference holds them (System::r_d, b_d,
 * k_d; System.cu:1502-1524, 1526-1580): r and b with 3 nc + nbil entries, the
 * bilateral rows first (dv_add_bilateral_dof), then 3 per contact; k with 3
 * per body.  Any pointer may be NULL.  System::exportMatrices writes them. */
DV_API int dv_get_step_vectors(dv_scene* s, double* r, double* b, double* k);

/* System::getCCPViolation (System.cu:1605-1643): out4 = (min gamma_n,
 * min v_n, gamma_n . v_n, ||cone violation||). */
DV_API int dv_ccp_violation(dv_scene* s, double* out4);
/* System::getKineticEnergy / getPotentialEnergy (System.cu:1645-1658). */
DV_API int dv_energies(dv_scene* s, double* kinetic, double* potential);
/* System::calculateContactForcePerCollision (System.cu:1259-1295): normal and
 * friction force per contact, 3 doubles each. */
DV_API int dv_contact_forces_per_collision(dv_scene* s, double* normal, double* friction);

DV_API int dv_get_step_stats(dv_scene* s, dv_step_stats* out);
DV_API const char* dv_status_string(int status);
/* Last CUDA error text recorded by the library (thread-local). */
DV_API const char* dv_last_error(void);
/* Number of kernel launches issued by this scene so far. */
DV_API int64_t dv_scene_launch_count(dv_scene* s);
/* Per-step reports since the last clear, oldest first (the per-step line the
 * reference prints at System.cu:592 and APGD.cu:351). */
DV_API int dv_get_step_history(dv_scene* s, dv_step_stats* out, int32_t cap, int32_t* n);
DV_API int dv_clear_step_history(dv_scene* s);
/* Device time of the solve kernel's phases summed over the steps so far (ns
 * between grid-barrier releases, 8 slots: setup, step, backtrack step, body
 * gather, product + residual, final) and how often each ran; reset != 0
 * clears the sums.  The reference's elapsedTime (System.cu:586-590) times the
 * whole step only. */
DV_API int dv_get_phase_times(dv_scene* s, double* ns, int64_t* counts, int32_t reset);

/* No counterpart in the reference.  dv_ccp_violation without any device
 * allocation, for callers that may not call cudaMalloc/cudaFree: an
 * application whose device memory belongs to its own pool allocator, or a
 * fixed-rate loop that cannot afford an allocation that may synchronise the
 * device.  All array arguments are caller-owned DEVICE pointers in the reference's
 * layouts: gamma 3 per contact (System::gamma_d), nP 4 per contact
 * (normalsAndPenetrations_d: normal B->A, gap), ida/idb per contact, v 3 per
 * body (System::v_d); out4 receives (min gamma_n, min v_n, gamma_n . v_n,
 * ||cone violation||) in device memory, queued on `stream` (a cudaStream_t,
 * NULL = legacy default stream).  Every ida/idb must be below nb: a contact
 * naming another body is not read, and all four outputs are NaN.  Results equal
 * dv_ccp_violation's for the same scene bit for bit, NaN inputs included.
 * Scratch is a fixed 1.75 MiB array in device memory that each CUDA context
 * (each GPU, for the runtime's own contexts) holds until the process exits; nc
 * above DV_NOALLOC_MAX_CONTACTS is rejected with DV_ERR_ARG.  The first call in
 * a context looks the array's device address up (cudaGetSymbolAddress) and
 * keeps it under the context's unique id; make that call before any stream
 * capture.  All calls share the array: calls that overlap on the GPU
 * (unordered streams) race. */
#define DV_NOALLOC_MAX_CONTACTS 16777216
DV_API int dv_ccp_violation_noalloc(int32_t nc, int32_t nb, const double* gamma, const double* nP,
                                    const uint32_t* ida, const uint32_t* idb, const double* v,
                                    double mu, double h, double* out4, void* stream);

/* ------------------------------------------------------------------------
 * Batched scenes.  No counterpart in the reference (DVIDE steps one System
 * per process).  A batch steps many independent scenes together: one
 * collision pipeline and ONE persistent solve kernel per step for all of
 * them, each scene with its own parameters, contact set, warm start and APGD
 * convergence (a converged scene stops iterating while the others go on).
 * Every reduction of a scene runs over that scene's own tiles in a fixed
 * order, so each scene's results are bit-identical to the same scene stepped
 * alone (dv_scene_* with the same precision) and independent of the launch
 * shape.  Bodies of all scenes are passed concatenated: scene i owns
 * counts[i] consecutive entries.  precision: DV_PREC_FP64 or DV_PREC_MIXED
 * for every scene of the batch (each dv_params' own precision is ignored).
 * ------------------------------------------------------------------------ */
typedef struct dv_batch dv_batch;

typedef struct dv_scene_stats {
  int32_t num_contacts;
  int32_t num_possible;
  int32_t iterations;
  int32_t backtracks;
  double residual;
  double objective;
  int32_t status;            /* DV_OK, DV_ERR_NAN or DV_ERR_NOCONV for this scene */
  int32_t sweeps;
  int32_t refine_iterations; /* DV_PREC_MIXED: FP64 refinement iterations (part of iterations) */
} dv_scene_stats;

typedef struct dv_tune_candidate {
  int32_t grid;              /* CTAs of the persistent solve kernel */
  int32_t chunk;             /* consecutive 512-contact tiles a CTA takes at a time */
  int32_t contiguous;        /* 1: each CTA owns one contiguous tile range (scenes per CTA) */
  int32_t blocks_per_sm;     /* 2 (128 registers per thread) or 3 (80; DV_PREC_MIXED only) */
  float ms_per_step;         /* measured device time per step */
} dv_tune_candidate;

typedef struct dv_tune_report {
  int32_t num_candidates;
  int32_t best;              /* index of the chosen candidate (now in effect) */
  int32_t identical;         /* 1: every candidate produced bit-identical states */
  int32_t steps_per_trial;
  dv_tune_candidate cand[16];
} dv_tune_report;

DV_API int dv_batch_create(const dv_body_desc* bodies, const int32_t* counts, int32_t nscenes,
                           const dv_params* params, int32_t precision, dv_batch** out);
DV_API int dv_batch_destroy(dv_batch* b);
DV_API int dv_batch_set_stream(dv_batch* b, void* cuda_stream);
/* nsteps time steps of every scene; returns the first engine-level error
 * (per-scene solver errors are reported in dv_batch_scene_stats). */
DV_API int dv_batch_step(dv_batch* b, int32_t nsteps);
DV_API int dv_batch_num_scenes(dv_batch* b, int32_t* nscenes, int32_t* nbodies);
/* p, v: 3 doubles per body of `scene`, or of all scenes concatenated when scene < 0. */
DV_API int dv_batch_get_state(dv_batch* b, int32_t scene, double* p, double* v);
DV_API int dv_batch_set_state(dv_batch* b, int32_t scene, const double* p, const double* v);
/* Per-scene report of the last step (nscenes entries). */
DV_API int dv_batch_scene_stats(dv_batch* b, dv_scene_stats* out);
/* Per-step, per-scene reports of the last dv_batch_step call: steps x nscenes
 * entries (step-major) and the device time of each step. */
DV_API int dv_batch_step_history(dv_batch* b, dv_scene_stats* out, float* step_ms, int32_t cap_steps,
                                 int32_t* nsteps);
DV_API int dv_batch_get_gamma(dv_batch* b, int32_t scene, double* gamma, int32_t cap, int32_t* n);
DV_API int dv_batch_ccp_violation(dv_batch* b, int32_t scene, double* out4);
/* Launch shape of the solve kernel (grid <= 0: default; blocks_per_sm 3 is
 * taken only by DV_PREC_MIXED batches). */
DV_API int dv_batch_set_launch(dv_batch* b, int32_t grid, int32_t chunk, int32_t contiguous,
                               int32_t blocks_per_sm);
DV_API int dv_batch_get_launch(dv_batch* b, int32_t* grid, int32_t* chunk, int32_t* contiguous,
                               int32_t* blocks_per_sm, int32_t* max_grid);
/* Replay each step from a captured CUDA graph (collision + solve); returns
 * DV_ERR_UNSUPPORTED and keeps stream launches if capture fails. */
DV_API int dv_batch_set_graph(dv_batch* b, int32_t enable);
/* Times candidate launch shapes on the batch's own scenes (steps_per_trial
 * steps each, state restored after every trial and at the end), checks that
 * all of them give bit-identical states, and keeps the fastest. */
DV_API int dv_batch_autotune(dv_batch* b, int32_t steps_per_trial, dv_tune_report* out);
DV_API int64_t dv_batch_launch_count(dv_batch* b);

/* ------------------------------------------------------------------------
 * Serving.  No counterpart in the reference.  A server keeps scenes (requests
 * for nsteps time steps each) resident on the device and steps every resident
 * scene together; requests that arrive while others run are admitted as
 * soon as a slot and the HBM budget allow, and a scene leaves when its steps
 * are done (continuous batching).  Membership changes move the resident
 * scenes' state device-to-device; a scene's results are bit-identical to the
 * same scene stepped alone with the same precision.  The caller drives it:
 * dv_server_submit when a request arrives, dv_server_round repeatedly (one
 * round = admissions, steps_per_round steps, retirements), dv_server_poll for
 * finished requests.  Times are seconds on the server's steady clock.
 * ------------------------------------------------------------------------ */
typedef struct dv_server dv_server;

typedef struct dv_server_config {
  double hbm_budget_bytes;   /* admission budget for resident scenes (estimate per scene) */
  int32_t max_active;        /* resident scenes at most */
  int32_t steps_per_round;   /* steps between admission and retirement checks */
  int32_t precision;         /* DV_PREC_FP64 or DV_PREC_MIXED for every scene */
  int32_t use_graph;         /* replay steps from a CUDA graph between membership changes */
  int32_t keep_states;       /* keep each finished scene's final p, v for dv_server_result_state */
  int32_t max_resident_bodies; /* resident bodies at most, 0 = no limit: bounds the work (and so
                                  the time) of each step; a scene larger than the limit is
                                  admitted alone */
} dv_server_config;

typedef struct dv_request_result {
  int64_t id;
  int32_t nb;
  int32_t nsteps;            /* steps done: the steps asked for, unless retired early */
  int32_t status;            /* first solver error of the scene, DV_OK otherwise; DV_ERR_ARG
                                when its scene went over the pair kernels' partner limits
                                (dv_step): retired at once, the others served on */
  int32_t rounds;
  int32_t solves;            /* its steps that solved (contacts or rows present) */
  int32_t solves_at_tolerance; /* ... whose solve ended below the solver tolerance */
  double t_submit, t_admit, t_done;
  double contact_steps;      /* contacts summed over its steps */
  double step_ms_mean, step_ms_p50, step_ms_p99;  /* device time of the steps it took part in */
  double bytes;              /* admission estimate */
  /* Solver work summed over its steps (for byte models): iterations in the
   * solve's working precision (FP32 under DV_PREC_MIXED, FP64 refinement
   * iterations counted apart), refinement iterations, backtracks, each also
   * weighted by the step's contacts; the contacts and count of its refined
   * solves. */
  double iterations, iteration_contacts;
  double refine_iterations, refine_iteration_contacts;
  double backtracks, backtrack_contacts;
  double refined_solves, refined_contacts;
} dv_request_result;

typedef struct dv_server_stats {
  int64_t submitted, admitted, completed, pending, active, rounds, reconfigures, steps;
  double bytes_in_use;
  double contact_steps;      /* contacts summed over every scene and step */
  double device_ms;          /* device time of all steps */
} dv_server_stats;

DV_API int dv_server_default_config(dv_server_config* cfg);
DV_API int dv_server_create(const dv_server_config* cfg, dv_server** out);
DV_API int dv_server_destroy(dv_server* s);
DV_API int dv_server_set_stream(dv_server* s, void* cuda_stream);
DV_API double dv_server_clock(dv_server* s);
/* Queues a request; bodies are copied.  Returns DV_ERR_OOM if the scene alone
 * exceeds the budget. */
DV_API int dv_server_submit(dv_server* s, const dv_body_desc* bodies, int32_t nb,
                            const dv_params* params, int32_t nsteps, int64_t* id);
/* One round; *busy = 0 when nothing is resident or pending after it. */
DV_API int dv_server_round(dv_server* s, int32_t* busy);
/* Finished requests since the last poll (up to cap; *n = how many written). */
DV_API int dv_server_poll(dv_server* s, dv_request_result* out, int32_t cap, int32_t* n);
/* Final positions / velocities of a finished request (keep_states); releases them. */
DV_API int dv_server_result_state(dv_server* s, int64_t id, double* p, double* v);
DV_API int dv_server_get_stats(dv_server* s, dv_server_stats* out);

/* Failure detection without a fault: runs the solve kernels' bounded waits
 * (grid barrier, bulk-copy mbarrier) against conditions that never become
 * true -- a CTA that never arrives, bytes no copy brings -- with a limit of
 * limit_ms, and reports whether each wait ended by its time limit
 * (*barrier_timed_out, *copy_timed_out = 1) and the error bits it left.  The
 * device stays usable afterwards. */
DV_API int dv_selftest_bounded_waits(int32_t limit_ms, int32_t* barrier_timed_out,
                                     int32_t* copy_timed_out, uint32_t* error_bits);

#ifdef __cplusplus
}
#endif
#endif /* DVIDE_H_ */
