// dv_internal.cuh -- device-side layout of an engine (one or many scenes) and
// the kernels' entry points.
//
// An engine steps S independent scenes ("segments") together.  A plain
// System is an engine with one segment; a batch or a server holds many.
// Every per-segment computation (collision grid, contact order, reductions,
// APGD control) depends only on that segment's own data, so a scene's
// results are bit-identical alone and in any mix.
//
// Data layout in HBM (all device-resident between calls):
//
//   bodies (nb, all segments concatenated, segment s owns [b0, b1)):
//                 p4, v4, k4, f4, fc4 as double4 (x, y, z, unused) so a body is
//                 one 32-byte sector for the random gathers of the narrowphase;
//                 w4 (Schur body vector; float4 in the mixed-precision solve);
//                 minv (double, 0 = fixed); geom4 (gx, gy, gz, 1 if box);
//                 family (int); bseg (segment of the body).
//   contacts:     per segment sorted by (A, B) like the reference's
//                 thrust::unique of 64-bit pair keys (CollisionDetector.cu:
//                 319-325); segment s owns [c0, c0 + nc), c0 a multiple of 256.
//                 ids A/B (uint32, global body ids), normal n as 3 planes (plus
//                 u, v for the frame accessors), gap, location (3 planes); every
//                 per-contact 3-vector is 3 planes of stride `ccap` (structure
//                 of arrays, coalesced loads).
//   tiles:        512 contacts; segment s owns tiles [t0, t0 + nt); tile k of
//                 a segment covers its contacts [512 k, 512 k + 512).  Per-tile
//                 partial sums are folded per segment in a fixed order.
//   incidence:    per body, its contacts in ascending contact order: those
//                 where it is B (bit 31 set), then those where it is A.
//   bilateral:    DOF rows (System::addBilateralConstraintDOF): segment s
//                 owns rows [bil0, bil0 + nbil) and the tiles after its
//                 contact tiles, ceil(nbil / 512) of them (a row is one item);
//                 per body, its rows in ascending order (bil_inc); iterates
//                 and products of the rows in 12 planes of nbil doubles.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "dv_common.cuh"

namespace dv {

constexpr int kContactAlign = 256;  // segment contact ranges start on this multiple

struct GridInfo {
  double ox, oy, oz;        // origin (AABB union min - 0.01, CollisionDetector.cu:566-568)
  double inv_w;             // 1 / cell width
  int dx, dy, dz;           // cells per axis
  int ncells;
  unsigned long long lo[3]; // ordered-bits AABB min accumulator
  unsigned long long hi[3]; // ordered-bits AABB max accumulator
};

// Read-only description of one segment (host-written).
struct SegParams {
  double h, mu, tol, env;
  double W;                 // grid cell lower bound: widest small AABB, 2 (r_max + env)
  int max_iter, max_bt, warm;
  int exact;                // 1: FP64 length/normalize in narrowphase and frame (opt-in)
  int active;               // 0: the segment is skipped entirely (free server slot)
  int b0, b1;               // bodies
  int s0, s1;               // small (gridded) bodies in small_ids
  int l0, l1;               // large bodies (boxes) in large_ids
  int cell_base, cell_cap;  // global cell ids [cell_base, cell_base + cell_cap)
  int wbase, wcap;          // warm-start region [wbase, wbase + wcap) of the gamma arena
  int bil0, nbil;           // bilateral DOF rows [bil0, bil0 + nbil) (System.cu:510-532)
  int ar;                   // APGD anti-relaxation (APGD.cu:335-345)
  int refine;               // mixed precision: FP64 iterations after a stalled FP32 phase (0: off)
};

// Scalar state of one APGD solve (APGD.cu:208-223, 266-332).  Iterates live in
// five rotating buffers G[0..4] with their Schur products NG[0..4]: cur =
// gamma_k, prev = gamma_{k-1}, nw = target of gamma_new, best = gamma_hat (-1
// before the first accepted iterate); the fifth holds the next iterate computed
// ahead.
struct ApgdCtl {
  double L, t, theta, theta_new, beta;
  double obj1, obj2, obj2_base;
  double residual;      // best residual so far (APGD.cu:214, 293-301)
  double objective;     // objective of the best iterate (APGD.cu:353-354)
  double gdiff, ginv;   // 1 / nc^2 and its reciprocal (APGD.cu:92, 98)
  double L0;
  double fx;            // PGJ: primal feasibility of the iterate computed last
  double yb;            // beta used for y_k = (1+yb) gamma_k - yb gamma_{k-1}
  int k;                // iteration index
  int mode;             // next contact pass: 0 full iteration, 1 backtrack
  int done;
  int restart;          // g.(gamma_new - gamma) > 0 for the current gamma_new
  int cur, prev, nw, best;
  int yr;               // y_k = gamma_k (first iteration or after a restart)
  int first;            // first iteration: N y_0 is a Schur product
  int backtracks;
  unsigned err;
  int iterations;
  int sweeps;           // iterations executed
  int rsel;             // anti-relaxation: plane of the current r_n and ar (the other: next)
  double objN;          // anti-relaxation: half of gamma_hat . N gamma_hat
  // mixed precision with FP64 refinement: accepted iterations since the best
  // residual last improved (FP32 phase); whether the FP64 phase refines this
  // solve (set at the end of the FP32 phase); the FP64 phase's iterations; the
  // FP32 phase's counts while the FP64 phase runs
  int since_best;
  int refined;
  int refine_it;
  int it_lo, bt_lo, sw_lo;
};

// Per-segment results of the current step (device-written).
struct SegState {
  int nc, npossible;
  int c0;               // first contact slot (multiple of kContactAlign)
  int t0, nt;           // tiles
  int delta;            // c0 - (unpadded global offset of the segment's first contact)
  int gsize;            // warm-start length (System::gamma_d / 3); kept when nc = 0
  unsigned arrive;      // tile arrivals in the current pass
  unsigned err;         // error bits of this segment's last step
  int pad_;
  ApgdCtl ctl;
};

// Engine-wide words (device).
struct EngineWords {
  int nc_total;         // unpadded contacts of all segments
  int nc_pad;           // padded contact slots in use
  int ntiles;           // tiles in use
  int npossible;
  int n_small;          // gridded bodies (constant)
  int stop_on_seg_err;  // 1: a segment's solver error also sets err (plain System semantics)
  unsigned err;         // error bits (kErr*); sticky: every kernel of a step skips its work while set
  int steps_done;       // steps completed since creation
  int active;           // segments still iterating (solve kernel)
  int step_count;       // segments that request a step pass next iteration
  int step_needed;      // latched step_count for the current iteration
  unsigned bar[4];      // grid barrier: [0] arrivals, [1] generation, [2] error bits
  unsigned long long last_release;
  unsigned long long phase_ns[8];
  unsigned long long phase_count[8];
  unsigned long long wait_limit_ns;  // every bounded wait (grid barrier, bulk copy) ends after this
  // Work lists of the iterating passes (solve kernel): once half the segments
  // that were iterating at the last rebuild have finished, the contact tiles
  // and body ranges of the segments still iterating are gathered into
  // SceneDev::act_tiles / act_bodies, and the passes walk those instead of
  // every tile and body.
  int act_on;           // 1: the lists are in use
  int act_nt;           // entries of act_tiles
  int act_nb;           // entries of act_bodies
  int act_base;         // segments iterating when the lists were last built (nseg before)
  int act_rebuild;      // 1: rebuild the lists before the next pass
  int n_wide;           // spheres of this step with more partners than the warp pair kernel lists
};

// Spheres per step whose partners (larger ids) exceed the warp pair kernel's
// list, the CTAs that take them in turn, and the partners one such sphere may
// have.
constexpr int kWideSpheres = 65536;
constexpr int kWideGrid = 256;
constexpr int kWidePartners = 8192;

struct SceneDev {
  int nb = 0, nseg = 0;
  int n_small = 0, n_large = 0;
  int precision = DV_PREC_FP64;
  int solver = DV_SOLVER_APGD;  // every segment of an engine uses the same solver
  // segments
  SegParams* seg = nullptr;     // nseg
  SegState* sst = nullptr;      // nseg
  GridInfo* grid = nullptr;     // nseg
  int* seg_tstart = nullptr;    // nseg + 1 tile starts (for tile -> segment lookup)
  int* tseg = nullptr;          // tile -> segment
  unsigned* donemask = nullptr; // (nseg + 31) / 32 words: segments not iterating
  EngineWords* ew = nullptr;
  // bodies
  double4 *p4 = nullptr, *v4 = nullptr, *k4 = nullptr, *f4 = nullptr, *w4 = nullptr, *fc4 = nullptr;
  double4* geom4 = nullptr;
  double* minv = nullptr;
  int* family = nullptr;
  int* bseg = nullptr;
  int* small_ids = nullptr;   // sphere bodies binned in the grid, grouped by segment
  int* large_ids = nullptr;   // boxes, tested against all bodies of their segment
  int max_seg_chunks = 0;     // largest ceil(segment bodies / 256)
  // collision scratch
  double4 *amin = nullptr, *amax = nullptr;   // shifted AABBs
  int4* cell = nullptr;                       // cell coords + global linear id
  uint32_t *keyA = nullptr, *valA = nullptr, *keyB = nullptr, *valB = nullptr;  // radix buffers
  size_t radix_cap = 0;
  uint32_t* radix_hist = nullptr;
  size_t radix_hist_cap = 0;
  int* cell_start = nullptr;
  int* cell_end = nullptr;
  int ncell_cap = 0;
  int* cnt_cont = nullptr;    // contacts with A = body
  int* cnt_cand = nullptr;    // candidate pairs with A = body
  int* wide_ids = nullptr;    // kWideSpheres: the spheres of EngineWords::n_wide
  int* cbase = nullptr;       // exclusive scan of cnt_cont (nb + 1), unpadded
  int* scan_tmp = nullptr;
  size_t scan_tmp_cap = 0;
  int* large_chunk = nullptr; // per (large body, chunk) counts
  int* large_chunk_off = nullptr;
  int large_chunks = 0;
  // contacts
  size_t ccap = 0;            // contact slots
  int tcap = 0;               // tiles
  uint32_t *ida = nullptr, *idb = nullptr;
  double* F = nullptr;        // 9 planes (n, u, v)
  float* nf = nullptr;        // 3 planes: n rounded to float (mixed-precision solve)
  double* gap = nullptr;
  double* loc = nullptr;      // 3 planes
  double* r = nullptr;        // 3 planes (float planes in the mixed solve)
  int* binc_start = nullptr;  // nb + 1
  uint32_t* binc = nullptr;   // contact ids sorted by B
  int* inc_start = nullptr;   // nb + 1
  uint32_t* inc = nullptr;    // 2 * ccap
  // APGD work: iterates and their Schur products, 3 planes each (stride ccap)
  double* G[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  double* NG[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  double4* q = nullptr;
  int* act_tiles = nullptr;   // tcap: contact tiles of the segments still iterating
  int4* act_bodies = nullptr; // act_bcap: (first body, end body, segment, 0), at most 256 bodies each
  size_t act_bcap = 0;
  double* part = nullptr;     // reduction partials, 9 x tcap
  // bilateral DOF rows (FP64 APGD only)
  int nbil = 0;               // rows of all segments
  int2* bil_off = nullptr;    // per row: element offsets 4 body + axis of DOF A, B (-1: none)
  double4* bil_info = nullptr;  // per row: velocity, start time, p0 (System.cu:1526-1544), 0
  int* bil_inc_start = nullptr; // nb + 1
  uint32_t* bil_inc = nullptr;  // (row << 3) | (axis << 1) | (1: the row's -1 entry)
  double* bil_work = nullptr; // 12 planes of nbil: G[0..4], NG[0..4], r, q
  double* bil_gam = nullptr;  // the rows' impulses of the last solve (System::gamma_d head)
  double* bil_b = nullptr;    // b of the rows at the last step
  double* seg_time = nullptr; // nseg: System::time at the step's start (rows with a velocity)
  // APGD anti-relaxation (one-scene engines, FP64): the normal component of r
  // and the anti-relaxation vector, current and next (2 planes of ccap each),
  // and v = Minv (k + D^T x) of the iterate x under test (nb)
  int anti_relax = 0;
  // mixed precision: some segment asks for FP64 refinement (a second,
  // FP64 solve launch follows the FP32 one in every step)
  int refine_any = 0;
  int refine_grid = 0;          // co-resident CTAs of the FP64 solve kernel
  double* ar_r0 = nullptr;
  double* ar_v = nullptr;
  double4* v_ar = nullptr;
  size_t v_ar_cap = 0;
  // warm-start arena (System::gamma_d of every segment): 3 planes of stride
  // wtotal; segment s owns [wbase, wbase + wcap), positional within it
  double* gamma = nullptr;
  size_t wtotal = 0;
  // matched warm start (warm_start 2): per warm slot the B body of its pair
  // (segment-relative); per body the segment-relative range of the contacts
  // where it was A at the last solve
  uint32_t* wid = nullptr;    // wtotal
  int* ws = nullptr;          // nb
  int* wc = nullptr;          // nb
  // host mirrors
  EngineWords* h_ew = nullptr;    // pinned
  SegState* h_sst = nullptr;      // pinned, nseg
};

// ---- sort / scan (dv_sort.cu) ----
size_t radix_hist_size(size_t n);
// Stable LSD radix sort of (key, value) by the low `bits` bits of key.  The
// item count is read on the device from *n_dev (at most n_cap).  On return the
// sorted data is in (k0, v0); k1/v1 are scratch.
void radix_sort_pairs(uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1, uint32_t* hist,
                      const int* n_dev, int n_cap, int bits, cudaStream_t st, int64_t* launches);
size_t scan_tmp_size(size_t n);
// out[i] = sum_{j<i} in[i]; out[n] = total.  n may be 0.
void exclusive_scan_i32(const int* in, int* out, int n, int* tmp, cudaStream_t st,
                        int64_t* launches);

// ---- collision (dv_collide.cu) ----
// The whole collision pipeline of one step: contacts of every active segment,
// their tiles and the body incidence.  Sizes are read on the device; a
// capacity overflow sets kErrCapacity in EngineWords::err and leaves the
// contact arrays unwritten.
void collide(SceneDev& sd, cudaStream_t st, int64_t* launches);

// ---- step (dv_apgd.cu) ----
struct SolveConfig {
  int grid;           // CTAs of the persistent kernel
  int chunk;          // tiles a CTA takes at a time (1, 2, 4)
  int contiguous;     // 1: CTA c takes a contiguous range of tiles; 0: round robin
  int blocks_per_sm;  // register budget: 2 (128 per thread) or 3 (80, FP32 iterates only)
};
int apgd_max_ctas(int precision, int blocks_per_sm);
// solve_only: System::DoTimeStep's solve without the update (the solver's
// own solve(): v, p, f_contact and the clock are left as they are)
void launch_step_solve(SceneDev& sd, const SolveConfig& cfg, cudaStream_t st, int64_t* launches,
                       bool solve_only = false);
// ---- PGJ (dv_pgj.cu) ----
int pgj_max_ctas(int precision);
void launch_pgj_solve(SceneDev& sd, const SolveConfig& cfg, cudaStream_t st, bool solve_only);
int pgs_max_ctas();
void launch_pgs_solve(SceneDev& sd, const SolveConfig& cfg, cudaStream_t st, bool solve_only);

}  // namespace dv
