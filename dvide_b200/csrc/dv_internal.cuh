// dv_internal.cuh -- device-side layout of one scene and the kernels' entry
// points.  Data layout in HBM (all device-resident between calls):
//
//   bodies (nb):  p4, v4, k4, f4, w4, fc4 as double4 (x, y, z, unused) so a
//                 body is one 32-byte sector for the random gathers of the
//                 narrowphase and the Schur product; minv (double, 0 = fixed);
//                 geom4 (gx, gy, gz, 1 if box); family (int).
//   contacts:     sorted by (A, B) like the reference's thrust::unique of
//                 64-bit pair keys (CollisionDetector.cu:319-325).  ids A/B
//                 (uint32), frame n,u,v as 9 planes, gap, location (3 planes),
//                 r (3 planes); every per-contact 3-vector is 3 planes of
//                 stride `ccap` (structure of arrays, coalesced 8-byte loads).
//   incidence:    contacts where a body is B, in ascending contact order
//                 (stable radix sort by B); contacts where it is A are the
//                 contiguous range [cbase[b], cbase[b+1]).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "dv_common.cuh"

namespace dv {

struct GridInfo {
  double ox, oy, oz;        // global origin (AABB union min - 0.01, CollisionDetector.cu:566-568)
  double inv_w;             // 1 / cell width
  int dx, dy, dz;           // cells per axis
  int ncells;
  unsigned long long lo[3]; // ordered-bits AABB min accumulator
  unsigned long long hi[3]; // ordered-bits AABB max accumulator
};

// Scalar state of one APGD solve, owned by the controller CTA of the
// persistent kernel (APGD.cu:208-223, 266-332).  Iterates live in five
// rotating buffers G[0..4] with their Schur products NG[0..4]: cur = gamma_k,
// prev = gamma_{k-1}, nw = target of gamma_new, best = gamma_hat (-1 before the
// first accepted iterate); the fifth holds the next iterate computed ahead.
struct ApgdCtl {
  double L, t, theta, theta_new, beta;
  double obj1, obj2, obj2_base;
  double residual;      // best residual so far (APGD.cu:214, 293-301)
  double objective;     // objective of the best iterate (APGD.cu:353-354)
  double gdiff, ginv;   // 1 / nc^2 and its reciprocal (APGD.cu:92, 98)
  double L0;
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
  // device time between consecutive grid-barrier releases, by the phase that
  // ended at the barrier (globaltimer ns): see kPhase* in dv_apgd.cu
  unsigned long long last_release;
  unsigned long long phase_ns[8];
  unsigned long long phase_count[8];
};

struct SceneDev {
  int nb = 0;
  int n_small = 0, n_large = 0;
  // bodies
  double4 *p4 = nullptr, *v4 = nullptr, *k4 = nullptr, *f4 = nullptr, *w4 = nullptr, *fc4 = nullptr;
  double4* geom4 = nullptr;
  double* minv = nullptr;
  int* family = nullptr;
  int* small_ids = nullptr;   // sphere bodies binned in the grid
  int* large_ids = nullptr;   // boxes, tested against all bodies
  // collision scratch
  double4 *amin = nullptr, *amax = nullptr;   // shifted AABBs
  int4* cell = nullptr;                       // cell coords + linear id (small bodies)
  uint32_t *keyA = nullptr, *valA = nullptr, *keyB = nullptr, *valB = nullptr;  // radix buffers
  size_t radix_cap = 0;
  uint32_t* radix_hist = nullptr;
  size_t radix_hist_cap = 0;
  int* cell_start = nullptr;
  int* cell_end = nullptr;
  int ncell_cap = 0;
  int* cnt_cont = nullptr;    // contacts with A = body
  int* cnt_cand = nullptr;    // candidate pairs with A = body
  int* cbase = nullptr;       // exclusive scan of cnt_cont (nb + 1)
  int* scan_tmp = nullptr;
  size_t scan_tmp_cap = 0;
  int* large_chunk = nullptr; // per (large body, chunk) counts
  int* large_chunk_off = nullptr;
  int large_chunks = 0;
  GridInfo* grid = nullptr;
  int* counters = nullptr;    // [0] nc, [1] npossible (device)
  int* h_counters = nullptr;  // pinned mirror
  double W = 0;               // widest small AABB (2 (r_max + envelope))
  // contacts
  size_t ccap = 0;
  int nc = 0, npossible = 0;
  uint32_t *ida = nullptr, *idb = nullptr;
  double* F = nullptr;        // 9 planes
  double* gap = nullptr;
  double* loc = nullptr;      // 3 planes
  double* r = nullptr;        // 3 planes
  int* binc_start = nullptr;  // nb + 1
  uint32_t* binc = nullptr;   // contact ids sorted by B
  // flat incidence per body in ascending contact order: B-side contacts with
  // bit 31 set (sign -1), then A-side contacts; body b owns [inc_start[b], inc_start[b+1])
  int* inc_start = nullptr;   // nb + 1
  uint32_t* inc = nullptr;    // 2 * ccap
  // APGD work: iterates and their Schur products, 3 planes each (stride ccap)
  double* G[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  double* NG[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  double4* q = nullptr;
  double* part = nullptr;     // reduction partials
  int part_tiles = 0;
  // warm-start buffer (System::gamma_d): 3 planes, stride gcap
  double* gamma = nullptr;
  size_t gcap = 0;
  int gsize = 0;
  ApgdCtl* ctl = nullptr;
  ApgdCtl* h_ctl = nullptr;   // pinned mirror
  unsigned* bar = nullptr;    // grid barrier words
};

// ---- sort / scan (dv_sort.cu) ----
size_t radix_hist_size(size_t n);
// Stable LSD radix sort of (key, value) by the low `bits` bits of key.
// On return the sorted data is in (k0, v0); k1/v1 are scratch.
void radix_sort_pairs(uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1, uint32_t* hist,
                      int n, int bits, cudaStream_t st, int64_t* launches);
size_t scan_tmp_size(size_t n);
// out[i] = sum_{j<i} in[i]; out[n] = total.  n may be 0.
void exclusive_scan_i32(const int* in, int* out, int n, int* tmp, cudaStream_t st,
                        int64_t* launches);

// ---- collision (dv_collide.cu) ----
// Counts candidates and contacts; leaves nc / npossible in sd.counters.
void collide_count(SceneDev& sd, double envelope, cudaStream_t st, int64_t* launches);
// Writes the sorted contact list, frames and the B-side incidence.
void collide_write(SceneDev& sd, double envelope, cudaStream_t st, int64_t* launches);

// ---- step (dv_apgd.cu) ----
struct SolveConfig {
  double h, mu, tol;
  int max_iter, max_bt, warm, precision;
  int grid;   // CTAs of the persistent kernel
};
int apgd_max_ctas(int precision);
void launch_step_solve(SceneDev& sd, const SolveConfig& cfg, cudaStream_t st, int64_t* launches);
void launch_step_nocontact(SceneDev& sd, double h, cudaStream_t st, int64_t* launches);

}  // namespace dv
