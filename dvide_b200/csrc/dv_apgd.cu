// dv_apgd.cu -- the time step after collision detection, as ONE persistent
// cooperative kernel per step:
//
//   applied impulse k = M v + h f             System.cu:1411-1417, 1502-1514
//   Schur vector r = D Minv k + b             System.cu:1516-1524, 1561-1580
//   APGD solve (all iterations)               APGD.cu:164-361
//   v = Minv (k + D^T gamma), p += h v        System.cu:570-583
//
// The reference runs each BLAS-1 call, SpMV and projection as its own launch
// and brings every dot/nrm2/nrmmax back to the host (APGD.cu:227-350).  Here
// the scalar control (step size, Lipschitz backtracking, restart, best
// iterate, convergence) runs on the device: the last CTA to reach each grid
// barrier folds the per-tile partial sums in a fixed order, executes the
// control logic and releases the others.
//
// Matrix-free N x = D Minv D^T x (D's block of contact c is [+F_c^T | -F_c^T],
// F_c = [n u v]):
//   contact pass: q_c = F_c x_c (written by the pass that produced x_c)
//   body pass:    w_b = minv_b * (sum of -q_c over contacts where b is B,
//                 then +q_c where b is A, ascending contact order; no atomics)
//   contact pass: (N x)_c = F_c^T (w_A - w_B), fused with the APGD vector
//                 updates, the cone projection and the reductions.
//
// One Schur product per iteration.  The reference evaluates N y_k with its own
// product (APGD.cu:229, 239) and N gamma_new twice more (:237, :276).  Since
// y_k = (1 + b) gamma_k - b gamma_{k-1} (APGD.cu:273) or gamma_k after a
// restart (:315), N y_k is formed here from the stored products of the two
// previous iterates; N gamma_new is computed once and serves the objective and
// the residual.  Iterates and their products rotate through four buffers, so
// y, g and gamma_hat are never copied.  The CPU oracle evaluates the same
// sequence (apgd_solve_fused), and bit-for-bit the same arithmetic.
//
// Work is split in tiles of 512 contacts (2 per thread) and 256 bodies;
// CTA b owns tiles b, b + G, ...  Every wait has a time limit.
#include <stdio.h>
#include <stdlib.h>

#include "dv_internal.cuh"

namespace dv {

namespace {

constexpr int kNQ = 7;      // partial-sum slots per tile
constexpr int kQMax = kNQ;  // slot of the per-tile maximum

// Phases timed between grid-barrier releases (ApgdCtl::phase_ns).
enum Phase : int {
  kPhaseSetup = 0,     // k, r, Lipschitz estimate
  kPhaseStep = 1,      // gamma_new = P(y - t g), full iteration
  kPhaseBacktrack = 2, // gamma_new recomputed after L doubled
  kPhaseBody = 3,      // body gather w = Minv D^T q
  kPhaseProduct = 4,   // N gamma_new, objective, residual
  kPhaseFinal = 5,     // gamma = gamma_hat, update
};

struct KArgs {
  int nb, nc;
  int nt, nbt;
  size_t S;    // plane stride of contact arrays
  size_t GS;   // plane stride of the warm-start buffer
  double4* p4;
  double4* v4;
  double4* k4;
  const double4* __restrict__ f4;
  double4* w4;
  double4* fc4;
  const double* __restrict__ minv;
  const uint32_t* __restrict__ ida;
  const uint32_t* __restrict__ idb;
  const double* __restrict__ F;
  const double* __restrict__ gap;
  double* r;
  const int* __restrict__ inc_start;
  const uint32_t* __restrict__ inc;
  double* G[5];
  double* NG[5];
  double4* q;
  double* gamma;
  double* part;
  int ptiles;
  ApgdCtl* ctl;
  unsigned* bar;   // [0] arrivals, [1] generation, [2] error bits
  double h, mu, tol;
  int max_iter, max_bt, warm;
};

struct Frame {
  double n0, n1, n2, u0, u1, u2, v0, v1, v2;
};

// Frame modes: 0 loads n, u, v; 1 recomputes u and v from n with the
// narrowphase's own function, so both modes see the same bits.
__device__ inline void complete_frame(Frame& f, int mode) {
  if (mode == 1) {
    d3 u, v;
    frame_from_normal(mk3(f.n0, f.n1, f.n2), &u, &v);
    f.u0 = u.x; f.u1 = u.y; f.u2 = u.z;
    f.v0 = v.x; f.v1 = v.y; f.v2 = v.z;
  }
}

template <int kMode>
__device__ inline Frame load_frame(const KArgs& a, int c) {
  const double* F = a.F;
  size_t S = a.S;
  Frame f;
  f.n0 = __ldg(F + 0 * S + c);
  f.n1 = __ldg(F + 1 * S + c);
  f.n2 = __ldg(F + 2 * S + c);
  if (kMode == 0) {
    f.u0 = __ldg(F + 3 * S + c); f.u1 = __ldg(F + 4 * S + c); f.u2 = __ldg(F + 5 * S + c);
    f.v0 = __ldg(F + 6 * S + c); f.v1 = __ldg(F + 7 * S + c); f.v2 = __ldg(F + 8 * S + c);
  }
  complete_frame(f, kMode);
  return f;
}

// q = F x : q_k = (n_k x0 + u_k x1) + v_k x2
__device__ inline double4 f_times(const Frame& f, double x0, double x1, double x2) {
  return make_double4((f.n0 * x0 + f.u0 * x1) + f.v0 * x2, (f.n1 * x0 + f.u1 * x1) + f.v1 * x2,
                      (f.n2 * x0 + f.u2 * x1) + f.v2 * x2, 0.0);
}

// (F^T d)_row = (f_x d_x + f_y d_y) + f_z d_z with d = w_A - w_B
__device__ inline void ft_times(const Frame& f, double4 wa, double4 wb, double* o0, double* o1,
                                double* o2) {
  double d0 = wa.x - wb.x, d1 = wa.y - wb.y, d2 = wa.z - wb.z;
  *o0 = (f.n0 * d0 + f.n1 * d1) + f.n2 * d2;
  *o1 = (f.u0 * d0 + f.u1 * d1) + f.u2 * d2;
  *o2 = (f.v0 * d0 + f.v1 * d1) + f.v2 * d2;
}

__device__ inline double dot3i(double a0, double a1, double a2, double b0, double b1, double b2) {
  return (a0 * b0 + a1 * b1) + a2 * b2;
}

// Folds NQ values of each thread; thread 0 gets the results.
template <int NQ>
__device__ inline void block_fold_multi(double (&v)[NQ], double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int qi = 0; qi < NQ; ++qi) v[qi] = warp_fold(v[qi]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int qi = 0; qi < NQ; ++qi) scratch[qi * 8 + warp] = v[qi];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int qi = 0; qi < NQ; ++qi) {
      double w = (lane < 8) ? scratch[qi * 8 + lane] : 0.0;
#pragma unroll
      for (int off = 4; off >= 1; off >>= 1) w = w + __shfl_down_sync(0xffffffffu, w, off);
      v[qi] = w;
    }
  }
  __syncthreads();
}

// Controller side: folds the per-tile partials of NQ quantities in the fixed
// order (slot j sums tiles j, j+256, ...; then the 256-slot tree).
template <int NQ>
__device__ inline void fold_tiles(const KArgs& a, double (&out)[NQ], double* scratch) {
  double v[NQ];
#pragma unroll
  for (int qi = 0; qi < NQ; ++qi) {
    double acc = 0.0;
    for (int t = threadIdx.x; t < a.nt; t += kThreads)
      acc = acc + __ldcg(a.part + (size_t)qi * a.ptiles + t);
    v[qi] = acc;
  }
  block_fold_multi<NQ>(v, scratch);
#pragma unroll
  for (int qi = 0; qi < NQ; ++qi) out[qi] = v[qi];
}

__device__ inline double fold_tiles_max(const KArgs& a, double* scratch) {
  double m = 0.0;
  for (int t = threadIdx.x; t < a.nt; t += kThreads)
    m = fmax(m, __ldcg(a.part + (size_t)kQMax * a.ptiles + t));
  double r = block_max256(m, scratch);
  __syncthreads();
  return r;
}

template <int NQ>
__device__ inline void write_partials(const KArgs& a, int tile, const double (&v)[NQ]) {
  if (threadIdx.x == 0) {
#pragma unroll
    for (int qi = 0; qi < NQ; ++qi) a.part[(size_t)qi * a.ptiles + tile] = v[qi];
  }
}

// Grid barrier.  The last CTA to arrive runs `ctl_fn` (all its threads),
// then releases the generation word.  Returns false after a timeout or an
// error raised by another CTA; the caller then leaves the kernel.
template <class Fn>
__device__ inline bool grid_sync(const KArgs& a, int phase, Fn ctl_fn) {
  __shared__ unsigned s_last, s_target;
  __shared__ int s_fail;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned ticket = atom_add_acq_rel(&a.bar[0], 1u);
    s_target = ticket / gridDim.x + 1u;
    s_last = (ticket % gridDim.x) == gridDim.x - 1u;
    s_fail = 0;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    ctl_fn();
    __syncthreads();
    if (threadIdx.x == 0) {
      ApgdCtl* C = a.ctl;
      unsigned long long now = global_ns();
      if (C->last_release) {
        C->phase_ns[phase] += now - C->last_release;
        C->phase_count[phase] += 1;
      }
      C->last_release = now;
      __threadfence();
      st_release(&a.bar[1], s_target);
    }
  } else if (threadIdx.x == 0) {
    uint64_t t0 = global_ns();
    unsigned polls = 0;
    while (ld_acquire(&a.bar[1]) < s_target) {
      __nanosleep(20);
      if ((++polls & 1023u) == 0u) {
        if (ld_acquire(&a.bar[2]) & (kErrBarrierTimeout | kErrCopyTimeout)) {
          s_fail = 1;
          break;
        }
        if (global_ns() - t0 > kBarrierTimeoutNs) {
          atomicOr(&a.bar[2], kErrBarrierTimeout);
          s_fail = 1;
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
  return !s_fail;
}

struct NoCtl {
  __device__ void operator()() const {}
};

// Sum of -q over B-side contacts, then +q over A-side contacts, ascending
// contact order (the flat incidence list); loads are issued in groups of
// eight, the additions stay in order.
__device__ inline double4 gather_q(const KArgs& a, int b) {
  double ax = 0.0, ay = 0.0, az = 0.0;
  const int s = __ldg(a.inc_start + b), e = __ldg(a.inc_start + b + 1);
  for (int i = s; i < e; i += 8) {
    uint32_t c[8];
    double4 q[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) c[j] = (i + j < e) ? __ldg(a.inc + i + j) : 0u;
#pragma unroll
    for (int j = 0; j < 8; ++j)
      q[j] = (i + j < e) ? a.q[c[j] & 0x7fffffffu] : make_double4(0, 0, 0, 0);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (i + j < e) {
        if (c[j] & 0x80000000u) {
          ax = ax - q[j].x; ay = ay - q[j].y; az = az - q[j].z;
        } else {
          ax = ax + q[j].x; ay = ay + q[j].y; az = az + q[j].z;
        }
      }
    }
  }
  return make_double4(ax, ay, az, 0.0);
}

// Schur body pass: w_b = minv_b * (D^T x)_b; fixed bodies keep w = 0.
__device__ inline void body_pass_schur(const KArgs& a) {
  for (int bt = blockIdx.x; bt < a.nbt; bt += gridDim.x) {
    int b = bt * kThreads + threadIdx.x;
    if (b < a.nb) {
      double mi = __ldg(a.minv + b);
      if (mi != 0.0) {
        double4 s = gather_q(a, b);
        a.w4[b] = make_double4(mi * s.x, mi * s.y, mi * s.z, 0.0);
      }
    }
  }
}

// A buffer holding none of the iterates in use (5 buffers, at most 4 in use).
__device__ inline int free_slot(int a, int b, int c, int d) {
  for (int i = 0; i < 5; ++i)
    if (i != a && i != b && i != c && i != d) return i;
  return 0;
}

// ---------------------------------------------------------------------------
// Shared-memory staging of the look-ahead pass, per warp.  A CTA walks its
// sub-tiles (256 consecutive contacts, kItemsPerThread per reduction tile) in
// order; warp w owns contacts [32w, 32w+32) of each sub-tile and two stages of
// its own.  While the warp computes sub-tile i from one stage, its lane 0 has
// already issued the bulk copies of sub-tile i+1's plane segments (256 bytes
// per plane) into the other stage, completed on the warp's own mbarrier, so
// warps never wait for each other except at the per-tile reduction.
// ---------------------------------------------------------------------------
constexpr int kWarps = kThreads / 32;
constexpr int kSub = kThreads;  // contacts per sub-tile
__host__ __device__ constexpr int kFramePlanes(int mode) { return mode == 0 ? 9 : 3; }
__host__ __device__ constexpr int kStagePlanesD(int mode) { return kFramePlanes(mode) + 12; }
__host__ __device__ constexpr unsigned kWarpStageBytes(int mode) {
  return (unsigned)kStagePlanesD(mode) * 32u * 8u + 2u * 32u * 4u;
}
__host__ __device__ constexpr size_t kDynSmem(int mode) {
  return (size_t)kWarps * 2 * kWarpStageBytes(mode) + (size_t)kWarps * 2 * 8;
}

struct Staging {
  unsigned char* base;  // warp w, stage s at base + (2w + s) * stage_bytes
  unsigned stage_bytes;
  uint64_t* bar;        // mbarrier of warp w, stage s: bar[2w + s]
  unsigned phase;       // bit s: parity the next wait on this warp's stage s expects
};

// Bounded wait for this warp's stage s; false after a timeout (error recorded).
__device__ inline bool wait_warp_stage(const KArgs& a, Staging& st, int s) {
  const int w = threadIdx.x >> 5;
  unsigned par = (st.phase >> s) & 1u;
  uint64_t* bar = st.bar + 2 * w + s;
  bool ok = mbar_try_wait(bar, par);
  if (!ok) {
    uint64_t t0 = global_ns();
    while (!(ok = mbar_try_wait(bar, par))) {
      if (global_ns() - t0 > kBarrierTimeoutNs) break;
    }
  }
  st.phase ^= (1u << s);
  if (!ok) atomicOr(&a.bar[2], kErrCopyTimeout);
  __syncwarp();
  return ok;
}

template <int kFrame, int kMinB>
__global__ void __launch_bounds__(kThreads, kMinB) k_step_solve(KArgs a) {
  __shared__ double scratch[kNQ * 8 + 8];
  extern __shared__ __align__(128) unsigned char dyn_smem[];
  const size_t S = a.S;
  const double h = a.h;
  Staging stg;
  stg.base = dyn_smem;
  stg.stage_bytes = kWarpStageBytes(kFrame);
  stg.bar = reinterpret_cast<uint64_t*>(dyn_smem + (size_t)kWarps * 2 * stg.stage_bytes);
  stg.phase = 0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < 2 * kWarps; ++i) mbar_init(stg.bar + i, 1);
    fence_mbar_init();
  }
  __syncthreads();

  // ---- applied impulse: k = m v + h f (m = 1/minv, 0 for fixed); w = minv k
  for (int bt = blockIdx.x; bt < a.nbt; bt += gridDim.x) {
    int b = bt * kThreads + threadIdx.x;
    if (b < a.nb) {
      double mi = __ldg(a.minv + b);
      double m = mi;
      if (m) m = 1.0 / m;
      double4 v = a.v4[b], f = a.f4[b];
      double4 k = make_double4(h * f.x + m * v.x, h * f.y + m * v.y, h * f.z + m * v.z, 0.0);
      a.k4[b] = k;
      a.w4[b] = make_double4(mi * k.x, mi * k.y, mi * k.z, 0.0);
    }
  }
  if (!grid_sync(a, kPhaseSetup, NoCtl{})) return;

  // ---- r = D (Minv k) + b; gamma_0 -> G[0]; e = gamma_0 - gamma_hat_0 (= gamma_0 - 1)
  for (int tile = blockIdx.x; tile < a.nt; tile += gridDim.x) {
    double acc[1] = {0.0};
    for (int m = 0; m < kItemsPerThread; ++m) {
      int c = tile * kTileItems + m * kThreads + threadIdx.x;
      if (c < a.nc) {
        Frame f = load_frame<kFrame>(a, c);
        double4 wa = a.w4[__ldg(a.ida + c)], wb = a.w4[__ldg(a.idb + c)];
        double d0, d1, d2;
        ft_times(f, wa, wb, &d0, &d1, &d2);
        double bn = __ldg(a.gap + c) / h;
        a.r[0 * S + c] = bn + d0;
        a.r[1 * S + c] = 0.0 + d1;
        a.r[2 * S + c] = 0.0 + d2;
        double g0, g1, g2;
        if (a.warm) {
          g0 = a.gamma[0 * a.GS + c];
          g1 = a.gamma[1 * a.GS + c];
          g2 = a.gamma[2 * a.GS + c];
        } else {
          g0 = 1.0; g1 = 0.0; g2 = 0.0;
        }
        a.G[0][0 * S + c] = g0; a.G[0][1 * S + c] = g1; a.G[0][2 * S + c] = g2;
        double e0 = g0 + (-1.0), e1 = g1 + (-1.0), e2 = g2 + (-1.0);
        acc[0] = acc[0] + dot3i(e0, e1, e2, e0, e1, e2);
        a.q[c] = f_times(f, e0, e1, e2);
      }
    }
    block_fold_multi<1>(acc, scratch);
    write_partials<1>(a, tile, acc);
  }
  if (!grid_sync(a, kPhaseSetup, [&]() {
        double s[1];
        fold_tiles<1>(a, s, scratch);
        if (threadIdx.x == 0) a.ctl->L0 = sqrt(s[0]);
      }))
    return;
  body_pass_schur(a);
  if (!grid_sync(a, kPhaseSetup, NoCtl{})) return;

  // ---- L = ||N e|| / ||e||; q = F gamma_0 for the first N y
  for (int tile = blockIdx.x; tile < a.nt; tile += gridDim.x) {
    double acc[1] = {0.0};
    for (int m = 0; m < kItemsPerThread; ++m) {
      int c = tile * kTileItems + m * kThreads + threadIdx.x;
      if (c < a.nc) {
        Frame f = load_frame<kFrame>(a, c);
        double4 wa = a.w4[__ldg(a.ida + c)], wb = a.w4[__ldg(a.idb + c)];
        double n0, n1, n2;
        ft_times(f, wa, wb, &n0, &n1, &n2);
        acc[0] = acc[0] + dot3i(n0, n1, n2, n0, n1, n2);
        double y0 = a.G[0][0 * S + c], y1 = a.G[0][1 * S + c], y2 = a.G[0][2 * S + c];
        a.q[c] = f_times(f, y0, y1, y2);
      }
    }
    block_fold_multi<1>(acc, scratch);
    write_partials<1>(a, tile, acc);
  }
  if (!grid_sync(a, kPhaseSetup, [&]() {
        double s[1];
        fold_tiles<1>(a, s, scratch);
        if (threadIdx.x == 0) {
          ApgdCtl* C = a.ctl;
          double L = sqrt(s[0]) / C->L0;
          C->L = L;
          C->t = 1.0 / L;
          C->theta = 1.0;
          double th = 1.0;
          C->theta_new = (-(th * th) + th * sqrt(th * th + 4.0)) / 2.0;
          C->beta = th * (1.0 - th) / (th * th + C->theta_new);
          C->residual = 10e30;
          C->objective = 0.0;
          double ncd = (double)a.nc;
          C->gdiff = 1.0 / (ncd * ncd);
          C->ginv = 1.0 / C->gdiff;
          C->k = 0;
          C->mode = 0;
          C->done = (a.max_iter <= 0) ? 1 : 0;
          C->iterations = 0;
          C->sweeps = 0;
          C->restart = 0;
          C->cur = 0;
          C->prev = -1;
          C->nw = 1;
          C->best = -1;
          C->yr = 1;
          C->yb = 0.0;
          C->first = 1;
          C->backtracks = 0;
          C->obj1 = C->obj2 = C->obj2_base = 0.0;
        }
      }))
    return;
  body_pass_schur(a);
  if (!grid_sync(a, kPhaseSetup, NoCtl{})) return;

  // ---- APGD iterations (APGD.cu:227-350)
  //
  // Each iteration is one body pass (w = Minv D^T q of gamma_new) and one
  // contact pass that computes N gamma_new, the objective and the residual of
  // iteration k, and -- assuming the Lipschitz test accepts gamma_new -- the
  // whole step of iteration k+1 (y, N y, g, gamma_new = P(y - t g), q).  When
  // the test fails (backtracking) the look-ahead is discarded and a step pass
  // recomputes gamma_new with the doubled L; the arithmetic of every value is
  // the same either way.
  bool step_pass = true;  // the first iteration's step: N y_0 is a product (w of gamma_0)
  for (;;) {
    if (__ldcg(&a.ctl->done)) break;  // maxIterations reached (0 included)
    if (step_pass) {
      const int first = __ldcg(&a.ctl->first);
      const int cur = __ldcg(&a.ctl->cur);
      const int prev = __ldcg(&a.ctl->prev);
      const int nw = __ldcg(&a.ctl->nw);
      const int yr = __ldcg(&a.ctl->yr);
      const double yb = __ldcg(&a.ctl->yb);
      const double ya = 1.0 + yb, ym = -yb;
      const double nt_ = -__ldcg(&a.ctl->t);
      const double* Gc = a.G[cur];
      const double* Gp = a.G[prev < 0 ? cur : prev];
      double* NGc = a.NG[cur];
      const double* NGp = a.NG[prev < 0 ? cur : prev];
      double* Gn = a.G[nw];
      for (int tile = blockIdx.x; tile < a.nt; tile += gridDim.x) {
        double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int m = 0; m < kItemsPerThread; ++m) {
          int c = tile * kTileItems + m * kThreads + threadIdx.x;
          if (c < a.nc) {
            Frame f = load_frame<kFrame>(a, c);
            double c0 = Gc[0 * S + c], c1 = Gc[1 * S + c], c2 = Gc[2 * S + c];
            double y0, y1, y2, N0, N1, N2;
            if (yr) {
              y0 = c0; y1 = c1; y2 = c2;
            } else {
              y0 = ya * c0 + ym * Gp[0 * S + c];
              y1 = ya * c1 + ym * Gp[1 * S + c];
              y2 = ya * c2 + ym * Gp[2 * S + c];
            }
            if (first) {
              double4 wa = a.w4[__ldg(a.ida + c)], wb = a.w4[__ldg(a.idb + c)];
              ft_times(f, wa, wb, &N0, &N1, &N2);
              NGc[0 * S + c] = N0; NGc[1 * S + c] = N1; NGc[2 * S + c] = N2;
            } else if (yr) {
              N0 = NGc[0 * S + c]; N1 = NGc[1 * S + c]; N2 = NGc[2 * S + c];
            } else {
              N0 = ya * NGc[0 * S + c] + ym * NGp[0 * S + c];
              N1 = ya * NGc[1 * S + c] + ym * NGp[1 * S + c];
              N2 = ya * NGc[2 * S + c] + ym * NGp[2 * S + c];
            }
            double r0 = a.r[0 * S + c], r1 = a.r[1 * S + c], r2 = a.r[2 * S + c];
            double g0 = N0 + r0, g1 = N1 + r1, g2 = N2 + r2;
            double x0 = y0 + nt_ * g0, x1 = y1 + nt_ * g1, x2 = y2 + nt_ * g2;
            project_cone<double>(x0, x1, x2, a.mu);
            Gn[0 * S + c] = x0; Gn[1 * S + c] = x1; Gn[2 * S + c] = x2;
            a.q[c] = f_times(f, x0, x1, x2);
            double t0 = x0 + (-1.0) * y0, t1 = x1 + (-1.0) * y1, t2 = x2 + (-1.0) * y2;
            double s0 = x0 + (-1.0) * c0, s1 = x1 + (-1.0) * c1, s2 = x2 + (-1.0) * c2;
            acc[0] = acc[0] + dot3i(g0, g1, g2, t0, t1, t2);
            acc[1] = acc[1] + dot3i(t0, t1, t2, t0, t1, t2);
            acc[2] = acc[2] + dot3i(g0, g1, g2, s0, s1, s2);
            if (first) {
              acc[3] = acc[3] + dot3i(y0, y1, y2, N0, N1, N2);
              acc[4] = acc[4] + dot3i(y0, y1, y2, r0, r1, r2);
            }
          }
        }
        block_fold_multi<5>(acc, scratch);
        write_partials<5>(a, tile, acc);
      }
      if (!grid_sync(a, first ? kPhaseStep : kPhaseBacktrack, [&]() {
            double s[5];
            fold_tiles<5>(a, s, scratch);
            if (threadIdx.x == 0) {
              ApgdCtl* C = a.ctl;
              if (C->first) C->obj2_base = 0.5 * s[3] + s[4];
              double nr = sqrt(s[1]);
              C->obj2 = C->obj2_base + (s[0] + 0.5 * C->L * (nr * nr));
              C->restart = (s[2] > 0) ? 1 : 0;
              C->first = 0;
            }
          }))
        return;
    }
    body_pass_schur(a);
    if (!grid_sync(a, kPhaseBody, NoCtl{})) return;

    // N gamma_new, objective (APGD.cu:237-238), residual (:90-102); then the
    // next iteration's step assuming gamma_new is accepted (:266-273, 312-332)
    {
      const int cur = __ldcg(&a.ctl->cur);
      const int prev = __ldcg(&a.ctl->prev);
      const int nw = __ldcg(&a.ctl->nw);
      const int best = __ldcg(&a.ctl->best);
      const int nw2 = free_slot(nw, cur, prev, best);
      const int restart = __ldcg(&a.ctl->restart);
      const double beta = __ldcg(&a.ctl->beta);
      const double ya = 1.0 + beta, ym = -beta;
      const double Lnext = 0.9 * __ldcg(&a.ctl->L);
      const double nt2 = -(1.0 / Lnext);
      const double gd = __ldcg(&a.ctl->gdiff);
      const double gA = __ldcg(&a.ctl->ginv);
      const double gB = -1.0 / gd;
      double* NGn = a.NG[nw];
      double* G2 = a.G[nw2];
      // staged planes: frame, gamma_new, r, gamma_k, N gamma_k; then ids A, B
      constexpr int FP = kFramePlanes(kFrame);
      constexpr int ND = kStagePlanesD(kFrame);
      const double* dsrc[ND];
#pragma unroll
      for (int p = 0; p < FP; ++p) dsrc[p] = a.F + p * S;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        dsrc[FP + k] = a.G[nw] + k * S;
        dsrc[FP + 3 + k] = a.r + k * S;
        dsrc[FP + 6 + k] = a.G[cur] + k * S;
        dsrc[FP + 9 + k] = a.NG[cur] + k * S;
      }
      const int nd_copy = restart ? FP + 6 : ND;
      const unsigned bytes = (unsigned)nd_copy * 32u * 8u + 2u * 32u * 4u;
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      const int my_tiles =
          (blockIdx.x < (unsigned)a.nt) ? (a.nt - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
      const int nsub = kItemsPerThread * my_tiles;
      // first contact of this warp's chunk of sub-tile i
      auto chunk_c0 = [&](int i) {
        return ((int)blockIdx.x + (i / kItemsPerThread) * (int)gridDim.x) * kTileItems +
               (i % kItemsPerThread) * kSub + warp * 32;
      };
      auto issue = [&](int i, int sidx) {
        int cw = chunk_c0(i);
        if (lane == 0 && cw < a.nc) {
          unsigned char* dst = stg.base + (size_t)(2 * warp + sidx) * stg.stage_bytes;
          uint64_t* bar = stg.bar + 2 * warp + sidx;
          // order this warp's earlier generic reads of the stage before the copies
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_arrive_expect_tx(bar, bytes);
          for (int p = 0; p < nd_copy; ++p) bulk_g2s(dst + (size_t)p * 256, dsrc[p] + cw, 256, bar);
          bulk_g2s(dst + (size_t)ND * 256, a.ida + cw, 128, bar);
          bulk_g2s(dst + (size_t)ND * 256 + 128, a.idb + cw, 128, bar);
        }
      };
      double acc[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      double mx = 0.0;
      bool bad = false, failed = false;
      if (nsub > 0) issue(0, 0);
      for (int i = 0; i < nsub; ++i) {
        const int sidx = i & 1;
        __syncwarp();  // the warp's reads of stage sidx^1 (sub-tile i-1) are done
        if (i + 1 < nsub) issue(i + 1, sidx ^ 1);
        const int cw = chunk_c0(i);
        if (cw < a.nc && !failed) {
          if (!wait_warp_stage(a, stg, sidx)) failed = true;
        }
        const int c = cw + lane;
        if (c < a.nc && !failed) {
          const double* sd =
              reinterpret_cast<const double*>(stg.base + (size_t)(2 * warp + sidx) * stg.stage_bytes);
          const uint32_t* su = reinterpret_cast<const uint32_t*>(sd + (size_t)ND * 32);
          const int j = lane;
          Frame f;
          f.n0 = sd[0 * 32 + j]; f.n1 = sd[1 * 32 + j]; f.n2 = sd[2 * 32 + j];
          if (kFrame == 0) {
            f.u0 = sd[3 * 32 + j]; f.u1 = sd[4 * 32 + j]; f.u2 = sd[5 * 32 + j];
            f.v0 = sd[6 * 32 + j]; f.v1 = sd[7 * 32 + j]; f.v2 = sd[8 * 32 + j];
          }
          complete_frame(f, kFrame);
          double4 wa = a.w4[su[j]], wb = a.w4[su[32 + j]];
          double N0, N1, N2;
          ft_times(f, wa, wb, &N0, &N1, &N2);
          NGn[0 * S + c] = N0; NGn[1 * S + c] = N1; NGn[2 * S + c] = N2;
          double x0 = sd[(FP + 0) * 32 + j], x1 = sd[(FP + 1) * 32 + j], x2 = sd[(FP + 2) * 32 + j];
          double r0 = sd[(FP + 3) * 32 + j], r1 = sd[(FP + 4) * 32 + j], r2 = sd[(FP + 5) * 32 + j];
          acc[0] = acc[0] + dot3i(x0, x1, x2, N0, N1, N2);
          acc[1] = acc[1] + dot3i(x0, x1, x2, r0, r1, r2);
          {
            double T0 = r0 + N0, T1 = r1 + N1, T2 = r2 + N2;
            T0 = x0 + (-gd) * T0; T1 = x1 + (-gd) * T1; T2 = x2 + (-gd) * T2;
            project_cone<double>(T0, T1, T2, a.mu);
            T0 = gA * x0 + gB * T0; T1 = gA * x1 + gB * T1; T2 = gA * x2 + gB * T2;
            double m0 = fabs(T0), m1 = fabs(T1), m2 = fabs(T2);
            bad |= (m0 != m0) || (m1 != m1) || (m2 != m2);
            mx = fmax(mx, fmax(m0, fmax(m1, m2)));
          }
          // look-ahead step of iteration k+1: y = (1+b) x - b gamma_k, or x after a restart
          double y0, y1, y2, M0, M1, M2;
          if (restart) {
            y0 = x0; y1 = x1; y2 = x2;
            M0 = N0; M1 = N1; M2 = N2;
          } else {
            double c0v = sd[(FP + 6) * 32 + j], c1v = sd[(FP + 7) * 32 + j], c2v = sd[(FP + 8) * 32 + j];
            y0 = ya * x0 + ym * c0v; y1 = ya * x1 + ym * c1v; y2 = ya * x2 + ym * c2v;
            M0 = ya * N0 + ym * sd[(FP + 9) * 32 + j];
            M1 = ya * N1 + ym * sd[(FP + 10) * 32 + j];
            M2 = ya * N2 + ym * sd[(FP + 11) * 32 + j];
          }
          double g0 = M0 + r0, g1 = M1 + r1, g2 = M2 + r2;
          double z0 = y0 + nt2 * g0, z1 = y1 + nt2 * g1, z2 = y2 + nt2 * g2;
          project_cone<double>(z0, z1, z2, a.mu);
          G2[0 * S + c] = z0; G2[1 * S + c] = z1; G2[2 * S + c] = z2;
          a.q[c] = f_times(f, z0, z1, z2);
          double t0 = z0 + (-1.0) * y0, t1 = z1 + (-1.0) * y1, t2 = z2 + (-1.0) * y2;
          double s0 = z0 + (-1.0) * x0, s1 = z1 + (-1.0) * x1, s2 = z2 + (-1.0) * x2;
          acc[2] = acc[2] + dot3i(g0, g1, g2, t0, t1, t2);
          acc[3] = acc[3] + dot3i(t0, t1, t2, t0, t1, t2);
          acc[4] = acc[4] + dot3i(g0, g1, g2, s0, s1, s2);
          acc[5] = acc[5] + dot3i(y0, y1, y2, M0, M1, M2);
          acc[6] = acc[6] + dot3i(y0, y1, y2, r0, r1, r2);
        }
        if ((i % kItemsPerThread) == kItemsPerThread - 1) {
          const int tile = (int)blockIdx.x + (i / kItemsPerThread) * (int)gridDim.x;
          if (__syncthreads_or(failed)) return;
          if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&a.bar[2], kErrNaN);
          block_fold_multi<7>(acc, scratch);
          write_partials<7>(a, tile, acc);
          double bm = block_max256(mx, scratch);
          if (threadIdx.x == 0) a.part[(size_t)kQMax * a.ptiles + tile] = bm;
          for (int qq = 0; qq < 7; ++qq) acc[qq] = 0.0;
          mx = 0.0;
          bad = false;
        }
      }
    }
    if (!grid_sync(a, kPhaseProduct, [&]() {
          double s[7];
          fold_tiles<7>(a, s, scratch);
          double res = fold_tiles_max(a, scratch);
          if (threadIdx.x == 0) {
            ApgdCtl* C = a.ctl;
            double obj1 = 0.5 * s[0] + s[1];
            C->obj1 = obj1;
            if (obj1 >= C->obj2) {
              // (10)-(14): double L and retry the projection
              if (C->backtracks >= a.max_bt) {
                atomicOr(&a.bar[2], kErrBacktrackCap);
                C->done = 1;
                C->iterations = C->k;
              } else {
                C->backtracks += 1;
                C->L = 2.0 * C->L;
                C->t = 1.0 / C->L;
                C->mode = 1;
              }
            } else {
              C->mode = 0;
              C->sweeps += 1;
              int old_best = C->best;
              if (res < C->residual) {
                C->residual = res;
                C->objective = obj1;
                C->best = C->nw;
              }
              if (C->residual < a.tol) {
                C->done = 1;
                C->iterations = C->k;
              } else {
                double th = C->restart ? 1.0 : C->theta_new;
                C->yb = C->beta;
                C->yr = C->restart;
                C->L = 0.9 * C->L;
                C->t = 1.0 / C->L;
                C->theta = th;
                int nw2 = free_slot(C->nw, C->cur, C->prev, old_best);
                C->prev = C->cur;
                C->cur = C->nw;
                C->nw = nw2;
                C->k += 1;
                if (C->k >= a.max_iter) {
                  C->done = 1;
                  C->iterations = C->k;
                } else {
                  C->theta_new = (-(th * th) + th * sqrt(th * th + 4.0)) / 2.0;
                  C->beta = th * (1.0 - th) / (th * th + C->theta_new);
                  // the look-ahead step is now iteration k's step
                  C->obj2_base = 0.5 * s[5] + s[6];
                  double nr = sqrt(s[3]);
                  C->obj2 = C->obj2_base + (s[2] + 0.5 * C->L * (nr * nr));
                  C->restart = (s[4] > 0) ? 1 : 0;
                }
              }
            }
          }
        }))
      return;
    if (__ldcg(&a.ctl->done)) break;
    step_pass = (__ldcg(&a.ctl->mode) == 1);
  }

  // ---- gamma = gamma_hat (APGD.cu:358); q = F gamma for D^T gamma
  {
    const int best = __ldcg(&a.ctl->best);
    const double* src = best >= 0 ? a.G[best] : nullptr;
    for (int tile = blockIdx.x; tile < a.nt; tile += gridDim.x) {
      for (int m = 0; m < kItemsPerThread; ++m) {
        int c = tile * kTileItems + m * kThreads + threadIdx.x;
        if (c < a.nc) {
          double x0 = 1.0, x1 = 1.0, x2 = 1.0;
          if (src) {
            x0 = src[0 * S + c]; x1 = src[1 * S + c]; x2 = src[2 * S + c];
          }
          a.gamma[0 * a.GS + c] = x0;
          a.gamma[1 * a.GS + c] = x1;
          a.gamma[2 * a.GS + c] = x2;
          Frame f = load_frame<kFrame>(a, c);
          a.q[c] = f_times(f, x0, x1, x2);
        }
      }
    }
  }
  if (!grid_sync(a, kPhaseFinal, NoCtl{})) return;

  // ---- f_c = D^T gamma; v = Minv (k + f_c); f_contact = f_c / h; p += h v
  const double invh = 1.0 / h;
  for (int bt = blockIdx.x; bt < a.nbt; bt += gridDim.x) {
    int b = bt * kThreads + threadIdx.x;
    if (b < a.nb) {
      double4 fc = gather_q(a, b);
      double4 k = a.k4[b];
      double mi = __ldg(a.minv + b);
      double4 v = make_double4(mi * (k.x + fc.x), mi * (k.y + fc.y), mi * (k.z + fc.z), 0.0);
      a.v4[b] = v;
      a.fc4[b] = make_double4(invh * fc.x, invh * fc.y, invh * fc.z, 0.0);
      double4 p = a.p4[b];
      a.p4[b] = make_double4(h * v.x + p.x, h * v.y + p.y, h * v.z + p.z, 0.0);
    }
  }
}

// System.cu:577-581: no contacts: v = Minv k, f_contact = 0, p += h v.
__global__ void __launch_bounds__(kThreads) k_step_nocontact(int nb, double h,
                                                             const double* __restrict__ minv,
                                                             const double4* __restrict__ f4,
                                                             double4* k4, double4* v4, double4* p4,
                                                             double4* fc4) {
  int b = blockIdx.x * kThreads + threadIdx.x;
  if (b >= nb) return;
  double mi = minv[b];
  double m = mi;
  if (m) m = 1.0 / m;
  double4 v = v4[b], f = f4[b];
  double4 k = make_double4(h * f.x + m * v.x, h * f.y + m * v.y, h * f.z + m * v.z, 0.0);
  k4[b] = k;
  v = make_double4(mi * k.x, mi * k.y, mi * k.z, 0.0);
  v4[b] = v;
  fc4[b] = make_double4(0.0, 0.0, 0.0, 0.0);
  double4 p = p4[b];
  p4[b] = make_double4(h * v.x + p.x, h * v.y + p.y, h * v.z + p.z, 0.0);
}

// Frame mode and register budget of the solve kernel; DVIDE_FRAME_MODE=0
// (frames loaded) and DVIDE_MIN_BLOCKS=3 select the other variants for timing
// comparisons.
int frame_mode_selected() {
  static int sel = -1;
  if (sel < 0) {
    const char* e = getenv("DVIDE_FRAME_MODE");
    sel = (e && e[0] == '0') ? 0 : 1;
  }
  return sel;
}

// CTAs per SM the register budget is set for (2: 128 registers; 3: 80);
// DVIDE_MIN_BLOCKS=3 selects the second for timing comparisons.
int min_blocks_selected() {
  static int sel = -1;
  if (sel < 0) {
    const char* e = getenv("DVIDE_MIN_BLOCKS");
    sel = (e && e[0] == '3') ? 3 : 2;
  }
  return sel;
}

const void* solve_kernel() {
  int fm = frame_mode_selected();
  if (min_blocks_selected() == 3)
    return fm == 0 ? (const void*)k_step_solve<0, 3> : (const void*)k_step_solve<1, 3>;
  return fm == 0 ? (const void*)k_step_solve<0, 2> : (const void*)k_step_solve<1, 2>;
}

size_t solve_smem() { return kDynSmem(frame_mode_selected()); }

void prepare_solve_kernel() {
  static bool done = false;
  if (done) return;
  cudaFuncSetAttribute(solve_kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)solve_smem());
  done = true;
}

}  // namespace

int apgd_max_ctas(int precision) {
  (void)precision;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  prepare_solve_kernel();
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, solve_kernel(), kThreads, solve_smem());
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

void launch_step_solve(SceneDev& sd, const SolveConfig& cfg, cudaStream_t st, int64_t* launches) {
  KArgs a;
  a.nb = sd.nb;
  a.nc = sd.nc;
  a.nt = (sd.nc + kTileItems - 1) / kTileItems;
  a.nbt = (sd.nb + kThreads - 1) / kThreads;
  a.S = sd.ccap;
  a.GS = sd.gcap;
  a.p4 = sd.p4;
  a.v4 = sd.v4;
  a.k4 = sd.k4;
  a.f4 = sd.f4;
  a.w4 = sd.w4;
  a.fc4 = sd.fc4;
  a.minv = sd.minv;
  a.ida = sd.ida;
  a.idb = sd.idb;
  a.F = sd.F;
  a.gap = sd.gap;
  a.r = sd.r;
  a.inc_start = sd.inc_start;
  a.inc = sd.inc;
  for (int k = 0; k < 5; ++k) {
    a.G[k] = sd.G[k];
    a.NG[k] = sd.NG[k];
  }
  a.q = sd.q;
  a.gamma = sd.gamma;
  a.part = sd.part;
  a.ptiles = sd.part_tiles;
  a.ctl = sd.ctl;
  a.bar = sd.bar;
  a.h = cfg.h;
  a.mu = cfg.mu;
  a.tol = cfg.tol;
  a.max_iter = cfg.max_iter;
  a.max_bt = cfg.max_bt;
  a.warm = cfg.warm;
  int grid = cfg.grid;
  cudaMemsetAsync(sd.bar, 0, 4 * sizeof(unsigned), st);
  cudaMemsetAsync(sd.ctl, 0, sizeof(ApgdCtl), st);
  void* params[] = {&a};
  prepare_solve_kernel();
  cudaLaunchCooperativeKernel(solve_kernel(), dim3(grid), dim3(kThreads), params, solve_smem(), st);
  ++*launches;
  cudaMemcpyAsync(sd.h_ctl, sd.ctl, sizeof(ApgdCtl), cudaMemcpyDeviceToHost, st);
}

void launch_step_nocontact(SceneDev& sd, double h, cudaStream_t st, int64_t* launches) {
  int nb = sd.nb;
  k_step_nocontact<<<(nb + kThreads - 1) / kThreads, kThreads, 0, st>>>(nb, h, sd.minv, sd.f4,
                                                                        sd.k4, sd.v4, sd.p4, sd.fc4);
  ++*launches;
}

}  // namespace dv
