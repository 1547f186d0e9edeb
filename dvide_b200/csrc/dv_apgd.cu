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
// The reference's per-iteration sequence calls the Schur product four times
// (APGD.cu:229, 237, 239, 276); the second N y and the residual's N gamma_new
// repeat a product of the same vector, so they are reused bit-for-bit here:
// two products per iteration and one per backtrack.
//
// Work is split in tiles of 1024 contacts (4 per thread) and 256 bodies;
// CTA b owns tiles b, b + G, ...  Every wait has a time limit.
#include <stdio.h>

#include "dv_internal.cuh"

namespace dv {

namespace {

constexpr int kNQ = 6;          // partial-sum slots per tile
constexpr int kQMax = kNQ;      // slot of the per-tile maximum

enum HatWhere { kHatNone = 0, kHatBuf = 1, kHatCur = 2, kHatNew = 3 };

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
  const int* __restrict__ abase;
  const int* __restrict__ bstart;
  const uint32_t* __restrict__ binc;
  double* G[2];
  double* Y[2];
  double* g;
  double* ghat;
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

__device__ inline Frame load_frame(const KArgs& a, int c) {
  const double* F = a.F;
  size_t S = a.S;
  Frame f;
  f.n0 = __ldg(F + 0 * S + c); f.n1 = __ldg(F + 1 * S + c); f.n2 = __ldg(F + 2 * S + c);
  f.u0 = __ldg(F + 3 * S + c); f.u1 = __ldg(F + 4 * S + c); f.u2 = __ldg(F + 5 * S + c);
  f.v0 = __ldg(F + 6 * S + c); f.v1 = __ldg(F + 7 * S + c); f.v2 = __ldg(F + 8 * S + c);
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

// Controller side: folds the per-tile partials of NQ quantities (slots
// qbase..qbase+NQ-1) in the fixed order; results valid in thread 0.
template <int NQ>
__device__ inline void fold_tiles(const KArgs& a, int qbase, double (&out)[NQ], double* scratch) {
  double v[NQ];
#pragma unroll
  for (int qi = 0; qi < NQ; ++qi) {
    double acc = 0.0;
    for (int t = threadIdx.x; t < a.nt; t += kThreads)
      acc = acc + __ldcg(a.part + (size_t)(qbase + qi) * a.ptiles + t);
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

// Grid barrier.  The last CTA to arrive runs `ctl_fn` (all its threads),
// then releases the generation word.  Returns false after a timeout or an
// error raised by another CTA; the caller then leaves the kernel.
template <class Fn>
__device__ inline bool grid_sync(const KArgs& a, Fn ctl_fn) {
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
      __threadfence();
      st_release(&a.bar[1], s_target);
    }
  } else if (threadIdx.x == 0) {
    uint64_t t0 = global_ns();
    unsigned polls = 0;
    while (ld_acquire(&a.bar[1]) < s_target) {
      __nanosleep(32);
      if ((++polls & 1023u) == 0u) {
        if (ld_acquire(&a.bar[2]) & kErrBarrierTimeout) {
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

__device__ inline double4 gather_q(const KArgs& a, int b) {
  double ax = 0.0, ay = 0.0, az = 0.0;
  int s = __ldg(a.bstart + b), e = __ldg(a.bstart + b + 1);
  for (int i = s; i < e; ++i) {
    int c = (int)__ldg(a.binc + i);
    double4 q = a.q[c];
    ax = ax - q.x; ay = ay - q.y; az = az - q.z;
  }
  s = __ldg(a.abase + b);
  e = __ldg(a.abase + b + 1);
  for (int c = s; c < e; ++c) {
    double4 q = a.q[c];
    ax = ax + q.x; ay = ay + q.y; az = az + q.z;
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

__device__ inline void write_partials(const KArgs& a, int tile, int qbase, const double* v, int nq) {
  if (threadIdx.x == 0)
    for (int qi = 0; qi < nq; ++qi) a.part[(size_t)(qbase + qi) * a.ptiles + tile] = v[qi];
}

__global__ void __launch_bounds__(kThreads) k_step_solve(KArgs a) {
  __shared__ double scratch[kNQ * 8 + 8];
  const size_t S = a.S;
  const double h = a.h;

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
  if (!grid_sync(a, NoCtl{})) return;

  // ---- r = D (Minv k) + b; gamma_0; y_0; d = gamma_0 - gamma_hat_0 (= gamma_0 - 1)
  for (int tile = blockIdx.x; tile < a.nt; tile += gridDim.x) {
    double acc[1] = {0.0};
    for (int m = 0; m < kItemsPerThread; ++m) {
      int c = tile * kTileItems + m * kThreads + threadIdx.x;
      if (c < a.nc) {
        Frame f = load_frame(a, c);
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
        a.Y[0][0 * S + c] = g0; a.Y[0][1 * S + c] = g1; a.Y[0][2 * S + c] = g2;
        double e0 = g0 + (-1.0), e1 = g1 + (-1.0), e2 = g2 + (-1.0);
        acc[0] = acc[0] + dot3i(e0, e1, e2, e0, e1, e2);
        a.q[c] = f_times(f, e0, e1, e2);
      }
    }
    block_fold_multi<1>(acc, scratch);
    write_partials(a, tile, 0, acc, 1);
  }
  if (!grid_sync(a, [&]() {
        double s[1];
        fold_tiles<1>(a, 0, s, scratch);
        if (threadIdx.x == 0) a.ctl->L0 = sqrt(s[0]);
      }))
    return;
  body_pass_schur(a);
  if (!grid_sync(a, NoCtl{})) return;

  // ---- L = ||N d|| / ||d||; q = F gamma_0 for the first N y
  for (int tile = blockIdx.x; tile < a.nt; tile += gridDim.x) {
    double acc[1] = {0.0};
    for (int m = 0; m < kItemsPerThread; ++m) {
      int c = tile * kTileItems + m * kThreads + threadIdx.x;
      if (c < a.nc) {
        Frame f = load_frame(a, c);
        double4 wa = a.w4[__ldg(a.ida + c)], wb = a.w4[__ldg(a.idb + c)];
        double n0, n1, n2;
        ft_times(f, wa, wb, &n0, &n1, &n2);
        acc[0] = acc[0] + dot3i(n0, n1, n2, n0, n1, n2);
        double y0 = a.Y[0][0 * S + c], y1 = a.Y[0][1 * S + c], y2 = a.Y[0][2 * S + c];
        a.q[c] = f_times(f, y0, y1, y2);
      }
    }
    block_fold_multi<1>(acc, scratch);
    write_partials(a, tile, 0, acc, 1);
  }
  if (!grid_sync(a, [&]() {
        double s[1];
        fold_tiles<1>(a, 0, s, scratch);
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
          C->hat = kHatNone;
          C->hat_pending = 0;
          C->backtracks = 0;
          C->obj1 = C->obj2 = C->obj2_base = 0.0;
        }
      }))
    return;
  body_pass_schur(a);
  if (!grid_sync(a, NoCtl{})) return;

  // ---- APGD iterations (APGD.cu:227-350)
  for (;;) {
    const int done = __ldcg(&a.ctl->done);
    if (done) break;
    const int mode = __ldcg(&a.ctl->mode);
    const int cur = __ldcg(&a.ctl->cur);
    const double t = __ldcg(&a.ctl->t);
    const double nt_ = -t;
    const double* Gc = a.G[cur];
    double* Gn = a.G[cur ^ 1];
    const double* Yc = a.Y[cur];
    if (mode == 0) {
      // g = N y + r; gamma_new = P(y - t g)
      const int copy_hat = __ldcg(&a.ctl->hat_pending);
      for (int tile = blockIdx.x; tile < a.nt; tile += gridDim.x) {
        double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int m = 0; m < kItemsPerThread; ++m) {
          int c = tile * kTileItems + m * kThreads + threadIdx.x;
          if (c < a.nc) {
            Frame f = load_frame(a, c);
            double4 wa = a.w4[__ldg(a.ida + c)], wb = a.w4[__ldg(a.idb + c)];
            double N0, N1, N2;
            ft_times(f, wa, wb, &N0, &N1, &N2);
            double r0 = a.r[0 * S + c], r1 = a.r[1 * S + c], r2 = a.r[2 * S + c];
            double y0 = Yc[0 * S + c], y1 = Yc[1 * S + c], y2 = Yc[2 * S + c];
            double c0 = Gc[0 * S + c], c1 = Gc[1 * S + c], c2 = Gc[2 * S + c];
            double g0 = N0 + r0, g1 = N1 + r1, g2 = N2 + r2;
            double x0 = y0 + nt_ * g0, x1 = y1 + nt_ * g1, x2 = y2 + nt_ * g2;
            project_cone<double>(x0, x1, x2, a.mu);
            a.g[0 * S + c] = g0; a.g[1 * S + c] = g1; a.g[2 * S + c] = g2;
            Gn[0 * S + c] = x0; Gn[1 * S + c] = x1; Gn[2 * S + c] = x2;
            a.q[c] = f_times(f, x0, x1, x2);
            if (copy_hat) {
              a.ghat[0 * S + c] = c0; a.ghat[1 * S + c] = c1; a.ghat[2 * S + c] = c2;
            }
            double t0 = x0 + (-1.0) * y0, t1 = x1 + (-1.0) * y1, t2 = x2 + (-1.0) * y2;
            double s0 = x0 + (-1.0) * c0, s1 = x1 + (-1.0) * c1, s2 = x2 + (-1.0) * c2;
            acc[0] = acc[0] + dot3i(y0, y1, y2, N0, N1, N2);
            acc[1] = acc[1] + dot3i(y0, y1, y2, r0, r1, r2);
            acc[2] = acc[2] + dot3i(g0, g1, g2, t0, t1, t2);
            acc[3] = acc[3] + dot3i(t0, t1, t2, t0, t1, t2);
            acc[4] = acc[4] + dot3i(g0, g1, g2, s0, s1, s2);
          }
        }
        block_fold_multi<5>(acc, scratch);
        write_partials(a, tile, 0, acc, 5);
      }
      if (!grid_sync(a, [&]() {
            double s[5];
            fold_tiles<5>(a, 0, s, scratch);
            if (threadIdx.x == 0) {
              ApgdCtl* C = a.ctl;
              double L = C->L;
              C->obj2_base = 0.5 * s[0] + s[1];
              double nr = sqrt(s[3]);
              C->obj2 = C->obj2_base + (s[2] + 0.5 * L * (nr * nr));
              C->restart = (s[4] > 0) ? 1 : 0;
              if (C->hat_pending) {
                C->hat_pending = 0;
                C->hat = kHatBuf;
              }
            }
          }))
        return;
    } else {
      // backtracking step: gamma_new = P(y - t g) with the halved step (APGD.cu:246-261)
      for (int tile = blockIdx.x; tile < a.nt; tile += gridDim.x) {
        double acc[3] = {0.0, 0.0, 0.0};
        for (int m = 0; m < kItemsPerThread; ++m) {
          int c = tile * kTileItems + m * kThreads + threadIdx.x;
          if (c < a.nc) {
            Frame f = load_frame(a, c);
            double y0 = Yc[0 * S + c], y1 = Yc[1 * S + c], y2 = Yc[2 * S + c];
            double c0 = Gc[0 * S + c], c1 = Gc[1 * S + c], c2 = Gc[2 * S + c];
            double g0 = a.g[0 * S + c], g1 = a.g[1 * S + c], g2 = a.g[2 * S + c];
            double x0 = y0 + nt_ * g0, x1 = y1 + nt_ * g1, x2 = y2 + nt_ * g2;
            project_cone<double>(x0, x1, x2, a.mu);
            Gn[0 * S + c] = x0; Gn[1 * S + c] = x1; Gn[2 * S + c] = x2;
            a.q[c] = f_times(f, x0, x1, x2);
            double t0 = x0 + (-1.0) * y0, t1 = x1 + (-1.0) * y1, t2 = x2 + (-1.0) * y2;
            double s0 = x0 + (-1.0) * c0, s1 = x1 + (-1.0) * c1, s2 = x2 + (-1.0) * c2;
            acc[0] = acc[0] + dot3i(g0, g1, g2, t0, t1, t2);
            acc[1] = acc[1] + dot3i(t0, t1, t2, t0, t1, t2);
            acc[2] = acc[2] + dot3i(g0, g1, g2, s0, s1, s2);
          }
        }
        block_fold_multi<3>(acc, scratch);
        write_partials(a, tile, 0, acc, 3);
      }
      if (!grid_sync(a, [&]() {
            double s[3];
            fold_tiles<3>(a, 0, s, scratch);
            if (threadIdx.x == 0) {
              ApgdCtl* C = a.ctl;
              double L = C->L;
              double nr = sqrt(s[1]);
              C->obj2 = C->obj2_base + (s[0] + 0.5 * L * (nr * nr));
              C->restart = (s[2] > 0) ? 1 : 0;
            }
          }))
        return;
    }
    body_pass_schur(a);
    if (!grid_sync(a, NoCtl{})) return;

    // N gamma_new: objective, residual (APGD.cu:90-102), speculative y_new
    {
      const double gd = __ldcg(&a.ctl->gdiff);
      const double gA = __ldcg(&a.ctl->ginv);
      const double gB = -1.0 / gd;
      const int restart = __ldcg(&a.ctl->restart);
      const double beta = __ldcg(&a.ctl->beta);
      const double opb = 1.0 + beta, mb = -beta;
      double* Yn = a.Y[cur ^ 1];
      for (int tile = blockIdx.x; tile < a.nt; tile += gridDim.x) {
        double acc[2] = {0.0, 0.0};
        double mx = 0.0;
        bool bad = false;
        for (int m = 0; m < kItemsPerThread; ++m) {
          int c = tile * kTileItems + m * kThreads + threadIdx.x;
          if (c < a.nc) {
            Frame f = load_frame(a, c);
            double4 wa = a.w4[__ldg(a.ida + c)], wb = a.w4[__ldg(a.idb + c)];
            double N0, N1, N2;
            ft_times(f, wa, wb, &N0, &N1, &N2);
            double r0 = a.r[0 * S + c], r1 = a.r[1 * S + c], r2 = a.r[2 * S + c];
            double x0 = Gn[0 * S + c], x1 = Gn[1 * S + c], x2 = Gn[2 * S + c];
            double c0 = Gc[0 * S + c], c1 = Gc[1 * S + c], c2 = Gc[2 * S + c];
            acc[0] = acc[0] + dot3i(x0, x1, x2, N0, N1, N2);
            acc[1] = acc[1] + dot3i(x0, x1, x2, r0, r1, r2);
            double T0 = r0 + N0, T1 = r1 + N1, T2 = r2 + N2;
            T0 = x0 + (-gd) * T0; T1 = x1 + (-gd) * T1; T2 = x2 + (-gd) * T2;
            project_cone<double>(T0, T1, T2, a.mu);
            T0 = gA * x0 + gB * T0; T1 = gA * x1 + gB * T1; T2 = gA * x2 + gB * T2;
            double m0 = fabs(T0), m1 = fabs(T1), m2 = fabs(T2);
            bad |= (m0 != m0) || (m1 != m1) || (m2 != m2);
            mx = fmax(mx, fmax(m0, fmax(m1, m2)));
            double y0, y1, y2;
            if (restart) {
              y0 = x0; y1 = x1; y2 = x2;
            } else {
              y0 = opb * x0 + mb * c0; y1 = opb * x1 + mb * c1; y2 = opb * x2 + mb * c2;
            }
            Yn[0 * S + c] = y0; Yn[1 * S + c] = y1; Yn[2 * S + c] = y2;
            a.q[c] = f_times(f, y0, y1, y2);
          }
        }
        if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&a.bar[2], kErrNaN);
        block_fold_multi<2>(acc, scratch);
        write_partials(a, tile, 0, acc, 2);
        double bm = block_max256(mx, scratch);
        if (threadIdx.x == 0) a.part[(size_t)kQMax * a.ptiles + tile] = bm;
        __syncthreads();
      }
    }
    if (!grid_sync(a, [&]() {
          double s[2];
          fold_tiles<2>(a, 0, s, scratch);
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
              if (res < C->residual) {
                C->residual = res;
                C->objective = obj1;
                C->hat = kHatNew;
              }
              if (C->residual < a.tol) {
                C->done = 1;
                C->iterations = C->k;
              } else {
                double th = C->restart ? 1.0 : C->theta_new;
                C->L = 0.9 * C->L;
                C->t = 1.0 / C->L;
                C->theta = th;
                C->cur ^= 1;
                if (C->hat == kHatNew) {
                  C->hat = kHatCur;
                  C->hat_pending = 1;
                }
                C->k += 1;
                if (C->k >= a.max_iter) {
                  C->done = 1;
                  C->iterations = C->k;
                } else {
                  C->theta_new = (-(th * th) + th * sqrt(th * th + 4.0)) / 2.0;
                  C->beta = th * (1.0 - th) / (th * th + C->theta_new);
                }
              }
            }
          }
        }))
      return;
    const int mode2 = __ldcg(&a.ctl->mode);
    const int done2 = __ldcg(&a.ctl->done);
    if (done2) break;
    if (mode2 == 1) continue;
    body_pass_schur(a);
    if (!grid_sync(a, NoCtl{})) return;
  }

  // ---- gamma = gamma_hat (APGD.cu:358); q = F gamma for D^T gamma
  {
    const int hat = __ldcg(&a.ctl->hat);
    const int cur = __ldcg(&a.ctl->cur);
    const double* src = nullptr;
    if (hat == kHatBuf) src = a.ghat;
    else if (hat == kHatCur) src = a.G[cur];
    else if (hat == kHatNew) src = a.G[cur ^ 1];
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
          Frame f = load_frame(a, c);
          a.q[c] = f_times(f, x0, x1, x2);
        }
      }
    }
  }
  if (!grid_sync(a, NoCtl{})) return;

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

}  // namespace

int apgd_max_ctas(int precision) {
  (void)precision;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_solve, kThreads, 0);
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
  a.abase = sd.cbase;
  a.bstart = sd.binc_start;
  a.binc = sd.binc;
  a.G[0] = sd.G0;
  a.G[1] = sd.G1;
  a.Y[0] = sd.Y0;
  a.Y[1] = sd.Y1;
  a.g = sd.gv;
  a.ghat = sd.ghat;
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
  void* params[] = {&a};
  cudaLaunchCooperativeKernel((const void*)k_step_solve, dim3(grid), dim3(kThreads), params, 0, st);
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
