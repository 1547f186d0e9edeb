// dv_apgd.cu -- the time step after collision detection, for every segment
// (scene) of an engine, as ONE persistent cooperative kernel per step:
//
//   applied impulse k = M v + h f             System.cu:1411-1417, 1502-1514
//   Schur vector r = D Minv k + b             System.cu:1516-1524, 1561-1580
//   APGD solve (all iterations)               APGD.cu:164-361
//   v = Minv (k + D^T gamma), p += h v        System.cu:570-583
//
// The reference runs each BLAS-1 call, SpMV and projection as its own launch
// and brings every dot/nrm2/nrmmax back to the host (APGD.cu:227-350).  Here
// the scalar control (step size, Lipschitz backtracking, restart, best
// iterate, convergence) runs on the device, per segment: the CTA that finishes
// a segment's last tile of a pass folds that segment's per-tile partial sums in
// a fixed order and executes its control logic; a grid barrier then starts the
// next pass.  Segments converge independently (their tiles and bodies are
// skipped once done); the kernel ends when every segment is done.
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
// the residual.  Iterates and their products rotate through five buffers, so
// y, g and gamma_hat are never copied.  The CPU oracle evaluates the same
// sequence (apgd_solve_fused), and bit-for-bit the same arithmetic.
//
// Precision: the kernel is a template on the iterate type T.  T = double is
// the FP64 path (bit-exact against the oracle).  T = float is the mixed path:
// frames, Jacobian and N gamma products, iterates and the cone projection in
// FP32; the Schur vector r (computed in FP64, stored in FP32), the objective
// and Lipschitz-test sums, the residual, the final D^T gamma and the
// integration in FP64.
//
// Work is split in tiles of 512 contacts (2 per thread) and 256 bodies.
// Every wait has a time limit.
#include <algorithm>

#include "dv_solve.cuh"

namespace dv {

namespace {

// Per-segment scalars of the step and product passes, kept in shared memory
// (written by thread 0 when the CTA moves to another segment) so that they
// take no registers in the contact loops.
struct ProdScalars {
  int cur, nw, nw2, restart, exact, rsel;
  double ya, ym, nt2, gd, gA, gB, mu;
};
struct StepScalars {
  int part, first, cur, prev, nw, yr, exact, rsel;
  double ya, ym, nt, mu;
};

// Mixed precision with refinement: the FP32 phase of a solve ends when its
// best residual has not improved for this many accepted iterations.
constexpr int kStallIterations = 50;

// What the segment controllers read and write, passed by value.
struct CtlArgs {
  double* part;
  int tcap;
  int mixed;  // FP32 iterates: the Lipschitz test allows float-noise differences
  int ar;     // anti-relaxation: an accepted, unconverged iterate moves r to the next plane
  int refine; // FP64 refinement launch: only the solves the FP32 launch marked, <= seg.refine iterations
  SegState* sst;
  const SegParams* seg;
  EngineWords* ew;
  unsigned* donemask;
};

// Segment controllers, run by the CTA that completes a segment's tiles of a
// pass (all its threads; thread 0 writes).  Kept out of line so that their
// registers do not weigh on the contact-pass loops.
__device__ __noinline__ void ctl_setup(CtlArgs a, int s, double* scratch) {
  double sm[1];
  fold_tiles<1>(a, a.sst[s].t0, a.sst[s].nt, sm, scratch);
  if (threadIdx.x == 0) a.sst[s].ctl.L0 = sqrt(sm[0]);
}

__device__ __noinline__ void ctl_lipschitz(CtlArgs a, int s, double* scratch) {
  double sm[1];
  fold_tiles<1>(a, a.sst[s].t0, a.sst[s].nt, sm, scratch);
  if (threadIdx.x == 0) {
    const SegParams& P = a.seg[s];
    ApgdCtl* C = &a.sst[s].ctl;
    // refinement launch: a solve the FP32 phase finished keeps its result
    if (a.refine && !__ldcg(&C->refined)) return;
    const double L = sqrt(sm[0]) / __ldcg(&C->L0);
    C->L = L;
    C->t = 1.0 / L;
    C->theta = 1.0;
    const double th = 1.0;
    const double tn = (-(th * th) + th * sqrt(th * th + 4.0)) / 2.0;
    C->theta_new = tn;
    C->beta = th * (1.0 - th) / (th * th + tn);
    C->residual = 10e30;
    C->objective = 0.0;
    // APGD.cu:92: 1 / (contacts + bilateral rows)^2
    const double ncd = (double)(a.sst[s].nc + a.seg[s].nbil);
    const double gd = 1.0 / (ncd * ncd);
    C->gdiff = gd;
    C->ginv = 1.0 / gd;
    C->k = 0;
    C->mode = 0;
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
    C->obj1 = 0.0;
    C->obj2 = 0.0;
    C->obj2_base = 0.0;
    C->rsel = 0;
    C->objN = 0.0;
    C->since_best = 0;
    if ((a.refine ? P.refine : P.max_iter) <= 0) {
      mark_done(a, s);
    } else {
      C->done = 0;
      atomicAdd(&a.ew->active, 1);
      atomicAdd(&a.ew->step_count, 1);
    }
  }
}

__device__ __noinline__ void ctl_step(CtlArgs a, int s, double* scratch) {
  double sm[5];
  fold_tiles<5>(a, a.sst[s].t0, a.sst[s].nt, sm, scratch);
  if (threadIdx.x == 0) {
    ApgdCtl* W = &a.sst[s].ctl;
    const int first = __ldcg(&W->first);
    const double L = __ldcg(&W->L);
    double ob = __ldcg(&W->obj2_base);
    if (first) {
      ob = 0.5 * sm[3] + sm[4];
      W->obj2_base = ob;
    }
    const double nr = sqrt(sm[1]);
    W->obj2 = ob + (sm[0] + 0.5 * L * (nr * nr));
    W->restart = (sm[2] > 0) ? 1 : 0;
    W->first = 0;
  }
}

// `direct`: an engine of one scene, whose controller runs at the product
// pass's barrier: it sets step_needed itself (no arrival counter to latch).
__device__ __noinline__ void ctl_product(CtlArgs a, int s, double* scratch, bool direct = false) {
  double sm[7], res;
  fold_tiles_sm<7, 1>(a, a.sst[s].t0, a.sst[s].nt, sm, &res, kQMax, scratch);
  if (threadIdx.x == 0) {
    const SegParams& P = a.seg[s];
    ApgdCtl* C = &a.sst[s].ctl;
    const ApgdCtl c = ctl_read(C);
    const double obj1 = 0.5 * sm[0] + sm[1];
    C->obj1 = obj1;
    bool finished = false;
    int k = c.k;
    // APGD.cu:240: obj1 >= obj2 means the step was too long.  With FP32
    // iterates both objectives carry rounding of order 1e-7 |f|; a difference
    // within that noise is not a failed test (else L doubles on noise alone).
    const double obj2 = c.obj2;
    const bool fail = a.mixed ? (obj1 - obj2 >= 1e-6 * (fabs(obj1) + fabs(obj2))) : (obj1 >= obj2);
    if (fail) {
      // (10)-(14): double L and retry the projection
      if (c.backtracks >= P.max_bt) {
        seg_error(a, s, kErrBacktrackCap);
        finished = true;
      } else {
        C->backtracks = c.backtracks + 1;
        const double L = 2.0 * c.L;
        C->L = L;
        C->t = 1.0 / L;
        C->mode = 1;
        if (direct) *(volatile int*)&a.ew->step_needed = 1;
        else atomicAdd(&a.ew->step_count, 1);
      }
    } else {
      C->mode = 0;
      if (direct) *(volatile int*)&a.ew->step_needed = 0;
      C->sweeps = c.sweeps + 1;
      double residual = c.residual;
      int since_best = c.since_best + 1;
      if (res < residual) {
        residual = res;
        C->residual = res;
        C->objective = obj1;
        if (a.ar) C->objN = 0.5 * sm[0];
        C->best = c.nw;
        since_best = 0;
      }
      C->since_best = since_best;
      if (residual < P.tol) {
        finished = true;
      } else if (a.mixed && P.refine > 0 && since_best >= kStallIterations) {
        // FP32 iterates no longer improve: the FP64 refinement continues
        // from gamma_hat
        finished = true;
      } else {
        // APGD.cu:335-345 after this iteration: r moves to the plane the
        // product pass wrote for the look-ahead
        if (a.ar) C->rsel = c.rsel ^ 1;
        const double th = c.restart ? 1.0 : c.theta_new;
        C->yb = c.beta;
        C->yr = c.restart;
        const double L = 0.9 * c.L;
        C->L = L;
        C->t = 1.0 / L;
        C->theta = th;
        C->prev = c.cur;
        C->cur = c.nw;
        C->nw = free_slot(c.nw, c.cur, c.prev, c.best);
        k += 1;
        C->k = k;
        if (k >= (a.refine ? P.refine : P.max_iter)) {
          finished = true;
        } else {
          const double tn = (-(th * th) + th * sqrt(th * th + 4.0)) / 2.0;
          C->theta_new = tn;
          C->beta = th * (1.0 - th) / (th * th + tn);
          // the look-ahead step is now iteration k's step
          const double ob = 0.5 * sm[5] + sm[6];
          C->obj2_base = ob;
          const double nr = sqrt(sm[3]);
          C->obj2 = ob + (sm[2] + 0.5 * L * (nr * nr));
          C->restart = (sm[4] > 0) ? 1 : 0;
        }
      }
    }
    if (finished) {
      C->iterations = k;
      mark_done(a, s);
      atomicSub(&a.ew->active, 1);
    }
  }
}

// The arrays of one bilateral tile in the product pass.
template <class T>
struct BilRows {
  const int2* off;
  const T* w;          // body vector (4 per body)
  const T* Gc;         // gamma_k
  const T* Gn;         // gamma_new
  T* G2;               // the look-ahead iterate
  const T* NGc;
  T* NGn;
  const T* r;
  T* q;
};

// Product pass on rows [r0, r0 + min(n, 512)): N gamma_new, the objective and
// residual items, the look-ahead step, without the cone projection; the tile's
// partials are parked in slot `slot`.  Called after the contact tiles (where
// it adds no registers to the contact loops).  Returns whether a residual
// item of this thread was NaN.
template <class T>
__device__ inline bool bil_product_tile(BilRows<T> R, const ProdScalars& ps, int r0, int n,
                                              bool has_contacts, DeferBuf* def, int slot, int tile) {
  const T ya = (T)ps.ya, ym = (T)ps.ym, nt2 = (T)ps.nt2;
  double acc[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  double mx = 0.0;
  bool bad = false;
  for (int m = 0; m < kItemsPerThread; ++m) {
    const int k = m * kThreads + threadIdx.x;
    if (k < n) {
      const int r = r0 + k;
      const T N0 = bil_dw<T>(__ldg(R.off + r), R.w);
      R.NGn[r] = N0;
      const T x0 = R.Gn[r], rr = R.r[r];
      acc[0] = acc[0] + (double)x0 * (double)N0;
      acc[1] = acc[1] + (double)x0 * (double)rr;
      // APGD.cu:90-102 on a row: no projection; without contacts the
      // residual is |N x + r| (the reference skips both axpby)
      double T0 = (double)rr + (double)N0;
      if (has_contacts) {
        const double X0 = x0;
        T0 = X0 + (-ps.gd) * T0;
        T0 = ps.gA * X0 + ps.gB * T0;
      }
      const double m0 = fabs(T0);
      bad |= (m0 != m0);
      mx = fmax(mx, m0);
      T y0, M0;
      if (ps.restart) {
        y0 = x0;
        M0 = N0;
      } else {
        y0 = ya * x0 + ym * R.Gc[r];
        M0 = ya * N0 + ym * R.NGc[r];
      }
      const T g0 = M0 + rr;
      const T z0 = y0 + nt2 * g0;
      R.G2[r] = z0;
      R.q[r] = z0;
      const T t0 = z0 + T(-1) * y0, s0 = z0 + T(-1) * x0;
      acc[2] = acc[2] + (double)g0 * (double)t0;
      acc[3] = acc[3] + (double)t0 * (double)t0;
      acc[4] = acc[4] + (double)g0 * (double)s0;
      acc[5] = acc[5] + (double)y0 * (double)M0;
      acc[6] = acc[6] + (double)y0 * (double)rr;
    }
  }
  park_tile<7, true>(*def, slot, tile, acc, mx);
  return bad;
}

// kAR: APGD's anti-relaxation (APGD.cu:335-345), FP64 one-scene engines.
template <class T, int kMinB, bool kAR>
__global__ void __launch_bounds__(kThreads, kMinB) k_step_solve(KArgs<T> a) {
  using V = typename Vec4<T>::type;
  __shared__ double scratch[kNQ * 8 + 8];
  __shared__ unsigned s_mask[kMaskWords];
  __shared__ ProdScalars s_ps;
  __shared__ StepScalars s_st;
  __shared__ DeferBuf s_def;
  extern __shared__ __align__(128) unsigned char dyn_smem[];
  const size_t S = a.S;
  V* wv = reinterpret_cast<V*>(a.wd);
  V* qv = reinterpret_cast<V*>(a.qd);
  Staging stg;
  stg.base = dyn_smem;
  stg.stage_bytes = warp_stage_bytes<T>();
  stg.bar = reinterpret_cast<uint64_t*>(dyn_smem + (size_t)kWarps * 2 * stg.stage_bytes);
  stg.phase = 0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < 2 * kWarps; ++i) mbar_init(stg.bar + i, 1);
    for (int w = 0; w < kWarps; ++w) reinterpret_cast<unsigned char*>(stg.bar + 2 * kWarps)[w] = 0;
    fence_mbar_init();
  }
  __syncthreads();
  if (ld_acquire(&a.ew->err)) return;  // an error of collision detection: nothing to do
  const int NT = a.ew->ntiles;
  const int nbt = (a.nb + kThreads - 1) / kThreads;
  const int mwords = (a.nseg + 31) >> 5;
  __shared__ SegCache s_sc;  // segment of the CTA's current tile
  SegCache& sc = s_sc;
  if (threadIdx.x == 0) {
    sc.s = -1;
    sc.t0 = sc.t1 = 0;
    s_def.fail = 0;
  }
  __syncthreads();
  const CtlArgs ca{a.part,  a.tcap, sizeof(T) != sizeof(double) ? 1 : 0, kAR ? 1 : 0, a.refine,
                   a.sst,   a.seg,  a.ew, a.donemask};

  // ---- work lists off; per-segment solve state; done mask (bit set: not iterating)
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.ew->act_on = 0;
    a.ew->act_rebuild = 0;
    a.ew->act_base = a.nseg;
  }
  for (int s = blockIdx.x * kThreads + threadIdx.x; s < a.nseg; s += gridDim.x * kThreads) {
    SegState& X = a.sst[s];
    X.arrive = 0u;
    ApgdCtl& C = X.ctl;
    // System.cu:560: a solve runs with contacts or bilateral rows
    const bool live = a.seg[s].active && (X.nc > 0 || a.seg[s].nbil > 0);
    if (a.refine) {
      // FP64 refinement: only the solves the FP32 launch marked; the others
      // keep their result, counts and error bits
      if (!(live && C.refined)) {
        C.done = 1;
        continue;
      }
      C.it_lo = C.iterations;
      C.bt_lo = C.backtracks;
      C.sw_lo = C.sweeps;
    } else {
      C.refined = 0;
      C.refine_it = 0;
    }
    X.err = 0u;
    C.done = live ? 0 : 1;
    C.iterations = 0;
    C.sweeps = 0;
    C.backtracks = 0;
    C.residual = 0.0;
    C.objective = 0.0;
    C.best = -1;
  }
  for (int wi = blockIdx.x * kThreads + threadIdx.x; wi < mwords; wi += gridDim.x * kThreads) {
    unsigned m = 0u;
    for (int j = 0; j < 32; ++j) {
      const int s = wi * 32 + j;
      if (s >= a.nseg || !(a.seg[s].active && (a.sst[s].nc > 0 || a.seg[s].nbil > 0)) ||
          (a.refine && !a.sst[s].ctl.refined))
        m |= 1u << j;
    }
    a.donemask[wi] = m;
  }

  // ---- applied impulse: k = m v + h f (m = 1/minv, 0 for fixed); w = minv k
  for (int bt = blockIdx.x; bt < nbt; bt += gridDim.x) {
    int b = bt * kThreads + threadIdx.x;
    if (b < a.nb) {
      const SegParams& P = a.seg[__ldg(a.bseg + b)];
      if (P.active) {
        const double h = P.h;
        double mi = __ldg(a.minv + b);
        double m = mi;
        if (m) m = 1.0 / m;
        double4 v = a.v4[b], f = a.f4[b];
        double4 k = make_double4(h * f.x + m * v.x, h * f.y + m * v.y, h * f.z + m * v.z, 0.0);
        a.k4[b] = k;
        a.wd[b] = make_double4(mi * k.x, mi * k.y, mi * k.z, 0.0);
      }
    }
  }
  if (!grid_sync(a, kPhaseSetup, [&]() {
        if (threadIdx.x == 0) {
          atomicExch(&a.ew->active, 0);
          atomicExch(&a.ew->step_count, 0);
          *(volatile int*)&a.ew->step_needed = 0;
        }
      }))
    return;

  // ---- r = D (Minv k) + b; gamma_0 -> G[0]; e = gamma_0 - gamma_hat_0 (= gamma_0 - 1)
  {
    SegRun run;
    int nslot = 0;
    auto ctl = [&](int s) { ctl_setup(ca, s, scratch); };
    for (int i = 0;; ++i) {
      const int t = cta_tile(a, NT, i);
      if (t < 0) break;
      locate(a, sc, t);
      const int s = sc.s;
      // refinement launch: a solve it does not refine needs no r, start or Lipschitz
      // estimate (its q and warm start from the FP32 launch stand)
      if (a.refine && !__ldcg(&a.sst[s].ctl.refined)) continue;
      if (s != run.s) {
        if (run.n) {
          fold_parked<1, false>(a, s_def, nslot);
          nslot = 0;
        }
        flush_run(a, run, ctl);
        run.s = s;
      }
      const SegParams& P = a.seg[s];
      const int k0 = (t - sc.t0) * kTileItems, nc = sc.nc, c0 = sc.c0, gsize = sc.gsize;
      const double h = P.h;
      double acc[1] = {0.0};
      const int kb = a.nbil ? bil_tile_k0(t, sc.t0, nc) : -1;
      if (kb >= 0) {
        // bilateral rows: b = violation / h (System.cu:1526-1544) at the
        // step's start time, r = b + (D Minv k)_row, gamma_0, e = gamma_0 - 1
        const double* pd = reinterpret_cast<const double*>(a.p4);
        const double* wdv = reinterpret_cast<const double*>(a.wd);
        const double tm = a.seg_time[s];
        for (int m = 0; m < kItemsPerThread; ++m) {
          const int k = kb + m * kThreads + threadIdx.x;
          if (k < P.nbil) {
            const int i = P.bil0 + k;
            const int2 o = __ldg(a.bil_off + i);
            const double4 inf = a.bil_info[i];  // velocity, start time, p0
            double velocity = inf.x;
            if (tm < inf.y) velocity = 0;
            const double pa = pd[o.x];
            const double viol = o.y >= 0 ? pa - pd[o.y] - velocity * (tm - inf.y)
                                         : pa - inf.z - velocity * (tm - inf.y);
            const double bb = viol / h;
            a.bil_b[i] = bb;
            a.br[i] = (T)(bb + bil_dw<double>(o, wdv));
            // warm start: the row's last impulse.  Without it the reference's
            // initialiser writes (1, 0, 0) over flat entries [0, 3 nc) with
            // the rows first (APGD.cu:114-120, 200): row k takes 1 if k is a
            // multiple of 3, 0 otherwise, and keeps its last impulse from 3 nc on.
            double g = a.bil_gam[i];
            if (!P.warm && k < 3 * nc) g = (k % 3 == 0) ? 1.0 : 0.0;
            const T x0 = (T)g;
            a.bG[0][i] = x0;
            const T e0 = x0 + T(-1);
            acc[0] = acc[0] + (double)e0 * (double)e0;
            a.bq[i] = e0;
          }
        }
      }
      for (int m = 0; m < kItemsPerThread && kb < 0; ++m) {
        int k = k0 + m * kThreads + threadIdx.x;
        if (k < nc) {
          const int c = c0 + k;
          Frame<double> fd = load_frame_fp64(a, c, P.exact != 0);
          double4 wa = a.wd[__ldg(a.ida + c)], wb = a.wd[__ldg(a.idb + c)];
          double d0, d1, d2;
          ft_times<double, double4>(fd, wa, wb, &d0, &d1, &d2);
          double bn = __ldg(a.gap + c) / h;
          a.r[0 * S + c] = (T)(bn + d0);
          if (kAR) {
            // r_n and the anti-relaxation vector (0 at the start, APGD.cu:196)
            a.ar_r0[c] = bn + d0;
            a.ar_v[c] = 0.0;
          }
          a.r[1 * S + c] = (T)(0.0 + d1);
          a.r[2 * S + c] = (T)(0.0 + d2);
          double g0, g1, g2;
          // refinement: positional, from the FP32 phase's gamma_hat of this step
          const int warm = a.refine ? 1 : P.warm;
          if (warm == 2) {
            // matched: the impulse the same (A, B) pair had at the last solve;
            // A's earlier contacts are sorted by B, so a binary search finds it
            const uint32_t ia = __ldg(a.ida + c);
            const uint32_t bl = __ldg(a.idb + c) - (uint32_t)P.b0;
            int lo = a.ws[ia], hi = lo + a.wc[ia];
            if (hi > gsize) hi = gsize;
            while (lo < hi) {
              const int mid = (lo + hi) >> 1;
              if (a.wid[(size_t)P.wbase + mid] < bl) lo = mid + 1;
              else hi = mid;
            }
            g0 = 0.0; g1 = 0.0; g2 = 0.0;
            if (lo < gsize && lo < a.ws[ia] + a.wc[ia] && a.wid[(size_t)P.wbase + lo] == bl) {
              const size_t wj = (size_t)P.wbase + lo;
              g0 = a.gamma[0 * a.WS + wj];
              g1 = a.gamma[1 * a.WS + wj];
              g2 = a.gamma[2 * a.WS + wj];
            }
          } else if (warm) {
            const size_t wi = (size_t)P.wbase + k;
            g0 = k < gsize ? a.gamma[0 * a.WS + wi] : 0.0;
            g1 = k < gsize ? a.gamma[1 * a.WS + wi] : 0.0;
            g2 = k < gsize ? a.gamma[2 * a.WS + wi] : 0.0;
          } else if (P.nbil == 0) {
            g0 = 1.0; g1 = 0.0; g2 = 0.0;
          } else {
            // the initialiser's (1, 0, 0) pattern over flat entries [0, 3 nc)
            // of a vector whose first nbil entries are the bilateral rows;
            // flat entries from 3 nc on keep what the resize kept
            const long long f = (long long)P.nbil + 3LL * k, lim = 3LL * nc;
            const size_t wi = (size_t)P.wbase + k;
            double gg[3];
#pragma unroll
            for (int d = 0; d < 3; ++d)
              gg[d] = (f + d < lim) ? (((f + d) % 3 == 0) ? 1.0 : 0.0)
                                    : (k < gsize ? a.gamma[d * a.WS + wi] : 0.0);
            g0 = gg[0]; g1 = gg[1]; g2 = gg[2];
          }
          const T x0 = (T)g0, x1 = (T)g1, x2 = (T)g2;
          a.G[0][0 * S + c] = x0; a.G[0][1 * S + c] = x1; a.G[0][2 * S + c] = x2;
          const T e0 = x0 + T(-1), e1 = x1 + T(-1), e2 = x2 + T(-1);
          acc[0] = acc[0] + dot3i(e0, e1, e2, e0, e1, e2);
          Frame<T> f = load_frame<T>(a, c, P.exact != 0);
          store_keep(qv + c, f_times<T, V>(f, e0, e1, e2));
        }
      }
      park_tile<1, false>(s_def, nslot, t, acc, 0.0);
      ++run.n;
      if (++nslot == kMaxDefer) {
        fold_parked<1, false>(a, s_def, nslot);
        nslot = 0;
      }
    }
    fold_parked<1, false>(a, s_def, nslot);
    flush_run(a, run, ctl);
  }
  if (!grid_sync(a, kPhaseSetup, NoCtl{})) return;
  load_mask(a, s_mask, mwords);
  body_pass_schur<T, kAR>(a, s_mask);
  if (!grid_sync(a, kPhaseSetup, NoCtl{})) return;

  // ---- L = ||N e|| / ||e||; q = F gamma_0 for the first N y
  {
    SegRun run;
    int nslot = 0;
    auto ctl = [&](int s) { ctl_lipschitz(ca, s, scratch); };
    for (int i = 0;; ++i) {
      const int t = cta_tile(a, NT, i);
      if (t < 0) break;
      locate(a, sc, t);
      const int s = sc.s;
      if (a.refine && !__ldcg(&a.sst[s].ctl.refined)) continue;
      if (s != run.s) {
        if (run.n) {
          fold_parked<1, false>(a, s_def, nslot);
          nslot = 0;
        }
        flush_run(a, run, ctl);
        run.s = s;
      }
      const int k0 = (t - sc.t0) * kTileItems, nc = sc.nc, c0 = sc.c0;
      double acc[1] = {0.0};
      const int kb = a.nbil ? bil_tile_k0(t, sc.t0, nc) : -1;
      if (kb >= 0) {
        // bilateral rows: (N e)_row; q = gamma_0 for the first N y
        const SegParams& P = a.seg[s];
        const T* wt = reinterpret_cast<const T*>(a.wd);
        for (int m = 0; m < kItemsPerThread; ++m) {
          const int k = kb + m * kThreads + threadIdx.x;
          if (k < P.nbil) {
            const int i = P.bil0 + k;
            const T n0 = bil_dw<T>(__ldg(a.bil_off + i), wt);
            acc[0] = acc[0] + (double)n0 * (double)n0;
            a.bq[i] = a.bG[0][i];
          }
        }
      }
      for (int m = 0; m < kItemsPerThread && kb < 0; ++m) {
        int k = k0 + m * kThreads + threadIdx.x;
        if (k < nc) {
          const int c = c0 + k;
          Frame<T> f = load_frame<T>(a, c, a.seg[s].exact != 0);
          V wa = wv[__ldg(a.ida + c)], wb = wv[__ldg(a.idb + c)];
          T n0, n1, n2;
          ft_times<T, V>(f, wa, wb, &n0, &n1, &n2);
          acc[0] = acc[0] + dot3i(n0, n1, n2, n0, n1, n2);
          T y0 = a.G[0][0 * S + c], y1 = a.G[0][1 * S + c], y2 = a.G[0][2 * S + c];
          store_keep(qv + c, f_times<T, V>(f, y0, y1, y2));
        }
      }
      park_tile<1, false>(s_def, nslot, t, acc, 0.0);
      ++run.n;
      if (++nslot == kMaxDefer) {
        fold_parked<1, false>(a, s_def, nslot);
        nslot = 0;
      }
    }
    fold_parked<1, false>(a, s_def, nslot);
    flush_run(a, run, ctl);
  }
  // step_count is raised by atomics of other CTAs: read and clear it atomically
  auto latch = [&]() {
    if (threadIdx.x == 0) {
      int n = atomicExch(&a.ew->step_count, 0);
      *(volatile int*)&a.ew->step_needed = n;
    }
  };
  if (!grid_sync(a, kPhaseSetup, latch)) return;
  load_mask(a, s_mask, mwords);
  body_pass_schur<T, kAR>(a, s_mask);
  if (!grid_sync(a, kPhaseSetup, NoCtl{})) return;

  // ---- APGD iterations (APGD.cu:227-350)
  //
  // Each iteration is one body pass (w = Minv D^T q of gamma_new) and one
  // contact pass that computes N gamma_new, the objective and the residual of
  // iteration k, and -- assuming the Lipschitz test accepts gamma_new -- the
  // whole step of iteration k+1 (y, N y, g, gamma_new = P(y - t g), q).  When
  // the test fails (backtracking) the look-ahead is discarded and a step pass
  // recomputes gamma_new with the doubled L; the arithmetic of every value is
  // the same either way.  A segment's first step is a step pass too (N y_0
  // is a product: w of gamma_0).  Segment scalars are loaded once per run of
  // consecutive tiles of one segment.
  // one segment: its step and product controllers run at the passes' barriers
  const bool single = a.nseg == 1;
  // the product pass's barrier also decides whether the work lists are rebuilt:
  // once half the segments iterating at the last build have finished
  auto latch_product = [&]() {
    if (single) {
      ctl_product(ca, 0, scratch, true);
      return;
    }
    if (threadIdx.x == 0) {
      volatile EngineWords* E = a.ew;
      const int n = atomicExch(&a.ew->step_count, 0);
      E->step_needed = n;
      const int act = E->active;
      if (a.nseg > 1 && act > 0 && 2 * act <= E->act_base) E->act_rebuild = 1;
    }
  };
  for (;;) {
    if (__ldcg(&a.ew->active) == 0) break;
    // the done mask at the start of a pass holds for every tile this CTA has
    // left in the pass: a segment finishes only after all its tiles
    load_mask(a, s_mask, mwords);
    const int lon = __ldcg(&a.ew->act_on);
    const int NTL = lon ? __ldcg(&a.ew->act_nt) : NT;
    const int NBL = lon ? __ldcg(&a.ew->act_nb) : 0;
    if (__ldcg(&a.ew->step_needed) > 0) {
      SegRun run;
      int nslot = 0;
      auto ctl = [&](int s) { ctl_step(ca, s, scratch); };
      int cs = -1;
      for (int i = 0;; ++i) {
        const int t = pass_tile(a, lon, NTL, i);
        if (t < 0) break;
        locate(a, sc, t);
        const int s = sc.s;
        if (s != cs) {
          cs = s;
          __syncthreads();
          if (threadIdx.x == 0) {
            int part = !mask_done(a, s_mask, mwords, s);
            if (part) {
              const ApgdCtl* C = &a.sst[s].ctl;
              const int first = __ldcg(&C->first);
              part = first || __ldcg(&C->mode) == 1;
              s_st.first = first;
              s_st.cur = __ldcg(&C->cur);
              s_st.prev = __ldcg(&C->prev);
              s_st.nw = __ldcg(&C->nw);
              s_st.yr = __ldcg(&C->yr);
              const double yb = __ldcg(&C->yb);
              s_st.ya = 1.0 + yb;
              s_st.ym = -yb;
              s_st.nt = -__ldcg(&C->t);
              s_st.mu = a.seg[s].mu;
              s_st.exact = a.seg[s].exact;
              if (kAR) s_st.rsel = __ldcg(&C->rsel);
            }
            s_st.part = part;
          }
          __syncthreads();
        }
        const bool part = s_st.part != 0;
        if (!part) continue;
        if (s != run.s) {
          if (run.n) {
            fold_parked<5, false>(a, s_def, nslot);
            nslot = 0;
          }
          flush_run(a, run, ctl, single);
          run.s = s;
        }
        const int cur = s_st.cur, prev = s_st.prev, first = s_st.first, yr = s_st.yr;
        const T ya = (T)s_st.ya, ym = (T)s_st.ym, nt_ = (T)s_st.nt, mu = (T)s_st.mu;
        const T* Gc = a.G[cur];
        const T* Gp = a.G[prev < 0 ? cur : prev];
        T* NGc = a.NG[cur];
        const T* NGp = a.NG[prev < 0 ? cur : prev];
        T* Gn = a.G[s_st.nw];
        const int k0 = (t - sc.t0) * kTileItems, nc = sc.nc, c0 = sc.c0;
        double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        const int kb = a.nbil ? bil_tile_k0(t, sc.t0, nc) : -1;
        if (kb >= 0) {
          // bilateral rows: the same step without the cone projection
          const SegParams& P = a.seg[s];
          const T* wt = reinterpret_cast<const T*>(a.wd);
          const T* bGc = a.bG[cur];
          const T* bGp = a.bG[prev < 0 ? cur : prev];
          T* bNGc = a.bNG[cur];
          const T* bNGp = a.bNG[prev < 0 ? cur : prev];
          T* bGn = a.bG[s_st.nw];
          for (int m = 0; m < kItemsPerThread; ++m) {
            const int k = kb + m * kThreads + threadIdx.x;
            if (k < P.nbil) {
              const int i = P.bil0 + k;
              const T c0v = bGc[i];
              T y0, N0;
              if (yr) y0 = c0v;
              else y0 = ya * c0v + ym * bGp[i];
              if (first) {
                N0 = bil_dw<T>(__ldg(a.bil_off + i), wt);
                bNGc[i] = N0;
              } else if (yr) {
                N0 = bNGc[i];
              } else {
                N0 = ya * bNGc[i] + ym * bNGp[i];
              }
              const T r0 = a.br[i];
              const T g0 = N0 + r0;
              const T x0 = y0 + nt_ * g0;
              bGn[i] = x0;
              a.bq[i] = x0;
              const T t0 = x0 + T(-1) * y0, s0 = x0 + T(-1) * c0v;
              acc[0] = acc[0] + (double)g0 * (double)t0;
              acc[1] = acc[1] + (double)t0 * (double)t0;
              acc[2] = acc[2] + (double)g0 * (double)s0;
              if (first) {
                acc[3] = acc[3] + (double)y0 * (double)N0;
                acc[4] = acc[4] + (double)y0 * (double)r0;
              }
            }
          }
        } else {
          // the second item's lines into L2 while the first one computes
          const int k = k0 + kThreads + threadIdx.x;
          if (k < nc) {
            const int c = c0 + k;
            const T* nrm = normal_planes<T>(a);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              prefetch_l2(nrm + d * S + c);
              prefetch_l2(Gc + d * S + c);
              prefetch_l2(a.r + d * S + c);
              if (!first) prefetch_l2(NGc + d * S + c);
              if (!yr) {
                prefetch_l2(Gp + d * S + c);
                if (!first) prefetch_l2(NGp + d * S + c);
              }
            }
          }
        }
        for (int m = 0; m < kItemsPerThread && kb < 0; ++m) {
          int k = k0 + m * kThreads + threadIdx.x;
          if (k < nc) {
            const int c = c0 + k;
            Frame<T> f = load_frame<T>(a, c, s_st.exact != 0);
            T c0v = Gc[0 * S + c], c1v = Gc[1 * S + c], c2v = Gc[2 * S + c];
            T y0, y1, y2, N0, N1, N2;
            if (yr) {
              y0 = c0v; y1 = c1v; y2 = c2v;
            } else {
              y0 = ya * c0v + ym * Gp[0 * S + c];
              y1 = ya * c1v + ym * Gp[1 * S + c];
              y2 = ya * c2v + ym * Gp[2 * S + c];
            }
            if (first) {
              V wa = wv[__ldg(a.ida + c)], wb = wv[__ldg(a.idb + c)];
              ft_times<T, V>(f, wa, wb, &N0, &N1, &N2);
              NGc[0 * S + c] = N0; NGc[1 * S + c] = N1; NGc[2 * S + c] = N2;
            } else if (yr) {
              N0 = NGc[0 * S + c]; N1 = NGc[1 * S + c]; N2 = NGc[2 * S + c];
            } else {
              N0 = ya * NGc[0 * S + c] + ym * NGp[0 * S + c];
              N1 = ya * NGc[1 * S + c] + ym * NGp[1 * S + c];
              N2 = ya * NGc[2 * S + c] + ym * NGp[2 * S + c];
            }
            T r0 = kAR ? (T)a.ar_r0[(size_t)s_st.rsel * S + c] : a.r[0 * S + c];
            T r1 = a.r[1 * S + c], r2 = a.r[2 * S + c];
            T g0 = N0 + r0, g1 = N1 + r1, g2 = N2 + r2;
            T x0 = y0 + nt_ * g0, x1 = y1 + nt_ * g1, x2 = y2 + nt_ * g2;
            project_cone<T>(x0, x1, x2, mu);
            Gn[0 * S + c] = x0; Gn[1 * S + c] = x1; Gn[2 * S + c] = x2;
            store_keep(qv + c, f_times<T, V>(f, x0, x1, x2));
            T t0 = x0 + T(-1) * y0, t1 = x1 + T(-1) * y1, t2 = x2 + T(-1) * y2;
            T s0 = x0 + T(-1) * c0v, s1 = x1 + T(-1) * c1v, s2 = x2 + T(-1) * c2v;
            acc[0] = acc[0] + dot3i(g0, g1, g2, t0, t1, t2);
            acc[1] = acc[1] + dot3i(t0, t1, t2, t0, t1, t2);
            acc[2] = acc[2] + dot3i(g0, g1, g2, s0, s1, s2);
            if (first) {
              acc[3] = acc[3] + dot3i(y0, y1, y2, N0, N1, N2);
              acc[4] = acc[4] + dot3i(y0, y1, y2, r0, r1, r2);
            }
          }
        }
        park_tile<5, false>(s_def, nslot, t, acc, 0.0);
        ++run.n;
        if (++nslot == kMaxDefer) {
          fold_parked<5, false>(a, s_def, nslot);
          nslot = 0;
        }
      }
      fold_parked<5, false>(a, s_def, nslot);
      flush_run(a, run, ctl, single);
      if (!grid_sync(a, kPhaseStep, [&]() {
            if (single) ctl_step(ca, 0, scratch);
          }))
        return;
    }
    body_pass_schur<T, kAR>(a, s_mask, lon, NBL);
    if (!grid_sync(a, kPhaseBody, NoCtl{})) return;

    // N gamma_new, objective (APGD.cu:237-238), residual (:90-102); then the
    // next iteration's step assuming gamma_new is accepted (:266-273, 312-332)
    {
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      // this CTA's next iterating tile at or after sequence index i (-1: none)
      auto next_tile = [&](int i, int* tile_out) {
        for (;; ++i) {
          int t = pass_tile(a, lon, NTL, i);
          if (t < 0) return -1;
          locate(a, sc, t);
          // contact tiles only (the bilateral rows' tiles have their own loop)
          if (!mask_done(a, s_mask, mwords, sc.s) &&
              (!a.nbil || (t - sc.t0) * kTileItems < sc.nc)) {
            *tile_out = t;
            return i;
          }
        }
      };
      // bulk copies of (tile t of segment s, sub-tile sub) for this warp into stage sidx
      auto issue = [&](int t, int st0, int sc0, int snc, int sub, int sidx, int cur, int nw,
                       int restart, int rsel) {
        const int kw = (t - st0) * kTileItems + sub * kSub + warp * 32;
        if (lane == 0 && kw < snc) {
          mark_stage_issued(stg, sidx);
          const int cw = sc0 + kw;
          const T* nrm = normal_planes<T>(a);
          const T* src[kStagePlanes];
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            src[k] = nrm + k * S;
            src[3 + k] = a.G[nw] + k * S;
            src[6 + k] = a.r + k * S;
            src[9 + k] = a.G[cur] + k * S;
            src[12 + k] = a.NG[cur] + k * S;
          }
          // anti-relaxation: the current plane of r_n
          if (kAR) src[6] = reinterpret_cast<const T*>(a.ar_r0 + (size_t)rsel * S);
          const int nd = restart ? 9 : kStagePlanes;
          const unsigned pbytes = 32u * (unsigned)sizeof(T);
          unsigned char* dst = stg.base + (size_t)(2 * warp + sidx) * stg.stage_bytes;
          uint64_t* bar = stg.bar + 2 * warp + sidx;
          // order this warp's earlier generic reads of the stage before the copies
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_arrive_expect_tx(bar, (unsigned)nd * pbytes + 256u);
          for (int p = 0; p < nd; ++p) bulk_g2s(dst + (size_t)p * pbytes, src[p] + cw, pbytes, bar);
          unsigned char* ids = dst + (size_t)kStagePlanes * pbytes;
          bulk_g2s(ids, a.ida + cw, 128, bar);
          bulk_g2s(ids + 128, a.idb + cw, 128, bar);
        }
      };
      auto load_ps = [&](int s) {
        __syncthreads();
        if (threadIdx.x == 0) {
          const ApgdCtl* C = &a.sst[s].ctl;
          const int cur = __ldcg(&C->cur), prev = __ldcg(&C->prev), nw = __ldcg(&C->nw);
          const int best = __ldcg(&C->best);
          const double beta = __ldcg(&C->beta), gd = __ldcg(&C->gdiff);
          s_ps.cur = cur;
          s_ps.nw = nw;
          s_ps.nw2 = free_slot(nw, cur, prev, best);
          s_ps.restart = __ldcg(&C->restart);
          s_ps.ya = 1.0 + beta;
          s_ps.ym = -beta;
          s_ps.nt2 = -(1.0 / (0.9 * __ldcg(&C->L)));
          s_ps.gd = gd;
          s_ps.gA = __ldcg(&C->ginv);
          s_ps.gB = -1.0 / gd;
          s_ps.mu = a.seg[s].mu;
          s_ps.exact = a.seg[s].exact;
          if (kAR) s_ps.rsel = __ldcg(&C->rsel);
        }
        __syncthreads();
      };
      SegRun run;
      int nslot = 0;
      auto ctl = [&](int s) { ctl_product(ca, s, scratch); };

      double acc[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      double mx = 0.0;
      bool bad = false, failed = false;
      int tcur = -1;
      int seq = next_tile(0, &tcur);
      int sub = 0, sidx = 0;
      const ProdScalars& ps = s_ps;
      int s = -1, sc0 = 0, st0 = 0, snc = 0;
      if (seq >= 0) {
        locate(a, sc, tcur);
        s = sc.s;
        load_ps(s);
        sc0 = sc.c0; st0 = sc.t0; snc = sc.nc;
        issue(tcur, st0, sc0, snc, 0, 0, ps.cur, ps.nw, ps.restart, kAR ? ps.rsel : 0);
      }
      while (seq >= 0) {
        const int ti = tcur;
        if (sub == 0 && s != run.s) {
          if (run.n) {
            if (!fold_parked<7, true>(a, s_def, nslot)) {
              drain_warp_stages(stg, &a.ew->wait_limit_ns);
              return;
            }
            nslot = 0;
          }
          flush_run(a, run, ctl, single);
          run.s = s;
        }
        // the following sub-tile: this tile's second half, or the next tile
        // (next_tile leaves that tile's segment in sc)
        int nseq = seq, ntile = tcur, nsub = sub + 1;
        if (nsub == kItemsPerThread) {
          nsub = 0;
          nseq = next_tile(seq + 1, &ntile);
        }
        const int ns = (nseq >= 0 && nsub == 0) ? sc.s : s;
        __syncwarp();  // the warp's reads of stage sidx^1 are done
        if (nseq >= 0 && !failed) {
          if (ns == s) {
            issue(ntile, st0, sc0, snc, nsub, sidx ^ 1, ps.cur, ps.nw, ps.restart,
                  kAR ? ps.rsel : 0);
          } else {
            const ApgdCtl* C = &a.sst[ns].ctl;
            issue(ntile, sc.t0, sc.c0, sc.nc, nsub, sidx ^ 1, __ldcg(&C->cur), __ldcg(&C->nw),
                  __ldcg(&C->restart), kAR ? __ldcg(&C->rsel) : 0);
          }
        }
        const int kw = (ti - st0) * kTileItems + sub * kSub + warp * 32;
        if (kw < snc && !failed) {
          if (!wait_warp_stage(a, stg, sidx)) failed = true;
        }
        const int k = kw + lane;
        if (k < snc && !failed) {
          const int c = sc0 + k;
          const T* sd =
              reinterpret_cast<const T*>(stg.base + (size_t)(2 * warp + sidx) * stg.stage_bytes);
          const uint32_t* su = reinterpret_cast<const uint32_t*>(sd + (size_t)kStagePlanes * 32);
          const int j = lane;
          Frame<T> f =
              make_frame<T>(sd[0 * 32 + j], sd[1 * 32 + j], sd[2 * 32 + j], ps.exact != 0);
          V wa = wv[su[j]], wb = wv[su[32 + j]];
          T N0, N1, N2;
          ft_times<T, V>(f, wa, wb, &N0, &N1, &N2);
          T* NGn = a.NG[ps.nw];
          NGn[0 * S + c] = N0; NGn[1 * S + c] = N1; NGn[2 * S + c] = N2;
          T x0 = sd[3 * 32 + j], x1 = sd[4 * 32 + j], x2 = sd[5 * 32 + j];
          T r0 = sd[6 * 32 + j], r1 = sd[7 * 32 + j], r2 = sd[8 * 32 + j];
          acc[0] = acc[0] + dot3i(x0, x1, x2, N0, N1, N2);
          acc[1] = acc[1] + dot3i(x0, x1, x2, r0, r1, r2);
          {
            // residual, FP64 in both paths (gd = 1/nc^2 is far below float
            // resolution).  The mixed path takes it at the FP64 projection of
            // the FP32 iterate: the residual divides by gd, which would
            // otherwise magnify the iterate's float rounding off the cone.
            double X0 = x0, X1 = x1, X2 = x2;
            if (sizeof(T) != sizeof(double)) project_cone<double>(X0, X1, X2, ps.mu);
            double T0 = (double)r0 + (double)N0, T1 = (double)r1 + (double)N1,
                   T2 = (double)r2 + (double)N2;
            T0 = X0 + (-ps.gd) * T0; T1 = X1 + (-ps.gd) * T1; T2 = X2 + (-ps.gd) * T2;
            project_cone<double>(T0, T1, T2, ps.mu);
            const double gA = ps.gA, gB = ps.gB;
            T0 = gA * X0 + gB * T0; T1 = gA * X1 + gB * T1; T2 = gA * X2 + gB * T2;
            double m0 = fabs(T0), m1 = fabs(T1), m2 = fabs(T2);
            bad |= (m0 != m0) || (m1 != m1) || (m2 != m2);
            mx = fmax(mx, fmax(m0, fmax(m1, m2)));
          }
          // look-ahead step of iteration k+1: y = (1+b) x - b gamma_k, or x after a restart
          const T ya = (T)ps.ya, ym = (T)ps.ym;
          const T nt2 = (T)ps.nt2;
          T y0, y1, y2, M0, M1, M2;
          if (ps.restart) {
            y0 = x0; y1 = x1; y2 = x2;
            M0 = N0; M1 = N1; M2 = N2;
          } else {
            T c0v = sd[9 * 32 + j], c1v = sd[10 * 32 + j], c2v = sd[11 * 32 + j];
            y0 = ya * x0 + ym * c0v; y1 = ya * x1 + ym * c1v; y2 = ya * x2 + ym * c2v;
            M0 = ya * N0 + ym * sd[12 * 32 + j];
            M1 = ya * N1 + ym * sd[13 * 32 + j];
            M2 = ya * N2 + ym * sd[14 * 32 + j];
          }
          T rn0 = r0;  // r_n of the next iteration
          if (kAR) {
            // APGD.cu:335-345 for gamma_new = x: v = Minv (k + D^T x) of the
            // body pass, s = (D v)_(u, v), ar = sqrt(s_u^2 + s_v^2) mu;
            // r_n' = ar + (-ar_old + r_n), into the next plane
            const double4 va = a.v_ar[su[j]], vb = a.v_ar[su[32 + j]];
            const double d0 = va.x - vb.x, d1 = va.y - vb.y, d2 = va.z - vb.z;
            const double s_u = (f.u0 * d0 + f.u1 * d1) + f.u2 * d2;
            const double s_v = (f.v0 * d0 + f.v1 * d1) + f.v2 * d2;
            const double arn = sqrt(s_u * s_u + s_v * s_v) * ps.mu;
            const size_t cur_p = (size_t)ps.rsel * S + c, nxt_p = (size_t)(ps.rsel ^ 1) * S + c;
            const double rnn = arn + (-a.ar_v[cur_p] + (double)r0);
            a.ar_r0[nxt_p] = rnn;
            a.ar_v[nxt_p] = arn;
            rn0 = (T)rnn;
          }
          T g0 = M0 + rn0, g1 = M1 + r1, g2 = M2 + r2;
          T z0 = y0 + nt2 * g0, z1 = y1 + nt2 * g1, z2 = y2 + nt2 * g2;
          project_cone<T>(z0, z1, z2, (T)ps.mu);
          T* G2 = a.G[ps.nw2];
          G2[0 * S + c] = z0; G2[1 * S + c] = z1; G2[2 * S + c] = z2;
          store_keep(qv + c, f_times<T, V>(f, z0, z1, z2));
          T t0 = z0 + T(-1) * y0, t1 = z1 + T(-1) * y1, t2 = z2 + T(-1) * y2;
          T s0 = z0 + T(-1) * x0, s1 = z1 + T(-1) * x1, s2 = z2 + T(-1) * x2;
          acc[2] = acc[2] + dot3i(g0, g1, g2, t0, t1, t2);
          acc[3] = acc[3] + dot3i(t0, t1, t2, t0, t1, t2);
          acc[4] = acc[4] + dot3i(g0, g1, g2, s0, s1, s2);
          acc[5] = acc[5] + dot3i(y0, y1, y2, M0, M1, M2);
          acc[6] = acc[6] + dot3i(y0, y1, y2, rn0, r1, r2);
        }
        if (sub == kItemsPerThread - 1) {
          if (__any_sync(0xffffffffu, bad) && lane == 0) seg_error(a, s, kErrNaN);
          if (failed && lane == 0) s_def.fail = 1;
          park_tile<7, true>(s_def, nslot, ti, acc, mx);
          for (int qq = 0; qq < 7; ++qq) acc[qq] = 0.0;
          mx = 0.0;
          bad = false;
          ++run.n;
          if (++nslot == kMaxDefer) {
            if (!fold_parked<7, true>(a, s_def, nslot)) {
              drain_warp_stages(stg, &a.ew->wait_limit_ns);
              return;
            }
            nslot = 0;
          }
        }
        seq = nseq;
        tcur = ntile;
        sub = nsub;
        sidx ^= 1;
        if (ns != s) {
          s = ns;
          load_ps(s);
          sc0 = sc.c0; st0 = sc.t0; snc = sc.nc;
        }
      }
      if (!fold_parked<7, true>(a, s_def, nslot)) {
        drain_warp_stages(stg, &a.ew->wait_limit_ns);
        return;
      }
      nslot = 0;
      flush_run(a, run, ctl, single);
      if (a.nbil) {
        // then the bilateral rows' tiles: N gamma_new, the objective and
        // residual items and the look-ahead step, without the cone projection
        const T* wt = reinterpret_cast<const T*>(a.wd);
        for (int i = 0;; ++i) {
          const int t = pass_tile(a, lon, NTL, i);
          if (t < 0) break;
          locate(a, sc, t);
          const int s = sc.s;
          if (mask_done(a, s_mask, mwords, s)) continue;
          const int kb = bil_tile_k0(t, sc.t0, sc.nc);
          if (kb < 0) continue;
          if (s != run.s) {
            if (run.n) {
              fold_parked<7, true>(a, s_def, nslot);
              nslot = 0;
            }
            flush_run(a, run, ctl, single);
            run.s = s;
          }
          load_ps(s);
          const SegParams& P = a.seg[s];
          const ProdScalars& ps = s_ps;
          BilRows<T> br_{a.bil_off, wt, a.bG[ps.cur], a.bG[ps.nw], a.bG[ps.nw2], a.bNG[ps.cur],
                         a.bNG[ps.nw], a.br, a.bq};
          const bool bad = bil_product_tile<T>(br_, ps, P.bil0 + kb, P.nbil - kb, sc.nc > 0,
                                               &s_def, nslot, t);
          if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) seg_error(a, s, kErrNaN);
          ++run.n;
          if (++nslot == kMaxDefer) {
            fold_parked<7, true>(a, s_def, nslot);
            nslot = 0;
          }
        }
        fold_parked<7, true>(a, s_def, nslot);
        nslot = 0;
        flush_run(a, run, ctl, single);
      }

    }
    if (!grid_sync(a, kPhaseProduct, latch_product)) {
      drain_warp_stages(stg, &a.ew->wait_limit_ns);
      return;
    }
    if (__ldcg(&a.ew->act_rebuild)) {
      if (blockIdx.x == 0) rebuild_work_lists(a, reinterpret_cast<int*>(scratch));
      if (!grid_sync(a, kPhaseRebuild, [&]() {
            if (threadIdx.x == 0) {
              volatile EngineWords* E = a.ew;
              E->act_rebuild = 0;
              E->act_on = 1;
              E->act_base = E->active;
            }
          }))
        return;
    }
  }

  // ---- anti-relaxation: objectiveCCP = 1/2 gamma_hat' N gamma_hat + gamma_hat' r
  // with the last r (APGD.cu:353-354); the first term was kept when gamma_hat was
  // found, the second is folded over the tiles here (one scene)
  if (kAR) {
    int nslot = 0;
    for (int i = 0;; ++i) {
      const int t = cta_tile(a, NT, i);
      if (t < 0) break;
      locate(a, sc, t);
      const ApgdCtl* C = &a.sst[sc.s].ctl;
      const int best = __ldcg(&C->best), rsel = __ldcg(&C->rsel);
      const int k0 = (t - sc.t0) * kTileItems, nc = sc.nc, c0 = sc.c0;
      double acc[1] = {0.0};
      if (best >= 0) {
        const T* B = a.G[best];
        for (int m = 0; m < kItemsPerThread; ++m) {
          const int k = k0 + m * kThreads + threadIdx.x;
          if (k < nc) {
            const int c = c0 + k;
            acc[0] = acc[0] + dot3i(B[c], B[S + c], B[2 * S + c], a.ar_r0[(size_t)rsel * S + c],
                                    (double)a.r[S + c], (double)a.r[2 * S + c]);
          }
        }
      }
      park_tile<1, false>(s_def, nslot, t, acc, 0.0);
      if (++nslot == kMaxDefer) {
        fold_parked<1, false>(a, s_def, nslot);
        nslot = 0;
      }
    }
    fold_parked<1, false>(a, s_def, nslot);
    if (!grid_sync(a, kPhaseFinal, [&]() {
          double sm[1];
          fold_tiles<1>(a, a.sst[0].t0, a.sst[0].nt, sm, scratch);
          if (threadIdx.x == 0) {
            ApgdCtl* C = &a.sst[0].ctl;
            if (__ldcg(&C->best) >= 0) C->objective = __ldcg(&C->objN) + sm[0];
          }
        }))
      return;
  }

  // ---- gamma = gamma_hat (APGD.cu:358) into the warm-start region; q = F gamma (FP64)
  {
    int cs = -1, cbest = -1;
    bool keep = false, skip = false;
    const T* src = nullptr;
    for (int i = 0;; ++i) {
      const int t = cta_tile(a, NT, i);
      if (t < 0) break;
      locate(a, sc, t);
      const int s = sc.s;
      if (s != cs) {
        cs = s;
        cbest = __ldcg(&a.sst[s].ctl.best);
        src = cbest >= 0 ? a.G[cbest] : nullptr;
        // refinement launch: a solve it did not refine keeps the FP32 launch's
        // gamma_hat and q = F gamma_hat, written by that launch's final pass; one
        // whose FP64 phase accepted no iterate keeps that gamma_hat, and q is
        // formed again (this launch's setup passes wrote over it)
        skip = a.refine && !__ldcg(&a.sst[s].ctl.refined);
        keep = a.refine && cbest < 0;
      }
      if (skip) continue;
      const SegParams& P = a.seg[s];
      const int k0 = (t - sc.t0) * kTileItems, nc = sc.nc, c0 = sc.c0;
      const int kb = a.nbil ? bil_tile_k0(t, sc.t0, nc) : -1;
      if (kb >= 0) {
        // the rows' gamma_hat (ones before the first accepted iterate)
        for (int m = 0; m < kItemsPerThread; ++m) {
          const int k = kb + m * kThreads + threadIdx.x;
          if (k < P.nbil) {
            const int r = P.bil0 + k;
            a.bil_gam[r] = cbest >= 0 ? (double)a.bG[cbest][r] : 1.0;
          }
        }
        continue;
      }
      for (int m = 0; m < kItemsPerThread; ++m) {
        int k = k0 + m * kThreads + threadIdx.x;
        if (k < nc) {
          const int c = c0 + k;
          double x0 = 1.0, x1 = 1.0, x2 = 1.0;
          const size_t wi = (size_t)P.wbase + k;
          if (keep) {
            x0 = a.gamma[0 * a.WS + wi]; x1 = a.gamma[1 * a.WS + wi]; x2 = a.gamma[2 * a.WS + wi];
          } else {
            if (src) {
              x0 = (double)src[0 * S + c]; x1 = (double)src[1 * S + c]; x2 = (double)src[2 * S + c];
            }
            a.gamma[0 * a.WS + wi] = x0;
            a.gamma[1 * a.WS + wi] = x1;
            a.gamma[2 * a.WS + wi] = x2;
          }
          a.wid[wi] = __ldg(a.idb + c) - (uint32_t)P.b0;
          Frame<double> f = load_frame_fp64(a, c, P.exact != 0);
          a.qd[c] = f_times<double, double4>(f, x0, x1, x2);
        }
      }
    }
  }
  if (!grid_sync(a, kPhaseFinal, [&]() {
        if (threadIdx.x == 0 && !a.solve_only) atomicAdd(&a.ew->steps_done, 1);
      }))
    return;

  // ---- f_c = D^T gamma; v = Minv (k + f_c); f_contact = f_c / h; p += h v.
  // Segments with neither contacts nor bilateral rows: v = Minv k, f_contact = 0
  // (System.cu:577-581); the rows' impulses enter f_c like the contacts'.
  for (int bt = blockIdx.x; bt < nbt && !a.solve_only; bt += gridDim.x) {
    int b = bt * kThreads + threadIdx.x;
    if (b < a.nb) {
      const int s = __ldg(a.bseg + b);
      const SegParams& P = a.seg[s];
      if (P.active) {
        const double h = P.h;
        const int nc = a.sst[s].nc;
        double4 k = a.k4[b];
        double mi = __ldg(a.minv + b);
        double4 v, fcv;
        if (nc > 0 || P.nbil > 0) {
          double4 fc = gather_q<double, double4>(a, a.qd, b);
          if (a.nbil) add_bilateral<double, double4>(a.bil_inc_start, a.bil_inc, a.bil_gam, b, fc);
          v = make_double4(mi * (k.x + fc.x), mi * (k.y + fc.y), mi * (k.z + fc.z), 0.0);
          const double invh = 1.0 / h;
          fcv = make_double4(invh * fc.x, invh * fc.y, invh * fc.z, 0.0);
        } else {
          v = make_double4(mi * k.x, mi * k.y, mi * k.z, 0.0);
          fcv = make_double4(0.0, 0.0, 0.0, 0.0);
        }
        a.v4[b] = v;
        a.fc4[b] = fcv;
        double4 p = a.p4[b];
        a.p4[b] = make_double4(h * v.x + p.x, h * v.y + p.y, h * v.z + p.z, 0.0);
      }
    }
  }
  // warm-start length of every segment that solved (System::gamma_d resize)
  for (int s = blockIdx.x * kThreads + threadIdx.x; s < a.nseg; s += gridDim.x * kThreads) {
    SegState& X = a.sst[s];
    const bool live = a.seg[s].active && (X.nc > 0 || a.seg[s].nbil > 0);
    if (live) X.gsize = X.nc;
    ApgdCtl& C = X.ctl;
    if (sizeof(T) != sizeof(double) && a.seg[s].refine > 0 && live) {
      // mixed precision: a solve that ended above the tolerance is refined
      // in FP64 by the launch that follows
      C.refined = (X.err == 0u && !(C.residual < a.seg[s].tol)) ? 1 : 0;
    }
    if (a.refine && live && C.refined) {
      C.refine_it = C.iterations;
      C.iterations += C.it_lo;
      C.backtracks += C.bt_lo;
      C.sweeps += C.sw_lo;
    }
    // System::time += h (System.cu:584), read by the next step's rows
    if (a.nbil && a.seg[s].active && !a.solve_only) a.seg_time[s] = a.seg_time[s] + a.seg[s].h;
  }
  // matched warm start: where each body's A-contacts went in the warm region
  for (int b = blockIdx.x * kThreads + threadIdx.x; b < a.nb; b += gridDim.x * kThreads) {
    const int s = __ldg(a.bseg + b);
    const SegState& X = a.sst[s];
    if (a.seg[s].active && (X.nc > 0 || a.seg[s].nbil > 0)) {
      a.ws[b] = a.cbase[b] + X.delta - X.c0;
      a.wc[b] = a.cnt_cont[b];
    }
  }
}

template <class T, int MB, bool AR>
void prepare_kernel() {
  static bool done = false;
  if (done) return;
  cudaFuncSetAttribute(k_step_solve<T, MB, AR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)dyn_smem_bytes<T>());
  done = true;
}


template <class T, int MB, bool AR = false>
void launch_typed(SceneDev& sd, const SolveConfig& cfg, cudaStream_t st, bool solve_only,
                  bool refine = false) {
  prepare_kernel<T, MB, AR>();
  KArgs<T> a = make_kargs<T>(sd, cfg);
  a.solve_only = solve_only ? 1 : 0;
  a.refine = refine ? 1 : 0;
  void* params[] = {&a};
  cudaLaunchCooperativeKernel((const void*)k_step_solve<T, MB, AR>, cfg.grid, kThreads, params,
                              dyn_smem_bytes<T>(), st);
}

template <class T, int MB>
int max_ctas_of() {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  prepare_kernel<T, MB, false>();
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_solve<T, MB, false>, kThreads,
                                                dyn_smem_bytes<T>());
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

}  // namespace

// Co-resident CTAs of the solve kernel for a precision and a register budget
// (blocks_per_sm 2: 128 registers per thread; 3: 80, FP32 iterates only).
int apgd_max_ctas(int precision, int blocks_per_sm) {
  if (precision == DV_PREC_MIXED)
    return blocks_per_sm == 3 ? max_ctas_of<float, 3>() : max_ctas_of<float, 2>();
  return max_ctas_of<double, 2>();
}

void launch_step_solve(SceneDev& sd, const SolveConfig& cfg, cudaStream_t st, int64_t* launches,
                       bool solve_only) {
  cudaMemsetAsync(sd.ew->bar, 0, sizeof(sd.ew->bar), st);
  cudaMemsetAsync(&sd.ew->last_release, 0, sizeof(unsigned long long), st);
  if (sd.solver == DV_SOLVER_PGJ) {
    launch_pgj_solve(sd, cfg, st, solve_only);
  } else if (sd.solver == DV_SOLVER_PGS) {
    launch_pgs_solve(sd, cfg, st, solve_only);
  } else if (sd.precision == DV_PREC_MIXED) {
    // with refinement the FP32 launch stops before the update, and an FP64
    // launch refines the solves it marked, then updates
    const bool refine = sd.refine_any != 0;
    if (cfg.blocks_per_sm == 3) launch_typed<float, 3>(sd, cfg, st, solve_only || refine);
    else launch_typed<float, 2>(sd, cfg, st, solve_only || refine);
    if (refine) {
      ++*launches;
      SolveConfig c2 = cfg;
      c2.blocks_per_sm = 2;
      c2.grid = std::min(cfg.grid, std::max(1, sd.refine_grid));
      cudaMemsetAsync(sd.ew->bar, 0, sizeof(sd.ew->bar), st);
      cudaMemsetAsync(&sd.ew->last_release, 0, sizeof(unsigned long long), st);
      launch_typed<double, 2>(sd, c2, st, solve_only, true);
    }
  } else if (sd.anti_relax) {
    launch_typed<double, 2, true>(sd, cfg, st, solve_only);
  } else {
    launch_typed<double, 2>(sd, cfg, st, solve_only);
  }
  ++*launches;
}

}  // namespace dv
