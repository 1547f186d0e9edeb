// dv_pgs.cu -- the time step with the PGS solver (System(6), PGS.cu:367-459)
// for every segment of an engine, as one persistent cooperative kernel per
// step: applied impulse, Schur vector, PGS iterations, update.  FP64 only.
//
// PGS: gamma starts at (1, 0, 0) per contact (:372, no warm start), the body
// velocities at v = Minv D^T gamma + Minv k (:376-379), B_c as in PGJ
// (buildB_PGS, :272-304), and each iteration is a Gauss-Seidel sweep over the
// contacts in their order (updateImpulseVector_CPU, :143-224): per contact
//   gamma_hat = P(gamma - omega B (D_c^T v + b_c))     (omega 0.3)
//   gamma     = lambda gamma_hat + (1 - lambda) gamma  (lambda 2/3)
//   v_A += minv_A F delta,  v_B -= minv_B F delta,  delta = lambda (gamma_hat - gamma_old)
// followed by the residual max(feasibleX(gamma), feasibleY(N gamma + r),
// max_c |(N gamma + r)_c . gamma_c|) (:402-426).  A sweep is sequential by
// definition -- every update reads the velocities the previous ones wrote --
// so one thread per scene runs it, in passes of at most kPgsChunk contacts
// (each pass ends at a grid barrier, which keeps every wait short); writing
// q = F gamma as it goes, it leaves the residual's Schur product to the
// parallel body and contact passes.  The working velocities live in v4,
// which the update at the end of the step overwrites, as the reference's
// sweep overwrites System::v.
#include "dv_solve.cuh"

namespace dv {

namespace {

constexpr double kPgsOmega = 0.3;
constexpr double kPgsLambda = 2.0 / 3.0;
constexpr int kPgsChunk = 32768;  // contacts one sweep pass updates per scene

struct PgsCtlArgs {
  double* part;
  int tcap;
  SegState* sst;
  const SegParams* seg;
  EngineWords* ew;
  unsigned* donemask;
};

// Scene controller after a residual pass: planes 0..2 hold the tile maxima of
// feasibleX(gamma), feasibleY(N gamma + r) and |(N gamma + r) . gamma|.
__device__ __noinline__ void pgs_ctl(PgsCtlArgs a, int s, double* scratch) {
  double m[3];
  fold_tiles_sm<0, 3>(a, a.sst[s].t0, a.sst[s].nt, nullptr, m, 0, scratch);
  if (threadIdx.x != 0) return;
  ApgdCtl* C = &a.sst[s].ctl;
  const SegParams& P = a.seg[s];
  const int k = __ldcg(&C->k);
  const double residual = fmax(fmax(m[0], m[1]), m[2]);
  C->residual = residual;
  bool finished = false;
  if (residual < P.tol) {
    finished = true;
    C->iterations = k;
  } else if (k + 1 >= P.max_iter) {
    finished = true;
    C->iterations = P.max_iter;
  }
  C->sweeps = k + 1;
  if (finished) {
    C->done = 1;
    atomicOr(a.donemask + (s >> 5), 1u << (s & 31));
    atomicSub(&a.ew->active, 1);
  } else {
    C->k = k + 1;
    C->mode = 0;  // next: sweep from the scene's first contact
  }
}

// One pass of the Gauss-Seidel sweep of scene s (thread-sequential): contacts
// [from, min(from + kPgsChunk, nc)) of the scene.  Returns the next start, or
// nc when the sweep is complete.
__device__ int pgs_sweep_chunk(const KArgs<double>& a, int s, int from) {
  const SegParams& P = a.seg[s];
  const SegState& X = a.sst[s];
  const size_t S = a.S;
  const int nc = X.nc, c0 = X.c0;
  const int to = min(nc, from + kPgsChunk);
  const double mu = P.mu, h = P.h;
  double* G = a.G[0];
  const double* Bc = a.G[4];
  double4* v = a.v4;
  double4* q = a.qd;
  for (int k = from; k < to; ++k) {
    const int c = c0 + k;
    const uint32_t ia = __ldg(a.ida + c), ib = __ldg(a.idb + c);
    const Frame<double> f = stored_frame(a, c);
    const double b = Bc[c];
    const double bn = __ldg(a.gap + c) / h;
    const double mia = __ldg(a.minv + ia), mib = __ldg(a.minv + ib);
    const double o0 = G[0 * S + c], o1 = G[1 * S + c], o2 = G[2 * S + c];
    const double4 va = v[ia], vb = v[ib];
    const double ob = kPgsOmega * b;
    double g0 = o0 - ob * (f.n0 * va.x + f.n1 * va.y + f.n2 * va.z - f.n0 * vb.x - f.n1 * vb.y -
                           f.n2 * vb.z + bn);
    double g1 = o1 - ob * (f.u0 * va.x + f.u1 * va.y + f.u2 * va.z - f.u0 * vb.x - f.u1 * vb.y -
                           f.u2 * vb.z);
    double g2 = o2 - ob * (f.v0 * va.x + f.v1 * va.y + f.v2 * va.z - f.v0 * vb.x - f.v1 * vb.y -
                           f.v2 * vb.z);
    project_cone<double>(g0, g1, g2, mu);
    const double la = kPgsLambda, lb = 1.0 - kPgsLambda;
    const double y0 = la * g0 + lb * o0, y1 = la * g1 + lb * o1, y2 = la * g2 + lb * o2;
    G[0 * S + c] = y0;
    G[1 * S + c] = y1;
    G[2 * S + c] = y2;
    const double d0 = la * (g0 - o0), d1 = la * (g1 - o1), d2 = la * (g2 - o2);
    const double ex = f.n0 * d0 + f.u0 * d1 + f.v0 * d2;
    const double ey = f.n1 * d0 + f.u1 * d1 + f.v1 * d2;
    const double ez = f.n2 * d0 + f.u2 * d1 + f.v2 * d2;
    v[ia] = make_double4(va.x + mia * ex, va.y + mia * ey, va.z + mia * ez, 0.0);
    // B after A: a contact's bodies differ, and B reads its velocity before A's write
    v[ib] = make_double4(vb.x - mib * ex, vb.y - mib * ey, vb.z - mib * ez, 0.0);
    q[c] = f_times<double, double4>(f, y0, y1, y2);
  }
  return to;
}

__global__ void __launch_bounds__(kThreads, 2) k_pgs_solve(KArgs<double> a) {
  using V = double4;
  __shared__ double scratch[kNQ * 8 + 8];
  __shared__ unsigned s_mask[kMaskWords];
  __shared__ DeferBuf s_def;
  __shared__ SegCache s_sc;
  const size_t S = a.S;
  V* wv = a.wd;
  V* qv = a.qd;
  SegCache& sc = s_sc;
  if (threadIdx.x == 0) {
    sc.s = -1;
    sc.t0 = sc.t1 = 0;
    s_def.fail = 0;
  }
  __syncthreads();
  if (ld_acquire(&a.ew->err)) return;
  const int NT = a.ew->ntiles;
  const int nbt = (a.nb + kThreads - 1) / kThreads;
  const int mwords = (a.nseg + 31) >> 5;
  const PgsCtlArgs ca{a.part, a.tcap, a.sst, a.seg, a.ew, a.donemask};
  double* Bc = a.G[4];  // per-contact B (plane 0)
  const int gtid = blockIdx.x * kThreads + threadIdx.x, gthreads = gridDim.x * kThreads;

  // ---- per-segment state, done mask
  for (int s = gtid; s < a.nseg; s += gthreads) {
    SegState& X = a.sst[s];
    X.err = 0u;
    X.arrive = 0u;
    ApgdCtl& C = X.ctl;
    const bool live = a.seg[s].active && X.nc > 0;
    C.done = (live && a.seg[s].max_iter > 0) ? 0 : 1;
    C.k = 0;
    C.cur = 0;
    C.best = 0;
    C.mode = 0;  // sweep start within the current iteration
    C.iterations = 0;
    C.sweeps = 0;
    C.backtracks = 0;
    C.residual = 0.0;
    C.objective = 0.0;
  }
  for (int wi = gtid; wi < mwords; wi += gthreads) {
    unsigned m = 0u;
    for (int j = 0; j < 32; ++j) {
      const int s = wi * 32 + j;
      if (s >= a.nseg || !(a.seg[s].active && a.sst[s].nc > 0 && a.seg[s].max_iter > 0))
        m |= 1u << j;
    }
    a.donemask[wi] = m;
  }

  // ---- applied impulse: k = m v + h f; w = minv k
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
          int n = 0;
          for (int s = 0; s < a.nseg; ++s) n += __ldcg(&a.sst[s].ctl.done) ? 0 : 1;
          atomicExch(&a.ew->active, n);
        }
      }))
    return;

  // ---- r = D (Minv k) + b; gamma_0 = (1, 0, 0) -> G[0]; B; q = F gamma_0
  for (int i = 0;; ++i) {
    const int t = cta_tile(a, NT, i);
    if (t < 0) break;
    locate(a, sc, t);
    const SegParams& P = a.seg[sc.s];
    const int k0 = (t - sc.t0) * kTileItems, nc = sc.nc, c0 = sc.c0;
    const double h = P.h;
    for (int m = 0; m < kItemsPerThread; ++m) {
      int k = k0 + m * kThreads + threadIdx.x;
      if (k < nc) {
        const int c = c0 + k;
        Frame<double> fd = load_frame_fp64(a, c, P.exact != 0);
        const uint32_t ia = __ldg(a.ida + c), ib = __ldg(a.idb + c);
        double4 wa = a.wd[ia], wb = a.wd[ib];
        double d0, d1, d2;
        ft_times<double, double4>(fd, wa, wb, &d0, &d1, &d2);
        double bn = __ldg(a.gap + c) / h;
        a.r[0 * S + c] = bn + d0;
        a.r[1 * S + c] = 0.0 + d1;
        a.r[2 * S + c] = 0.0 + d2;
        a.G[0][0 * S + c] = 1.0;
        a.G[0][1 * S + c] = 0.0;
        a.G[0][2 * S + c] = 0.0;
        // buildB_PGS: the nine frame entries squared and summed in row order n, u, v
        double sum = fd.n0 * fd.n0;
        sum = sum + fd.n1 * fd.n1;
        sum = sum + fd.n2 * fd.n2;
        sum = sum + fd.u0 * fd.u0;
        sum = sum + fd.u1 * fd.u1;
        sum = sum + fd.u2 * fd.u2;
        sum = sum + fd.v0 * fd.v0;
        sum = sum + fd.v1 * fd.v1;
        sum = sum + fd.v2 * fd.v2;
        const double mia = __ldg(a.minv + ia), mib = __ldg(a.minv + ib);
        Bc[c] = 3.0 / ((mia + mib) * sum);
        qv[c] = f_times<double, double4>(fd, 1.0, 0.0, 0.0);
      }
    }
  }
  if (!grid_sync(a, kPhaseSetup, NoCtl{})) return;

  // ---- v = Minv (D^T gamma_0) + Minv k for the bodies of scenes that iterate
  // (PGS.cu:376-379: two products, then the sum)
  load_mask(a, s_mask, mwords);
  for (int bt = blockIdx.x; bt < nbt; bt += gridDim.x) {
    int b = bt * kThreads + threadIdx.x;
    if (b < a.nb && !mask_done(a, s_mask, mwords, __ldg(a.bseg + b))) {
      const double mi = __ldg(a.minv + b);
      const double4 fc = gather_q<double, double4>(a, qv, b);
      const double4 k = a.k4[b];
      const double4 t = make_double4(mi * k.x, mi * k.y, mi * k.z, 0.0);
      a.v4[b] = make_double4(t.x + mi * fc.x, t.y + mi * fc.y, t.z + mi * fc.z, 0.0);
    }
  }
  if (!grid_sync(a, kPhaseSetup, NoCtl{})) return;

  // ---- iterations: sweep passes (one thread per scene), then the residual:
  // one body pass (w of q = F gamma) and one contact pass (N gamma + r).  The
  // controllers change `active` only in the contact pass, which a grid barrier
  // separates from every CTA's check at the top of the loop.
  for (;;) {
    if (__ldcg(&a.ew->active) == 0) break;
    load_mask(a, s_mask, mwords);
    // sweep passes until every iterating scene has swept all its contacts
    for (;;) {
      int more = 0;
      for (int s = gtid; s < a.nseg; s += gthreads) {
        if (mask_done(a, s_mask, mwords, s)) continue;
        ApgdCtl* C = &a.sst[s].ctl;
        const int from = __ldcg(&C->mode);
        const int nc = a.sst[s].nc;
        if (from >= nc) continue;
        const int to = pgs_sweep_chunk(a, s, from);
        C->mode = to;
        if (to < nc) more = 1;
      }
      if (more) atomicOr(&a.ew->step_count, 1);
      if (!grid_sync(a, kPhaseStep, [&]() {
            if (threadIdx.x == 0) {
              const int n = atomicExch(&a.ew->step_count, 0);
              *(volatile int*)&a.ew->step_needed = n;
            }
          }))
        return;
      if (__ldcg(&a.ew->step_needed) == 0) break;
    }
    body_pass_schur(a, s_mask);
    if (!grid_sync(a, kPhaseBody, NoCtl{})) return;
    {
      SegRun run;
      int nslot = 0;
      auto ctl = [&](int s) { pgs_ctl(ca, s, scratch); };
      int cs = -1;
      double mu = 0.0;
      bool ex = false;
      for (int i = 0;; ++i) {
        const int t = cta_tile(a, NT, i);
        if (t < 0) break;
        locate(a, sc, t);
        const int s = sc.s;
        if (mask_done(a, s_mask, mwords, s)) continue;
        if (s != cs) {
          cs = s;
          mu = a.seg[s].mu;
          ex = a.seg[s].exact != 0;
        }
        if (s != run.s) {
          if (run.n) {
            fold_parked_max<3>(a, s_def, nslot);
            nslot = 0;
          }
          flush_run(a, run, ctl);
          run.s = s;
        }
        const double* G = a.G[0];
        const int k0 = (t - sc.t0) * kTileItems, nc = sc.nc, c0 = sc.c0;
        double mx[3] = {0.0, 0.0, 0.0};
        for (int m = 0; m < kItemsPerThread; ++m) {
          int k = k0 + m * kThreads + threadIdx.x;
          if (k < nc) {
            const int c = c0 + k;
            Frame<double> f = load_frame<double>(a, c, ex);
            V wa = wv[__ldg(a.ida + c)], wb = wv[__ldg(a.idb + c)];
            double N0, N1, N2;
            ft_times<double, V>(f, wa, wb, &N0, &N1, &N2);
            const double x0 = G[0 * S + c], x1 = G[1 * S + c], x2 = G[2 * S + c];
            const double g0 = a.r[0 * S + c] + N0, g1 = a.r[1 * S + c] + N1,
                         g2 = a.r[2 * S + c] + N2;
            mx[0] = fmax(mx[0], pgj_feasible(x0, x1, x2, mu));
            mx[1] = fmax(mx[1], pgj_feasible(g0, g1, g2, 1.0 / mu));
            const double d = (g0 * x0 + g1 * x1) + g2 * x2;
            mx[2] = fmax(mx[2], fabs(d));
          }
        }
        park_max<3>(s_def, nslot, t, mx);
        ++run.n;
        if (++nslot == kMaxDefer) {
          fold_parked_max<3>(a, s_def, nslot);
          nslot = 0;
        }
      }
      fold_parked_max<3>(a, s_def, nslot);
      flush_run(a, run, ctl);
    }
    if (!grid_sync(a, kPhaseProduct, NoCtl{})) return;
  }

  // ---- gamma -> warm-start region (System::gamma_d); q = F gamma (FP64)
  for (int i = 0;; ++i) {
    const int t = cta_tile(a, NT, i);
    if (t < 0) break;
    locate(a, sc, t);
    const SegParams& P = a.seg[sc.s];
    const int k0 = (t - sc.t0) * kTileItems, nc = sc.nc, c0 = sc.c0;
    for (int m = 0; m < kItemsPerThread; ++m) {
      int k = k0 + m * kThreads + threadIdx.x;
      if (k < nc) {
        const int c = c0 + k;
        const double x0 = a.G[0][0 * S + c], x1 = a.G[0][1 * S + c], x2 = a.G[0][2 * S + c];
        const size_t wi = (size_t)P.wbase + k;
        a.gamma[0 * a.WS + wi] = x0;
        a.gamma[1 * a.WS + wi] = x1;
        a.gamma[2 * a.WS + wi] = x2;
        Frame<double> f = load_frame_fp64(a, c, P.exact != 0);
        a.qd[c] = f_times<double, double4>(f, x0, x1, x2);
      }
    }
  }
  if (!grid_sync(a, kPhaseFinal, [&]() {
        if (threadIdx.x == 0 && !a.solve_only) atomicAdd(&a.ew->steps_done, 1);
      }))
    return;

  // ---- f_c = D^T gamma; v = Minv (k + f_c); f_contact = f_c / h; p += h v
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
        if (nc > 0) {
          double4 fc = gather_q<double, double4>(a, a.qd, b);
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
  for (int s = gtid; s < a.nseg; s += gthreads) {
    SegState& X = a.sst[s];
    if (a.seg[s].active && X.nc > 0) X.gsize = X.nc;
  }
}

}  // namespace

int pgs_max_ctas() {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pgs_solve, kThreads, 0);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

void launch_pgs_solve(SceneDev& sd, const SolveConfig& cfg, cudaStream_t st, bool solve_only) {
  const int grid = std::min(cfg.grid, pgs_max_ctas());
  KArgs<double> a = make_kargs<double>(sd, cfg);
  a.solve_only = solve_only ? 1 : 0;
  void* params[] = {&a};
  cudaLaunchCooperativeKernel((const void*)k_pgs_solve, grid, kThreads, params, 0, st);
}

}  // namespace dv
