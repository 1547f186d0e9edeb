// dv_pgj.cu -- the time step with the PGJ solver (System(5), PGJ.cu:152-224)
// for every segment of an engine, as one persistent cooperative kernel per
// step: applied impulse, Schur vector, PGJ iterations, update.
//
// PGJ: gamma starts at (1, 0, 0) per contact (PGJ.cu:170, no warm start),
// B_c = 3 / ((minv_A + minv_B) |F_c|^2) (buildB, :73-89), and each iteration
//   gamma_hat = P(gamma - omega B (N gamma + r))
//   gamma     = lambda gamma_hat + (1 - lambda) gamma       (omega 0.3, lambda 2/3)
// stops when max(feasibleX, feasibleY, max_c |(N gamma + r)_c . gamma_c|) of
// the new gamma is below the tolerance (:188-214).  N of the new iterate
// serves its residual and the next iteration, so an iteration is one body
// pass and one contact pass: the contact pass forms N gamma_k, the residual
// terms of gamma_k and the step to gamma_{k+1} (its feasibleX and q = F
// gamma_{k+1}); the scene's controller then decides on gamma_k.  Only maxima
// are reduced, so the result does not depend on any summation order.
#include "dv_solve.cuh"

namespace dv {

namespace {

constexpr double kPgjOmega = 0.3;
constexpr double kPgjLambda = 2.0 / 3.0;

struct PgjCtlArgs {
  double* part;
  int tcap;
  SegState* sst;
  const SegParams* seg;
  EngineWords* ew;
  unsigned* donemask;
};

// Scene controller after a PGJ contact pass: planes 0..2 hold the tile maxima
// of feasibleX (of the new iterate), feasibleY and res3 (of the current one).
__device__ __noinline__ void pgj_ctl(PgjCtlArgs a, int s, double* scratch) {
  double m[3];
  fold_tiles_sm<0, 3>(a, a.sst[s].t0, a.sst[s].nt, nullptr, m, 0, scratch);
  if (threadIdx.x != 0) return;
  ApgdCtl* C = &a.sst[s].ctl;
  const ApgdCtl c = ctl_read(C);
  const SegParams& P = a.seg[s];
  const int k = c.k;
  bool finished = false;
  if (k >= 1) {
    const double residual = fmax(fmax(c.fx, m[1]), m[2]);
    C->residual = residual;
    if (residual < P.tol) {
      finished = true;
      C->iterations = k - 1;
    } else if (k >= P.max_iter) {
      finished = true;
      C->iterations = P.max_iter;
    }
  }
  if (finished) {
    C->best = c.cur;  // gamma_k
    C->done = 1;
    atomicOr(a.donemask + (s >> 5), 1u << (s & 31));
    atomicSub(&a.ew->active, 1);
  } else {
    C->fx = m[0];
    C->cur = c.cur ^ 1;
    C->k = k + 1;
    C->sweeps = c.sweeps + 1;
  }
}

template <class T>
__global__ void __launch_bounds__(kThreads, 2) k_pgj_solve(KArgs<T> a) {
  using V = typename Vec4<T>::type;
  __shared__ double scratch[kNQ * 8 + 8];
  __shared__ unsigned s_mask[kMaskWords];
  __shared__ DeferBuf s_def;
  __shared__ SegCache s_sc;
  const size_t S = a.S;
  V* wv = reinterpret_cast<V*>(a.wd);
  V* qv = reinterpret_cast<V*>(a.qd);
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
  const PgjCtlArgs ca{a.part, a.tcap, a.sst, a.seg, a.ew, a.donemask};
  T* Bc = a.G[4];  // per-contact B (plane 0)

  // ---- per-segment state, done mask
  for (int s = blockIdx.x * kThreads + threadIdx.x; s < a.nseg; s += gridDim.x * kThreads) {
    SegState& X = a.sst[s];
    X.err = 0u;
    X.arrive = 0u;
    ApgdCtl& C = X.ctl;
    const bool live = a.seg[s].active && X.nc > 0;
    C.done = (live && a.seg[s].max_iter > 0) ? 0 : 1;
    C.k = 0;
    C.cur = 0;
    C.best = 0;
    C.iterations = 0;
    C.sweeps = 0;
    C.backtracks = 0;
    C.residual = 0.0;
    C.objective = 0.0;
    C.fx = 0.0;
  }
  for (int wi = blockIdx.x * kThreads + threadIdx.x; wi < mwords; wi += gridDim.x * kThreads) {
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
        a.r[0 * S + c] = (T)(bn + d0);
        a.r[1 * S + c] = (T)(0.0 + d1);
        a.r[2 * S + c] = (T)(0.0 + d2);
        a.G[0][0 * S + c] = T(1);
        a.G[0][1 * S + c] = T(0);
        a.G[0][2 * S + c] = T(0);
        // buildB: the nine frame entries squared and summed in row order n, u, v
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
        Bc[c] = (T)(3.0 / ((mia + mib) * sum));
        Frame<T> f = load_frame<T>(a, c, P.exact != 0);
        qv[c] = f_times<T, V>(f, T(1), T(0), T(0));
      }
    }
  }
  if (!grid_sync(a, kPhaseSetup, NoCtl{})) return;

  // ---- iterations: one body pass (w of q = F gamma_k) and one contact pass
  // (N gamma_k, residual terms of gamma_k, step to gamma_{k+1}) each.  The
  // controllers change `active` only in the contact pass, which a grid
  // barrier separates from every CTA's check at the top of the loop.
  for (;;) {
    if (__ldcg(&a.ew->active) == 0) break;
    load_mask(a, s_mask, mwords);
    body_pass_schur(a, s_mask);
    if (!grid_sync(a, kPhaseBody, NoCtl{})) return;
    {
      SegRun run;
      int nslot = 0;
      auto ctl = [&](int s) { pgj_ctl(ca, s, scratch); };
      int cs = -1, cur = 0, kk = 0;
      T mu = T(0);
      double mud = 0.0;
      bool ex = false;
      for (int i = 0;; ++i) {
        const int t = cta_tile(a, NT, i);
        if (t < 0) break;
        locate(a, sc, t);
        const int s = sc.s;
        if (mask_done(a, s_mask, mwords, s)) continue;
        if (s != cs) {
          cs = s;
          cur = __ldcg(&a.sst[s].ctl.cur);
          kk = __ldcg(&a.sst[s].ctl.k);
          mud = a.seg[s].mu;
          mu = (T)mud;
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
        const T* Gc = a.G[cur];
        T* Gn = a.G[cur ^ 1];
        const int k0 = (t - sc.t0) * kTileItems, nc = sc.nc, c0 = sc.c0;
        double mx[3] = {0.0, 0.0, 0.0};
        for (int m = 0; m < kItemsPerThread; ++m) {
          int k = k0 + m * kThreads + threadIdx.x;
          if (k < nc) {
            const int c = c0 + k;
            Frame<T> f = load_frame<T>(a, c, ex);
            V wa = wv[__ldg(a.ida + c)], wb = wv[__ldg(a.idb + c)];
            T N0, N1, N2;
            ft_times<T, V>(f, wa, wb, &N0, &N1, &N2);
            const T x0 = Gc[0 * S + c], x1 = Gc[1 * S + c], x2 = Gc[2 * S + c];
            const T r0 = a.r[0 * S + c], r1 = a.r[1 * S + c], r2 = a.r[2 * S + c];
            const T g0 = N0 + r0, g1 = N1 + r1, g2 = N2 + r2;
            if (kk >= 1) {
              const double d = ((double)g0 * (double)x0 + (double)g1 * (double)x1) +
                               (double)g2 * (double)x2;
              mx[2] = fmax(mx[2], fabs(d));
              mx[1] = fmax(mx[1], pgj_feasible(g0, g1, g2, 1.0 / mud));
            }
            // gamma_hat = gamma + (-omega) (B (N gamma + r)), projected
            const T b = Bc[c];
            const T om = (T)(-kPgjOmega);
            T h0 = x0 + om * (b * g0), h1 = x1 + om * (b * g1), h2 = x2 + om * (b * g2);
            project_cone<T>(h0, h1, h2, mu);
            const T la = (T)kPgjLambda, lb = (T)(1.0 - kPgjLambda);
            const T y0 = la * h0 + lb * x0, y1 = la * h1 + lb * x1, y2 = la * h2 + lb * x2;
            Gn[0 * S + c] = y0; Gn[1 * S + c] = y1; Gn[2 * S + c] = y2;
            mx[0] = fmax(mx[0], pgj_feasible(y0, y1, y2, mud));
            qv[c] = f_times<T, V>(f, y0, y1, y2);
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

  // ---- gamma -> warm-start region; q = F gamma (FP64)
  {
    int cs = -1;
    const T* src = nullptr;
    for (int i = 0;; ++i) {
      const int t = cta_tile(a, NT, i);
      if (t < 0) break;
      locate(a, sc, t);
      const int s = sc.s;
      if (s != cs) {
        cs = s;
        src = a.G[__ldcg(&a.sst[s].ctl.best)];
      }
      const SegParams& P = a.seg[s];
      const int k0 = (t - sc.t0) * kTileItems, nc = sc.nc, c0 = sc.c0;
      for (int m = 0; m < kItemsPerThread; ++m) {
        int k = k0 + m * kThreads + threadIdx.x;
        if (k < nc) {
          const int c = c0 + k;
          const double x0 = (double)src[0 * S + c], x1 = (double)src[1 * S + c],
                       x2 = (double)src[2 * S + c];
          const size_t wi = (size_t)P.wbase + k;
          a.gamma[0 * a.WS + wi] = x0;
          a.gamma[1 * a.WS + wi] = x1;
          a.gamma[2 * a.WS + wi] = x2;
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
  for (int s = blockIdx.x * kThreads + threadIdx.x; s < a.nseg; s += gridDim.x * kThreads) {
    SegState& X = a.sst[s];
    if (a.seg[s].active && X.nc > 0) X.gsize = X.nc;
  }
}


template <class T>
int pgj_ctas() {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pgj_solve<T>, kThreads, 0);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

}  // namespace

int pgj_max_ctas(int precision) {
  return precision == DV_PREC_MIXED ? pgj_ctas<float>() : pgj_ctas<double>();
}

void launch_pgj_solve(SceneDev& sd, const SolveConfig& cfg, cudaStream_t st, bool solve_only) {
  const int grid = std::min(cfg.grid, pgj_max_ctas(sd.precision));
  if (sd.precision == DV_PREC_MIXED) {
    KArgs<float> a = make_kargs<float>(sd, cfg);
    a.solve_only = solve_only ? 1 : 0;
    void* params[] = {&a};
    cudaLaunchCooperativeKernel((const void*)k_pgj_solve<float>, grid, kThreads, params, 0, st);
  } else {
    KArgs<double> a = make_kargs<double>(sd, cfg);
    a.solve_only = solve_only ? 1 : 0;
    void* params[] = {&a};
    cudaLaunchCooperativeKernel((const void*)k_pgj_solve<double>, grid, kThreads, params, 0, st);
  }
}

}  // namespace dv
