// dv_engine.cu -- host side of an engine (see dv_engine.h).
//
// One step on the engine's stream (System::DoTimeStep, System.cu:544-602, for
// every active segment):
//   collide         AABBs, per-segment grids, radix sort, candidate/contact
//                   counts, contact layout and tiles, sorted contacts +
//                   frames, body incidence -- sizes read on the device
//   k_step_solve    one cooperative persistent kernel: k, r, APGD of every
//                   segment, update
// Nothing waits for the host inside a step, so n steps are enqueued at once
// (or replayed from a captured CUDA graph) and the host synchronizes once.
// When a step overflows a buffer the device flags it and skips the rest of
// the step (and every later step) without touching the state; the host grows
// the buffer and re-runs from the failed step.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <numeric>

#include "dv_engine.h"

namespace dv {

int status_from_bits(unsigned bits) {
  if (bits & (kErrBarrierTimeout | kErrCopyTimeout)) return DV_ERR_TIMEOUT;
  if (bits & kErrNaN) return DV_ERR_NAN;
  if (bits & kErrBacktrackCap) return DV_ERR_NOCONV;
  if (bits & (kErrCapacity | kErrPartners)) return DV_ERR_ARG;
  if (bits & kErrAborted) return DV_ERR_ABORTED;
  return DV_OK;
}

void fill_step_stats(const StepRecord& r, int s, dv_step_stats* out) {
  memset(out, 0, sizeof(*out));
  const SegState& X = r.sst[s];
  out->num_contacts = X.nc;
  out->num_possible = X.npossible;
  out->iterations = X.ctl.iterations;
  out->backtracks = X.ctl.backtracks;
  out->residual = X.ctl.residual;
  out->objective = X.ctl.objective;
  out->sweeps = X.ctl.sweeps;
  out->refine_iterations = X.ctl.refine_it;
  out->elapsed_ms = r.ms_total;
  out->collide_ms = r.ms_collide;
  out->solve_ms = r.ms_solve;
  out->time = r.time;
  out->time_index = r.time_index;
  int st = status_from_bits(r.ew.err);
  if (st == DV_OK) st = status_from_bits(X.err);
  out->status = st;
}

#define TRY(x)                    \
  do {                            \
    int rc_ = (x);                \
    if (rc_ != DV_OK) return rc_; \
  } while (0)

Engine::~Engine() {
  if (st_) cudaStreamSynchronize(st_);
  drop_graph();
  for (void* p : allocs_) cudaFree(p);
  allocs_.clear();
  if (h_ew_) cudaFreeHost(h_ew_);
  if (h_sst_) cudaFreeHost(h_sst_);
  if (h_ew_ring_) cudaFreeHost(h_ew_ring_);
  if (h_sst_ring_) cudaFreeHost(h_sst_ring_);
  if (h_red_) cudaFreeHost(h_red_);
  for (cudaEvent_t e : ev_) cudaEventDestroy(e);
  if (own_stream_ && st_) cudaStreamDestroy(st_);
}

static const char* const kPartnerLimitText =
    "a sphere has more than 8192 contact partners with larger ids, or more than 65536 spheres "
    "have over 128 in one step";

static int check_params(const dv_params& p) {
  if (!(p.h > 0) || !(p.envelope >= 0) || !(p.mu >= 0) || !(p.tolerance >= 0)) return DV_ERR_ARG;
  if (p.max_iterations < 0 || p.max_backtracks < 0) return DV_ERR_ARG;
  if (p.solver != DV_SOLVER_APGD && p.solver != DV_SOLVER_PGJ && p.solver != DV_SOLVER_PGS)
    return DV_ERR_UNSUPPORTED;
  if (p.precision != DV_PREC_FP64 && p.precision != DV_PREC_MIXED) return DV_ERR_UNSUPPORTED;
  if (p.solver == DV_SOLVER_PGS && p.precision != DV_PREC_FP64) return DV_ERR_UNSUPPORTED;
  if (p.warm_start < 0 || p.warm_start > 2) return DV_ERR_ARG;
  if (p.fp64_narrowphase != 0 && p.fp64_narrowphase != 1) return DV_ERR_ARG;
  if (p.anti_relaxation != 0 && p.anti_relaxation != 1) return DV_ERR_ARG;
  if (p.refine_iterations < 0) return DV_ERR_ARG;
  // anti-relaxation: an APGD option, FP64 only
  if (p.anti_relaxation && (p.solver != DV_SOLVER_APGD || p.precision != DV_PREC_FP64))
    return DV_ERR_UNSUPPORTED;
  return DV_OK;
}

int Engine::alloc_contacts(size_t cap) {
  SceneDev& q = d;
  // segment ranges start on multiples of 256 and the solve kernel copies
  // 32-contact plane segments with bulk asynchronous copies
  cap = (cap + kContactAlign - 1) / kContactAlign * kContactAlign;
  dfree(q.ida); dfree(q.idb); dfree(q.F); dfree(q.nf); dfree(q.gap); dfree(q.loc);
  dfree(q.r);
  for (int k = 0; k < 5; ++k) {
    dfree(q.G[k]);
    dfree(q.NG[k]);
  }
  dfree(q.q); dfree(q.inc); dfree(q.part); dfree(q.tseg); dfree(q.act_tiles);
  dfree(q.ar_r0); dfree(q.ar_v);
  q.ccap = cap;
  q.tcap = (int)(cap / kTileItems) + q.nseg + 1 + (q.nbil + kTileItems - 1) / kTileItems;
  TRY(dalloc(&q.ida, cap));
  TRY(dalloc(&q.idb, cap));
  TRY(dalloc(&q.F, 9 * cap));
  TRY(dalloc(&q.nf, 3 * cap));
  TRY(dalloc(&q.gap, cap));
  TRY(dalloc(&q.loc, 3 * cap));
  TRY(dalloc(&q.r, 3 * cap));
  for (int k = 0; k < 5; ++k) {
    TRY(dalloc(&q.G[k], 3 * cap));
    TRY(dalloc(&q.NG[k], 3 * cap));
  }
  TRY(dalloc(&q.q, cap));
  TRY(dalloc(&q.inc, 2 * cap));
  if (q.anti_relax) {
    TRY(dalloc(&q.ar_r0, 2 * cap));
    TRY(dalloc(&q.ar_v, 2 * cap));
  }
  TRY(dalloc(&q.part, (size_t)8 * q.tcap));
  TRY(dalloc(&q.tseg, (size_t)q.tcap));
  TRY(dalloc(&q.act_tiles, (size_t)q.tcap));
  size_t rc = std::max((size_t)q.nb, cap);
  if (rc > q.radix_cap) {
    dfree(q.keyA); dfree(q.valA); dfree(q.keyB); dfree(q.valB); dfree(q.radix_hist);
    q.radix_cap = rc;
    TRY(dalloc(&q.keyA, rc));
    TRY(dalloc(&q.valA, rc));
    TRY(dalloc(&q.keyB, rc));
    TRY(dalloc(&q.valB, rc));
    q.radix_hist_cap = radix_hist_size(rc);
    TRY(dalloc(&q.radix_hist, q.radix_hist_cap));
  }
  return DV_OK;
}

int Engine::upload_segments() {
  DV_CUDA_TRY(cudaMemcpyAsync(d.seg, hseg_.data(), sizeof(SegParams) * hseg_.size(),
                              cudaMemcpyHostToDevice, st_));
  // a second (FP64) solve launch per step when a segment asks for refinement
  int ra = 0;
  for (const SegParams& G : hseg_) ra |= (G.active && G.refine > 0) ? 1 : 0;
  if (ra != d.refine_any) {
    d.refine_any = ra;
    if (ra && !d.refine_grid) d.refine_grid = apgd_max_ctas(DV_PREC_FP64, 2);
    drop_graph();
  }
  return DV_OK;
}

namespace {

// Carried body arrays of the new layout: body b' takes old body map[b'] (>= 0)
// or staged new body -(map[b'] + 1).
__global__ void __launch_bounds__(kThreads) k_gather_bodies(
    int nb, const int* __restrict__ map, const double4* __restrict__ op, const double4* __restrict__ ov,
    const double4* __restrict__ of, const double4* __restrict__ og, const double* __restrict__ om,
    const int* __restrict__ ofam, const int* __restrict__ ows, const int* __restrict__ owc,
    const double4* __restrict__ sp, const double4* __restrict__ sv,
    const double4* __restrict__ sf, const double4* __restrict__ sg, const double* __restrict__ sm,
    const int* __restrict__ sfam, double4* __restrict__ np, double4* __restrict__ nv,
    double4* __restrict__ nf, double4* __restrict__ ng, double* __restrict__ nm,
    int* __restrict__ nfam, int* __restrict__ nws, int* __restrict__ nwc) {
  int b = blockIdx.x * kThreads + threadIdx.x;
  if (b >= nb) return;
  int m = map[b];
  if (m >= 0) {
    np[b] = op[m]; nv[b] = ov[m]; nf[b] = of[m]; ng[b] = og[m]; nm[b] = om[m]; nfam[b] = ofam[m];
    nws[b] = ows[m]; nwc[b] = owc[m];
  } else {
    int k = -(m + 1);
    np[b] = sp[k]; nv[b] = sv[k]; nf[b] = sf[k]; ng[b] = sg[k]; nm[b] = sm[k]; nfam[b] = sfam[k];
    nws[b] = 0; nwc[b] = 0;
  }
}

// Warm-start regions of carried segments: 3 planes of `n[s]` values from
// src[s] in the old arena to dst[s] in the new one (blockIdx.y = segment).
__global__ void __launch_bounds__(kThreads) k_gather_warm(const int* __restrict__ src,
                                                         const int* __restrict__ dst,
                                                         const int* __restrict__ n,
                                                         const double* __restrict__ og, size_t ows,
                                                         const uint32_t* __restrict__ oid,
                                                         double* __restrict__ ng, size_t nws,
                                                         uint32_t* __restrict__ nid) {
  const int s = blockIdx.y;
  const int cnt = n[s];
  if (src[s] < 0) return;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < cnt; i += gridDim.x * kThreads) {
    for (int k = 0; k < 3; ++k) ng[k * nws + dst[s] + i] = og[k * ows + src[s] + i];
    nid[dst[s] + i] = oid[src[s] + i];
  }
}

}  // namespace

static int validate_scene(const SceneInput& sc) {
  if (sc.nb < 0 || (sc.nb > 0 && !sc.bodies)) return DV_ERR_ARG;
  TRY(check_params(sc.P));
  for (int i = 0; i < sc.nb; ++i) {
    const dv_body_desc& b = sc.bodies[i];
    if (!(b.mass > 0) && !b.fixed) return DV_ERR_ARG;
    if (b.geom[1] == 0 && !(b.geom[0] >= 0)) return DV_ERR_ARG;
  }
  return DV_OK;
}

int Engine::init(const std::vector<SceneInput>& scenes, int precision) {
  if (scenes.empty()) return DV_ERR_ARG;
  if (precision != DV_PREC_FP64 && precision != DV_PREC_MIXED) return DV_ERR_UNSUPPORTED;
  // arguments first: nothing touches the device for an invalid scene
  for (const SceneInput& sc : scenes) TRY(validate_scene(sc));
  if (cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking) != cudaSuccess)
    return dv_record_cuda_error(cudaGetLastError(), "cudaStreamCreate", __FILE__, __LINE__);
  own_stream_ = true;
  d.precision = precision;
  TRY(dalloc(&d.ew, 1));
  TRY(dalloc(&d.wide_ids, kWideSpheres));
  if (cudaMallocHost(&h_ew_, sizeof(EngineWords)) != cudaSuccess)
    return dv_record_cuda_error(cudaErrorMemoryAllocation, "cudaMallocHost", __FILE__, __LINE__);
  memset(h_ew_, 0, sizeof(EngineWords));
  h_ew_->wait_limit_ns = kBarrierTimeoutNs;
  DV_CUDA_TRY(cudaMemcpyAsync(d.ew, h_ew_, sizeof(EngineWords), cudaMemcpyHostToDevice, st_));
  std::vector<SlotSpec> slots(scenes.size());
  for (size_t i = 0; i < scenes.size(); ++i) slots[i].in = scenes[i];
  TRY(reconfigure(slots));
  if (scenes.size() == 1 && scenes[0].P.anti_relaxation) TRY(enable_anti_relax());
  max_ctas_ = apgd_max_ctas(precision, 2);
  DV_CUDA_TRY(cudaGetLastError());
  cfg_.grid = std::max(1, std::min(max_ctas_, (d.nb + kThreads - 1) / kThreads));
  cfg_.chunk = 1;
  cfg_.contiguous = 0;
  cfg_.blocks_per_sm = 2;
  return DV_OK;
}

template <class T>
int Engine::ensure(T** p, int* cap, size_t need) {
  if ((size_t)*cap >= need && *p) return DV_OK;
  size_t n = std::max(need, (size_t)*cap + (size_t)*cap / 4);
  dfree(*p);
  TRY(dalloc(p, n));
  *cap = (int)n;
  return DV_OK;
}

int Engine::reconfigure(const std::vector<SlotSpec>& slots) {
  const int nseg2 = (int)slots.size();
  if (nseg2 == 0) return DV_ERR_ARG;
  for (const SlotSpec& sl : slots) {
    if (sl.keep >= d.nseg) return DV_ERR_ARG;
    if (sl.keep < 0) TRY(validate_scene(sl.in));
    // anti-relaxation: the first layout of a one-scene engine only
    if (sl.keep < 0 && sl.in.P.anti_relaxation && !(nseg2 == 1 && d.nseg == 0))
      return DV_ERR_UNSUPPORTED;
  }
  // one solver for every segment of an engine
  int solver = -1;
  for (const SlotSpec& sl : slots) {
    const int sv = sl.keep >= 0 ? P_[sl.keep].solver : sl.in.P.solver;
    if (solver < 0) solver = sv;
    if (sv != solver) {
      dv_set_error_text("the scenes of one batch must use the same solver");
      return DV_ERR_UNSUPPORTED;
    }
  }
  if (d.nseg > 0) TRY(sync_words());

  // ---- host layout of the new segment list
  std::vector<SegParams> hs2(nseg2);
  std::vector<dv_params> P2(nseg2);
  std::vector<double> t2(nseg2, 0.0);
  std::vector<int> ti2(nseg2, 0);
  std::vector<int> bseg2, small2, large2, map2, gsize2(nseg2), wsrc(nseg2, -1), wdst(nseg2);
  std::vector<double4> sp4, sv4, sf4, sg4;
  std::vector<double> sminv;
  std::vector<int> sfam;
  size_t ccap2 = 0, wtotal2 = 0;
  long long cell_total = 0;
  int max_chunks = 1, nb2 = 0;
  for (int s2 = 0; s2 < nseg2; ++s2) {
    const SlotSpec& sl = slots[s2];
    SegParams G;
    int n;
    if (sl.keep >= 0) {
      const SegParams& O = hseg_[sl.keep];
      G = O;
      n = O.b1 - O.b0;
      G.b0 = nb2;
      G.b1 = nb2 + n;
      G.s0 = (int)small2.size();
      for (int k = O.s0; k < O.s1; ++k) small2.push_back(small_h_[k] - O.b0 + nb2);
      G.s1 = (int)small2.size();
      G.l0 = (int)large2.size();
      for (int k = O.l0; k < O.l1; ++k) large2.push_back(large_h_[k] - O.b0 + nb2);
      G.l1 = (int)large2.size();
      for (int i = 0; i < n; ++i) map2.push_back(O.b0 + i);
      gsize2[s2] = h_sst_[sl.keep].gsize;
      wsrc[s2] = O.wbase;
      P2[s2] = P_[sl.keep];
      t2[s2] = time_[sl.keep];
      ti2[s2] = time_index_[sl.keep];
    } else {
      const SceneInput& sc = sl.in;
      const dv_params& P = sc.P;
      n = sc.nb;
      P2[s2] = P;
      G = SegParams{};
      G.h = P.h;
      G.mu = P.mu;
      G.tol = P.tolerance;
      G.env = P.envelope;
      G.max_iter = P.max_iterations;
      G.max_bt = P.max_backtracks;
      G.warm = P.warm_start;
      G.exact = P.fp64_narrowphase;
      G.ar = P.anti_relaxation;
      G.refine = P.refine_iterations;
      G.active = 1;
      G.b0 = nb2;
      G.b1 = nb2 + n;
      // spheres up to 4x the median radius go in the grid; larger spheres and
      // boxes are tested against every body of the segment
      std::vector<double> radii;
      for (int i = 0; i < n; ++i)
        if (sc.bodies[i].geom[1] == 0) radii.push_back(sc.bodies[i].geom[0]);
      double rlimit = 0;
      if (!radii.empty()) {
        std::nth_element(radii.begin(), radii.begin() + radii.size() / 2, radii.end());
        rlimit = 4.0 * radii[radii.size() / 2];
      }
      double rmax = 0;
      G.s0 = (int)small2.size();
      G.l0 = (int)large2.size();
      for (int i = 0; i < n; ++i) {
        const dv_body_desc& b = sc.bodies[i];
        if (b.geom[1] == 0 && b.geom[0] <= rlimit) {
          small2.push_back(nb2 + i);
          rmax = std::max(rmax, b.geom[0]);
        } else {
          large2.push_back(nb2 + i);
        }
        map2.push_back(-(int)sp4.size() - 1);
        sp4.push_back(make_double4(b.pos[0], b.pos[1], b.pos[2], 0.0));
        sv4.push_back(make_double4(b.vel[0], b.vel[1], b.vel[2], 0.0));
        // System.cu:368-376, 409-417: f = m g and Minv = 1/m, both 0 for fixed bodies
        if (b.fixed) {
          sf4.push_back(make_double4(0.0, 0.0, 0.0, 0.0));
          sminv.push_back(0.0);
        } else {
          sf4.push_back(make_double4(b.mass * P.gravity[0], b.mass * P.gravity[1],
                                     b.mass * P.gravity[2], 0.0));
          sminv.push_back(1.0 / b.mass);
        }
        sg4.push_back(make_double4(b.geom[0], b.geom[1], b.geom[2], b.geom[1] != 0 ? 1.0 : 0.0));
        sfam.push_back(b.family);
      }
      G.s1 = (int)small2.size();
      G.l1 = (int)large2.size();
      G.W = 2.0 * (rmax + P.envelope);
      G.cell_cap = std::max(64, 4 * (G.s1 - G.s0));
      // warm-start region: System.cu:185, gamma_d starts as 3 nb zeros
      G.wcap = (std::max(1024, 6 * n) + 31) / 32 * 32;
      gsize2[s2] = n;
    }
    for (int i = 0; i < n; ++i) bseg2.push_back(s2);
    G.cell_base = (int)cell_total;
    cell_total += G.cell_cap;
    G.wbase = (int)wtotal2;
    wdst[s2] = G.wbase;
    wtotal2 += (size_t)G.wcap;
    size_t c = (size_t)std::max(4 * n, 256);
    ccap2 += (c + kContactAlign - 1) / kContactAlign * kContactAlign;
    max_chunks = std::max(max_chunks, (n + kThreads - 1) / kThreads);
    nb2 += n;
    hs2[s2] = G;
  }
  if (nb2 == 0) return DV_ERR_ARG;
  if ((long long)wtotal2 > 0x7fffffffLL || ccap2 > 0x3fffffffULL || cell_total > 0x7ffffff0LL)
    return DV_ERR_ARG;
  const int n_small2 = (int)small2.size(), n_large2 = (int)large2.size();
  if (n_large2 > 65535) {
    dv_set_error_text("more than 65535 boxes / large spheres in one engine");
    return DV_ERR_ARG;
  }
  drop_graph();
  recs_.clear();

  // ---- carried arrays: gather into fresh buffers
  cudaStream_t st = st_;
  const size_t nbz = (size_t)nb2;
  double4 *np4 = nullptr, *nv4 = nullptr, *nf4 = nullptr, *ng4 = nullptr;
  double* nminv = nullptr;
  int* nfam = nullptr;
  TRY(dalloc(&np4, nbz));
  TRY(dalloc(&nv4, nbz));
  TRY(dalloc(&nf4, nbz));
  TRY(dalloc(&ng4, nbz));
  TRY(dalloc(&nminv, nbz));
  TRY(dalloc(&nfam, nbz));
  int *nws = nullptr, *nwc = nullptr;
  TRY(dalloc(&nws, nbz));
  TRY(dalloc(&nwc, nbz));
  {
    const size_t ns = std::max<size_t>(sp4.size(), 1);
    double4 *tp = nullptr, *tv = nullptr, *tf = nullptr, *tg = nullptr;
    double* tm = nullptr;
    int *tfam = nullptr, *tmap = nullptr;
    TRY(dalloc(&tp, ns));
    TRY(dalloc(&tv, ns));
    TRY(dalloc(&tf, ns));
    TRY(dalloc(&tg, ns));
    TRY(dalloc(&tm, ns));
    TRY(dalloc(&tfam, ns));
    TRY(dalloc(&tmap, nbz));
    const size_t k = sp4.size();
    if (k) {
      DV_CUDA_TRY(cudaMemcpyAsync(tp, sp4.data(), sizeof(double4) * k, cudaMemcpyHostToDevice, st));
      DV_CUDA_TRY(cudaMemcpyAsync(tv, sv4.data(), sizeof(double4) * k, cudaMemcpyHostToDevice, st));
      DV_CUDA_TRY(cudaMemcpyAsync(tf, sf4.data(), sizeof(double4) * k, cudaMemcpyHostToDevice, st));
      DV_CUDA_TRY(cudaMemcpyAsync(tg, sg4.data(), sizeof(double4) * k, cudaMemcpyHostToDevice, st));
      DV_CUDA_TRY(cudaMemcpyAsync(tm, sminv.data(), sizeof(double) * k, cudaMemcpyHostToDevice, st));
      DV_CUDA_TRY(cudaMemcpyAsync(tfam, sfam.data(), sizeof(int) * k, cudaMemcpyHostToDevice, st));
    }
    DV_CUDA_TRY(cudaMemcpyAsync(tmap, map2.data(), sizeof(int) * nbz, cudaMemcpyHostToDevice, st));
    k_gather_bodies<<<(nb2 + kThreads - 1) / kThreads, kThreads, 0, st>>>(
        nb2, tmap, d.p4, d.v4, d.f4, d.geom4, d.minv, d.family, d.ws, d.wc, tp, tv, tf, tg, tm,
        tfam, np4, nv4, nf4, ng4, nminv, nfam, nws, nwc);
    ++launches_;
    DV_CUDA_TRY(cudaGetLastError());
    // warm-start arena
    double* ng = nullptr;
    uint32_t* nid = nullptr;
    TRY(dalloc(&ng, 3 * std::max<size_t>(wtotal2, 1)));
    TRY(dalloc(&nid, std::max<size_t>(wtotal2, 1)));
    DV_CUDA_TRY(cudaMemsetAsync(ng, 0, sizeof(double) * 3 * std::max<size_t>(wtotal2, 1), st));
    DV_CUDA_TRY(cudaMemsetAsync(nid, 0, sizeof(uint32_t) * std::max<size_t>(wtotal2, 1), st));
    bool any_keep = false;
    for (int s2 = 0; s2 < nseg2; ++s2) any_keep |= (wsrc[s2] >= 0 && gsize2[s2] > 0);
    if (any_keep) {
      int *tsrc = nullptr, *tdst = nullptr, *tn = nullptr;
      std::vector<int> nn(nseg2);
      int mx = 1;
      for (int s2 = 0; s2 < nseg2; ++s2) {
        nn[s2] = wsrc[s2] >= 0 ? std::min(gsize2[s2], hs2[s2].wcap) : 0;
        mx = std::max(mx, nn[s2]);
      }
      TRY(dalloc(&tsrc, nseg2));
      TRY(dalloc(&tdst, nseg2));
      TRY(dalloc(&tn, nseg2));
      DV_CUDA_TRY(cudaMemcpyAsync(tsrc, wsrc.data(), sizeof(int) * nseg2, cudaMemcpyHostToDevice, st));
      DV_CUDA_TRY(cudaMemcpyAsync(tdst, wdst.data(), sizeof(int) * nseg2, cudaMemcpyHostToDevice, st));
      DV_CUDA_TRY(cudaMemcpyAsync(tn, nn.data(), sizeof(int) * nseg2, cudaMemcpyHostToDevice, st));
      dim3 g(std::min((mx + kThreads - 1) / kThreads, 64), nseg2);
      k_gather_warm<<<g, kThreads, 0, st>>>(tsrc, tdst, tn, d.gamma, d.wtotal, d.wid, ng, wtotal2,
                                             nid);
      ++launches_;
      DV_CUDA_TRY(cudaGetLastError());
      DV_CUDA_TRY(cudaStreamSynchronize(st));
      dfree(tsrc);
      dfree(tdst);
      dfree(tn);
    }
    DV_CUDA_TRY(cudaStreamSynchronize(st));
    dfree(tp); dfree(tv); dfree(tf); dfree(tg); dfree(tm); dfree(tfam); dfree(tmap);
    dfree(d.p4); dfree(d.v4); dfree(d.f4); dfree(d.geom4); dfree(d.minv); dfree(d.family);
    dfree(d.gamma); dfree(d.wid); dfree(d.ws); dfree(d.wc);
    d.p4 = np4; d.v4 = nv4; d.f4 = nf4; d.geom4 = ng4; d.minv = nminv; d.family = nfam;
    d.gamma = ng;
    d.wid = nid;
    d.ws = nws;
    d.wc = nwc;
    d.wtotal = wtotal2;
  }

  // ---- per-body scratch, segment tables, collision and contact capacity
  if (nb2 > nb_cap_) {
    int cap = std::max(nb2, nb_cap_ + nb_cap_ / 4);
    dfree(d.k4); dfree(d.w4); dfree(d.fc4); dfree(d.amin); dfree(d.amax); dfree(d.cell);
    dfree(d.cnt_cont); dfree(d.cnt_cand); dfree(d.cbase); dfree(d.binc_start); dfree(d.inc_start);
    dfree(d.bseg);
    TRY(dalloc(&d.k4, cap));
    TRY(dalloc(&d.w4, cap));
    TRY(dalloc(&d.fc4, cap));
    TRY(dalloc(&d.amin, cap));
    TRY(dalloc(&d.amax, cap));
    TRY(dalloc(&d.cell, cap));
    TRY(dalloc(&d.cnt_cont, cap));
    TRY(dalloc(&d.cnt_cand, cap));
    TRY(dalloc(&d.cbase, (size_t)cap + 1));
    TRY(dalloc(&d.binc_start, (size_t)cap + 1));
    TRY(dalloc(&d.inc_start, (size_t)cap + 1));
    TRY(dalloc(&d.bseg, cap));
    nb_cap_ = cap;
  }
  // body ranges of the solve's work lists: at most one partial range per segment
  const size_t need_ab = (size_t)nb2 / kThreads + (size_t)nseg2 + 1;
  if (need_ab > d.act_bcap) {
    dfree(d.act_bodies);
    TRY(dalloc(&d.act_bodies, need_ab));
    d.act_bcap = need_ab;
  }
  DV_CUDA_TRY(cudaMemsetAsync(d.k4, 0, sizeof(double4) * nbz, st));
  DV_CUDA_TRY(cudaMemsetAsync(d.w4, 0, sizeof(double4) * nbz, st));
  DV_CUDA_TRY(cudaMemsetAsync(d.fc4, 0, sizeof(double4) * nbz, st));
  if (nseg2 > seg_cap_) {
    int cap = std::max(nseg2, seg_cap_ + seg_cap_ / 4);
    dfree(d.seg); dfree(d.sst); dfree(d.grid); dfree(d.seg_tstart); dfree(d.donemask);
    TRY(dalloc(&d.seg, cap));
    TRY(dalloc(&d.sst, cap));
    TRY(dalloc(&d.grid, cap));
    TRY(dalloc(&d.seg_tstart, (size_t)cap + 1));
    TRY(dalloc(&d.donemask, (size_t)(cap + 31) / 32));
    if (h_sst_) cudaFreeHost(h_sst_);
    h_sst_ = nullptr;
    if (cudaMallocHost(&h_sst_, sizeof(SegState) * cap) != cudaSuccess)
      return dv_record_cuda_error(cudaErrorMemoryAllocation, "cudaMallocHost", __FILE__, __LINE__);
    seg_cap_ = cap;
    ring_cap_ = 0;  // per-step staging is sized by the segment count
    if (h_ew_ring_) cudaFreeHost(h_ew_ring_);
    if (h_sst_ring_) cudaFreeHost(h_sst_ring_);
    h_ew_ring_ = nullptr;
    h_sst_ring_ = nullptr;
  }
  TRY(ensure(&d.small_ids, &small_cap_, std::max<size_t>(n_small2, 1)));
  TRY(ensure(&d.large_ids, &large_cap_, std::max<size_t>(n_large2, 1)));
  const int ncell2 = (int)cell_total + 1;  // + the parking cell
  if (ncell2 > ncell_alloc_) {
    int cap = std::max(ncell2, ncell_alloc_ + ncell_alloc_ / 4);
    dfree(d.cell_start);
    dfree(d.cell_end);
    TRY(dalloc(&d.cell_start, cap));
    TRY(dalloc(&d.cell_end, cap));
    DV_CUDA_TRY(cudaMemsetAsync(d.cell_end, 0, sizeof(int) * cap, st));
    ncell_alloc_ = cap;
  }
  const int large_chunks2 = max_chunks * std::max(n_large2, 1);
  if (large_chunks2 + 1 > chunk_cap_) {
    int cap = std::max(large_chunks2 + 1, chunk_cap_ + chunk_cap_ / 4);
    dfree(d.large_chunk);
    dfree(d.large_chunk_off);
    TRY(dalloc(&d.large_chunk, cap));
    TRY(dalloc(&d.large_chunk_off, cap));
    chunk_cap_ = cap;
  }
  size_t stmp = scan_tmp_size(std::max((size_t)nb_cap_ + 1, (size_t)chunk_cap_));
  if (stmp > d.scan_tmp_cap) {
    dfree(d.scan_tmp);
    TRY(dalloc(&d.scan_tmp, stmp));
    d.scan_tmp_cap = stmp;
  }

  // ---- engine dimensions, then the contact buffers (their tile count depends on nseg)
  d.nb = nb2;
  d.nseg = nseg2;
  d.solver = solver;
  d.n_small = n_small2;
  d.n_large = n_large2;
  d.max_seg_chunks = max_chunks;
  d.large_chunks = large_chunks2;
  d.ncell_cap = ncell2;
  if (ccap2 > d.ccap || (int)(d.ccap / kTileItems) + nseg2 + 1 > d.tcap || !d.ida)
    TRY(alloc_contacts(std::max(ccap2, d.ccap)));
  hseg_ = hs2;
  P_ = P2;
  time_ = t2;
  time_index_ = ti2;
  small_h_ = small2;
  large_h_ = large2;
  memset(h_sst_, 0, sizeof(SegState) * nseg2);
  for (int s2 = 0; s2 < nseg2; ++s2) h_sst_[s2].gsize = gsize2[s2];
  h_ew_->n_small = n_small2;
  DV_CUDA_TRY(cudaMemcpyAsync(&d.ew->n_small, &h_ew_->n_small, sizeof(int), cudaMemcpyHostToDevice, st));
  DV_CUDA_TRY(cudaMemcpyAsync(d.sst, h_sst_, sizeof(SegState) * nseg2, cudaMemcpyHostToDevice, st));
  DV_CUDA_TRY(cudaMemsetAsync(d.grid, 0, sizeof(GridInfo) * nseg2, st));
  DV_CUDA_TRY(cudaMemcpyAsync(d.bseg, bseg2.data(), sizeof(int) * nbz, cudaMemcpyHostToDevice, st));
  if (n_small2)
    DV_CUDA_TRY(cudaMemcpyAsync(d.small_ids, small2.data(), sizeof(int) * n_small2,
                                cudaMemcpyHostToDevice, st));
  if (n_large2)
    DV_CUDA_TRY(cudaMemcpyAsync(d.large_ids, large2.data(), sizeof(int) * n_large2,
                                cudaMemcpyHostToDevice, st));
  TRY(upload_segments());
  DV_CUDA_TRY(cudaStreamSynchronize(st));
  DV_CUDA_TRY(cudaGetLastError());
  if (!cfg_user_ && max_ctas_ > 0)
    cfg_.grid = std::max(1, std::min(max_ctas_, (d.nb + kThreads - 1) / kThreads));
  return DV_OK;
}

int Engine::max_ctas_for(int blocks_per_sm) const {
  if (blocks_per_sm == 3 && d.precision == DV_PREC_MIXED) return apgd_max_ctas(d.precision, 3);
  return max_ctas_;
}

void Engine::set_launch(int grid, int chunk, int contiguous, int blocks_per_sm) {
  const int bps = (blocks_per_sm == 3 && d.precision == DV_PREC_MIXED) ? 3 : 2;
  const int mx = max_ctas_for(bps);
  if (grid <= 0) {
    cfg_user_ = false;
    cfg_.grid = std::max(1, std::min(mx, (d.nb + kThreads - 1) / kThreads));
  } else {
    cfg_user_ = true;
    cfg_.grid = std::min(grid, mx);
  }
  cfg_.chunk = std::max(1, chunk);
  cfg_.contiguous = contiguous ? 1 : 0;
  cfg_.blocks_per_sm = bps;
  drop_graph();
}

int Engine::set_stream(cudaStream_t s) {
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  if (s) {
    if (own_stream_) cudaStreamDestroy(st_);
    own_stream_ = false;
    st_ = s;
  }
  return DV_OK;
}

int Engine::set_segment_params(int s, const dv_params& P) {
  if (s < 0 || s >= d.nseg) return DV_ERR_ARG;
  TRY(check_params(P));
  // bilateral rows: APGD only (the reference's PGJ and PGS size their vectors 3 nc)
  if (hseg_[s].nbil > 0 && P.solver != DV_SOLVER_APGD) return DV_ERR_UNSUPPORTED;
  // anti-relaxation: one-scene engines without bilateral rows (the reference's
  // anti-relaxation vector is indexed without the rows' offset, APGD.cu:104-112)
  if (P.anti_relaxation && (d.nseg != 1 || hseg_[s].nbil > 0)) return DV_ERR_UNSUPPORTED;
  if (P.anti_relaxation && !d.anti_relax) TRY(enable_anti_relax());
  if (!P.anti_relaxation && d.anti_relax) {
    d.anti_relax = 0;
    drop_graph();
  }
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  SegParams& G = hseg_[s];
  if (P.envelope > P_[s].envelope) {
    // the grid cell must stay wider than every sphere AABB
    G.W = G.W - 2.0 * P_[s].envelope + 2.0 * P.envelope;
  }
  G.h = P.h;
  G.mu = P.mu;
  G.tol = P.tolerance;
  G.env = P.envelope;
  G.max_iter = P.max_iterations;
  G.max_bt = P.max_backtracks;
  G.warm = P.warm_start;
  G.exact = P.fp64_narrowphase;
  G.ar = P.anti_relaxation;
  G.refine = P.refine_iterations;
  if (P.solver != P_[s].solver) {
    if (d.nseg != 1) return DV_ERR_UNSUPPORTED;
    d.solver = P.solver;
    drop_graph();
  }
  P_[s] = P;
  TRY(upload_segments());
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  return DV_OK;
}

int Engine::set_precision(int precision) {
  if (precision != DV_PREC_FP64 && precision != DV_PREC_MIXED) return DV_ERR_UNSUPPORTED;
  if (precision == d.precision) return DV_OK;
  if (d.nbil > 0 && precision != DV_PREC_FP64) return DV_ERR_UNSUPPORTED;  // rows: FP64 only
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  d.precision = precision;
  max_ctas_ = apgd_max_ctas(precision, 2);
  cfg_.blocks_per_sm = 2;
  if (cfg_.grid > max_ctas_) cfg_.grid = max_ctas_;
  drop_graph();
  return DV_OK;
}

int Engine::ensure_records(int n) {
  if (n <= ring_cap_) return DV_OK;
  int cap = std::max(n, 2 * ring_cap_);
  if (h_ew_ring_) cudaFreeHost(h_ew_ring_);
  if (h_sst_ring_) cudaFreeHost(h_sst_ring_);
  h_ew_ring_ = nullptr;
  h_sst_ring_ = nullptr;
  // sized by the segment capacity, not the current count: a later layout with
  // more segments that still fit the capacity keeps this ring
  if (cudaMallocHost(&h_ew_ring_, sizeof(EngineWords) * cap) != cudaSuccess ||
      cudaMallocHost(&h_sst_ring_, sizeof(SegState) * (size_t)cap * std::max(seg_cap_, d.nseg)) !=
          cudaSuccess)
    return dv_record_cuda_error(cudaErrorMemoryAllocation, "cudaMallocHost", __FILE__, __LINE__);
  while ((int)ev_.size() < 3 * cap) {
    cudaEvent_t e;
    DV_CUDA_TRY(cudaEventCreate(&e));
    ev_.push_back(e);
  }
  ring_cap_ = cap;
  return DV_OK;
}

void Engine::drop_graph() {
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  if (graph_) cudaGraphDestroy(graph_);
  graph_exec_ = nullptr;
  graph_ = nullptr;
}

int Engine::capture_graph() {
  drop_graph();
  int64_t dummy = 0;
  cudaError_t e = cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return DV_ERR_UNSUPPORTED;
  }
  collide(d, st_, &dummy);
  launch_step_solve(d, cfg_, st_, &dummy);
  e = cudaStreamEndCapture(st_, &graph_);
  if (e != cudaSuccess || !graph_) {
    cudaGetLastError();
    graph_ = nullptr;
    return DV_ERR_UNSUPPORTED;
  }
  e = cudaGraphInstantiate(&graph_exec_, graph_, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(graph_);
    graph_ = nullptr;
    graph_exec_ = nullptr;
    return DV_ERR_UNSUPPORTED;
  }
  graph_kernels_ = dummy;
  return DV_OK;
}

int Engine::set_graph(bool on) {
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  use_graph_ = false;
  graph_failed_ = false;
  drop_graph();
  if (!on) return DV_OK;
  int rc = capture_graph();
  if (rc != DV_OK) {
    graph_failed_ = true;
    dv_set_error_text("CUDA graph capture of the step failed");
    return rc;
  }
  use_graph_ = true;
  return DV_OK;
}

int Engine::enqueue_step(int i) {
  cudaStream_t st = st_;
  DV_CUDA_TRY(cudaEventRecord(ev_[3 * i], st));
  if (use_graph_) {
    if (!graph_exec_) TRY(capture_graph());
    DV_CUDA_TRY(cudaGraphLaunch(graph_exec_, st));
    launches_ += graph_kernels_;
    DV_CUDA_TRY(cudaEventRecord(ev_[3 * i + 1], st));
  } else {
    collide(d, st, &launches_);
    DV_CUDA_TRY(cudaEventRecord(ev_[3 * i + 1], st));
    launch_step_solve(d, cfg_, st, &launches_);
  }
  DV_CUDA_TRY(cudaGetLastError());
  DV_CUDA_TRY(cudaEventRecord(ev_[3 * i + 2], st));
  DV_CUDA_TRY(cudaMemcpyAsync(h_ew_ring_ + i, d.ew, sizeof(EngineWords), cudaMemcpyDeviceToHost, st));
  DV_CUDA_TRY(cudaMemcpyAsync(h_sst_ring_ + (size_t)i * d.nseg, d.sst, sizeof(SegState) * d.nseg,
                              cudaMemcpyDeviceToHost, st));
  return DV_OK;
}

int Engine::grow_warm(double factor, int min_seg_cap, int which) {
  // new regions: every segment keeps its capacity except `which` (or every
  // segment whose last contact count overflowed when which < 0)
  std::vector<SegParams> ns = hseg_;
  size_t total = 0;
  for (int s = 0; s < d.nseg; ++s) {
    int cap = hseg_[s].wcap;
    bool grow = (which == s) || (which < 0 && h_sst_[s].nc > cap);
    if (grow) cap = std::max((int)(cap * factor), min_seg_cap);
    cap = (cap + 31) / 32 * 32;
    ns[s].wbase = (int)total;
    ns[s].wcap = cap;
    total += (size_t)cap;
  }
  if ((long long)total > 0x7fffffffLL) return DV_ERR_OOM;
  double* g = nullptr;
  uint32_t* id = nullptr;
  TRY(dalloc(&g, 3 * total));
  TRY(dalloc(&id, total));
  DV_CUDA_TRY(cudaMemsetAsync(g, 0, sizeof(double) * 3 * total, st_));
  DV_CUDA_TRY(cudaMemsetAsync(id, 0, sizeof(uint32_t) * total, st_));
  for (int s = 0; s < d.nseg; ++s) {
    int n = std::min(h_sst_[s].gsize, hseg_[s].wcap);
    if (n <= 0) continue;
    for (int k = 0; k < 3; ++k)
      DV_CUDA_TRY(cudaMemcpyAsync(g + k * total + ns[s].wbase, d.gamma + k * d.wtotal + hseg_[s].wbase,
                                  sizeof(double) * n, cudaMemcpyDeviceToDevice, st_));
    DV_CUDA_TRY(cudaMemcpyAsync(id + ns[s].wbase, d.wid + hseg_[s].wbase, sizeof(uint32_t) * n,
                                cudaMemcpyDeviceToDevice, st_));
  }
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  dfree(d.gamma);
  dfree(d.wid);
  d.gamma = g;
  d.wid = id;
  d.wtotal = total;
  hseg_ = ns;
  TRY(upload_segments());
  drop_graph();
  return DV_OK;
}

int Engine::sync_words() {
  DV_CUDA_TRY(cudaMemcpyAsync(h_ew_, d.ew, sizeof(EngineWords), cudaMemcpyDeviceToHost, st_));
  DV_CUDA_TRY(cudaMemcpyAsync(h_sst_, d.sst, sizeof(SegState) * d.nseg, cudaMemcpyDeviceToHost, st_));
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  return DV_OK;
}

int Engine::sync_state() { return sync_words(); }

int Engine::step(int n) {
  recs_.clear();
  if (n <= 0) return DV_OK;
  int done = 0;
  int retries = 0;
  while (done < n) {
    const int m = n - done;
    TRY(ensure_records(m));
    DV_CUDA_TRY(cudaMemsetAsync(&d.ew->err, 0, sizeof(unsigned), st_));
    // the bilateral rows' clock: System::time of every segment at the first
    // step (the solve kernel advances it by h per step)
    if (d.nbil)
      DV_CUDA_TRY(cudaMemcpyAsync(d.seg_time, time_.data(), sizeof(double) * d.nseg,
                                  cudaMemcpyHostToDevice, st_));
    for (int i = 0; i < m; ++i) TRY(enqueue_step(i));
    DV_CUDA_TRY(cudaStreamSynchronize(st_));
    DV_CUDA_TRY(cudaGetLastError());
    int failed = -1;
    for (int i = 0; i < m; ++i) {
      const EngineWords& w = h_ew_ring_[i];
      const SegState* ss = h_sst_ring_ + (size_t)i * d.nseg;
      // a step counts when its solve reached the update (steps_done advanced)
      // or, for engine-level errors, not at all
      unsigned hard = w.err & (kErrCapacity | kErrPartners | kErrBarrierTimeout | kErrCopyTimeout);
      if (hard) {
        failed = i;
        memcpy(h_ew_, &w, sizeof(EngineWords));
        memcpy(h_sst_, ss, sizeof(SegState) * d.nseg);
        break;
      }
      StepRecord r;
      r.ew = w;
      r.sst.assign(ss, ss + d.nseg);
      cudaEventElapsedTime(&r.ms_total, ev_[3 * i], ev_[3 * i + 2]);
      if (!use_graph_) {
        cudaEventElapsedTime(&r.ms_collide, ev_[3 * i], ev_[3 * i + 1]);
        cudaEventElapsedTime(&r.ms_solve, ev_[3 * i + 1], ev_[3 * i + 2]);
      } else {
        r.ms_solve = r.ms_total;
      }
      for (int s = 0; s < d.nseg; ++s) {
        if (!hseg_[s].active) continue;
        time_[s] += P_[s].h;
        time_index_[s] += 1;
      }
      r.time = time_[0];
      r.time_index = time_index_[0];
      recs_.push_back(std::move(r));
      memcpy(h_ew_, &w, sizeof(EngineWords));
      memcpy(h_sst_, ss, sizeof(SegState) * d.nseg);
      // a solver error of a plain scene ends the call (System semantics)
      if (stop_on_segment_error_) {
        for (int s = 0; s < d.nseg; ++s)
          if (status_from_bits(ss[s].err) != DV_OK) return status_from_bits(ss[s].err);
      }
    }
    if (failed < 0) {
      done += m;
      continue;
    }
    done += failed;
    const EngineWords& w = *h_ew_;
    if (w.err & kErrPartners) {
      dv_set_error_text(kPartnerLimitText);
      return DV_ERR_ARG;
    }
    if (w.err & (kErrBarrierTimeout | kErrCopyTimeout)) {
      dv_set_error_text("a bounded wait of the solve kernel expired");
      return DV_ERR_TIMEOUT;
    }
    // capacity: contact slots / tiles, or a segment's warm-start region
    if (++retries > 16) return DV_ERR_OOM;
    bool warm_over = false;
    for (int s = 0; s < d.nseg; ++s)
      if (hseg_[s].active && h_sst_[s].nc > hseg_[s].wcap) warm_over = true;
    if (warm_over) TRY(grow_warm(1.5, 0, -1));
    if ((size_t)w.nc_pad > d.ccap || w.ntiles > d.tcap || !warm_over) {
      size_t need = std::max((size_t)w.nc_pad + (size_t)w.nc_pad / 4, d.ccap + d.ccap / 2);
      DV_CUDA_TRY(cudaStreamSynchronize(st_));
      TRY(alloc_contacts(need));
      drop_graph();
    }
  }
  return DV_OK;
}

int Engine::collide_only() {
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  for (int attempt = 0; attempt < 16; ++attempt) {
    DV_CUDA_TRY(cudaMemsetAsync(&d.ew->err, 0, sizeof(unsigned), st_));
    collide(d, st_, &launches_);
    DV_CUDA_TRY(cudaGetLastError());
    TRY(sync_words());
    const EngineWords& w = *h_ew_;
    if (w.err & kErrPartners) {
      dv_set_error_text(kPartnerLimitText);
      return DV_ERR_ARG;
    }
    if (!(w.err & kErrCapacity)) return DV_OK;
    if ((size_t)w.nc_pad > d.ccap || w.ntiles > d.tcap) {
      TRY(alloc_contacts(std::max((size_t)w.nc_pad + (size_t)w.nc_pad / 4, d.ccap + d.ccap / 2)));
      drop_graph();
    } else {
      TRY(grow_warm(1.5, 0, -1));
    }
  }
  return DV_ERR_OOM;
}

// Turns the anti-relaxation kernel on, with its buffers for the current
// contact capacity (alloc_contacts keeps them sized while it is on).
int Engine::enable_anti_relax() {
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  d.anti_relax = 1;
  dfree(d.ar_r0);
  dfree(d.ar_v);
  TRY(dalloc(&d.ar_r0, 2 * d.ccap));
  TRY(dalloc(&d.ar_v, 2 * d.ccap));
  if (d.v_ar_cap < (size_t)d.nb) {
    dfree(d.v_ar);
    TRY(dalloc(&d.v_ar, (size_t)d.nb));
    d.v_ar_cap = d.nb;
  }
  drop_graph();
  return DV_OK;
}

int Engine::add_bilateral(int s, int dof_a, int dof_b, double velocity, double start_time) {
  if (s < 0 || s >= d.nseg) return DV_ERR_ARG;
  if (d.nseg != 1) return DV_ERR_UNSUPPORTED;
  const int nbs = hseg_[s].b1 - hseg_[s].b0;
  if (dof_a < 0 || dof_a >= 3 * nbs || dof_b >= 3 * nbs) {
    dv_set_error_text("bilateral DOF index out of range");
    return DV_ERR_ARG;
  }
  if (time_index_[s] > 0) {
    // System::processConstraints copies the rows to the device once, at
    // initializeSystem (System.cu:292-296, 303-315)
    dv_set_error_text("bilateral constraints are added before the first step");
    return DV_ERR_ARG;
  }
  if (P_[s].solver != DV_SOLVER_APGD || d.precision != DV_PREC_FP64 || P_[s].anti_relaxation)
    return DV_ERR_UNSUPPORTED;
  if (dof_b < 0) dof_b = -1;
  double p0 = 0.0;
  if (dof_b < 0) {
    // the DOF's position now (infoConstraintBilateralDOF.z, System.cu:310)
    double p[3];
    TRY(copy_state_out(hseg_[s].b0 + dof_a / 3, 1, p, nullptr));
    p0 = p[dof_a % 3];
  }
  bil_a_.push_back(3 * hseg_[s].b0 + dof_a);
  bil_b_.push_back(dof_b < 0 ? -1 : 3 * hseg_[s].b0 + dof_b);
  bil_vel_.push_back(velocity);
  bil_t0_.push_back(start_time);
  bil_p0_.push_back(p0);
  return upload_bilateral();
}

int Engine::upload_bilateral() {
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  const int n = (int)bil_a_.size();
  const int nb = d.nb;
  std::vector<int2> off(n);
  std::vector<double4> info(n);
  std::vector<std::vector<uint32_t>> per(nb);
  for (int i = 0; i < n; ++i) {
    const int a = bil_a_[i], b = bil_b_[i];
    off[i] = make_int2(4 * (a / 3) + a % 3, b >= 0 ? 4 * (b / 3) + b % 3 : -1);
    info[i] = make_double4(bil_vel_[i], bil_t0_[i], bil_p0_[i], 0.0);
    per[a / 3].push_back(((uint32_t)i << 3) | ((uint32_t)(a % 3) << 1));
    if (b >= 0) per[b / 3].push_back(((uint32_t)i << 3) | ((uint32_t)(b % 3) << 1) | 1u);
  }
  std::vector<int> start(nb + 1, 0);
  std::vector<uint32_t> inc;
  for (int b = 0; b < nb; ++b) {
    start[b] = (int)inc.size();
    inc.insert(inc.end(), per[b].begin(), per[b].end());
  }
  start[nb] = (int)inc.size();
  dfree(d.bil_off); dfree(d.bil_info); dfree(d.bil_inc_start); dfree(d.bil_inc);
  dfree(d.bil_work); dfree(d.bil_gam); dfree(d.bil_b);
  TRY(dalloc(&d.bil_off, n));
  TRY(dalloc(&d.bil_info, n));
  TRY(dalloc(&d.bil_inc_start, (size_t)nb + 1));
  TRY(dalloc(&d.bil_inc, inc.size()));
  TRY(dalloc(&d.bil_work, 12 * (size_t)n));
  TRY(dalloc(&d.bil_gam, n));
  TRY(dalloc(&d.bil_b, n));
  if (!d.seg_time) TRY(dalloc(&d.seg_time, (size_t)d.nseg));
  DV_CUDA_TRY(cudaMemcpyAsync(d.bil_off, off.data(), sizeof(int2) * n, cudaMemcpyHostToDevice, st_));
  DV_CUDA_TRY(cudaMemcpyAsync(d.bil_info, info.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, st_));
  DV_CUDA_TRY(cudaMemcpyAsync(d.bil_inc_start, start.data(), sizeof(int) * (nb + 1),
                              cudaMemcpyHostToDevice, st_));
  if (!inc.empty())
    DV_CUDA_TRY(cudaMemcpyAsync(d.bil_inc, inc.data(), sizeof(uint32_t) * inc.size(),
                                cudaMemcpyHostToDevice, st_));
  // System::gamma_d starts as zeros (System.cu:185); b is set by the first step
  DV_CUDA_TRY(cudaMemsetAsync(d.bil_gam, 0, sizeof(double) * n, st_));
  DV_CUDA_TRY(cudaMemsetAsync(d.bil_b, 0, sizeof(double) * n, st_));
  DV_CUDA_TRY(cudaMemsetAsync(d.bil_work, 0, sizeof(double) * 12 * n, st_));
  d.nbil = n;
  hseg_[0].bil0 = 0;
  hseg_[0].nbil = n;
  TRY(upload_segments());
  if ((int)(d.ccap / kTileItems) + d.nseg + 1 + (n + kTileItems - 1) / kTileItems > d.tcap)
    TRY(alloc_contacts(d.ccap));
  drop_graph();
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  return DV_OK;
}

int Engine::get_bilateral_gamma(int s, std::vector<double>& g) {
  const int n = hseg_[s].nbil;
  g.assign(n, 0.0);
  if (n == 0) return DV_OK;
  return download(g.data(), d.bil_gam + hseg_[s].bil0, sizeof(double) * n);
}

int Engine::solve_only() {
  // the reference's anti-relaxation leaves its own velocities in System::v
  if (d.anti_relax) return DV_ERR_UNSUPPORTED;
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  DV_CUDA_TRY(cudaMemsetAsync(&d.ew->err, 0, sizeof(unsigned), st_));
  if (d.nbil)
    DV_CUDA_TRY(cudaMemcpyAsync(d.seg_time, time_.data(), sizeof(double) * d.nseg,
                                cudaMemcpyHostToDevice, st_));
  launch_step_solve(d, cfg_, st_, &launches_, true);
  DV_CUDA_TRY(cudaGetLastError());
  TRY(sync_words());
  const EngineWords& w = *h_ew_;
  if (w.err & (kErrBarrierTimeout | kErrCopyTimeout)) {
    dv_set_error_text("a bounded wait of the solve kernel expired");
    return DV_ERR_TIMEOUT;
  }
  if (w.err & kErrCapacity) return DV_ERR_OOM;
  return DV_OK;
}

int Engine::get_gamma(int s, std::vector<double>& g, int* n) {
  TRY(sync_words());
  int m = h_sst_[s].gsize;
  if (n) *n = m;
  g.assign(3 * (size_t)m, 0.0);
  std::vector<double> planes;
  TRY(download_planes(d.gamma, d.wtotal, 3, hseg_[s].wbase, std::min(m, hseg_[s].wcap), planes));
  int mm = std::min(m, hseg_[s].wcap);
  for (int i = 0; i < mm; ++i)
    for (int k = 0; k < 3; ++k) g[3 * (size_t)i + k] = planes[k * (size_t)mm + i];
  return DV_OK;
}

int Engine::set_gamma(int s, const double* g, int n) {
  TRY(sync_words());
  if (n > hseg_[s].wcap) TRY(grow_warm(1.0, n, s));
  std::vector<double> h(3 * (size_t)std::max(n, 1));
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) h[k * (size_t)n + i] = g[3 * (size_t)i + k];
  for (int k = 0; k < 3; ++k)
    if (n > 0)
      DV_CUDA_TRY(cudaMemcpyAsync(d.gamma + k * d.wtotal + hseg_[s].wbase, h.data() + k * (size_t)n,
                                  sizeof(double) * n, cudaMemcpyHostToDevice, st_));
  DV_CUDA_TRY(cudaMemcpyAsync(&d.sst[s].gsize, &n, sizeof(int), cudaMemcpyHostToDevice, st_));
  // a positional warm start carries no pairs: the matched lookup finds none
  DV_CUDA_TRY(cudaMemsetAsync(d.wc + hseg_[s].b0, 0, sizeof(int) * (hseg_[s].b1 - hseg_[s].b0), st_));
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  h_sst_[s].gsize = n;
  return DV_OK;
}

int Engine::set_stop_on_segment_error(bool on) {
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  stop_on_segment_error_ = on;
  int v = on ? 1 : 0;
  h_ew_->stop_on_seg_err = v;
  DV_CUDA_TRY(cudaMemcpyAsync(&d.ew->stop_on_seg_err, &v, sizeof(int), cudaMemcpyHostToDevice, st_));
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  return DV_OK;
}

namespace {
__global__ void __launch_bounds__(kThreads) k_pack3(const double4* __restrict__ src, int n,
                                                   double* __restrict__ dst) {
  int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  double4 x = src[i];
  dst[3 * i] = x.x;
  dst[3 * i + 1] = x.y;
  dst[3 * i + 2] = x.z;
}
__global__ void __launch_bounds__(kThreads) k_unpack3(const double* __restrict__ src, int n,
                                                     double4* __restrict__ dst) {
  int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= n) return;
  dst[i] = make_double4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.0);
}
}  // namespace

int Engine::copy_state_out(int b0, int n, double* p, double* v) {
  if (n <= 0) return DV_OK;
  if (b0 < 0 || b0 + n > d.nb) return DV_ERR_ARG;
  const size_t need = 3 * (size_t)n * ((p && v) ? 2 : 1);
  if (need > stage3_cap_) {
    dfree(stage3_);
    TRY(dalloc(&stage3_, need));
    stage3_cap_ = need;
  }
  const int g = (n + kThreads - 1) / kThreads;
  double* sp = stage3_;
  double* sv = stage3_ + ((p && v) ? 3 * (size_t)n : 0);
  if (p) k_pack3<<<g, kThreads, 0, st_>>>(d.p4 + b0, n, sp);
  if (v) k_pack3<<<g, kThreads, 0, st_>>>(d.v4 + b0, n, sv);
  if (p) DV_CUDA_TRY(cudaMemcpyAsync(p, sp, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, st_));
  if (v) DV_CUDA_TRY(cudaMemcpyAsync(v, sv, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, st_));
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  DV_CUDA_TRY(cudaGetLastError());
  return DV_OK;
}

int Engine::copy_state_in(int b0, int n, const double* p, const double* v) {
  if (n <= 0) return DV_OK;
  if (b0 < 0 || b0 + n > d.nb) return DV_ERR_ARG;
  const size_t need = 3 * (size_t)n * ((p && v) ? 2 : 1);
  if (need > stage3_cap_) {
    dfree(stage3_);
    TRY(dalloc(&stage3_, need));
    stage3_cap_ = need;
  }
  const int g = (n + kThreads - 1) / kThreads;
  double* sp = stage3_;
  double* sv = stage3_ + ((p && v) ? 3 * (size_t)n : 0);
  if (p) DV_CUDA_TRY(cudaMemcpyAsync(sp, p, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st_));
  if (v) DV_CUDA_TRY(cudaMemcpyAsync(sv, v, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st_));
  if (p) k_unpack3<<<g, kThreads, 0, st_>>>(sp, n, d.p4 + b0);
  if (v) k_unpack3<<<g, kThreads, 0, st_>>>(sv, n, d.v4 + b0);
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  DV_CUDA_TRY(cudaGetLastError());
  return DV_OK;
}

int Engine::snapshot() {
  TRY(sync_words());
  if (!snap_p_ || snap_nb_ != d.nb) {
    dfree(snap_p_);
    dfree(snap_v_);
    dfree(snap_ws_);
    dfree(snap_wc_);
    TRY(dalloc(&snap_p_, (size_t)d.nb));
    TRY(dalloc(&snap_v_, (size_t)d.nb));
    TRY(dalloc(&snap_ws_, (size_t)d.nb));
    TRY(dalloc(&snap_wc_, (size_t)d.nb));
    snap_nb_ = d.nb;
  }
  if (snap_wtotal_ != d.wtotal) {
    dfree(snap_g_);
    dfree(snap_id_);
    TRY(dalloc(&snap_g_, 3 * d.wtotal));
    TRY(dalloc(&snap_id_, d.wtotal));
    snap_wtotal_ = d.wtotal;
  }
  DV_CUDA_TRY(cudaMemcpyAsync(snap_p_, d.p4, sizeof(double4) * d.nb, cudaMemcpyDeviceToDevice, st_));
  DV_CUDA_TRY(cudaMemcpyAsync(snap_v_, d.v4, sizeof(double4) * d.nb, cudaMemcpyDeviceToDevice, st_));
  DV_CUDA_TRY(cudaMemcpyAsync(snap_g_, d.gamma, sizeof(double) * 3 * d.wtotal,
                              cudaMemcpyDeviceToDevice, st_));
  DV_CUDA_TRY(cudaMemcpyAsync(snap_id_, d.wid, sizeof(uint32_t) * d.wtotal, cudaMemcpyDeviceToDevice,
                              st_));
  DV_CUDA_TRY(cudaMemcpyAsync(snap_ws_, d.ws, sizeof(int) * d.nb, cudaMemcpyDeviceToDevice, st_));
  DV_CUDA_TRY(cudaMemcpyAsync(snap_wc_, d.wc, sizeof(int) * d.nb, cudaMemcpyDeviceToDevice, st_));
  snap_gsize_.resize(d.nseg);
  for (int s = 0; s < d.nseg; ++s) snap_gsize_[s] = h_sst_[s].gsize;
  snap_time_ = time_;
  snap_time_index_ = time_index_;
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  return DV_OK;
}

int Engine::restore() {
  if (!snap_p_ || snap_wtotal_ != d.wtotal || snap_nb_ != d.nb) return DV_ERR_ARG;
  DV_CUDA_TRY(cudaMemcpyAsync(d.p4, snap_p_, sizeof(double4) * d.nb, cudaMemcpyDeviceToDevice, st_));
  DV_CUDA_TRY(cudaMemcpyAsync(d.v4, snap_v_, sizeof(double4) * d.nb, cudaMemcpyDeviceToDevice, st_));
  DV_CUDA_TRY(cudaMemcpyAsync(d.gamma, snap_g_, sizeof(double) * 3 * d.wtotal,
                              cudaMemcpyDeviceToDevice, st_));
  DV_CUDA_TRY(cudaMemcpyAsync(d.wid, snap_id_, sizeof(uint32_t) * d.wtotal, cudaMemcpyDeviceToDevice,
                              st_));
  DV_CUDA_TRY(cudaMemcpyAsync(d.ws, snap_ws_, sizeof(int) * d.nb, cudaMemcpyDeviceToDevice, st_));
  DV_CUDA_TRY(cudaMemcpyAsync(d.wc, snap_wc_, sizeof(int) * d.nb, cudaMemcpyDeviceToDevice, st_));
  DV_CUDA_TRY(cudaMemcpy2DAsync(&d.sst[0].gsize, sizeof(SegState), snap_gsize_.data(), sizeof(int),
                                sizeof(int), d.nseg, cudaMemcpyHostToDevice, st_));
  time_ = snap_time_;
  time_index_ = snap_time_index_;
  TRY(sync_words());
  return DV_OK;
}

int Engine::state_hash(uint64_t* h) {
  std::vector<double4> p(d.nb), v(d.nb);
  TRY(download(p.data(), d.p4, sizeof(double4) * d.nb));
  TRY(download(v.data(), d.v4, sizeof(double4) * d.nb));
  uint64_t x = 1469598103934665603ull;
  auto mix = [&](const void* data, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < n; ++i) {
      x ^= c[i];
      x *= 1099511628211ull;
    }
  };
  for (int i = 0; i < d.nb; ++i) {
    mix(&p[i], 3 * sizeof(double));
    mix(&v[i], 3 * sizeof(double));
  }
  *h = x;
  return DV_OK;
}

void Engine::clear_phase_times() {
  cudaStreamSynchronize(st_);
  cudaMemsetAsync(d.ew->phase_ns, 0, sizeof(d.ew->phase_ns) + sizeof(d.ew->phase_count), st_);
  cudaStreamSynchronize(st_);
  memset(h_ew_->phase_ns, 0, sizeof(h_ew_->phase_ns));
  memset(h_ew_->phase_count, 0, sizeof(h_ew_->phase_count));
}

int Engine::download(void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return DV_OK;
  DV_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st_));
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  return DV_OK;
}

int Engine::download_planes(const double* dev, size_t stride, int k, int first, int n,
                            std::vector<double>& out) {
  out.assign((size_t)k * std::max(n, 0), 0.0);
  if (n <= 0) return DV_OK;
  for (int c = 0; c < k; ++c)
    DV_CUDA_TRY(cudaMemcpyAsync(out.data() + (size_t)c * n, dev + c * stride + first,
                                sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, st_));
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  return DV_OK;
}

int Engine::download_planes_f(const float* dev, size_t stride, int k, int first, int n,
                              std::vector<double>& out) {
  std::vector<float> tmp((size_t)k * std::max(n, 0));
  out.assign((size_t)k * std::max(n, 0), 0.0);
  if (n <= 0) return DV_OK;
  for (int c = 0; c < k; ++c)
    DV_CUDA_TRY(cudaMemcpyAsync(tmp.data() + (size_t)c * n, dev + c * stride + first,
                                sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, st_));
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  for (size_t i = 0; i < tmp.size(); ++i) out[i] = tmp[i];
  return DV_OK;
}

}  // namespace dv
