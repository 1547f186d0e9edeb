// dv_scene.cu -- the C ABI of include/dvide.h: scene lifetime, the time step
// orchestration (System::DoTimeStep, System.cu:544-602) and the diagnostics
// of System.cu:1259-1295, 1590-1658.
//
// One step on the scene's stream:
//   collide_count   AABBs, grid, radix sort, candidate/contact counts, scan
//   (host waits for the contact count: the only synchronisation of a step)
//   collide_write   sorted contacts + frames, B-side incidence
//   k_step_solve    one cooperative persistent kernel: k, r, APGD, update
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "dv_internal.cuh"

using namespace dv;

static thread_local std::string g_last_error;

int dv_record_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s failed at %s:%d: %s", what, file, line, cudaGetErrorString(e));
  g_last_error = buf;
  if (e == cudaErrorMemoryAllocation) return DV_ERR_OOM;
  return DV_ERR_CUDA;
}

void dv_set_error_text(const char* text) { g_last_error = text; }

struct dv_scene {
  SceneDev d;
  dv_params P;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaEvent_t ev_count = nullptr;
  // per-step timing events, double-buffered: step k uses set k & 1 so the
  // previous step's events survive until its report is folded in
  cudaEvent_t ev_t0[2] = {nullptr, nullptr}, ev_t1[2] = {nullptr, nullptr};
  cudaEvent_t ev_c[2] = {nullptr, nullptr}, ev_s[2] = {nullptr, nullptr};
  int ev_cur = 0;
  int64_t launches = 0;
  int max_ctas = 1;
  double time = 0;
  int time_index = 0;
  dv_step_stats last;
  bool solve_pending = false;
  bool step_open = false;
  std::vector<dv_step_stats> history;
  double phase_ns[8] = {0};       // accumulated since the last dv_get_phase_times reset
  long long phase_count[8] = {0};
  unsigned* h_bar = nullptr;
  double* h_red = nullptr;     // pinned results of diagnostic reductions
  double* d_red = nullptr;     // device partials for diagnostics
  size_t d_red_cap = 0;
  std::vector<void*> allocs;
};

namespace {

template <class T>
int dalloc(dv_scene* s, T** p, size_t n) {
  if (n == 0) n = 1;
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    return dv_record_cuda_error(e, "cudaMalloc", __FILE__, __LINE__);
  }
  s->allocs.push_back(q);
  *p = reinterpret_cast<T*>(q);
  return DV_OK;
}

template <class T>
void dfree(dv_scene* s, T*& p) {
  if (!p) return;
  cudaFree(p);
  auto it = std::find(s->allocs.begin(), s->allocs.end(), (void*)p);
  if (it != s->allocs.end()) s->allocs.erase(it);
  p = nullptr;
}

#define TRY(x)                  \
  do {                          \
    int rc_ = (x);              \
    if (rc_ != DV_OK) return rc_; \
  } while (0)

int alloc_contacts(dv_scene* s, size_t cap) {
  SceneDev& d = s->d;
  // planes start on 2 KiB boundaries: the solve kernel copies 256-contact
  // plane segments with bulk asynchronous copies (16-byte alignment rule)
  cap = (cap + 255) / 256 * 256;
  dfree(s, d.ida); dfree(s, d.idb); dfree(s, d.F); dfree(s, d.gap); dfree(s, d.loc);
  dfree(s, d.r);
  for (int k = 0; k < 5; ++k) {
    dfree(s, d.G[k]);
    dfree(s, d.NG[k]);
  }
  dfree(s, d.q); dfree(s, d.binc); dfree(s, d.inc); dfree(s, d.part);
  d.ccap = cap;
  TRY(dalloc(s, &d.ida, cap));
  TRY(dalloc(s, &d.idb, cap));
  TRY(dalloc(s, &d.F, 9 * cap));
  TRY(dalloc(s, &d.gap, cap));
  TRY(dalloc(s, &d.loc, 3 * cap));
  TRY(dalloc(s, &d.r, 3 * cap));
  for (int k = 0; k < 5; ++k) {
    TRY(dalloc(s, &d.G[k], 3 * cap));
    TRY(dalloc(s, &d.NG[k], 3 * cap));
  }
  TRY(dalloc(s, &d.q, cap));
  TRY(dalloc(s, &d.binc, cap));
  TRY(dalloc(s, &d.inc, 2 * cap));
  d.part_tiles = (int)((cap + kTileItems - 1) / kTileItems) + 1;
  TRY(dalloc(s, &d.part, (size_t)(9) * d.part_tiles));
  size_t rc = std::max((size_t)d.nb, cap);
  if (rc > d.radix_cap) {
    dfree(s, d.keyA); dfree(s, d.valA); dfree(s, d.keyB); dfree(s, d.valB);
    dfree(s, d.radix_hist);
    d.radix_cap = rc;
    TRY(dalloc(s, &d.keyA, rc));
    TRY(dalloc(s, &d.valA, rc));
    TRY(dalloc(s, &d.keyB, rc));
    TRY(dalloc(s, &d.valB, rc));
    d.radix_hist_cap = radix_hist_size(rc);
    TRY(dalloc(s, &d.radix_hist, d.radix_hist_cap));
  }
  return DV_OK;
}

int ensure_gamma(dv_scene* s, size_t n) {
  SceneDev& d = s->d;
  if (n <= d.gcap) return DV_OK;
  size_t cap = std::max(n, d.gcap + d.gcap / 2);
  double* g = nullptr;
  TRY(dalloc(s, &g, 3 * cap));
  DV_CUDA_TRY(cudaMemsetAsync(g, 0, sizeof(double) * 3 * cap, s->stream));
  if (d.gamma && d.gsize > 0) {
    for (int k = 0; k < 3; ++k)
      DV_CUDA_TRY(cudaMemcpyAsync(g + k * cap, d.gamma + k * d.gcap,
                                  sizeof(double) * (size_t)d.gsize, cudaMemcpyDeviceToDevice,
                                  s->stream));
  }
  dfree(s, d.gamma);
  d.gamma = g;
  d.gcap = cap;
  return DV_OK;
}

int status_from_bits(unsigned bits) {
  if (bits & kErrBarrierTimeout) return DV_ERR_TIMEOUT;
  if (bits & kErrNaN) return DV_ERR_NAN;
  if (bits & kErrBacktrackCap) return DV_ERR_NOCONV;
  if (bits & kErrCapacity) return DV_ERR_ARG;
  return DV_OK;
}

// Folds the previous step's solver report (already copied to pinned memory)
// and appends the step to the history.
int absorb_solve(dv_scene* s) {
  int st = DV_OK;
  if (s->solve_pending) {
    s->solve_pending = false;
    const ApgdCtl& c = *s->d.h_ctl;
    s->last.iterations = c.iterations;
    s->last.backtracks = c.backtracks;
    s->last.residual = c.residual;
    s->last.objective = c.objective;
    s->last.sweeps = c.sweeps;
    for (int i = 0; i < 8; ++i) {
      s->phase_ns[i] += (double)c.phase_ns[i];
      s->phase_count[i] += (long long)c.phase_count[i];
    }
    int e = s->ev_cur;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, s->ev_t0[e], s->ev_c[e]) == cudaSuccess) s->last.collide_ms = ms;
    if (cudaEventElapsedTime(&ms, s->ev_c[e], s->ev_s[e]) == cudaSuccess) s->last.solve_ms = ms;
    st = status_from_bits(s->h_bar[2]);
    if (st != DV_OK) s->last.status = st;
  }
  if (s->step_open) {
    s->step_open = false;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, s->ev_t0[s->ev_cur], s->ev_t1[s->ev_cur]) == cudaSuccess)
      s->last.elapsed_ms = ms;
    s->last.time = s->time;
    s->last.time_index = s->time_index;
    s->history.push_back(s->last);
  }
  return st;
}

int one_step(dv_scene* s) {
  SceneDev& d = s->d;
  cudaStream_t st = s->stream;
  const int e = s->ev_cur ^ 1;   // the previous step (if any) used ev_cur
  DV_CUDA_TRY(cudaEventRecord(s->ev_t0[e], st));
  collide_count(d, s->P.envelope, st, &s->launches);
  DV_CUDA_TRY(cudaEventRecord(s->ev_count, st));
  DV_CUDA_TRY(cudaEventSynchronize(s->ev_count));
  DV_CUDA_TRY(cudaGetLastError());
  int prev = absorb_solve(s);
  s->ev_cur = e;
  if (prev != DV_OK) return prev;
  int nc = d.h_counters[0];
  int np = d.h_counters[1];
  unsigned cerr = (unsigned)d.h_counters[2];
  if (cerr) {
    g_last_error = "a sphere has more than 128 contact partners with larger ids";
    return status_from_bits(cerr);
  }
  if ((size_t)nc > d.ccap) TRY(alloc_contacts(s, std::max((size_t)nc, d.ccap + d.ccap / 2)));
  d.nc = nc;
  d.npossible = np;
  collide_write(d, s->P.envelope, st, &s->launches);
  memset(&s->last, 0, sizeof(s->last));
  s->last.num_contacts = nc;
  s->last.num_possible = np;
  if (nc > 0) {
    TRY(ensure_gamma(s, (size_t)nc));
    // thrust::device_vector::resize keeps the prefix and zero-fills the growth
    // (APGD.cu:166): positional warm start.
    if (d.gsize < nc) {
      for (int k = 0; k < 3; ++k)
        DV_CUDA_TRY(cudaMemsetAsync(d.gamma + k * d.gcap + d.gsize, 0,
                                    sizeof(double) * (size_t)(nc - d.gsize), st));
    }
    d.gsize = nc;
    SolveConfig cfg;
    cfg.h = s->P.h;
    cfg.mu = s->P.mu;
    cfg.tol = s->P.tolerance;
    cfg.max_iter = s->P.max_iterations;
    cfg.max_bt = s->P.max_backtracks;
    cfg.warm = s->P.warm_start;
    cfg.precision = s->P.precision;
    int nt = (nc + kTileItems - 1) / kTileItems;
    int nbt = (d.nb + kThreads - 1) / kThreads;
    cfg.grid = std::max(1, std::min(s->max_ctas, std::max(nt, nbt)));
    DV_CUDA_TRY(cudaEventRecord(s->ev_c[e], st));
    launch_step_solve(d, cfg, st, &s->launches);
    DV_CUDA_TRY(cudaGetLastError());
    DV_CUDA_TRY(cudaEventRecord(s->ev_s[e], st));
    DV_CUDA_TRY(cudaMemcpyAsync(s->h_bar, d.bar, 4 * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    s->solve_pending = true;
  } else {
    launch_step_nocontact(d, s->P.h, st, &s->launches);
    DV_CUDA_TRY(cudaGetLastError());
  }
  DV_CUDA_TRY(cudaEventRecord(s->ev_t1[e], st));
  s->time += s->P.h;
  s->time_index += 1;
  s->step_open = true;
  return DV_OK;
}

int finish(dv_scene* s) {
  DV_CUDA_TRY(cudaStreamSynchronize(s->stream));
  int st = absorb_solve(s);
  s->last.time = s->time;
  s->last.time_index = s->time_index;
  if (s->P.verbose)
    printf("Time: %f (Exec. Time: %f), Collisions: %d (%d possible)\n  Iterations: %d Residual: %g\n",
           s->time, s->last.elapsed_ms, s->last.num_contacts, s->last.num_possible,
           s->last.iterations, s->last.residual);
  return st;
}

// Interleaves 3 planes (stride S) into n rows of 3 (or 4 with an extra plane).
void interleave(const std::vector<double>& planes, size_t S, int n, int k, double* out, int width) {
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < k; ++c) out[(size_t)i * width + c] = planes[c * S + i];
}

int download_planes(dv_scene* s, const double* dev, size_t S, int k, int n, std::vector<double>& h) {
  h.assign((size_t)k * S, 0.0);
  for (int c = 0; c < k; ++c)
    DV_CUDA_TRY(cudaMemcpyAsync(h.data() + c * S, dev + c * S, sizeof(double) * (size_t)n,
                                cudaMemcpyDeviceToHost, s->stream));
  DV_CUDA_TRY(cudaStreamSynchronize(s->stream));
  return DV_OK;
}

// ---- ordered reductions for diagnostics (same fold order as the solver) ----
__global__ void __launch_bounds__(kThreads) k_items_partials(const double* __restrict__ items, int n,
                                                             double* __restrict__ part, int nt) {
  __shared__ double scratch[8];
  int tile = blockIdx.x;
  double acc = 0.0;
  for (int m = 0; m < kItemsPerThread; ++m) {
    int c = tile * kTileItems + m * kThreads + threadIdx.x;
    if (c < n) acc = acc + items[c];
  }
  double v = block_fold256(acc, scratch);
  if (threadIdx.x == 0) part[tile] = v;
}

__global__ void __launch_bounds__(kThreads) k_items_final(const double* __restrict__ part, int nt,
                                                          double* __restrict__ out) {
  __shared__ double scratch[8];
  double acc = 0.0;
  for (int t = threadIdx.x; t < nt; t += kThreads) acc = acc + part[t];
  double v = block_fold256(acc, scratch);
  if (threadIdx.x == 0) *out = v;
}

// System.cu:1590-1643 per-contact items: gamma_n, v_n, gamma_n v_n, cone violation^2.
__global__ void __launch_bounds__(kThreads) k_violation_items(
    int nc, size_t S, size_t GS, const double* __restrict__ gamma, const double* __restrict__ F,
    const double* __restrict__ gap, const uint32_t* __restrict__ ida,
    const uint32_t* __restrict__ idb, const double4* __restrict__ v4, double h, double mu,
    double* __restrict__ items) {
  int c = blockIdx.x * kThreads + threadIdx.x;
  if (c >= nc) return;
  double g0 = gamma[c], g1 = gamma[GS + c], g2 = gamma[2 * GS + c];
  double4 va = v4[ida[c]], vb = v4[idb[c]];
  double d0 = va.x - vb.x, d1 = va.y - vb.y, d2 = va.z - vb.z;
  double dv = (F[c] * d0 + F[S + c] * d1) + F[2 * S + c] * d2;
  double vn = gap[c] / h + dv;
  double gt = sqrt(g1 * g1 + g2 * g2);
  double cv = mu * g0 - gt;
  if (cv > 0) cv = 0;
  items[c] = g0;
  items[(size_t)nc + c] = vn;
  items[2 * (size_t)nc + c] = g0 * vn;
  items[3 * (size_t)nc + c] = cv * cv;
}

__global__ void __launch_bounds__(kThreads) k_energy_items(int nb, const double4* __restrict__ p4,
                                                           const double4* __restrict__ v4,
                                                           const double4* __restrict__ f4,
                                                           const double* __restrict__ minv,
                                                           double* __restrict__ items) {
  int b = blockIdx.x * kThreads + threadIdx.x;
  if (b >= nb) return;
  double m = minv[b];
  if (m) m = 1.0 / m;
  double4 v = v4[b], p = p4[b], f = f4[b];
  items[b] = (v.x * (m * v.x) + v.y * (m * v.y)) + v.z * (m * v.z);
  items[(size_t)nb + b] = (f.x * p.x + f.y * p.y) + f.z * p.z;
}

int ensure_red(dv_scene* s, size_t n) {
  if (n <= s->d_red_cap) return DV_OK;
  dfree(s, s->d_red);
  s->d_red_cap = n;
  return dalloc(s, &s->d_red, n);
}

// Ordered sum of `n` device items; result lands in h_red[slot] after sync.
void ordered_sum_dev(dv_scene* s, const double* items, int n, double* part, int slot) {
  int nt = std::max(1, (n + kTileItems - 1) / kTileItems);
  k_items_partials<<<nt, kThreads, 0, s->stream>>>(items, n, part, nt);
  k_items_final<<<1, kThreads, 0, s->stream>>>(part, nt, part + nt);
  cudaMemcpyAsync(s->h_red + slot, part + nt, sizeof(double), cudaMemcpyDeviceToHost, s->stream);
  s->launches += 2;
}

}  // namespace

extern "C" {

DV_API int dv_params_default(dv_params* p) {
  if (!p) return DV_ERR_ARG;
  memset(p, 0, sizeof(*p));
  p->h = 1e-3;
  p->mu = 0.25;
  p->gravity[0] = 0.0;
  p->gravity[1] = -9.81;
  p->gravity[2] = 0.0;
  p->envelope = 1e-3;
  p->tolerance = 1e-4;
  p->max_iterations = 100000;
  p->warm_start = 0;
  p->solver = DV_SOLVER_APGD;
  p->precision = DV_PREC_FP64;
  p->max_backtracks = 4096;
  p->verbose = 0;
  return DV_OK;
}

DV_API const char* dv_status_string(int status) {
  switch (status) {
    case DV_OK: return "ok";
    case DV_ERR_ARG: return "invalid argument";
    case DV_ERR_CUDA: return "CUDA error";
    case DV_ERR_NAN: return "non-finite value in the solve";
    case DV_ERR_NOCONV: return "Lipschitz backtracking limit reached";
    case DV_ERR_OOM: return "out of device memory";
    case DV_ERR_TIMEOUT: return "device wait timed out";
    case DV_ERR_UNSUPPORTED: return "unsupported";
    case DV_ERR_ABORTED: return "aborted";
    default: return "unknown status";
  }
}

DV_API const char* dv_last_error(void) { return g_last_error.c_str(); }

static int check_params(const dv_params* p) {
  if (!p) return DV_ERR_ARG;
  if (!(p->h > 0) || !(p->envelope >= 0) || !(p->mu >= 0) || !(p->tolerance >= 0)) return DV_ERR_ARG;
  if (p->max_iterations < 0 || p->max_backtracks < 0) return DV_ERR_ARG;
  if (p->solver != DV_SOLVER_APGD) return DV_ERR_UNSUPPORTED;
  if (p->precision != DV_PREC_FP64) return DV_ERR_UNSUPPORTED;
  return DV_OK;
}

DV_API int dv_scene_create(const dv_body_desc* bodies, int32_t nb, const dv_params* params,
                           dv_scene** out) {
  if (!out || nb < 0 || (nb > 0 && !bodies)) return DV_ERR_ARG;
  *out = nullptr;
  int pc = check_params(params);
  if (pc != DV_OK) return pc;
  for (int i = 0; i < nb; ++i) {
    const dv_body_desc& b = bodies[i];
    if (!(b.mass > 0) && !b.fixed) return DV_ERR_ARG;
    if (b.geom[1] == 0 && !(b.geom[0] >= 0)) return DV_ERR_ARG;
  }
  dv_scene* s = new dv_scene();
  s->P = *params;
  SceneDev& d = s->d;
  d.nb = nb;
  int rc = DV_OK;
  auto fail = [&](int code) {
    dv_scene_destroy(s);
    return code;
  };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(dv_record_cuda_error(cudaGetLastError(), "cudaStreamCreate", __FILE__, __LINE__));
  s->own_stream = true;
  cudaEventCreate(&s->ev_count);
  for (int k = 0; k < 2; ++k) {
    cudaEventCreate(&s->ev_t0[k]);
    cudaEventCreate(&s->ev_t1[k]);
    cudaEventCreate(&s->ev_c[k]);
    cudaEventCreate(&s->ev_s[k]);
  }

  // classify: spheres go in the grid, boxes are tested against all bodies
  std::vector<int> small, large;
  std::vector<double> radii;
  for (int i = 0; i < nb; ++i)
    if (bodies[i].geom[1] == 0) radii.push_back(bodies[i].geom[0]);
  double rlimit = 0;
  if (!radii.empty()) {
    std::vector<double> r2 = radii;
    std::nth_element(r2.begin(), r2.begin() + r2.size() / 2, r2.end());
    rlimit = 4.0 * r2[r2.size() / 2];
  }
  double rmax = 0;
  for (int i = 0; i < nb; ++i) {
    if (bodies[i].geom[1] == 0 && bodies[i].geom[0] <= rlimit) {
      small.push_back(i);
      rmax = std::max(rmax, bodies[i].geom[0]);
    } else {
      large.push_back(i);
    }
  }
  d.n_small = (int)small.size();
  d.n_large = (int)large.size();
  d.W = 2.0 * (rmax + params->envelope);

  std::vector<double4> p4(nb), v4(nb), f4(nb), g4(nb);
  std::vector<double> minv(nb);
  std::vector<int> fam(nb);
  for (int i = 0; i < nb; ++i) {
    const dv_body_desc& b = bodies[i];
    p4[i] = make_double4(b.pos[0], b.pos[1], b.pos[2], 0.0);
    v4[i] = make_double4(b.vel[0], b.vel[1], b.vel[2], 0.0);
    // System.cu:368-376, 409-417: f = m g and Minv = 1/m, both 0 for fixed bodies
    if (b.fixed) {
      f4[i] = make_double4(0.0, 0.0, 0.0, 0.0);
      minv[i] = 0.0;
    } else {
      f4[i] = make_double4(b.mass * params->gravity[0], b.mass * params->gravity[1],
                           b.mass * params->gravity[2], 0.0);
      minv[i] = 1.0 / b.mass;
    }
    g4[i] = make_double4(b.geom[0], b.geom[1], b.geom[2], b.geom[1] != 0 ? 1.0 : 0.0);
    fam[i] = b.family;
  }
  size_t nbz = std::max(nb, 1);
  if ((rc = dalloc(s, &d.p4, nbz)) || (rc = dalloc(s, &d.v4, nbz)) || (rc = dalloc(s, &d.k4, nbz)) ||
      (rc = dalloc(s, &d.f4, nbz)) || (rc = dalloc(s, &d.w4, nbz)) || (rc = dalloc(s, &d.fc4, nbz)) ||
      (rc = dalloc(s, &d.geom4, nbz)) || (rc = dalloc(s, &d.minv, nbz)) ||
      (rc = dalloc(s, &d.family, nbz)) || (rc = dalloc(s, &d.small_ids, std::max(d.n_small, 1))) ||
      (rc = dalloc(s, &d.large_ids, std::max(d.n_large, 1))) || (rc = dalloc(s, &d.amin, nbz)) ||
      (rc = dalloc(s, &d.amax, nbz)) || (rc = dalloc(s, &d.cell, nbz)) ||
      (rc = dalloc(s, &d.cnt_cont, nbz)) || (rc = dalloc(s, &d.cnt_cand, nbz)) ||
      (rc = dalloc(s, &d.cbase, nbz + 1)) || (rc = dalloc(s, &d.binc_start, nbz + 1)) ||
      (rc = dalloc(s, &d.inc_start, nbz + 1)) ||
      (rc = dalloc(s, &d.grid, 1)) || (rc = dalloc(s, &d.counters, 4)) ||
      (rc = dalloc(s, &d.ctl, 1)) || (rc = dalloc(s, &d.bar, 4)))
    return fail(rc);
  d.ncell_cap = std::max(4 * d.n_small, 64);
  if ((rc = dalloc(s, &d.cell_start, d.ncell_cap)) || (rc = dalloc(s, &d.cell_end, d.ncell_cap)))
    return fail(rc);
  int nchunks = (nb + kThreads - 1) / kThreads;
  d.large_chunks = nchunks * std::max(d.n_large, 1);
  if ((rc = dalloc(s, &d.large_chunk, d.large_chunks + 1)) ||
      (rc = dalloc(s, &d.large_chunk_off, d.large_chunks + 1)))
    return fail(rc);
  d.scan_tmp_cap = scan_tmp_size(std::max((size_t)nbz + 1, (size_t)d.large_chunks + 1));
  if ((rc = dalloc(s, &d.scan_tmp, d.scan_tmp_cap))) return fail(rc);
  if (cudaMallocHost(&d.h_counters, 4 * sizeof(int)) != cudaSuccess ||
      cudaMallocHost(&d.h_ctl, sizeof(ApgdCtl)) != cudaSuccess ||
      cudaMallocHost(&s->h_bar, 4 * sizeof(unsigned)) != cudaSuccess ||
      cudaMallocHost(&s->h_red, 16 * sizeof(double)) != cudaSuccess)
    return fail(dv_record_cuda_error(cudaErrorMemoryAllocation, "cudaMallocHost", __FILE__, __LINE__));
  memset(s->h_bar, 0, 4 * sizeof(unsigned));
  if ((rc = alloc_contacts(s, std::max((size_t)4 * nb, (size_t)1024)))) return fail(rc);
  // System.cu:185: gamma_d starts as 3 nb zeros
  if ((rc = ensure_gamma(s, std::max((size_t)nb, (size_t)1024)))) return fail(rc);
  d.gsize = nb;
  cudaStream_t st = s->stream;
  cudaMemcpyAsync(d.p4, p4.data(), sizeof(double4) * nb, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d.v4, v4.data(), sizeof(double4) * nb, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d.f4, f4.data(), sizeof(double4) * nb, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d.geom4, g4.data(), sizeof(double4) * nb, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d.minv, minv.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d.family, fam.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, st);
  if (d.n_small)
    cudaMemcpyAsync(d.small_ids, small.data(), sizeof(int) * d.n_small, cudaMemcpyHostToDevice, st);
  if (d.n_large)
    cudaMemcpyAsync(d.large_ids, large.data(), sizeof(int) * d.n_large, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(d.fc4, 0, sizeof(double4) * nbz, st);
  cudaMemsetAsync(d.k4, 0, sizeof(double4) * nbz, st);
  cudaMemsetAsync(d.w4, 0, sizeof(double4) * nbz, st);
  cudaMemsetAsync(d.cell_end, 0, sizeof(int) * d.ncell_cap, st);
  if (cudaStreamSynchronize(st) != cudaSuccess)
    return fail(dv_record_cuda_error(cudaGetLastError(), "scene upload", __FILE__, __LINE__));
  s->max_ctas = apgd_max_ctas(params->precision);
  memset(&s->last, 0, sizeof(s->last));
  *out = s;
  return DV_OK;
}

DV_API int dv_scene_destroy(dv_scene* s) {
  if (!s) return DV_ERR_ARG;
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (void* p : s->allocs) cudaFree(p);
  s->allocs.clear();
  if (s->d.h_counters) cudaFreeHost(s->d.h_counters);
  if (s->d.h_ctl) cudaFreeHost(s->d.h_ctl);
  if (s->h_bar) cudaFreeHost(s->h_bar);
  if (s->h_red) cudaFreeHost(s->h_red);
  if (s->ev_count) cudaEventDestroy(s->ev_count);
  for (int k = 0; k < 2; ++k) {
    if (s->ev_t0[k]) cudaEventDestroy(s->ev_t0[k]);
    if (s->ev_t1[k]) cudaEventDestroy(s->ev_t1[k]);
    if (s->ev_c[k]) cudaEventDestroy(s->ev_c[k]);
    if (s->ev_s[k]) cudaEventDestroy(s->ev_s[k]);
  }
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return DV_OK;
}

DV_API int dv_scene_set_stream(dv_scene* s, void* cuda_stream) {
  if (!s) return DV_ERR_ARG;
  DV_CUDA_TRY(cudaStreamSynchronize(s->stream));
  if (cuda_stream) {
    if (s->own_stream) cudaStreamDestroy(s->stream);
    s->own_stream = false;
    s->stream = (cudaStream_t)cuda_stream;
  }
  return DV_OK;
}

DV_API int dv_set_params(dv_scene* s, const dv_params* params) {
  if (!s) return DV_ERR_ARG;
  int pc = check_params(params);
  if (pc != DV_OK) return pc;
  if (params->envelope > s->P.envelope) {
    // the grid cell must stay wider than every sphere AABB
    s->d.W = s->d.W - 2.0 * s->P.envelope + 2.0 * params->envelope;
  }
  s->P = *params;
  return DV_OK;
}

DV_API int dv_step(dv_scene* s, int32_t nsteps) {
  if (!s || nsteps < 0) return DV_ERR_ARG;
  for (int i = 0; i < nsteps; ++i) {
    int rc = one_step(s);
    if (rc != DV_OK) {
      finish(s);
      s->last.status = rc;
      return rc;
    }
  }
  int rc = finish(s);
  s->last.status = rc;
  return rc;
}

DV_API int dv_collide(dv_scene* s) {
  if (!s) return DV_ERR_ARG;
  SceneDev& d = s->d;
  DV_CUDA_TRY(cudaStreamSynchronize(s->stream));
  absorb_solve(s);
  collide_count(d, s->P.envelope, s->stream, &s->launches);
  DV_CUDA_TRY(cudaStreamSynchronize(s->stream));
  int nc = d.h_counters[0];
  if (d.h_counters[2]) return status_from_bits((unsigned)d.h_counters[2]);
  if ((size_t)nc > d.ccap) TRY(alloc_contacts(s, std::max((size_t)nc, d.ccap + d.ccap / 2)));
  d.nc = nc;
  d.npossible = d.h_counters[1];
  collide_write(d, s->P.envelope, s->stream, &s->launches);
  DV_CUDA_TRY(cudaStreamSynchronize(s->stream));
  DV_CUDA_TRY(cudaGetLastError());
  s->last.num_contacts = nc;
  s->last.num_possible = d.npossible;
  return DV_OK;
}

DV_API int dv_get_state(dv_scene* s, double* p, double* v) {
  if (!s) return DV_ERR_ARG;
  int nb = s->d.nb;
  if (nb == 0) return DV_OK;
  if (p)
    DV_CUDA_TRY(cudaMemcpy2DAsync(p, 3 * sizeof(double), s->d.p4, sizeof(double4), 3 * sizeof(double),
                                  nb, cudaMemcpyDeviceToHost, s->stream));
  if (v)
    DV_CUDA_TRY(cudaMemcpy2DAsync(v, 3 * sizeof(double), s->d.v4, sizeof(double4), 3 * sizeof(double),
                                  nb, cudaMemcpyDeviceToHost, s->stream));
  DV_CUDA_TRY(cudaStreamSynchronize(s->stream));
  return DV_OK;
}

DV_API int dv_set_state(dv_scene* s, const double* p, const double* v) {
  if (!s) return DV_ERR_ARG;
  int nb = s->d.nb;
  if (nb == 0) return DV_OK;
  if (p)
    DV_CUDA_TRY(cudaMemcpy2DAsync(s->d.p4, sizeof(double4), p, 3 * sizeof(double), 3 * sizeof(double),
                                  nb, cudaMemcpyHostToDevice, s->stream));
  if (v)
    DV_CUDA_TRY(cudaMemcpy2DAsync(s->d.v4, sizeof(double4), v, 3 * sizeof(double), 3 * sizeof(double),
                                  nb, cudaMemcpyHostToDevice, s->stream));
  DV_CUDA_TRY(cudaStreamSynchronize(s->stream));
  return DV_OK;
}

DV_API int dv_get_contact_force(dv_scene* s, double* f) {
  if (!s || !f) return DV_ERR_ARG;
  int nb = s->d.nb;
  if (nb == 0) return DV_OK;
  DV_CUDA_TRY(cudaMemcpy2DAsync(f, 3 * sizeof(double), s->d.fc4, sizeof(double4), 3 * sizeof(double),
                                nb, cudaMemcpyDeviceToHost, s->stream));
  DV_CUDA_TRY(cudaStreamSynchronize(s->stream));
  return DV_OK;
}

DV_API int dv_get_num_contacts(dv_scene* s, int32_t* nc, int32_t* npossible) {
  if (!s) return DV_ERR_ARG;
  if (nc) *nc = s->d.nc;
  if (npossible) *npossible = s->d.npossible;
  return DV_OK;
}

DV_API int dv_get_contacts(dv_scene* s, uint32_t* a, uint32_t* b, double* nP, double* loc) {
  if (!s) return DV_ERR_ARG;
  SceneDev& d = s->d;
  int nc = d.nc;
  if (nc == 0) return DV_OK;
  if (a) DV_CUDA_TRY(cudaMemcpyAsync(a, d.ida, sizeof(uint32_t) * nc, cudaMemcpyDeviceToHost, s->stream));
  if (b) DV_CUDA_TRY(cudaMemcpyAsync(b, d.idb, sizeof(uint32_t) * nc, cudaMemcpyDeviceToHost, s->stream));
  std::vector<double> h;
  if (nP) {
    TRY(download_planes(s, d.F, d.ccap, 3, nc, h));
    interleave(h, d.ccap, nc, 3, nP, 4);
    std::vector<double> g(nc);
    DV_CUDA_TRY(cudaMemcpy(g.data(), d.gap, sizeof(double) * nc, cudaMemcpyDeviceToHost));
    for (int i = 0; i < nc; ++i) nP[4 * (size_t)i + 3] = g[i];
  }
  if (loc) {
    TRY(download_planes(s, d.loc, d.ccap, 3, nc, h));
    interleave(h, d.ccap, nc, 3, loc, 3);
  }
  DV_CUDA_TRY(cudaStreamSynchronize(s->stream));
  return DV_OK;
}

DV_API int dv_get_frames(dv_scene* s, double* F) {
  if (!s || !F) return DV_ERR_ARG;
  std::vector<double> h;
  TRY(download_planes(s, s->d.F, s->d.ccap, 9, s->d.nc, h));
  interleave(h, s->d.ccap, s->d.nc, 9, F, 9);
  return DV_OK;
}

DV_API int dv_get_schur_vector(dv_scene* s, double* r) {
  if (!s || !r) return DV_ERR_ARG;
  std::vector<double> h;
  TRY(download_planes(s, s->d.r, s->d.ccap, 3, s->d.nc, h));
  interleave(h, s->d.ccap, s->d.nc, 3, r, 3);
  return DV_OK;
}

DV_API int dv_get_gamma(dv_scene* s, double* gamma, int32_t cap, int32_t* n) {
  if (!s) return DV_ERR_ARG;
  SceneDev& d = s->d;
  if (n) *n = d.gsize;
  if (!gamma || cap <= 0) return DV_OK;
  int m = std::min(cap, d.gsize);
  std::vector<double> h;
  TRY(download_planes(s, d.gamma, d.gcap, 3, m, h));
  interleave(h, d.gcap, m, 3, gamma, 3);
  return DV_OK;
}

DV_API int dv_set_gamma(dv_scene* s, const double* gamma, int32_t n) {
  if (!s || n < 0 || (n > 0 && !gamma)) return DV_ERR_ARG;
  SceneDev& d = s->d;
  DV_CUDA_TRY(cudaStreamSynchronize(s->stream));
  TRY(ensure_gamma(s, (size_t)std::max(n, 1)));
  std::vector<double> h(3 * (size_t)n);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) h[k * (size_t)n + i] = gamma[3 * (size_t)i + k];
  for (int k = 0; k < 3; ++k)
    DV_CUDA_TRY(cudaMemcpyAsync(d.gamma + k * d.gcap, h.data() + k * (size_t)n,
                                sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, s->stream));
  DV_CUDA_TRY(cudaStreamSynchronize(s->stream));
  d.gsize = n;
  return DV_OK;
}

DV_API int dv_ccp_violation(dv_scene* s, double* out4) {
  if (!s || !out4) return DV_ERR_ARG;
  SceneDev& d = s->d;
  out4[0] = out4[1] = out4[2] = out4[3] = 0.0;
  int nc = d.nc;
  if (nc == 0) return DV_OK;
  int nt = (nc + kTileItems - 1) / kTileItems;
  TRY(ensure_red(s, 4 * (size_t)nc + 2 * (size_t)(nt + 2)));
  double* items = s->d_red;
  double* part = s->d_red + 4 * (size_t)nc;
  k_violation_items<<<(nc + kThreads - 1) / kThreads, kThreads, 0, s->stream>>>(
      nc, d.ccap, d.gcap, d.gamma, d.F, d.gap, d.ida, d.idb, d.v4, s->P.h, s->P.mu, items);
  ++s->launches;
  ordered_sum_dev(s, items + 2 * (size_t)nc, nc, part, 0);
  ordered_sum_dev(s, items + 3 * (size_t)nc, nc, part + nt + 2, 1);
  std::vector<double> gn(nc), vn(nc);
  DV_CUDA_TRY(cudaMemcpyAsync(gn.data(), items, sizeof(double) * nc, cudaMemcpyDeviceToHost, s->stream));
  DV_CUDA_TRY(cudaMemcpyAsync(vn.data(), items + nc, sizeof(double) * nc, cudaMemcpyDeviceToHost,
                              s->stream));
  DV_CUDA_TRY(cudaStreamSynchronize(s->stream));
  DV_CUDA_TRY(cudaGetLastError());
  double x = gn[0], y = vn[0];
  for (int i = 1; i < nc; ++i) {
    x = std::min(x, gn[i]);
    y = std::min(y, vn[i]);
  }
  if (x > 0) x = 0;
  if (y > 0) y = 0;
  out4[0] = x;
  out4[1] = y;
  out4[2] = s->h_red[0];
  out4[3] = sqrt(s->h_red[1]);
  return DV_OK;
}

DV_API int dv_energies(dv_scene* s, double* kinetic, double* potential) {
  if (!s) return DV_ERR_ARG;
  SceneDev& d = s->d;
  int nb = d.nb;
  if (nb == 0) {
    if (kinetic) *kinetic = 0;
    if (potential) *potential = 0;
    return DV_OK;
  }
  int nt = (nb + kTileItems - 1) / kTileItems;
  TRY(ensure_red(s, 2 * (size_t)nb + 2 * (size_t)(nt + 2)));
  double* items = s->d_red;
  double* part = s->d_red + 2 * (size_t)nb;
  k_energy_items<<<(nb + kThreads - 1) / kThreads, kThreads, 0, s->stream>>>(nb, d.p4, d.v4, d.f4,
                                                                            d.minv, items);
  ++s->launches;
  ordered_sum_dev(s, items, nb, part, 2);
  ordered_sum_dev(s, items + nb, nb, part + nt + 2, 3);
  DV_CUDA_TRY(cudaStreamSynchronize(s->stream));
  DV_CUDA_TRY(cudaGetLastError());
  if (kinetic) *kinetic = 0.5 * s->h_red[2];
  if (potential) *potential = -s->h_red[3];
  return DV_OK;
}

DV_API int dv_contact_forces_per_collision(dv_scene* s, double* normal, double* friction) {
  if (!s) return DV_ERR_ARG;
  SceneDev& d = s->d;
  int nc = d.nc;
  if (nc == 0) return DV_OK;
  std::vector<double> F, g;
  TRY(download_planes(s, d.F, d.ccap, 9, nc, F));
  TRY(download_planes(s, d.gamma, d.gcap, 3, nc, g));
  double h = s->P.h;
  for (int c = 0; c < nc; ++c) {
    double g0 = g[c], g1 = g[d.gcap + c], g2 = g[2 * d.gcap + c];
    for (int k = 0; k < 3; ++k) {
      double n = F[k * d.ccap + c], u = F[(3 + k) * d.ccap + c], v = F[(6 + k) * d.ccap + c];
      if (normal) normal[3 * (size_t)c + k] = (g0 * n) / h;
      if (friction) friction[3 * (size_t)c + k] = (g1 * u + g2 * v) / h;
    }
  }
  return DV_OK;
}

DV_API int dv_get_step_stats(dv_scene* s, dv_step_stats* out) {
  if (!s || !out) return DV_ERR_ARG;
  int rc = finish(s);
  *out = s->last;
  return rc;
}

DV_API int64_t dv_scene_launch_count(dv_scene* s) { return s ? s->launches : -1; }

DV_API int dv_get_step_history(dv_scene* s, dv_step_stats* out, int32_t cap, int32_t* n) {
  if (!s) return DV_ERR_ARG;
  int rc = finish(s);
  int m = (int)s->history.size();
  if (n) *n = m;
  if (out)
    for (int i = 0; i < std::min(cap, m); ++i) out[i] = s->history[i];
  return rc;
}

DV_API int dv_get_phase_times(dv_scene* s, double* ns, int64_t* counts, int32_t reset) {
  if (!s) return DV_ERR_ARG;
  int rc = finish(s);
  for (int i = 0; i < 8; ++i) {
    if (ns) ns[i] = s->phase_ns[i];
    if (counts) counts[i] = s->phase_count[i];
    if (reset) {
      s->phase_ns[i] = 0;
      s->phase_count[i] = 0;
    }
  }
  return rc;
}

DV_API int dv_clear_step_history(dv_scene* s) {
  if (!s) return DV_ERR_ARG;
  s->history.clear();
  return DV_OK;
}

}  // extern "C"
