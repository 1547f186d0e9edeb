// dv_scene.cu -- the plain-scene C ABI of include/dvide.h: one DVIDE System
// is an engine with one segment.  Scene lifetime, System::DoTimeStep
// (System.cu:544-602), the state accessors and the diagnostics of
// System.cu:1259-1295, 1590-1658.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "dv_engine.h"

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
  Engine E;
  dv_params P;
  dv_step_stats last;
  std::vector<dv_step_stats> history;
};

namespace {

#define TRY(x)                    \
  do {                            \
    int rc_ = (x);                \
    if (rc_ != DV_OK) return rc_; \
  } while (0)

// Interleaves k planes of n values into n rows of `width`.
void interleave(const std::vector<double>& planes, int n, int k, double* out, int width) {
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < k; ++c) out[(size_t)i * width + c] = planes[(size_t)c * n + i];
}

void absorb_records(dv_scene* s) {
  for (const StepRecord& r : s->E.records()) {
    dv_step_stats st;
    fill_step_stats(r, 0, &st);
    s->history.push_back(st);
    s->last = st;
  }
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

DV_API int dv_scene_create(const dv_body_desc* bodies, int32_t nb, const dv_params* params,
                           dv_scene** out) {
  if (!out || !params || nb < 0 || (nb > 0 && !bodies)) return DV_ERR_ARG;
  *out = nullptr;
  dv_scene* s = new dv_scene();
  s->P = *params;
  SceneInput in;
  in.bodies = bodies;
  in.nb = nb;
  in.P = *params;
  int rc = nb == 0 ? DV_ERR_ARG : s->E.init({in}, params->precision);
  if (rc == DV_OK) rc = s->E.set_stop_on_segment_error(true);
  if (rc != DV_OK) {
    delete s;
    return rc;
  }
  memset(&s->last, 0, sizeof(s->last));
  *out = s;
  return DV_OK;
}

DV_API int dv_scene_destroy(dv_scene* s) {
  if (!s) return DV_ERR_ARG;
  delete s;
  return DV_OK;
}

DV_API int dv_scene_set_stream(dv_scene* s, void* cuda_stream) {
  if (!s) return DV_ERR_ARG;
  return s->E.set_stream((cudaStream_t)cuda_stream);
}

DV_API int dv_set_params(dv_scene* s, const dv_params* params) {
  if (!s || !params) return DV_ERR_ARG;
  TRY(s->E.set_segment_params(0, *params));
  TRY(s->E.set_precision(params->precision));
  s->P = *params;
  return DV_OK;
}

DV_API int dv_step(dv_scene* s, int32_t nsteps) {
  if (!s || nsteps < 0) return DV_ERR_ARG;
  int rc = s->E.step(nsteps);
  absorb_records(s);
  if (rc == DV_OK) rc = s->last.status;
  if (rc != DV_OK) s->last.status = rc;
  if (s->P.verbose && !s->E.records().empty())
    printf("Time: %f (Exec. Time: %f), Collisions: %d (%d possible)\n  Iterations: %d Residual: %g\n",
           s->last.time, s->last.elapsed_ms, s->last.num_contacts, s->last.num_possible,
           s->last.iterations, s->last.residual);
  return rc;
}

DV_API int dv_collide(dv_scene* s) {
  if (!s) return DV_ERR_ARG;
  TRY(s->E.collide_only());
  const SegState& X = s->E.seg_state(0);
  s->last.num_contacts = X.nc;
  s->last.num_possible = X.npossible;
  return DV_OK;
}

DV_API int dv_apgd_solve(dv_scene* s) {
  if (!s) return DV_ERR_ARG;
  TRY(s->E.solve_only());
  const SegState& X = s->E.seg_state(0);
  dv_step_stats& L = s->last;
  L.num_contacts = X.nc;
  L.num_possible = X.npossible;
  L.iterations = X.ctl.iterations;
  L.backtracks = X.ctl.backtracks;
  L.residual = X.ctl.residual;
  L.objective = X.ctl.objective;
  L.sweeps = X.ctl.sweeps;
  L.refine_iterations = X.ctl.refine_it;
  L.status = status_from_bits(X.err);
  return L.status;
}

DV_API int dv_get_state(dv_scene* s, double* p, double* v) {
  if (!s) return DV_ERR_ARG;
  return s->E.copy_state_out(0, s->E.d.nb, p, v);
}

DV_API int dv_set_state(dv_scene* s, const double* p, const double* v) {
  if (!s) return DV_ERR_ARG;
  return s->E.copy_state_in(0, s->E.d.nb, p, v);
}

DV_API int dv_get_contact_force(dv_scene* s, double* f) {
  if (!s || !f) return DV_ERR_ARG;
  Engine& E = s->E;
  DV_CUDA_TRY(cudaMemcpy2DAsync(f, 3 * sizeof(double), E.d.fc4, sizeof(double4), 3 * sizeof(double),
                                E.d.nb, cudaMemcpyDeviceToHost, E.stream()));
  DV_CUDA_TRY(cudaStreamSynchronize(E.stream()));
  return DV_OK;
}

DV_API int dv_get_num_contacts(dv_scene* s, int32_t* nc, int32_t* npossible) {
  if (!s) return DV_ERR_ARG;
  TRY(s->E.sync_state());
  if (nc) *nc = s->E.seg_state(0).nc;
  if (npossible) *npossible = s->E.seg_state(0).npossible;
  return DV_OK;
}

DV_API int dv_get_contacts(dv_scene* s, uint32_t* a, uint32_t* b, double* nP, double* loc) {
  if (!s) return DV_ERR_ARG;
  Engine& E = s->E;
  TRY(E.sync_state());
  const int nc = E.seg_state(0).nc, c0 = E.seg_state(0).c0;
  if (nc == 0) return DV_OK;
  if (a) TRY(E.download(a, E.d.ida + c0, sizeof(uint32_t) * nc));
  if (b) TRY(E.download(b, E.d.idb + c0, sizeof(uint32_t) * nc));
  std::vector<double> h;
  if (nP) {
    TRY(E.download_planes(E.d.F, E.d.ccap, 3, c0, nc, h));
    interleave(h, nc, 3, nP, 4);
    std::vector<double> g(nc);
    TRY(E.download(g.data(), E.d.gap + c0, sizeof(double) * nc));
    for (int i = 0; i < nc; ++i) nP[4 * (size_t)i + 3] = g[i];
  }
  if (loc) {
    TRY(E.download_planes(E.d.loc, E.d.ccap, 3, c0, nc, h));
    interleave(h, nc, 3, loc, 3);
  }
  return DV_OK;
}

DV_API int dv_get_frames(dv_scene* s, double* F) {
  if (!s || !F) return DV_ERR_ARG;
  Engine& E = s->E;
  TRY(E.sync_state());
  const int nc = E.seg_state(0).nc, c0 = E.seg_state(0).c0;
  std::vector<double> h;
  TRY(E.download_planes(E.d.F, E.d.ccap, 9, c0, nc, h));
  interleave(h, nc, 9, F, 9);
  return DV_OK;
}

DV_API int dv_get_schur_vector(dv_scene* s, double* r) {
  if (!s || !r) return DV_ERR_ARG;
  Engine& E = s->E;
  TRY(E.sync_state());
  const int nc = E.seg_state(0).nc, c0 = E.seg_state(0).c0;
  std::vector<double> h;
  if (E.precision() == DV_PREC_MIXED)
    TRY(E.download_planes_f(reinterpret_cast<const float*>(E.d.r), E.d.ccap, 3, c0, nc, h));
  else
    TRY(E.download_planes(E.d.r, E.d.ccap, 3, c0, nc, h));
  interleave(h, nc, 3, r, 3);
  return DV_OK;
}

DV_API int dv_get_step_vectors(dv_scene* s, double* r, double* b, double* k) {
  if (!s) return DV_ERR_ARG;
  Engine& E = s->E;
  TRY(E.sync_state());
  const int nc = E.seg_state(0).nc, c0 = E.seg_state(0).c0, nbil = E.num_bilateral(0);
  const double h = s->P.h;
  std::vector<double> hv;
  if (r) {
    if (nc) {
      if (E.precision() == DV_PREC_MIXED)
        TRY(E.download_planes_f(reinterpret_cast<const float*>(E.d.r), E.d.ccap, 3, c0, nc, hv));
      else
        TRY(E.download_planes(E.d.r, E.d.ccap, 3, c0, nc, hv));
      interleave(hv, nc, 3, r + nbil, 3);
    }
    if (nbil) TRY(E.download(r, E.d.bil_work + 10 * (size_t)E.d.nbil, sizeof(double) * nbil));
  }
  if (b) {
    // System.cu:1516-1524: (gap / h, 0, 0) per contact, as the solve kernel forms it
    std::vector<double> g(nc);
    if (nc) TRY(E.download(g.data(), E.d.gap + c0, sizeof(double) * nc));
    for (int i = 0; i < nc; ++i) {
      b[nbil + 3 * (size_t)i] = g[i] / h;
      b[nbil + 3 * (size_t)i + 1] = 0.0;
      b[nbil + 3 * (size_t)i + 2] = 0.0;
    }
    if (nbil) TRY(E.download(b, E.d.bil_b, sizeof(double) * nbil));
  }
  if (k) {
    const int nb = E.d.nb;
    std::vector<double4> k4(nb);
    TRY(E.download(k4.data(), E.d.k4, sizeof(double4) * nb));
    for (int i = 0; i < nb; ++i) {
      k[3 * (size_t)i] = k4[i].x;
      k[3 * (size_t)i + 1] = k4[i].y;
      k[3 * (size_t)i + 2] = k4[i].z;
    }
  }
  return DV_OK;
}

DV_API int dv_get_gamma(dv_scene* s, double* gamma, int32_t cap, int32_t* n) {
  if (!s) return DV_ERR_ARG;
  std::vector<double> g;
  int m = 0;
  TRY(s->E.get_gamma(0, g, &m));
  if (n) *n = m;
  if (!gamma || cap <= 0) return DV_OK;
  int k = std::min(cap, m);
  memcpy(gamma, g.data(), sizeof(double) * 3 * (size_t)k);
  return DV_OK;
}

DV_API int dv_set_gamma(dv_scene* s, const double* gamma, int32_t n) {
  if (!s || n < 0 || (n > 0 && !gamma)) return DV_ERR_ARG;
  return s->E.set_gamma(0, gamma, n);
}

DV_API int dv_add_bilateral_dof(dv_scene* s, int32_t dof_a, int32_t dof_b, double velocity,
                                double start_time) {
  if (!s) return DV_ERR_ARG;
  return s->E.add_bilateral(0, dof_a, dof_b, velocity, start_time);
}

DV_API int dv_get_bilateral_gamma(dv_scene* s, double* gamma, int32_t cap, int32_t* n) {
  if (!s) return DV_ERR_ARG;
  std::vector<double> g;
  TRY(s->E.get_bilateral_gamma(0, g));
  if (n) *n = (int32_t)g.size();
  if (gamma && cap > 0) memcpy(gamma, g.data(), sizeof(double) * std::min((size_t)cap, g.size()));
  return DV_OK;
}

DV_API int dv_ccp_violation(dv_scene* s, double* out4) {
  if (!s || !out4) return DV_ERR_ARG;
  return s->E.ccp_violation(0, out4);
}

DV_API int dv_energies(dv_scene* s, double* kinetic, double* potential) {
  if (!s) return DV_ERR_ARG;
  return s->E.energies(0, kinetic, potential);
}

DV_API int dv_contact_forces_per_collision(dv_scene* s, double* normal, double* friction) {
  if (!s) return DV_ERR_ARG;
  Engine& E = s->E;
  TRY(E.sync_state());
  const int nc = E.seg_state(0).nc, c0 = E.seg_state(0).c0;
  if (nc == 0) return DV_OK;
  std::vector<double> F, g;
  TRY(E.download_planes(E.d.F, E.d.ccap, 9, c0, nc, F));
  int m = 0;
  TRY(E.get_gamma(0, g, &m));
  const double h = s->P.h;
  for (int c = 0; c < nc; ++c) {
    double g0 = c < m ? g[3 * (size_t)c] : 0.0, g1 = c < m ? g[3 * (size_t)c + 1] : 0.0,
           g2 = c < m ? g[3 * (size_t)c + 2] : 0.0;
    for (int k = 0; k < 3; ++k) {
      double nn = F[(size_t)k * nc + c], u = F[(size_t)(3 + k) * nc + c],
             v = F[(size_t)(6 + k) * nc + c];
      if (normal) normal[3 * (size_t)c + k] = (g0 * nn) / h;
      if (friction) friction[3 * (size_t)c + k] = (g1 * u + g2 * v) / h;
    }
  }
  return DV_OK;
}

DV_API int dv_get_step_stats(dv_scene* s, dv_step_stats* out) {
  if (!s || !out) return DV_ERR_ARG;
  *out = s->last;
  return out->status;
}

DV_API int64_t dv_scene_launch_count(dv_scene* s) { return s ? s->E.launches() : -1; }

DV_API int dv_get_step_history(dv_scene* s, dv_step_stats* out, int32_t cap, int32_t* n) {
  if (!s) return DV_ERR_ARG;
  int m = (int)s->history.size();
  if (n) *n = m;
  if (out)
    for (int i = 0; i < std::min(cap, m); ++i) out[i] = s->history[i];
  return DV_OK;
}

DV_API int dv_get_phase_times(dv_scene* s, double* ns, int64_t* counts, int32_t reset) {
  if (!s) return DV_ERR_ARG;
  const EngineWords& w = s->E.words();
  for (int i = 0; i < 8; ++i) {
    if (ns) ns[i] = (double)w.phase_ns[i];
    if (counts) counts[i] = (int64_t)w.phase_count[i];
  }
  if (reset) s->E.clear_phase_times();
  return DV_OK;
}

DV_API int dv_clear_step_history(dv_scene* s) {
  if (!s) return DV_ERR_ARG;
  s->history.clear();
  return DV_OK;
}

}  // extern "C"
