// dv_batch.cu -- the batch C ABI of include/dvide.h: many independent scenes
// stepped by one engine (one collision pipeline and one persistent solve
// kernel per step), optional CUDA-graph replay, and the launch-shape
// autotuner.  No counterpart in the reference (DVIDE steps one System).
#include <string.h>

#include <algorithm>
#include <vector>

#include "dv_engine.h"

using namespace dv;

struct dv_batch {
  Engine E;
  std::vector<int> counts;
};

namespace {

void to_scene_stats(const SegState& X, unsigned ew_err, dv_scene_stats* o) {
  memset(o, 0, sizeof(*o));
  o->num_contacts = X.nc;
  o->num_possible = X.npossible;
  o->iterations = X.ctl.iterations;
  o->backtracks = X.ctl.backtracks;
  o->residual = X.ctl.residual;
  o->objective = X.ctl.objective;
  o->sweeps = X.ctl.sweeps;
  o->refine_iterations = X.ctl.refine_it;
  int st = status_from_bits(ew_err & (kErrBarrierTimeout | kErrCopyTimeout | kErrCapacity | kErrPartners));
  if (st == DV_OK) st = status_from_bits(X.err);
  o->status = st;
}

int copy_state(dv_batch* b, int32_t scene, double* p, double* v, bool upload) {
  Engine& E = b->E;
  int b0 = 0, n = E.d.nb;
  if (scene >= 0) {
    if (scene >= E.nseg()) return DV_ERR_ARG;
    b0 = E.seg_b0(scene);
    n = E.seg_nb(scene);
  }
  return upload ? E.copy_state_in(b0, n, p, v) : E.copy_state_out(b0, n, p, v);
}

}  // namespace

extern "C" {

DV_API int dv_batch_create(const dv_body_desc* bodies, const int32_t* counts, int32_t nscenes,
                           const dv_params* params, int32_t precision, dv_batch** out) {
  if (!out || !bodies || !counts || !params || nscenes <= 0) return DV_ERR_ARG;
  *out = nullptr;
  std::vector<SceneInput> in(nscenes);
  size_t off = 0;
  for (int s = 0; s < nscenes; ++s) {
    if (counts[s] < 0) return DV_ERR_ARG;
    in[s].bodies = bodies + off;
    in[s].nb = counts[s];
    in[s].P = params[s];
    in[s].P.precision = precision;
    off += (size_t)counts[s];
  }
  dv_batch* b = new dv_batch();
  b->counts.assign(counts, counts + nscenes);
  int rc = b->E.init(in, precision);
  if (rc == DV_OK) {
    b->E.set_launch(b->E.max_ctas(), 1, 0, 2);
  } else {
    delete b;
    return rc;
  }
  *out = b;
  return DV_OK;
}

DV_API int dv_batch_destroy(dv_batch* b) {
  if (!b) return DV_ERR_ARG;
  delete b;
  return DV_OK;
}

DV_API int dv_batch_set_stream(dv_batch* b, void* cuda_stream) {
  if (!b) return DV_ERR_ARG;
  return b->E.set_stream((cudaStream_t)cuda_stream);
}

DV_API int dv_batch_step(dv_batch* b, int32_t nsteps) {
  if (!b || nsteps < 0) return DV_ERR_ARG;
  return b->E.step(nsteps);
}

DV_API int dv_batch_num_scenes(dv_batch* b, int32_t* nscenes, int32_t* nbodies) {
  if (!b) return DV_ERR_ARG;
  if (nscenes) *nscenes = b->E.nseg();
  if (nbodies) *nbodies = b->E.d.nb;
  return DV_OK;
}

DV_API int dv_batch_get_state(dv_batch* b, int32_t scene, double* p, double* v) {
  if (!b) return DV_ERR_ARG;
  return copy_state(b, scene, p, v, false);
}

DV_API int dv_batch_set_state(dv_batch* b, int32_t scene, const double* p, const double* v) {
  if (!b) return DV_ERR_ARG;
  return copy_state(b, scene, const_cast<double*>(p), const_cast<double*>(v), true);
}

DV_API int dv_batch_scene_stats(dv_batch* b, dv_scene_stats* out) {
  if (!b || !out) return DV_ERR_ARG;
  const EngineWords& w = b->E.words();
  for (int s = 0; s < b->E.nseg(); ++s) to_scene_stats(b->E.seg_state(s), w.err, out + s);
  return DV_OK;
}

DV_API int dv_batch_step_history(dv_batch* b, dv_scene_stats* out, float* step_ms, int32_t cap_steps,
                                 int32_t* nsteps) {
  if (!b) return DV_ERR_ARG;
  const std::vector<StepRecord>& R = b->E.records();
  const int n = (int)R.size();
  if (nsteps) *nsteps = n;
  const int m = std::min(n, std::max(cap_steps, 0));
  const int ns = b->E.nseg();
  for (int i = 0; i < m; ++i) {
    if (step_ms) step_ms[i] = R[i].ms_total;
    if (out)
      for (int s = 0; s < ns; ++s) to_scene_stats(R[i].sst[s], R[i].ew.err, out + (size_t)i * ns + s);
  }
  return DV_OK;
}

DV_API int dv_batch_get_gamma(dv_batch* b, int32_t scene, double* gamma, int32_t cap, int32_t* n) {
  if (!b || scene < 0 || scene >= b->E.nseg()) return DV_ERR_ARG;
  std::vector<double> g;
  int m = 0;
  int rc = b->E.get_gamma(scene, g, &m);
  if (rc != DV_OK) return rc;
  if (n) *n = m;
  if (gamma && cap > 0) memcpy(gamma, g.data(), sizeof(double) * 3 * (size_t)std::min(cap, m));
  return DV_OK;
}

DV_API int dv_batch_ccp_violation(dv_batch* b, int32_t scene, double* out4) {
  if (!b || !out4 || scene < 0 || scene >= b->E.nseg()) return DV_ERR_ARG;
  return b->E.ccp_violation(scene, out4);
}

DV_API int dv_batch_set_launch(dv_batch* b, int32_t grid, int32_t chunk, int32_t contiguous,
                               int32_t blocks_per_sm) {
  if (!b || chunk < 0) return DV_ERR_ARG;
  b->E.set_launch(grid, chunk, contiguous, blocks_per_sm);
  if (b->E.graph_on()) return b->E.set_graph(true);
  return DV_OK;
}

DV_API int dv_batch_get_launch(dv_batch* b, int32_t* grid, int32_t* chunk, int32_t* contiguous,
                               int32_t* blocks_per_sm, int32_t* max_grid) {
  if (!b) return DV_ERR_ARG;
  SolveConfig c = b->E.launch();
  if (grid) *grid = c.grid;
  if (chunk) *chunk = c.chunk;
  if (contiguous) *contiguous = c.contiguous;
  if (blocks_per_sm) *blocks_per_sm = c.blocks_per_sm;
  if (max_grid) *max_grid = b->E.max_ctas_for(c.blocks_per_sm);
  return DV_OK;
}

DV_API int dv_batch_set_graph(dv_batch* b, int32_t enable) {
  if (!b) return DV_ERR_ARG;
  return b->E.set_graph(enable != 0);
}

DV_API int dv_batch_autotune(dv_batch* b, int32_t steps_per_trial, dv_tune_report* out) {
  if (!b || steps_per_trial <= 0) return DV_ERR_ARG;
  Engine& E = b->E;
  const bool graph = E.graph_on();
  const int G = E.max_ctas();
  const int sms = std::max(1, G / 2);
  struct Cand { int grid, chunk, contiguous, bps; };
  std::vector<Cand> cands = {
      {G, 1, 0, 2}, {G, 2, 0, 2}, {G, 4, 0, 2}, {G, 1, 1, 2}, {sms, 1, 0, 2}, {sms, 2, 0, 2},
      {sms, 1, 1, 2},
  };
  if (E.precision() == DV_PREC_MIXED) {
    const int G3 = E.max_ctas_for(3);
    cands.push_back({G3, 1, 0, 3});
    cands.push_back({G3, 2, 0, 3});
    cands.push_back({G3, 1, 1, 3});
  }
  dv_tune_report rep;
  memset(&rep, 0, sizeof(rep));
  rep.steps_per_trial = steps_per_trial;
  rep.identical = 1;
  int rc = E.snapshot();
  if (rc != DV_OK) return rc;
  uint64_t ref_hash = 0;
  float best_ms = 1e30f;
  int best = 0;
  for (size_t i = 0; i < cands.size() && i < 16; ++i) {
    E.set_launch(cands[i].grid, cands[i].chunk, cands[i].contiguous, cands[i].bps);
    if (graph && E.set_graph(true) != DV_OK) E.set_graph(false);
    if ((rc = E.restore()) != DV_OK) return rc;
    if ((rc = E.step(steps_per_trial)) != DV_OK) return rc;
    float ms = 0;
    for (const StepRecord& r : E.records()) ms += r.ms_total;
    ms /= (float)steps_per_trial;
    uint64_t h = 0;
    if ((rc = E.state_hash(&h)) != DV_OK) return rc;
    if (i == 0) ref_hash = h;
    else if (h != ref_hash) rep.identical = 0;
    dv_tune_candidate& c = rep.cand[rep.num_candidates++];
    c.grid = E.launch().grid;
    c.chunk = cands[i].chunk;
    c.contiguous = cands[i].contiguous;
    c.blocks_per_sm = E.launch().blocks_per_sm;
    c.ms_per_step = ms;
    if (ms < best_ms) {
      best_ms = ms;
      best = (int)i;
    }
  }
  rep.best = best;
  E.set_launch(cands[best].grid, cands[best].chunk, cands[best].contiguous, cands[best].bps);
  if (graph) E.set_graph(true);
  if ((rc = E.restore()) != DV_OK) return rc;
  if (out) *out = rep;
  return rep.identical ? DV_OK : DV_ERR_ARG;
}

DV_API int64_t dv_batch_launch_count(dv_batch* b) { return b ? b->E.launches() : -1; }

}  // extern "C"
