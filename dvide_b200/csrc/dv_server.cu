// dv_server.cu -- serving (continuous batching) over an engine: the serving
// C ABI of include/dvide.h.  No counterpart in the reference.
//
// A round: admit pending requests (FIFO) while a slot, the HBM budget and
// the resident-body limit allow; if the resident set changed, reconfigure the engine (resident
// scenes keep their state on the device); run `steps_per_round` steps of
// every resident scene (fewer when a resident scene needs fewer to finish);
// retire the scenes whose steps are done, copying their final state out.
#include <string.h>

#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <memory>
#include <vector>

#include "dv_engine.h"

using namespace dv;

namespace {

struct Request {
  int64_t id = 0;
  std::vector<dv_body_desc> bodies;
  dv_params P{};
  int nsteps = 0, done = 0, status = DV_OK, rounds = 0;
  int solves = 0, solves_at_tol = 0;
  bool failed = false;  // its scene made a step fail for every scene: retired early
  double t_submit = 0, t_admit = 0, t_done = 0;
  double contact_steps = 0, bytes = 0;
  double it = 0, it_c = 0, rit = 0, rit_c = 0, bt = 0, bt_c = 0, refined = 0, refined_c = 0;
  std::vector<float> step_ms;
  int seg = -1;  // segment index in the current engine layout
};

// Admission estimate of a resident scene's device memory: carried body
// arrays and per-body scratch, contact slots (4 per body) with their solver
// vectors, and the warm-start region (6 per body).
double estimate_bytes(int nb) {
  const double per_body = 6 * 32 + 3 * 32 + 2 * 32 + 16 + 4 * 8;
  const double per_contact = 8 + 72 + 12 + 8 + 24 + 24 + 10 * 24 + 32 + 8 + 16;
  const double per_warm = 24;
  return (double)nb * (per_body + 4.0 * per_contact + 6.0 * per_warm) + 64.0 * 1024.0;
}

double pct(std::vector<float> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  double pos = q * (double)(v.size() - 1);
  size_t i = (size_t)pos;
  double f = pos - (double)i;
  if (i + 1 < v.size()) return v[i] * (1.0 - f) + v[i + 1] * f;
  return v[i];
}

}  // namespace

struct dv_server {
  dv_server_config cfg;
  std::unique_ptr<Engine> E;
  cudaStream_t user_stream = nullptr;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  int64_t next_id = 1;
  std::deque<std::unique_ptr<Request>> pending;
  std::vector<std::unique_ptr<Request>> active;  // engine segment order
  std::vector<dv_request_result> finished;
  std::map<int64_t, std::pair<std::vector<double>, std::vector<double>>> states;
  double bytes_in_use = 0;
  bool departed = false;  // scenes left since the engine layout was built
  dv_server_stats st{};

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  // Rebuilds the engine for `next`: kept[i] = segment index of next[i] in the
  // current engine, or -1 for a newly admitted request.
  int rebuild(std::vector<std::unique_ptr<Request>>& next, const std::vector<int>& kept) {
    std::vector<SlotSpec> slots(next.size());
    for (size_t i = 0; i < next.size(); ++i) {
      slots[i].keep = kept[i];
      if (kept[i] < 0) {
        slots[i].in.bodies = next[i]->bodies.data();
        slots[i].in.nb = (int)next[i]->bodies.size();
        slots[i].in.P = next[i]->P;
        slots[i].in.P.precision = cfg.precision;
      }
    }
    int rc;
    if (!E) {
      std::vector<SceneInput> in(slots.size());
      for (size_t i = 0; i < slots.size(); ++i) in[i] = slots[i].in;
      E.reset(new Engine());
      rc = E->init(in, cfg.precision);
      if (rc == DV_OK && user_stream) rc = E->set_stream(user_stream);
      // FP32 iterates fit three CTAs per SM (80 registers); results do not
      // depend on the launch shape
      if (rc == DV_OK) {
        if (cfg.precision == DV_PREC_MIXED) E->set_launch(E->max_ctas_for(3), 1, 1, 3);
        else E->set_launch(E->max_ctas(), 1, 0, 2);
      }
    } else {
      rc = E->reconfigure(slots);
    }
    if (rc == DV_OK && cfg.use_graph) E->set_graph(true);  // falls back to launches on failure
    st.reconfigures += 1;
    return rc;
  }

  int round(int32_t* busy) {
    // ---- admissions; one engine layout change covers them and the scenes
    // that left in the previous round
    std::vector<std::unique_ptr<Request>> next;
    std::vector<int> kept;
    for (auto& r : active) {
      kept.push_back(r->seg);
      next.push_back(std::move(r));
    }
    active.clear();
    bool changed = departed;
    long long bodies = 0;
    for (auto& r : next) bodies += (long long)r->bodies.size();
    const long long body_cap = cfg.max_resident_bodies;
    while (!pending.empty() && (int)next.size() < cfg.max_active &&
           (next.empty() || bytes_in_use + pending.front()->bytes <= cfg.hbm_budget_bytes) &&
           (body_cap <= 0 || next.empty() ||
            bodies + (long long)pending.front()->bodies.size() <= body_cap)) {
      bodies += (long long)pending.front()->bodies.size();
      std::unique_ptr<Request> r = std::move(pending.front());
      pending.pop_front();
      r->t_admit = now();
      bytes_in_use += r->bytes;
      st.admitted += 1;
      next.push_back(std::move(r));
      kept.push_back(-1);
      changed = true;
    }
    if (next.empty()) {
      E.reset();  // nothing resident: free the device memory
      departed = false;
      if (busy) *busy = 0;
      return DV_OK;
    }
    if (changed || !E) {
      if (!E)
        for (int& k : kept) k = -1;
      int rc = rebuild(next, kept);
      if (rc != DV_OK) {
        active = std::move(next);
        return rc;
      }
      for (size_t i = 0; i < next.size(); ++i) next[i]->seg = (int)i;
      departed = false;
    }
    active = std::move(next);
    // ---- steps
    int k = cfg.steps_per_round;
    for (auto& r : active) k = std::min(k, r->nsteps - r->done);
    k = std::max(k, 1);
    int rc = E->step(k);
    if (rc == DV_ERR_ARG) {
      // a scene over the pair kernels' partner limits fails the step for every
      // scene: retire the requests whose scenes did it (with DV_ERR_ARG and
      // the steps done before), and serve the others from the next round
      bool any = false;
      for (auto& r : active)
        if (E->seg_state(r->seg).err & kErrPartners) {
          r->failed = true;
          r->status = DV_ERR_ARG;
          any = true;
        }
      if (!any) return rc;
    } else if (rc != DV_OK) {
      return rc;
    }
    const std::vector<StepRecord>& R = E->records();
    for (const StepRecord& rec : R) {
      st.steps += 1;
      st.device_ms += rec.ms_total;
      for (auto& r : active) {
        Request& q = *r;
        const SegState& X = rec.sst[q.seg];
        q.contact_steps += X.nc;
        st.contact_steps += X.nc;
        if (X.nc > 0) {
          q.solves += 1;
          if (X.ctl.residual < q.P.tolerance) q.solves_at_tol += 1;
          const double nc = X.nc, ri = X.ctl.refine_it, i0 = X.ctl.iterations - ri;
          q.it += i0;
          q.it_c += i0 * nc;
          q.rit += ri;
          q.rit_c += ri * nc;
          q.bt += X.ctl.backtracks;
          q.bt_c += X.ctl.backtracks * nc;
          if (ri > 0) {
            q.refined += 1;
            q.refined_c += nc;
          }
        }
        q.step_ms.push_back(rec.ms_total);
        if (q.status == DV_OK) q.status = status_from_bits(X.err);
      }
    }
    st.rounds += 1;
    // ---- retirements (their segments stay in the engine until the next layout change)
    std::vector<std::unique_ptr<Request>> stay;
    for (auto& r : active) {
      Request& q = *r;
      q.done += (int)R.size();
      q.rounds += 1;
      if (q.done < q.nsteps && !q.failed) {
        stay.push_back(std::move(r));
        continue;
      }
      q.t_done = now();
      dv_request_result o;
      memset(&o, 0, sizeof(o));
      o.id = q.id;
      o.nb = (int)q.bodies.size();
      o.nsteps = q.done;
      o.status = q.status;
      o.rounds = q.rounds;
      o.solves = q.solves;
      o.solves_at_tolerance = q.solves_at_tol;
      o.t_submit = q.t_submit;
      o.t_admit = q.t_admit;
      o.t_done = q.t_done;
      o.contact_steps = q.contact_steps;
      o.iterations = q.it;
      o.iteration_contacts = q.it_c;
      o.refine_iterations = q.rit;
      o.refine_iteration_contacts = q.rit_c;
      o.backtracks = q.bt;
      o.backtrack_contacts = q.bt_c;
      o.refined_solves = q.refined;
      o.refined_contacts = q.refined_c;
      double sum = 0;
      for (float m : q.step_ms) sum += m;
      o.step_ms_mean = q.step_ms.empty() ? 0.0 : sum / q.step_ms.size();
      o.step_ms_p50 = pct(q.step_ms, 0.50);
      o.step_ms_p99 = pct(q.step_ms, 0.99);
      o.bytes = q.bytes;
      if (cfg.keep_states) {
        const int n = o.nb;
        std::vector<double> p(3 * (size_t)n), v(3 * (size_t)n);
        int rc3 = E->copy_state_out(E->seg_b0(q.seg), n, p.data(), v.data());
        if (rc3 != DV_OK) return rc3;
        states[q.id] = {std::move(p), std::move(v)};
      }
      finished.push_back(o);
      bytes_in_use -= q.bytes;
      st.completed += 1;
      departed = true;
    }
    active = std::move(stay);
    if (active.empty() && departed) {
      E.reset();
      departed = false;
    }
    if (busy) *busy = (!active.empty() || !pending.empty()) ? 1 : 0;
    return DV_OK;
  }
};

extern "C" {

DV_API int dv_server_default_config(dv_server_config* c) {
  if (!c) return DV_ERR_ARG;
  memset(c, 0, sizeof(*c));
  c->hbm_budget_bytes = 150e9;
  c->max_active = 4096;
  c->steps_per_round = 4;
  c->precision = DV_PREC_MIXED;
  c->use_graph = 1;
  c->keep_states = 1;
  return DV_OK;
}

DV_API int dv_server_create(const dv_server_config* cfg, dv_server** out) {
  if (!cfg || !out || cfg->max_active <= 0 || cfg->steps_per_round <= 0 ||
      !(cfg->hbm_budget_bytes > 0) || cfg->max_resident_bodies < 0)
    return DV_ERR_ARG;
  if (cfg->precision != DV_PREC_FP64 && cfg->precision != DV_PREC_MIXED) return DV_ERR_UNSUPPORTED;
  dv_server* s = new dv_server();
  s->cfg = *cfg;
  *out = s;
  return DV_OK;
}

DV_API int dv_server_destroy(dv_server* s) {
  if (!s) return DV_ERR_ARG;
  delete s;
  return DV_OK;
}

DV_API int dv_server_set_stream(dv_server* s, void* cuda_stream) {
  if (!s) return DV_ERR_ARG;
  s->user_stream = (cudaStream_t)cuda_stream;
  if (s->E && cuda_stream) return s->E->set_stream((cudaStream_t)cuda_stream);
  return DV_OK;
}

DV_API double dv_server_clock(dv_server* s) { return s ? s->now() : 0.0; }

DV_API int dv_server_submit(dv_server* s, const dv_body_desc* bodies, int32_t nb,
                            const dv_params* params, int32_t nsteps, int64_t* id) {
  if (!s || !params || nb <= 0 || !bodies || nsteps <= 0) return DV_ERR_ARG;
  std::unique_ptr<Request> r(new Request());
  r->id = s->next_id++;
  r->bodies.assign(bodies, bodies + nb);
  r->P = *params;
  r->nsteps = nsteps;
  r->t_submit = s->now();
  r->bytes = estimate_bytes(nb);
  if (r->bytes > s->cfg.hbm_budget_bytes) return DV_ERR_OOM;
  if (id) *id = r->id;
  s->pending.push_back(std::move(r));
  s->st.submitted += 1;
  return DV_OK;
}

DV_API int dv_server_round(dv_server* s, int32_t* busy) {
  if (!s) return DV_ERR_ARG;
  return s->round(busy);
}

DV_API int dv_server_poll(dv_server* s, dv_request_result* out, int32_t cap, int32_t* n) {
  if (!s) return DV_ERR_ARG;
  int m = std::min((int)s->finished.size(), std::max(cap, 0));
  if (out)
    for (int i = 0; i < m; ++i) out[i] = s->finished[i];
  else
    m = 0;
  s->finished.erase(s->finished.begin(), s->finished.begin() + m);
  if (n) *n = m;
  return DV_OK;
}

DV_API int dv_server_result_state(dv_server* s, int64_t id, double* p, double* v) {
  if (!s) return DV_ERR_ARG;
  auto it = s->states.find(id);
  if (it == s->states.end()) return DV_ERR_ARG;
  if (p) memcpy(p, it->second.first.data(), sizeof(double) * it->second.first.size());
  if (v) memcpy(v, it->second.second.data(), sizeof(double) * it->second.second.size());
  s->states.erase(it);
  return DV_OK;
}

DV_API int dv_server_get_stats(dv_server* s, dv_server_stats* out) {
  if (!s || !out) return DV_ERR_ARG;
  *out = s->st;
  out->pending = (int64_t)s->pending.size();
  out->active = (int64_t)s->active.size();
  out->bytes_in_use = s->bytes_in_use;
  return DV_OK;
}

}  // extern "C"
