// dv_engine.h -- host side of an engine: the segments (scenes) it steps
// together, device memory, the step loop, optional CUDA-graph replay and the
// per-step records the C ABI reports from.  Used by the plain scene ABI
// (one segment), the batch ABI and the server.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "dv_internal.cuh"

namespace dv {

// One scene handed to an engine: its bodies and parameters.
struct SceneInput {
  const dv_body_desc* bodies = nullptr;
  int nb = 0;
  dv_params P{};
};

// One segment of a new layout: an existing segment carried over (its device
// state, warm start and clock move with it) or a new scene.
struct SlotSpec {
  int keep = -1;
  SceneInput in;
};

// Host copy of what a step left on the device.
struct StepRecord {
  EngineWords ew;
  std::vector<SegState> sst;
  float ms_total = 0, ms_collide = 0, ms_solve = 0;
  double time = 0;
  int time_index = 0;
};

class Engine {
 public:
  Engine() = default;
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  // Allocates and uploads every segment.  Returns DV_OK or an error code.
  int init(const std::vector<SceneInput>& scenes, int precision);

  // Replaces the segment list: carried segments keep their state on the
  // device (gathered into the new layout), new scenes are uploaded.
  int reconfigure(const std::vector<SlotSpec>& slots);

  // Enqueues and runs n steps of every active segment; waits for them.
  // Capacity overflows are repaired (buffers grown) and the failed steps
  // re-run.  Returns the first error status (per-segment solver errors are
  // reported in the records, not here).
  int step(int n);
  // Collision detection only (System::DoTimeStep's first half), synchronous.
  int collide_only();
  // The solve of a step on the current state and the contacts of the last
  // collision detection, without the update (the solver's own solve()):
  // k, r, the solve, gamma into the warm start; v, p, f_contact and the
  // clock are left as they are (PGS leaves its working velocities in v, as
  // the reference's PGS::solve does).  Synchronous.
  int solve_only();

  // Per-step records of the last step() call (one per step, in order).
  const std::vector<StepRecord>& records() const { return recs_; }
  // The last synchronized device words and segment states.
  const EngineWords& words() const { return *h_ew_; }
  const SegState& seg_state(int s) const { return h_sst_[s]; }
  int sync_state();  // waits and refreshes words()/seg_state()

  // Launch shape of the persistent solve kernel (blocks_per_sm 3 only with
  // FP32 iterates; grid <= 0: one CTA per 256 bodies up to the co-resident maximum).
  void set_launch(int grid, int chunk, int contiguous, int blocks_per_sm = 2);
  int max_ctas_for(int blocks_per_sm) const;
  SolveConfig launch() const { return cfg_; }
  int max_ctas() const { return max_ctas_; }
  // CUDA-graph replay of the step (collision + solve); false if capture failed.
  int set_graph(bool on);
  bool graph_on() const { return use_graph_; }
  bool graph_failed() const { return graph_failed_; }

  int set_stream(cudaStream_t s);
  cudaStream_t stream() const { return st_; }
  int set_segment_params(int s, const dv_params& P);
  const dv_params& segment_params(int s) const { return P_[s]; }
  int precision() const { return d.precision; }
  int set_precision(int precision);

  // Bilateral DOF row of segment s (System::addBilateralConstraintDOF,
  // System.cu:510-532): DOF dof_a (3 body + axis) minus DOF dof_b (< 0: dof_a
  // against its position now) at `velocity` from `start_time` on.  Engines of
  // one segment, FP64 APGD, before the first step.
  int add_bilateral(int s, int dof_a, int dof_b, double velocity, double start_time);
  int num_bilateral(int s) const { return hseg_[s].nbil; }
  // The rows' impulses of the last solve (System::gamma_d's first entries).
  int get_bilateral_gamma(int s, std::vector<double>& g);

  // Warm-start (System::gamma_d) of segment s.
  int get_gamma(int s, std::vector<double>& g, int* n);
  int set_gamma(int s, const double* g, int n);

  void clear_phase_times();
  // Plain System semantics: a solver error (NaN, backtracking limit) ends the
  // step() call after the failing step.  Batches keep stepping other scenes.
  int set_stop_on_segment_error(bool on);
  int64_t launches() const { return launches_; }

  // Positions / velocities of bodies [b0, b0 + n) as 3 doubles per body,
  // between host arrays and the device's double4 layout: one contiguous copy
  // plus a pack/unpack kernel (synchronous).  p or v may be null.
  int copy_state_out(int b0, int n, double* p, double* v);
  int copy_state_in(int b0, int n, const double* p, const double* v);

  // Download helpers (synchronous).
  int download(void* dst, const void* src, size_t bytes);
  int download_planes(const double* dev, size_t stride, int k, int first, int n,
                      std::vector<double>& out);  // out: k x n
  int download_planes_f(const float* dev, size_t stride, int k, int first, int n,
                        std::vector<double>& out);

  // System::getCCPViolation (System.cu:1590-1643) and the energies
  // (System.cu:1645-1658) of segment s, with the solver's reduction order.
  int ccp_violation(int s, double* out4);
  int energies(int s, double* kinetic, double* potential);

  // Device copy of the dynamic state (positions, velocities, warm starts,
  // clocks) for trial runs; restore() puts it back.
  int snapshot();
  int restore();
  // FNV-1a hash of the positions and velocities of every body (downloads).
  int state_hash(uint64_t* h);

  double time(int s) const { return time_[s]; }
  int time_index(int s) const { return time_index_[s]; }
  int nseg() const { return d.nseg; }
  int seg_b0(int s) const { return hseg_[s].b0; }
  int seg_nb(int s) const { return hseg_[s].b1 - hseg_[s].b0; }

  SceneDev d;

 private:
  template <class T>
  int dalloc(T** p, size_t n);
  template <class T>
  void dfree(T*& p);
  int alloc_contacts(size_t cap);
  template <class T>
  int ensure(T** p, int* cap, size_t need);
  int grow_warm(double factor, int min_seg_cap, int which);
  int enqueue_step(int rec_index);
  int capture_graph();
  void drop_graph();
  int ensure_records(int n);
  int upload_segments();
  int upload_bilateral();
  int enable_anti_relax();
  int sync_words();
  int ensure_red(size_t n);
  void ordered_sum_dev(const double* items, int n, double* part, int slot);

  cudaStream_t st_ = nullptr;
  bool own_stream_ = false;
  std::vector<void*> allocs_;
  std::vector<SegParams> hseg_;
  std::vector<dv_params> P_;
  std::vector<double> time_;
  std::vector<int> time_index_;
  // bilateral rows (host copy; segment 0 of a one-segment engine)
  std::vector<int> bil_a_, bil_b_;
  std::vector<double> bil_vel_, bil_t0_, bil_p0_;
  int max_ctas_ = 1;
  SolveConfig cfg_{1, 1, 0, 2};
  bool cfg_user_ = false;
  int64_t launches_ = 0;
  // graph
  bool use_graph_ = false, graph_failed_ = false;
  int64_t graph_kernels_ = 0;
  bool stop_on_segment_error_ = false;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t graph_exec_ = nullptr;
  // per-step records and their pinned staging
  std::vector<StepRecord> recs_;
  EngineWords* h_ew_ = nullptr;       // pinned: last synchronized
  SegState* h_sst_ = nullptr;         // pinned: last synchronized
  EngineWords* h_ew_ring_ = nullptr;  // pinned ring, one per step in flight
  SegState* h_sst_ring_ = nullptr;
  int ring_cap_ = 0;
  std::vector<cudaEvent_t> ev_;       // 3 per step in flight
  // capacities and host copies of the layout
  std::vector<int> small_h_, large_h_;
  int nb_cap_ = 0, seg_cap_ = 0, small_cap_ = 0, large_cap_ = 0, ncell_alloc_ = 0, chunk_cap_ = 0;
  // snapshot
  double4* snap_p_ = nullptr;
  double4* snap_v_ = nullptr;
  double* snap_g_ = nullptr;
  uint32_t* snap_id_ = nullptr;
  int* snap_ws_ = nullptr;
  int* snap_wc_ = nullptr;
  size_t snap_wtotal_ = 0;
  int snap_nb_ = 0;
  std::vector<int> snap_gsize_;
  std::vector<double> snap_time_;
  std::vector<int> snap_time_index_;
  // state transfer staging (3 doubles per body)
  double* stage3_ = nullptr;
  size_t stage3_cap_ = 0;
  // diagnostics scratch
  double* d_red_ = nullptr;
  size_t d_red_cap_ = 0;
  double* h_red_ = nullptr;           // pinned, 16 slots
};

template <class T>
inline int Engine::dalloc(T** p, size_t n) {
  if (n == 0) n = 1;
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return dv_record_cuda_error(e, "cudaMalloc", __FILE__, __LINE__);
  }
  allocs_.push_back(q);
  *p = reinterpret_cast<T*>(q);
  return DV_OK;
}

template <class T>
inline void Engine::dfree(T*& p) {
  if (!p) return;
  cudaFree(p);
  auto it = std::find(allocs_.begin(), allocs_.end(), (void*)p);
  if (it != allocs_.end()) allocs_.erase(it);
  p = nullptr;
}

// Host-side helpers shared by the ABI files.
int status_from_bits(unsigned bits);
void fill_step_stats(const StepRecord& r, int s, dv_step_stats* out);

}  // namespace dv
