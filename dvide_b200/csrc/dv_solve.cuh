// dv_solve.cuh -- device machinery shared by the persistent solve kernels
// (APGD in dv_apgd.cu, PGJ in dv_pgj.cu): kernel arguments, the tangent frame
// and the matrix-free products with the frame, the ordered tile reductions
// (per-warp shuffle folds parked in shared memory, per-scene tile folds), the
// per-scene arrival counters, the grid barrier, the CTA tile sequence and
// segment cache, the body gather, the done mask, and the per-warp staging of
// bulk asynchronous copies.  Every wait has a time limit.
#pragma once

#include <stdio.h>
#include <stdlib.h>

#include "dv_internal.cuh"

namespace dv {

namespace {

constexpr int kNQ = 7;      // partial-sum slots per tile
constexpr int kQMax = kNQ;  // slot of the per-tile maximum
constexpr int kWarps = kThreads / 32;
constexpr int kSub = kThreads;  // contacts per sub-tile

// Phases timed between grid-barrier releases (EngineWords::phase_ns).
enum Phase : int {
  kPhaseSetup = 0,     // k, r, Lipschitz estimate
  kPhaseStep = 1,      // gamma_new = P(y - t g): first iteration or backtrack
  kPhaseRebuild = 2,   // work lists of the segments still iterating
  kPhaseBody = 3,      // body gather w = Minv D^T q
  kPhaseProduct = 4,   // N gamma_new, objective, residual, look-ahead step
  kPhaseFinal = 5,     // gamma = gamma_hat, update
};

template <class T> struct Vec4;
template <> struct Vec4<double> { using type = double4; };
template <> struct Vec4<float> { using type = float4; };

template <class T>
struct KArgs {
  int nb, nseg;
  int solve_only;     // 1: the solve without the update (v, p, f_contact, clock untouched)
  int refine;         // 1: FP64 refinement of the solves a mixed-precision launch marked
  int tcap;           // plane stride of the partials
  int chunk, contiguous;
  size_t S;           // plane stride of contact arrays
  size_t WS;          // plane stride of the warm-start arena
  double4* p4;
  double4* v4;
  double4* k4;
  const double4* __restrict__ f4;
  double4* fc4;
  double4* wd;        // body vector, double4 (setup); reinterpreted as Vec4<T> in iterations
  const double* __restrict__ minv;
  const int* __restrict__ bseg;
  const uint32_t* __restrict__ ida;
  const uint32_t* __restrict__ idb;
  const double* __restrict__ F;
  const float* __restrict__ nf;
  const double* __restrict__ gap;
  T* r;
  const int* __restrict__ inc_start;
  const uint32_t* __restrict__ inc;
  T* G[5];
  T* NG[5];
  double4* qd;        // contact vector q, double4 (final pass); Vec4<T> in iterations
  double* gamma;
  uint32_t* wid;      // matched warm start: B of the pair per warm slot (segment-relative)
  int* ws;            // matched warm start: per body, first warm slot of its A-contacts
  int* wc;            // ... and their count
  const int* __restrict__ cbase;     // this step's contact offsets (unpadded) per body
  const int* __restrict__ cnt_cont;  // this step's contacts with A = body
  double* part;
  const SegParams* __restrict__ seg;
  SegState* sst;
  const int* __restrict__ tseg;
  unsigned* donemask;
  EngineWords* ew;
  int* act_tiles;          // work lists of the iterating passes (EngineWords::act_on)
  int4* act_bodies;
  // bilateral DOF rows (nbil = 0: none; FP64 iterates only)
  int nbil;
  const int2* __restrict__ bil_off;
  const double4* __restrict__ bil_info;
  const int* __restrict__ bil_inc_start;
  const uint32_t* __restrict__ bil_inc;
  T* bG[5];            // iterates of the rows (the contacts' G[k] slot k)
  T* bNG[5];           // their products
  T* br;               // Schur vector of the rows
  T* bq;               // the rows' share of the body gather (the contacts' q)
  double* bil_gam;     // warm start / solution of the rows
  double* bil_b;       // b of the rows (for the CCP violation)
  double* seg_time;    // System::time of each segment at the step's start
  // APGD anti-relaxation (the kAR kernel): r_n and ar planes (current, next;
  // stride S), v = Minv (k + D^T x) of the iterate under test
  double* ar_r0;
  double* ar_v;
  double4* v_ar;
};

template <class T>
struct Frame {
  T n0, n1, n2, u0, u1, u2, v0, v1, v2;
};

// System.cu:753-762 in float arithmetic (mixed path).
__device__ inline void frame_from_normal_f(float n0, float n1, float n2, Frame<float>& f) {
  float ux, uy, uz;
  if (n2 != 0.0f) {
    ux = 1.0f; uy = 0.0f; uz = __fdiv_rn(-n0, n2);
  } else if (n0 != 0.0f) {
    ux = __fdiv_rn(-n2, n0); uy = 0.0f; uz = 1.0f;
  } else {
    ux = 1.0f; uy = __fdiv_rn(-n0, n1); uz = 0.0f;
  }
  float iu = __fdiv_rn(1.0f, __fsqrt_rn(ux * ux + uy * uy + uz * uz));
  ux *= iu; uy *= iu; uz *= iu;
  float vx = n1 * uz - n2 * uy, vy = n2 * ux - n0 * uz, vz = n0 * uy - n1 * ux;
  float iv = __fdiv_rn(1.0f, __fsqrt_rn(vx * vx + vy * vy + vz * vz));
  f.n0 = n0; f.n1 = n1; f.n2 = n2;
  f.u0 = ux; f.u1 = uy; f.u2 = uz;
  f.v0 = vx * iv; f.v1 = vy * iv; f.v2 = vz * iv;
}

// The FP64 frame, recomputed from the stored normal with the narrowphase's own
// function and the scene's mode (same bits as the stored u, v planes).
__device__ inline Frame<double> frame_d(double n0, double n1, double n2, bool exact) {
  d3 u, v;
  frame_from_normal(mk3(n0, n1, n2), &u, &v, exact);
  Frame<double> f;
  f.n0 = n0; f.n1 = n1; f.n2 = n2;
  f.u0 = u.x; f.u1 = u.y; f.u2 = u.z;
  f.v0 = v.x; f.v1 = v.y; f.v2 = v.z;
  return f;
}

// `exact`: the scene's FP64 narrowphase mode (the FP32 frame ignores it).
template <class T> __device__ inline Frame<T> make_frame(T n0, T n1, T n2, bool exact);
template <>
__device__ inline Frame<double> make_frame<double>(double n0, double n1, double n2, bool exact) {
  return frame_d(n0, n1, n2, exact);
}
template <> __device__ inline Frame<float> make_frame<float>(float n0, float n1, float n2, bool) {
  Frame<float> f;
  frame_from_normal_f(n0, n1, n2, f);
  return f;
}

// Normal planes in the solve's precision.
template <class T> __device__ inline const T* normal_planes(const KArgs<T>& a);
template <> __device__ inline const double* normal_planes<double>(const KArgs<double>& a) {
  return a.F;
}
template <> __device__ inline const float* normal_planes<float>(const KArgs<float>& a) {
  return a.nf;
}

template <class T>
__device__ inline Frame<T> load_frame(const KArgs<T>& a, int c, bool exact) {
  const T* n = normal_planes<T>(a);
  return make_frame<T>(n[c], n[a.S + c], n[2 * a.S + c], exact);
}

template <class T>
__device__ inline Frame<double> load_frame_fp64(const KArgs<T>& a, int c, bool exact) {
  return frame_d(__ldg(a.F + c), __ldg(a.F + a.S + c), __ldg(a.F + 2 * a.S + c), exact);
}

// The nine stored frame planes (n, u, v) of contact c, as the narrowphase
// wrote them: the same bits as load_frame_fp64, read instead of rebuilt.
template <class T>
__device__ inline Frame<double> stored_frame(const KArgs<T>& a, int c) {
  const double* F = a.F;
  const size_t S = a.S;
  Frame<double> f;
  f.n0 = __ldg(F + c); f.n1 = __ldg(F + S + c); f.n2 = __ldg(F + 2 * S + c);
  f.u0 = __ldg(F + 3 * S + c); f.u1 = __ldg(F + 4 * S + c); f.u2 = __ldg(F + 5 * S + c);
  f.v0 = __ldg(F + 6 * S + c); f.v1 = __ldg(F + 7 * S + c); f.v2 = __ldg(F + 8 * S + c);
  return f;
}

// Stores of the vectors a pass writes and the next pass reads at once (q for
// the body pass, w for the contact pass's gathers), with an L2 evict-last
// priority: each contact pass streams more contact data than L2 holds, and
// without the hint these lines are the first to go.  A hint, not a value
// change.
__device__ inline uint64_t l2_evict_last_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ inline void store_keep(double4* addr, const double4& v) {
  const uint64_t pol = l2_evict_last_policy();
  asm volatile(
      "st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %5;\n\t"
      "st.global.L2::cache_hint.v2.f64 [%0+16], {%3, %4}, %5;" ::"l"(addr),
      "d"(v.x), "d"(v.y), "d"(v.z), "d"(v.w), "l"(pol)
      : "memory");
}
__device__ inline void store_keep(float4* addr, const float4& v) {
  const uint64_t pol = l2_evict_last_policy();
  asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(addr),
               "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "l"(pol)
               : "memory");
}

// q = F x : q_k = (n_k x0 + u_k x1) + v_k x2
template <class T, class V>
__device__ inline V f_times(const Frame<T>& f, T x0, T x1, T x2) {
  V q;
  q.x = (f.n0 * x0 + f.u0 * x1) + f.v0 * x2;
  q.y = (f.n1 * x0 + f.u1 * x1) + f.v1 * x2;
  q.z = (f.n2 * x0 + f.u2 * x1) + f.v2 * x2;
  q.w = T(0);
  return q;
}

// (F^T d)_row = (f_x d_x + f_y d_y) + f_z d_z with d = w_A - w_B
template <class T, class V>
__device__ inline void ft_times(const Frame<T>& f, V wa, V wb, T* o0, T* o1, T* o2) {
  T d0 = wa.x - wb.x, d1 = wa.y - wb.y, d2 = wa.z - wb.z;
  *o0 = (f.n0 * d0 + f.n1 * d1) + f.n2 * d2;
  *o1 = (f.u0 * d0 + f.u1 * d1) + f.u2 * d2;
  *o2 = (f.v0 * d0 + f.v1 * d1) + f.v2 * d2;
}

// Dot products of the reductions, always in FP64.
template <class A, class B>
__device__ inline double dot3i(A a0, A a1, A a2, B b0, B b1, B b2) {
  return ((double)a0 * (double)b0 + (double)a1 * (double)b1) + (double)a2 * (double)b2;
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

// Folds NS sums (the order of block_fold_multi) and NM maxima of each thread
// with one exchange through shared memory (NS + NM <= 8); thread 0 gets the
// results.
template <int NS, int NM>
__device__ inline void block_fold_sums_maxes(double* v, double* m, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int qi = 0; qi < NS; ++qi) v[qi] = warp_fold(v[qi]);
#pragma unroll
  for (int qi = 0; qi < NM; ++qi) m[qi] = warp_max(m[qi]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int qi = 0; qi < NS; ++qi) scratch[qi * 8 + warp] = v[qi];
#pragma unroll
    for (int qi = 0; qi < NM; ++qi) scratch[(NS + qi) * 8 + warp] = m[qi];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int qi = 0; qi < NS; ++qi) {
      double w = (lane < 8) ? scratch[qi * 8 + lane] : 0.0;
#pragma unroll
      for (int off = 4; off >= 1; off >>= 1) w = w + __shfl_down_sync(0xffffffffu, w, off);
      v[qi] = w;
    }
#pragma unroll
    for (int qi = 0; qi < NM; ++qi) {
      double w = (lane < 8) ? scratch[(NS + qi) * 8 + lane] : 0.0;
#pragma unroll
      for (int off = 4; off >= 1; off >>= 1) w = fmax(w, __shfl_down_sync(0xffffffffu, w, off));
      m[qi] = w;
    }
  }
  __syncthreads();
}

// Segment controller side: folds the segment's per-tile partials, NS sums
// (planes 0..NS-1) in the fixed order -- slot j sums the segment's tiles j,
// j+256, ... in turn, then the 256-slot tree -- and NM maxima (planes
// mplane0, mplane0+1, ...).  All loads of a chunk of U tiles are in flight
// before its sums, which keep the slot order: one L2 round trip per chunk.
template <int NS, int NM, class K>
__device__ inline void fold_tiles_sm(const K& a, int t0, int nt, double* sum_out, double* max_out,
                                     int mplane0, double* scratch) {
  constexpr int U = (NS + NM) <= 2 ? 8 : 4;
  constexpr int AS = NS > 0 ? NS : 1, AM = NM > 0 ? NM : 1;
  const double* p = a.part + t0;
  const size_t tc = (size_t)a.tcap;
  double sum[AS], mx[AM];
#pragma unroll
  for (int qi = 0; qi < AS; ++qi) sum[qi] = 0.0;
#pragma unroll
  for (int qi = 0; qi < AM; ++qi) mx[qi] = 0.0;
  int t = threadIdx.x;
  for (; t + (U - 1) * kThreads < nt; t += U * kThreads) {
    double xs[AS][U], xm[AM][U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
#pragma unroll
      for (int qi = 0; qi < NS; ++qi) xs[qi][u] = __ldcg(p + qi * tc + t + u * kThreads);
#pragma unroll
      for (int qi = 0; qi < NM; ++qi)
        xm[qi][u] = __ldcg(p + (size_t)(mplane0 + qi) * tc + t + u * kThreads);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
#pragma unroll
      for (int qi = 0; qi < NS; ++qi) sum[qi] = sum[qi] + xs[qi][u];
#pragma unroll
      for (int qi = 0; qi < NM; ++qi) mx[qi] = fmax(mx[qi], xm[qi][u]);
    }
  }
  for (; t < nt; t += kThreads) {
#pragma unroll
    for (int qi = 0; qi < NS; ++qi) sum[qi] = sum[qi] + __ldcg(p + qi * tc + t);
#pragma unroll
    for (int qi = 0; qi < NM; ++qi) mx[qi] = fmax(mx[qi], __ldcg(p + (size_t)(mplane0 + qi) * tc + t));
  }
  block_fold_sums_maxes<NS, NM>(sum, mx, scratch);
#pragma unroll
  for (int qi = 0; qi < NS; ++qi) sum_out[qi] = sum[qi];
#pragma unroll
  for (int qi = 0; qi < NM; ++qi) max_out[qi] = mx[qi];
}

template <int NQ, class K>
__device__ inline void fold_tiles(const K& a, int t0, int nt, double (&out)[NQ], double* scratch) {
  fold_tiles_sm<NQ, 0>(a, t0, nt, out, nullptr, 0, scratch);
}

template <int NQ, class K>
__device__ inline void write_partials(const K& a, int tile, const double (&v)[NQ]) {
  if (threadIdx.x == 0) {
#pragma unroll
    for (int qi = 0; qi < NQ; ++qi) a.part[(size_t)qi * a.tcap + tile] = v[qi];
  }
}

// Deferred tile folds.  At the end of a tile each warp folds its partial sums
// with shuffles (strides 16..1) and parks the eight warp results in shared
// memory; fold_parked() later completes the 8-warp tree of every parked tile
// ((w0+w4)+(w2+w6)) + ((w1+w5)+(w3+w7)) -- the order of block_fold_multi --
// and writes the tile partials.  Warps thus run their copy pipelines across
// tiles without a CTA barrier per tile.
constexpr int kMaxDefer = 16;
struct DeferBuf {
  double w[kMaxDefer][kNQ + 1][kWarps];  // [slot][quantity][warp]
  int tile[kMaxDefer];
  int fail;                              // a warp's copy wait timed out
};

template <int NQ, bool kMax>
__device__ inline void park_tile(DeferBuf& B, int slot, int tile, const double (&acc)[NQ], double mx) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    const double v = warp_fold(acc[q]);
    if (lane == 0) B.w[slot][q][warp] = v;
  }
  if (kMax) {
    const double m = warp_max(mx);
    if (lane == 0) B.w[slot][NQ][warp] = m;
  }
  if (threadIdx.x == 0) B.tile[slot] = tile;
}

// Completes the parked tiles (NQ sums into planes 0..NQ-1, the max into
// plane kQMax); returns false if a warp's copy wait had timed out.
template <int NQ, bool kMax, class K>
__device__ inline bool fold_parked(const K& a, DeferBuf& B, int n) {
  __syncthreads();
  const int nq = NQ + (kMax ? 1 : 0);
  for (int i = threadIdx.x; i < n * nq; i += kThreads) {
    const int slot = i / nq, q = i - slot * nq;
    const double* w = B.w[slot][q];
    double r;
    if (kMax && q == NQ)
      r = fmax(fmax(fmax(w[0], w[4]), fmax(w[2], w[6])), fmax(fmax(w[1], w[5]), fmax(w[3], w[7])));
    else
      r = ((w[0] + w[4]) + (w[2] + w[6])) + ((w[1] + w[5]) + (w[3] + w[7]));
    const int plane = (kMax && q == NQ) ? kQMax : q;
    a.part[(size_t)plane * a.tcap + B.tile[slot]] = r;
  }
  __threadfence();
  __syncthreads();
  return B.fail == 0;
}

// Tile arrivals of one segment: a CTA delivers the count of its consecutive
// tiles of segment s at once (after their partials are written).  True, in
// every thread, in the CTA whose delivery completes the segment's tiles.
// ---- maxima reductions of PGJ and PGS (only maxima: no summation order) ----
// max_c -min(0, scale * x_n - |x_t|), a NaN term counting 0 (PGJ.cu:112-142, PGS.cu:335-365)
__device__ inline double pgj_feasible(double xn, double xt1, double xt2, double scale) {
  double v = scale * xn - sqrt(xt1 * xt1 + xt2 * xt2);
  if (v != v) v = 0.0;
  return -fmin(0.0, v);
}

// Per-tile maxima: each warp folds (exact, order-free) and parks them; the
// CTA completes the 8-warp fold later and writes planes 0..NQ-1.
template <int NQ>
__device__ inline void park_max(DeferBuf& B, int slot, int tile, const double (&m)[NQ]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    const double v = warp_max(m[q]);
    if (lane == 0) B.w[slot][q][warp] = v;
  }
  if (threadIdx.x == 0) B.tile[slot] = tile;
}

template <int NQ, class K>
__device__ inline void fold_parked_max(const K& a, DeferBuf& B, int n) {
  __syncthreads();
  for (int i = threadIdx.x; i < n * NQ; i += kThreads) {
    const int slot = i / NQ, q = i - slot * NQ;
    const double* w = B.w[slot][q];
    double r = w[0];
    for (int k = 1; k < kWarps; ++k) r = fmax(r, w[k]);
    a.part[(size_t)q * a.tcap + B.tile[slot]] = r;
  }
  __threadfence();
  __syncthreads();
}


template <class K>
__device__ inline bool seg_arrive(const K& a, int s, int n) {
  __shared__ int s_flag;
  // the tiles' partials were written (and fenced) before the CTA barrier that
  // ends fold_parked
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned nt = (unsigned)a.sst[s].nt;
    unsigned old = atom_add_acq_rel(&a.sst[s].arrive, (unsigned)n);
    int last = (old + (unsigned)n == nt);
    if (last) a.sst[s].arrive = 0u;  // the next pass starts after a grid barrier
    s_flag = last;
  }
  __syncthreads();
  const bool last = s_flag != 0;
  if (last) __threadfence();
  return last;
}

// The segment of a tile and its ranges, cached per CTA for the whole kernel
// (they do not change during a step): tiles of the cached segment need no
// loads to find their contacts.
struct SegCache {
  int s;
  int t0, t1;   // tiles [t0, t1)
  int c0, nc;   // contacts [c0, c0 + nc)
  int gsize;
};

// c is in shared memory; every thread of the CTA calls this with the same t.
template <class K>
__device__ inline void locate(const K& a, SegCache& c, int t) {
  if (t >= c.t0 && t < c.t1) return;
  __syncthreads();
  if (threadIdx.x == 0) {
    const int s = a.tseg[t];
    const SegState& X = a.sst[s];
    c.s = s;
    c.t0 = X.t0;
    c.t1 = X.t0 + X.nt;
    c.c0 = X.c0;
    c.nc = X.nc;
    c.gsize = X.gsize;
  }
  __syncthreads();
}

struct SegRun {
  int s = -1;  // segment of the current run of tiles
  int n = 0;   // tiles of it processed since the last delivery
};

// Delivers the run's arrivals; the CTA that completes the segment runs ctl(s).
template <class K, class Fn>
// `deferred`: the pass's grid barrier runs the controller instead (an engine
// with one segment: its controller follows the last arrival anyway, so the
// arrival counter would only add a serialized atomic to every CTA's exit).
__device__ inline void flush_run(const K& a, SegRun& run, Fn ctl, bool deferred = false) {
  if (run.n == 0) return;
  const int s = run.s, n = run.n;
  run.n = 0;
  if (deferred) return;
  if (seg_arrive(a, s, n)) ctl(s);
}

// Grid barrier.  The last CTA to arrive runs `ctl_fn` (all its threads),
// then releases the generation word.  Returns false after a timeout or an
// error raised by another CTA; the caller then leaves the kernel.
template <class K, class Fn>
__device__ inline bool grid_sync(const K& a, int phase, Fn ctl_fn) {
  __shared__ unsigned s_last, s_target;
  __shared__ int s_fail;
  unsigned* bar = a.ew->bar;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned ticket = atom_add_acq_rel(&bar[0], 1u);
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
      const unsigned long long now = global_ns();
      __threadfence();
      st_release(&bar[1], s_target);
      // Phase timers, after the release so that their round trips to L2 are
      // off the barrier's critical path.  Written by whichever CTA arrives
      // last (no L1-cached copies); the next barrier's last CTA reads them
      // only after this CTA's next arrival, which follows in program order.
      volatile EngineWords* E = a.ew;
      const unsigned long long prev = E->last_release;
      if (prev) {
        E->phase_ns[phase] += now - prev;
        E->phase_count[phase] += 1;
      }
      E->last_release = now;
    }
  } else if (threadIdx.x == 0) {
    const uint64_t limit = a.ew->wait_limit_ns;
    uint64_t t0 = global_ns();
    unsigned polls = 0;
    while (ld_acquire(&bar[1]) < s_target) {
      __nanosleep(20);
      if ((++polls & 1023u) == 0u) {
        if (ld_acquire(&a.ew->err) & (kErrBarrierTimeout | kErrCopyTimeout)) {
          s_fail = 1;
          break;
        }
        if (global_ns() - t0 > limit) {
          atomicOr(&a.ew->err, kErrBarrierTimeout);
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

// Tile i of this CTA's sequence (-1 past the end): round robin in chunks of
// `chunk` consecutive tiles, or one contiguous range per CTA.
template <class K>
__device__ inline int cta_tile(const K& a, int nt, int i) {
  if (a.contiguous) {
    long long lo = (long long)nt * blockIdx.x / gridDim.x;
    long long hi = (long long)nt * (blockIdx.x + 1) / gridDim.x;
    long long t = lo + i;
    return t < hi ? (int)t : -1;
  }
  const int k = a.chunk;
  long long t = ((long long)blockIdx.x + (long long)(i / k) * gridDim.x) * k + (i % k);
  return t < nt ? (int)t : -1;
}

// Tile at sequence index i of this CTA in an iterating pass: position i of the
// work list when it is in use (n = its length; the list is rewritten inside
// the kernel, so it is read through L2), else tile i of all n tiles.
template <class K>
__device__ inline int pass_tile(const K& a, int lon, int n, int i) {
  const int t = cta_tile(a, n, i);
  return (t < 0 || !lon) ? t : __ldcg(a.act_tiles + t);
}

// Eight incidence entries c[0, n) of a body's run (n <= 8): their q gathered
// together, then added to (ax, ay, az) in order, -q for a B side.
template <class T, class V>
__device__ inline void add_q8(const V* q, const uint32_t* c, int n, T& ax, T& ay, T& az) {
  V qq[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    if (j < n) {
      qq[j] = q[c[j] & 0x7fffffffu];
    } else {
      qq[j].x = T(0); qq[j].y = T(0); qq[j].z = T(0); qq[j].w = T(0);
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    if (j < n) {
      if (c[j] & 0x80000000u) {
        ax = ax - qq[j].x; ay = ay - qq[j].y; az = az - qq[j].z;
      } else {
        ax = ax + qq[j].x; ay = ay + qq[j].y; az = az + qq[j].z;
      }
    }
  }
}

// Sum of -q over B-side contacts, then +q over A-side contacts, ascending
// contact order (the flat incidence list).  Sixteen incidence entries are
// read at once (a settled body has about seven contacts, often more than
// eight), their q in two groups of eight; the additions stay in order.
template <class T, class V, class K>
__device__ inline V gather_q(const K& a, const V* q, int s, int e) {
  T ax = T(0), ay = T(0), az = T(0);
  for (int i = s; i < e; i += 16) {
    uint32_t c[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) c[j] = (i + j < e) ? __ldg(a.inc + i + j) : 0u;
    add_q8<T, V>(q, c, e - i, ax, ay, az);
    if (i + 8 < e) add_q8<T, V>(q, c + 8, e - i - 8, ax, ay, az);
  }
  V r;
  r.x = ax; r.y = ay; r.z = az; r.w = T(0);
  return r;
}

// gather_q with the run's first eight entries already loaded (c0; zero past
// the run): entries 8..15 load alongside the first group's q.  The same sums
// in the same order.
template <class T, class V, class K>
__device__ inline V gather_q_pre(const K& a, const V* q, int s, int e, const uint32_t* c0) {
  T ax = T(0), ay = T(0), az = T(0);
  uint32_t c1[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) c1[j] = (s + 8 + j < e) ? __ldg(a.inc + s + 8 + j) : 0u;
  add_q8<T, V>(q, c0, e - s, ax, ay, az);
  if (s + 8 < e) add_q8<T, V>(q, c1, e - s - 8, ax, ay, az);
  for (int i = s + 16; i < e; i += 16) {
    uint32_t c[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) c[j] = (i + j < e) ? __ldg(a.inc + i + j) : 0u;
    add_q8<T, V>(q, c, e - i, ax, ay, az);
    if (i + 8 < e) add_q8<T, V>(q, c + 8, e - i - 8, ax, ay, az);
  }
  V r;
  r.x = ax; r.y = ay; r.z = az; r.w = T(0);
  return r;
}

template <class T, class V, class K>
__device__ inline V gather_q(const K& a, const V* q, int b) {
  return gather_q<T, V>(a, q, __ldg(a.inc_start + b), __ldg(a.inc_start + b + 1));
}

// Bilateral DOF rows.  Tile t of a segment with contacts [0, nc) and tiles
// starting at t0 is a tile of its rows when it lies past the contact tiles;
// returns the tile's first row (segment-relative), else -1.
__device__ inline int bil_tile_k0(int t, int t0, int nc) {
  const int ntc = (nc + kTileItems - 1) / kTileItems;
  return (t - t0) >= ntc ? (t - t0 - ntc) * kTileItems : -1;
}

// Row i of D w (System.cu:622-638): w[A] - w[B], or w[A] for one DOF.  o holds
// the DOFs' element offsets (4 body + axis) into a 4-wide body vector.
template <class T>
__device__ inline T bil_dw(int2 o, const T* w) {
  const T wa = w[o.x];
  return o.y >= 0 ? wa - w[o.y] : wa;
}

// The rows' part of (D^T x)_b, added after the contacts' part: +x_i at DOF A,
// -x_i at DOF B, ascending rows.  x is written inside the kernel (read through L2).
template <class T, class V>
__device__ inline void add_bilateral(const int* __restrict__ start, const uint32_t* __restrict__ inc,
                                     const T* x, int b, V& s) {
  const int e0 = __ldg(start + b), e1 = __ldg(start + b + 1);
  for (int e = e0; e < e1; ++e) {
    const uint32_t code = __ldg(inc + e);
    const T v = __ldcg(x + (code >> 3));
    const int k = (code >> 1) & 3;
    if (code & 1u) {
      if (k == 0) s.x = s.x - v; else if (k == 1) s.y = s.y - v; else s.z = s.z - v;
    } else {
      if (k == 0) s.x = s.x + v; else if (k == 1) s.y = s.y + v; else s.z = s.z + v;
    }
  }
}

// A solver error of segment s; with stop_on_seg_err it also stops the steps
// that follow (every kernel checks EngineWords::err first).
// A segment's APGD words as its controller finds them: controllers of earlier
// passes ran on other CTAs, so every field is read through L2, with all the
// loads in flight together (one round trip instead of one per field).
__device__ inline ApgdCtl ctl_read(const ApgdCtl* C) {
  ApgdCtl c;
  c.L = __ldcg(&C->L); c.t = __ldcg(&C->t); c.theta = __ldcg(&C->theta);
  c.theta_new = __ldcg(&C->theta_new); c.beta = __ldcg(&C->beta);
  c.obj1 = __ldcg(&C->obj1); c.obj2 = __ldcg(&C->obj2); c.obj2_base = __ldcg(&C->obj2_base);
  c.residual = __ldcg(&C->residual); c.objective = __ldcg(&C->objective);
  c.gdiff = __ldcg(&C->gdiff); c.ginv = __ldcg(&C->ginv); c.L0 = __ldcg(&C->L0);
  c.fx = __ldcg(&C->fx); c.yb = __ldcg(&C->yb);
  c.k = __ldcg(&C->k); c.mode = __ldcg(&C->mode); c.done = __ldcg(&C->done);
  c.restart = __ldcg(&C->restart); c.cur = __ldcg(&C->cur); c.prev = __ldcg(&C->prev);
  c.nw = __ldcg(&C->nw); c.best = __ldcg(&C->best); c.yr = __ldcg(&C->yr);
  c.first = __ldcg(&C->first); c.backtracks = __ldcg(&C->backtracks); c.err = __ldcg(&C->err);
  c.iterations = __ldcg(&C->iterations); c.sweeps = __ldcg(&C->sweeps);
  c.rsel = __ldcg(&C->rsel);
  c.since_best = __ldcg(&C->since_best);
  return c;
}

template <class K>
__device__ inline void seg_error(const K& a, int s, unsigned bit) {
  atomicOr(&a.sst[s].err, bit);
  if (a.ew->stop_on_seg_err) atomicOr(&a.ew->err, bit);
}

// Done mask: bit s set when segment s is not iterating.  Each pass starts
// with a copy in shared memory (segments beyond kMaskWords * 32 read it from
// global memory).
constexpr int kMaskWords = 256;

template <class K>
__device__ inline void load_mask(const K& a, unsigned* s_mask, int mwords) {
  if (a.nseg == 1) return;  // a single segment iterates while the loop runs
  __syncthreads();
  for (int i = threadIdx.x; i < mwords && i < kMaskWords; i += kThreads)
    s_mask[i] = __ldcg(a.donemask + i);
  __syncthreads();
}

template <class K>
__device__ inline bool mask_done(const K& a, const unsigned* s_mask, int mwords, int s) {
  if (a.nseg == 1) return false;
  const int w = s >> 5;
  const unsigned m = (w < kMaskWords) ? s_mask[w] : __ldcg(a.donemask + w);
  return (m >> (s & 31)) & 1u;
}

// Segment s stops iterating (controller thread).
template <class K>
__device__ inline void mark_done(const K& a, int s) {
  volatile ApgdCtl* C = &a.sst[s].ctl;
  C->done = 1;
  atomicOr(a.donemask + (s >> 5), 1u << (s & 31));
}

// Schur body pass: w_b = minv_b * (D^T x)_b for bodies of iterating
// segments; fixed bodies keep w = 0.
// w_b of one body of an iterating segment.
// kAR: also v = Minv (k + D^T x) for the anti-relaxation (APGD.cu:338-340;
// 0 for fixed bodies, whose v enters only as squares).
// The words a body's gather starts from: its inverse mass, the bounds of its
// incidence run and (batches) its segment, loaded together so that they cost
// one memory round trip, and loaded a round ahead by the body pass.
struct BodyHead {
  double mi;
  int s, e, seg;
};

template <class K>
__device__ inline BodyHead body_head(const K& a, int b) {
  BodyHead h;
  h.mi = __ldg(a.minv + b);
  h.s = __ldg(a.inc_start + b);
  h.e = __ldg(a.inc_start + b + 1);
  h.seg = a.nseg > 1 ? __ldg(a.bseg + b) : 0;
  return h;
}

// kPre: c0 holds the body's first eight incidence entries, loaded a round
// ahead by the body pass (zero past its run).
template <class T, bool kAR = false, bool kPre = false>
__device__ inline void body_w(const KArgs<T>& a, int b, const BodyHead& h,
                              const uint32_t* c0 = nullptr) {
  using V = typename Vec4<T>::type;
  V* w = reinterpret_cast<V*>(a.wd);
  const V* q = reinterpret_cast<const V*>(a.qd);
  const double mi = h.mi;
  if (mi != 0.0) {
    V s = kPre ? gather_q_pre<T, V>(a, q, h.s, h.e, c0) : gather_q<T, V>(a, q, h.s, h.e);
    if (a.nbil) add_bilateral<T, V>(a.bil_inc_start, a.bil_inc, a.bq, b, s);
    T m = (T)mi;
    V o;
    o.x = m * s.x; o.y = m * s.y; o.z = m * s.z; o.w = T(0);
    store_keep(w + b, o);
    if (kAR) {
      const double4 k = a.k4[b];
      a.v_ar[b] = make_double4(mi * (k.x + (double)s.x), mi * (k.y + (double)s.y),
                               mi * (k.z + (double)s.z), 0.0);
    }
  } else if (kAR) {
    a.v_ar[b] = make_double4(0.0, 0.0, 0.0, 0.0);
  } else if (sizeof(T) != sizeof(double)) {
    // the FP32 view of w overlays the FP64 setup values: store the zero
    V o;
    o.x = T(0); o.y = T(0); o.z = T(0); o.w = T(0);
    store_keep(w + b, o);
  }
}

// Schur body pass: w_b = minv_b * (D^T x)_b for bodies of iterating
// segments; fixed bodies keep w = 0.  With the work lists in use (lon), over
// the listed body ranges (one segment each) instead of every body.
template <class T, bool kAR = false>
__device__ inline void body_pass_schur(const KArgs<T>& a, const unsigned* s_mask, int lon = 0,
                                       int nlist = 0) {
  const int mwords = (a.nseg + 31) >> 5;
  if (lon) {
    for (int p = blockIdx.x; p < nlist; p += gridDim.x) {
      const int4 r = __ldcg(a.act_bodies + p);
      if (mask_done(a, s_mask, mwords, r.z)) continue;
      const int b = r.x + threadIdx.x;
      if (b < r.y) body_w<T, kAR>(a, b, body_head(a, b));
    }
    return;
  }
  // heads load into registers two rounds ahead, and each body's first eight
  // incidence entries one round ahead, while the current round gathers
  const int stride = gridDim.x * kThreads;
  int b = blockIdx.x * kThreads + threadIdx.x;
  BodyHead h{0.0, 0, 0, 0}, hn{0.0, 0, 0, 0};
  if (b < a.nb) h = body_head(a, b);
  if (b + stride < a.nb) hn = body_head(a, b + stride);
  uint32_t c[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) c[j] = (h.s + j < h.e) ? __ldg(a.inc + h.s + j) : 0u;
  for (; b < a.nb; b += stride) {
    const int bnn = b + 2 * stride;
    BodyHead hnn{0.0, 0, 0, 0};
    if (bnn < a.nb) hnn = body_head(a, bnn);
    uint32_t cn[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) cn[j] = (hn.s + j < hn.e) ? __ldg(a.inc + hn.s + j) : 0u;
    if (a.nseg == 1 || !mask_done(a, s_mask, mwords, h.seg)) body_w<T, kAR, true>(a, b, h, c);
    h = hn;
    hn = hnn;
#pragma unroll
    for (int j = 0; j < 8; ++j) c[j] = cn[j];
  }
}

// Work lists of the segments still iterating (CTA 0, all its threads): their
// contact tiles in segment order into act_tiles and their bodies, in ranges of
// at most kThreads within one segment, into act_bodies.  Reads the done mask
// as the last product pass left it.
template <class T>
__device__ inline void rebuild_work_lists(const KArgs<T>& a, int* sbuf) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int base_t = 0, base_b = 0;
  for (int s0 = 0; s0 < a.nseg; s0 += kThreads) {
    const int s = s0 + tid;
    int ct = 0, cb = 0, t0 = 0, b0 = 0, b1 = 0;
    if (s < a.nseg && !((__ldcg(a.donemask + (s >> 5)) >> (s & 31)) & 1u)) {
      ct = a.sst[s].nt;
      t0 = a.sst[s].t0;
      b0 = a.seg[s].b0;
      b1 = a.seg[s].b1;
      cb = (b1 - b0 + kThreads - 1) / kThreads;
    }
    // exclusive scans of ct and cb over the block (warp shuffles, then warp totals)
    int it = ct, ib = cb;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int ut = __shfl_up_sync(0xffffffffu, it, off);
      const int ub = __shfl_up_sync(0xffffffffu, ib, off);
      if (lane >= off) {
        it += ut;
        ib += ub;
      }
    }
    __syncthreads();
    if (lane == 31) {
      sbuf[warp] = it;
      sbuf[kWarps + warp] = ib;
    }
    __syncthreads();
    int wt = 0, wb = 0, tt = 0, tb = 0;
    for (int k = 0; k < kWarps; ++k) {
      if (k < warp) {
        wt += sbuf[k];
        wb += sbuf[kWarps + k];
      }
      tt += sbuf[k];
      tb += sbuf[kWarps + k];
    }
    const int et = base_t + wt + it - ct, eb = base_b + wb + ib - cb;
    for (int j = 0; j < ct; ++j) a.act_tiles[et + j] = t0 + j;
    for (int j = 0; j < cb; ++j) {
      const int lo = b0 + j * kThreads;
      a.act_bodies[eb + j] = make_int4(lo, min(b1, lo + kThreads), s, 0);
    }
    base_t += tt;
    base_b += tb;
  }
  __threadfence();
  if (tid == 0) {
    a.ew->act_nt = base_t;
    a.ew->act_nb = base_b;
  }
}

// A buffer holding none of the iterates in use (5 buffers, at most 4 in use).
__device__ inline int free_slot(int a, int b, int c, int d) {
  for (int i = 0; i < 5; ++i)
    if (i != a && i != b && i != c && i != d) return i;
  return 0;
}

// ---------------------------------------------------------------------------
// Shared-memory staging of the look-ahead pass, per warp.  A CTA walks its
// sub-tiles (256 consecutive contacts, kItemsPerThread per reduction tile) in
// order; warp w owns contacts [32w, 32w+32) of each sub-tile and two stages of
// its own.  While the warp computes sub-tile i from one stage, its lane 0 has
// already issued the bulk copies of sub-tile i+1's plane segments (32 values
// per plane) into the other stage, completed on the warp's own mbarrier, so
// warps never wait for each other except at the per-tile reduction.
// Planes: n (3), gamma_new (3), r (3), gamma_k (3), N gamma_k (3); ids A, B.
// A segment's contacts start on a multiple of 256, so every copy starts on a
// 128-byte boundary.
// ---------------------------------------------------------------------------
constexpr int kStagePlanes = 15;
template <class T>
__host__ __device__ constexpr unsigned warp_stage_bytes() {
  return (unsigned)kStagePlanes * 32u * (unsigned)sizeof(T) + 2u * 32u * 4u;
}
template <class T>
__host__ __device__ constexpr size_t dyn_smem_bytes() {
  return (size_t)kWarps * 2 * warp_stage_bytes<T>() + (size_t)kWarps * 2 * 8 + 16;
}

struct Staging {
  unsigned char* base;  // warp w, stage s at base + (2w + s) * stage_bytes
  unsigned stage_bytes;
  uint64_t* bar;        // mbarrier of warp w, stage s: bar[2w + s]
  unsigned phase;       // bit s: parity the next wait on this warp's stage s expects
};

// Per warp, bit s: copies issued into stage s and not yet seen complete; one
// byte per warp after the mbarriers (lane 0 writes it).
__device__ inline volatile unsigned char* stage_pending(const Staging& st) {
  return reinterpret_cast<volatile unsigned char*>(st.bar + 2 * kWarps) + (threadIdx.x >> 5);
}
__device__ inline void mark_stage_issued(const Staging& st, int s) {
  if ((threadIdx.x & 31) == 0) *stage_pending(st) |= (unsigned char)(1u << s);
}

// Waits for the phase of parity `parity` of an mbarrier to complete; false
// after `*limit_ns` (read only if the first test fails).
__device__ inline bool bounded_mbar_wait(uint64_t* bar, unsigned parity,
                                         const unsigned long long* limit_ns) {
  bool ok = mbar_try_wait(bar, parity);
  if (!ok) {
    const uint64_t limit = *limit_ns;
    const uint64_t t0 = global_ns();
    while (!(ok = mbar_try_wait(bar, parity))) {
      if (global_ns() - t0 > limit) break;
    }
  }
  return ok;
}

// Bounded wait on this warp's stage s.
__device__ inline bool bounded_stage_wait(Staging& st, int s, const unsigned long long* limit_ns) {
  const int w = threadIdx.x >> 5;
  const unsigned par = (st.phase >> s) & 1u;
  uint64_t* bar = st.bar + 2 * w + s;
  const bool ok = bounded_mbar_wait(bar, par, limit_ns);
  if (ok) {
    st.phase ^= (1u << s);
    if ((threadIdx.x & 31) == 0) *stage_pending(st) &= (unsigned char)~(1u << s);
  }
  return ok;
}

// Waits for this warp's stage s; false after a timeout (error recorded, the
// stage left pending for drain_warp_stages).
template <class K>
__device__ inline bool wait_warp_stage(const K& a, Staging& st, int s) {
  const bool ok = bounded_stage_wait(st, s, &a.ew->wait_limit_ns);
  if (!ok && (threadIdx.x & 31) == 0) atomicOr(&a.ew->err, kErrCopyTimeout);
  __syncwarp();
  return ok;
}

// Before a CTA leaves the kernel early: waits once more, again with a time
// limit, for the copies this warp still has in flight into its stages.
__device__ __noinline__ void drain_warp_stages(Staging st, const unsigned long long* limit_ns) {
  __syncwarp();
  const unsigned pend = __shfl_sync(0xffffffffu, (unsigned)*stage_pending(st), 0);
  for (int s = 0; s < 2; ++s)
    if ((pend >> s) & 1u) bounded_stage_wait(st, s, limit_ns);
  __syncwarp();
}

// Kernel arguments of the solve kernels for an engine and a launch shape.
template <class T>
KArgs<T> make_kargs(SceneDev& sd, const SolveConfig& cfg) {
  KArgs<T> a;
  a.nb = sd.nb;
  a.nseg = sd.nseg;
  a.solve_only = 0;
  a.refine = 0;
  a.tcap = sd.tcap;
  a.chunk = cfg.chunk > 0 ? cfg.chunk : 1;
  a.contiguous = cfg.contiguous;
  a.S = sd.ccap;
  a.WS = sd.wtotal;
  a.p4 = sd.p4;
  a.v4 = sd.v4;
  a.k4 = sd.k4;
  a.f4 = sd.f4;
  a.fc4 = sd.fc4;
  a.wd = sd.w4;
  a.minv = sd.minv;
  a.bseg = sd.bseg;
  a.ida = sd.ida;
  a.idb = sd.idb;
  a.F = sd.F;
  a.nf = sd.nf;
  a.gap = sd.gap;
  a.r = reinterpret_cast<T*>(sd.r);
  a.inc_start = sd.inc_start;
  a.inc = sd.inc;
  for (int k = 0; k < 5; ++k) {
    a.G[k] = reinterpret_cast<T*>(sd.G[k]);
    a.NG[k] = reinterpret_cast<T*>(sd.NG[k]);
  }
  a.qd = sd.q;
  a.gamma = sd.gamma;
  a.wid = sd.wid;
  a.ws = sd.ws;
  a.wc = sd.wc;
  a.cbase = sd.cbase;
  a.cnt_cont = sd.cnt_cont;
  a.part = sd.part;
  a.seg = sd.seg;
  a.sst = sd.sst;
  a.tseg = sd.tseg;
  a.donemask = sd.donemask;
  a.ew = sd.ew;
  a.act_tiles = sd.act_tiles;
  a.act_bodies = sd.act_bodies;
  a.nbil = sizeof(T) == sizeof(double) ? sd.nbil : 0;
  a.bil_off = sd.bil_off;
  a.bil_info = sd.bil_info;
  a.bil_inc_start = sd.bil_inc_start;
  a.bil_inc = sd.bil_inc;
  T* bw = a.nbil ? reinterpret_cast<T*>(sd.bil_work) : nullptr;
  const size_t nbl = (size_t)sd.nbil;
  for (int k = 0; k < 5; ++k) {
    a.bG[k] = bw ? bw + k * nbl : nullptr;
    a.bNG[k] = bw ? bw + (5 + k) * nbl : nullptr;
  }
  a.br = bw ? bw + 10 * nbl : nullptr;
  a.bq = bw ? bw + 11 * nbl : nullptr;
  a.bil_gam = sd.bil_gam;
  a.bil_b = sd.bil_b;
  a.seg_time = sd.seg_time;
  a.ar_r0 = sd.ar_r0;
  a.ar_v = sd.ar_v;
  a.v_ar = sd.v_ar;
  return a;
}

}  // namespace

}  // namespace dv
