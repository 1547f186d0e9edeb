// dv_common.cuh -- shared device helpers for the DVIDE B200 contact step.
//
// Arithmetic here is written so that every result is bit-identical to the
// CPU restatement of the reference (no fused multiply-add: the library is
// compiled with -fmad=false; float square roots and divisions use the
// correctly rounded intrinsics, matching the host sqrtf / float division
// that the reference's helper_math_double.h:58-61, 576-597 performs).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dvide.h"

namespace dv {

constexpr int kThreads = 256;       // threads per CTA in every pass
constexpr int kTileItems = 512;     // items per reduction tile (2 per thread)
constexpr int kItemsPerThread = 2;

// ---------------------------------------------------------------------------
// helper_math_double.h semantics (host build): length = (double)sqrtf(float),
// normalize = v * (double)(1.0f / sqrtf(float(dot))).
// ---------------------------------------------------------------------------
struct d3 {
  double x, y, z;
};

__host__ __device__ inline d3 mk3(double x, double y, double z) { return d3{x, y, z}; }
__device__ inline d3 add3(d3 a, d3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ inline d3 sub3(d3 a, d3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ inline d3 scale3(d3 a, double s) { return mk3(a.x * s, a.y * s, a.z * s); }
__device__ inline d3 neg3(d3 a) { return mk3(-a.x, -a.y, -a.z); }
__device__ inline double dot3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ inline double length3(d3 a) {
  return (double)__fsqrt_rn((float)dot3(a, a));
}
__device__ inline d3 normalize3(d3 a) {
  float s = __fsqrt_rn((float)dot3(a, a));
  double inv = (double)__fdiv_rn(1.0f, s);
  return scale3(a, inv);
}
// The opt-in FP64 forms (not the reference's semantics): double sqrt, then
// 1 / length and a scale, as normalize3 does in float.
__device__ inline double length3x(d3 a, bool exact) {
  return exact ? sqrt(dot3(a, a)) : length3(a);
}
__device__ inline d3 normalize3x(d3 a, bool exact) {
  if (!exact) return normalize3(a);
  const double inv = 1.0 / sqrt(dot3(a, a));
  return scale3(a, inv);
}
__device__ inline d3 cross3(d3 a, d3 b) {
  return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// System.cu:753-762: tangent frame from the stored (B -> A) normal.
__device__ inline void frame_from_normal(d3 n, d3* u, d3* v, bool exact = false) {
  d3 uu;
  if (n.z != 0) {
    uu = normalize3x(mk3(1, 0, -n.x / n.z), exact);
  } else if (n.x != 0) {
    uu = normalize3x(mk3(-n.z / n.x, 0, 1), exact);
  } else {
    uu = normalize3x(mk3(1, -n.x / n.y, 0), exact);
  }
  *u = uu;
  *v = normalize3x(cross3(n, uu), exact);
}

// APGD.cu:47-78: projection of one contact impulse onto the friction cone.
// pow(x, 2.0) is evaluated as x * x.
template <class R>
__device__ inline void project_cone(R& g0, R& g1, R& g2, R mu) {
  R gn = g0;
  R gt = sqrt(g1 * g1 + g2 * g2);
  if (mu == R(0)) {
    g1 = R(0);
    g2 = R(0);
    if (gn < R(0)) g0 = R(0);
  } else if (gt < mu * gn) {
    // inside the cone
  } else if ((gt < -(R(1) / mu) * gn) || (fabs(gn) < R(10e-15))) {
    g0 = R(0);
    g1 = R(0);
    g2 = R(0);
  } else {
    R gnp = (gt * mu + gn) / (mu * mu + R(1));
    R gtp = gnp * mu;
    R ratio = gtp / gt;
    g0 = gnp;
    g1 = ratio * g1;
    g2 = ratio * g2;
  }
}

// ---------------------------------------------------------------------------
// Ordered reduction: the 256 per-thread partials of a CTA are folded as 8
// warps by shuffle-down strides 16..1, then the 8 warp sums by strides 4,2,1.
// The CPU oracle (ordered_sum) folds in exactly this order.
// ---------------------------------------------------------------------------
__device__ inline double warp_fold(double v) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, off);
  return v;
}

// Folds one value per thread of a 256-thread CTA; result valid in thread 0.
// scratch must hold 8 doubles of shared memory.
__device__ inline double block_fold256(double v, double* scratch) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_fold(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    double w = (lane < 8) ? scratch[lane] : 0.0;
#pragma unroll
    for (int off = 4; off >= 1; off >>= 1) w = w + __shfl_down_sync(0xffffffffu, w, off);
    r = w;
  }
  return r;
}

__device__ inline double warp_max(double v) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
  return v;
}

__device__ inline double block_max256(double v, double* scratch) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    double w = (lane < 8) ? scratch[lane] : 0.0;
#pragma unroll
    for (int off = 4; off >= 1; off >>= 1) w = fmax(w, __shfl_down_sync(0xffffffffu, w, off));
    r = w;
  }
  return r;
}

// ---------------------------------------------------------------------------
// Memory-model helpers for the persistent kernels.
// ---------------------------------------------------------------------------
__device__ inline unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ inline void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ inline unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;"
               : "=r"(old)
               : "l"(p), "r"(v)
               : "memory");
  return old;
}
__device__ inline uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---------------------------------------------------------------------------
// Bulk asynchronous copies (TMA, no multicast) into shared memory, completed
// on an mbarrier.  Addresses and sizes must be multiples of 16 bytes.
// ---------------------------------------------------------------------------
__device__ inline uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ inline void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ inline void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ inline void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ inline void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// A hint to bring the line holding *p into L2 (no register, no value).
__device__ inline void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
__device__ inline bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Error bits recorded by kernels (host reads them after the step).
enum : unsigned {
  kErrBarrierTimeout = 1u,
  kErrNaN = 2u,
  kErrBacktrackCap = 4u,
  kErrCapacity = 8u,
  kErrAborted = 16u,
  kErrCopyTimeout = 32u,
  kErrPartners = 64u,     // a sphere has more contact partners than the pair kernel keeps
};

// Longest a CTA waits at a grid barrier before it records a timeout and
// leaves the kernel (a barrier normally completes in microseconds).
constexpr uint64_t kBarrierTimeoutNs = 2000000000ull;

}  // namespace dv

#define DV_CUDA_TRY(expr)                                   \
  do {                                                      \
    cudaError_t e_ = (expr);                                \
    if (e_ != cudaSuccess) return dv_record_cuda_error(e_, #expr, __FILE__, __LINE__); \
  } while (0)

int dv_record_cuda_error(cudaError_t e, const char* what, const char* file, int line);
void dv_set_error_text(const char* text);
