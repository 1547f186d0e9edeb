// dv_noalloc.cu -- dv_ccp_violation_noalloc: the CCP-violation diagnostic of
// dv_ccp_violation computed from caller-owned device arrays, without any
// device allocation.
//
// Who needs it: callers that may not call cudaMalloc/cudaFree.  An application
// that reserves the device memory up front and hands out sub-buffers from its
// own pool cannot let a library allocate behind its back (the allocation may
// fail, or fragment the pool it manages); a fixed-rate control or serving loop
// cannot afford cudaMalloc/cudaFree, which may synchronise the whole device
// and take milliseconds.  Such a caller passes its own input and output
// buffers; the only scratch is the fixed-size array below, which exists once
// per CUDA context (per device, for the runtime's primary contexts) for the
// lifetime of the process.
//
// Scratch: s_tile_scratch holds 7 values per reduction tile of 512 contacts
// (two sums, two minima with the contact index each holds, a bad-id flag), so
// one call handles at most DV_NOALLOC_MAX_CONTACTS contacts (16,777,216, i.e.
// 32,768 tiles; 1.75 MiB of device memory).  Every slot a call reads is
// written earlier in the same call, so no state carries over between calls
// and nothing needs clearing; but all calls share the one array, so two calls
// whose kernels overlap on the GPU (different streams, no ordering between
// them) race and give wrong results.
//
// Results equal dv_ccp_violation's bit for bit: the sums use the same tile
// fold, and each minimum is the one the allocating path's sequential host
// loop (x = item 0, then x = min(x, item i) in order) returns -- the first
// item, in contact order, holding the smallest value; NaN items after the
// first are passed over, and a NaN first item is the result.
//
// Set-up: host code may not use the array's name as a device address (it is a
// host-side stand-in).  The first call in each CUDA context, with that
// context current, looks the address up with cudaGetSymbolAddress; the
// address is cached under the context's unique id (cuCtxGetId), so a
// context created later -- after cudaDeviceReset, or a driver-API context
// made current by the caller -- gets its own lookup.  Make the first call in
// a context before any stream capture begins in it.
#include <cuda.h>

#include <mutex>

#include "dv_internal.cuh"

namespace {

constexpr int kMaxTiles = DV_NOALLOC_MAX_CONTACTS / dv::kTileItems;
// per tile: sum gamma_n v_n, sum cone^2, min gamma_n, its contact index,
// min v_n, its contact index, bad body id seen (1) or not (0)
constexpr int kSlots = 7;
constexpr int kCacheEntries = 64;

static __device__ __align__(256) double s_tile_scratch[kSlots * kMaxTiles];

// Per-contact items of System::getCCPViolation (System.cu:1605-1643), with
// the stored normal n (B -> A) and the gap taken from normalsAndPenetrations
// (4 doubles per contact) and gamma / v in the reference's 3-per-item layout.
// Returns false (and reads no body) when a body id is not below nb.
__device__ inline bool violation_items(int c, int nb, const double* __restrict__ gamma,
                                       const double* __restrict__ nP,
                                       const uint32_t* __restrict__ ida,
                                       const uint32_t* __restrict__ idb,
                                       const double* __restrict__ v, double mu, double h,
                                       double* gn, double* vn, double* cv2) {
  size_t a = ida[c], b = idb[c];
  if (a >= (size_t)nb || b >= (size_t)nb) return false;
  double g0 = gamma[3 * (size_t)c], g1 = gamma[3 * (size_t)c + 1], g2 = gamma[3 * (size_t)c + 2];
  double d0 = v[3 * a] - v[3 * b], d1 = v[3 * a + 1] - v[3 * b + 1], d2 = v[3 * a + 2] - v[3 * b + 2];
  const double* n = nP + 4 * (size_t)c;
  double dv = (n[0] * d0 + n[1] * d1) + n[2] * d2;
  *gn = g0;
  *vn = n[3] / h + dv;
  double gt = sqrt(g1 * g1 + g2 * g2);
  double cv = mu * g0 - gt;
  if (cv > 0) cv = 0;
  *cv2 = cv * cv;
  return true;
}

// A running minimum with the contact index holding it.  take() keeps the
// earlier item on ties (-0 and +0 compare equal) and never takes a NaN, as
// the sequential loop x = (y < x) ? y : x does after its first item.
struct ArgMin {
  double v;
  int i;  // -1: nothing taken yet
};
__device__ inline void take(ArgMin& m, double v, int i) {
  if (i < 0) return;
  if (m.i < 0 ? !(v != v) : (v < m.v || (v == m.v && i < m.i))) {
    m.v = v;
    m.i = i;
  }
}
__device__ inline ArgMin warp_argmin(ArgMin m) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    const double v = __shfl_down_sync(0xffffffffu, m.v, off);
    const int i = __shfl_down_sync(0xffffffffu, m.i, off);
    take(m, v, i);
  }
  return m;
}
// Result in thread 0.
__device__ inline ArgMin block_argmin(ArgMin m, double* sv, int* si) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  m = warp_argmin(m);
  __syncthreads();
  if (lane == 0) {
    sv[warp] = m.v;
    si[warp] = m.i;
  }
  __syncthreads();
  ArgMin r{0.0, -1};
  if (threadIdx.x == 0)
    for (int w = 0; w < dv::kThreads / 32; ++w) take(r, sv[w], si[w]);
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(dv::kThreads) k_violation_tiles(
    int nc, int nb, const double* __restrict__ gamma, const double* __restrict__ nP,
    const uint32_t* __restrict__ ida, const uint32_t* __restrict__ idb,
    const double* __restrict__ v, double mu, double h, double* __restrict__ tiles) {
  __shared__ double scratch[8];
  __shared__ int iscratch[8];
  __shared__ int s_bad;
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  const int tile = blockIdx.x;
  double s_gv = 0.0, s_cv = 0.0;
  ArgMin m_gn{0.0, -1}, m_vn{0.0, -1};
  for (int m = 0; m < dv::kItemsPerThread; ++m) {
    int c = tile * dv::kTileItems + m * dv::kThreads + threadIdx.x;
    if (c < nc) {
      double gn, vn, cv2;
      if (violation_items(c, nb, gamma, nP, ida, idb, v, mu, h, &gn, &vn, &cv2)) {
        s_gv = s_gv + gn * vn;
        s_cv = s_cv + cv2;
        take(m_gn, gn, c);
        take(m_vn, vn, c);
      } else {
        s_bad = 1;
      }
    }
  }
  double a = dv::block_fold256(s_gv, scratch);
  __syncthreads();
  double b = dv::block_fold256(s_cv, scratch);
  __syncthreads();
  ArgMin c = block_argmin(m_gn, scratch, iscratch);
  ArgMin d = block_argmin(m_vn, scratch, iscratch);
  if (threadIdx.x == 0) {
    tiles[0 * kMaxTiles + tile] = a;
    tiles[1 * kMaxTiles + tile] = b;
    tiles[2 * kMaxTiles + tile] = c.v;
    tiles[3 * kMaxTiles + tile] = (double)c.i;
    tiles[4 * kMaxTiles + tile] = d.v;
    tiles[5 * kMaxTiles + tile] = (double)d.i;
    tiles[6 * kMaxTiles + tile] = s_bad ? 1.0 : 0.0;
  }
}

__global__ void __launch_bounds__(dv::kThreads) k_violation_final(
    int nc, int nb, int nt, const double* tiles, const double* __restrict__ gamma,
    const double* __restrict__ nP, const uint32_t* __restrict__ ida,
    const uint32_t* __restrict__ idb, const double* __restrict__ v, double mu, double h,
    double* __restrict__ out4) {
  __shared__ double scratch[8];
  __shared__ int iscratch[8];
  __shared__ int s_bad;
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  double s_gv = 0.0, s_cv = 0.0;
  ArgMin m_gn{0.0, -1}, m_vn{0.0, -1};
  for (int t = threadIdx.x; t < nt; t += dv::kThreads) {
    s_gv = s_gv + tiles[0 * kMaxTiles + t];
    s_cv = s_cv + tiles[1 * kMaxTiles + t];
    take(m_gn, tiles[2 * kMaxTiles + t], (int)tiles[3 * kMaxTiles + t]);
    take(m_vn, tiles[4 * kMaxTiles + t], (int)tiles[5 * kMaxTiles + t]);
    if (tiles[6 * kMaxTiles + t] != 0.0) s_bad = 1;
  }
  double a = dv::block_fold256(s_gv, scratch);
  __syncthreads();
  double b = dv::block_fold256(s_cv, scratch);
  __syncthreads();
  ArgMin c = block_argmin(m_gn, scratch, iscratch);
  ArgMin d = block_argmin(m_vn, scratch, iscratch);
  if (threadIdx.x == 0) {
    if (s_bad) {
      // a body id not below nb: no item was read for it, the result is void
      const double q = __longlong_as_double(0x7ff8000000000000ll);
      out4[0] = q; out4[1] = q; out4[2] = q; out4[3] = q;
      return;
    }
    // the sequential minimum starts from item 0 itself: a NaN there is the result
    double gn0, vn0, cv0;
    violation_items(0, nb, gamma, nP, ida, idb, v, mu, h, &gn0, &vn0, &cv0);
    double x = (gn0 != gn0) ? gn0 : (c.i < 0 ? gn0 : c.v);
    double y = (vn0 != vn0) ? vn0 : (d.i < 0 ? vn0 : d.v);
    if (x > 0) x = 0;
    if (y > 0) y = 0;
    out4[0] = x;
    out4[1] = y;
    out4[2] = a;
    out4[3] = sqrt(b);
  }
}

__global__ void k_violation_zero(double* out4) {
  out4[0] = 0.0;
  out4[1] = 0.0;
  out4[2] = 0.0;
  out4[3] = 0.0;
}

// ---- the scratch array's device address, per CUDA context ----
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

std::mutex g_setup_mutex;
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;
bool g_fns_tried = false;
struct CacheEntry {
  unsigned long long ctx_id;
  void* addr;
};
CacheEntry g_cache[kCacheEntries];
int g_cache_n = 0, g_cache_next = 0;

// Unique id of the context current on this thread (created for the current
// device if there is none yet).  Caller holds g_setup_mutex.
int current_context_id(unsigned long long* id) {
  if (!g_fns_tried) {
    g_fns_tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(p);
    p = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      g_ctx_id = reinterpret_cast<CtxGetIdFn>(p);
    cudaGetLastError();
  }
  if (!g_ctx_current || !g_ctx_id) {
    dv_set_error_text("dv_ccp_violation_noalloc: the driver offers no cuCtxGetCurrent/cuCtxGetId");
    return DV_ERR_CUDA;
  }
  CUcontext ctx = nullptr;
  if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) {
    // no context yet on this thread: bind the current device's primary context
    int dev = 0;
    DV_CUDA_TRY(cudaGetDevice(&dev));
    DV_CUDA_TRY(cudaSetDevice(dev));
    if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return DV_ERR_CUDA;
  }
  if (g_ctx_id(ctx, id) != CUDA_SUCCESS) return DV_ERR_CUDA;
  return DV_OK;
}

// Device address of s_tile_scratch in the current context.
int scratch_address(double** out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  unsigned long long id = 0;
  int rc = current_context_id(&id);
  if (rc != DV_OK) return rc;
  for (int i = 0; i < g_cache_n; ++i) {
    if (g_cache[i].ctx_id == id) {
      *out = static_cast<double*>(g_cache[i].addr);
      return DV_OK;
    }
  }
  void* p = nullptr;
  DV_CUDA_TRY(cudaGetSymbolAddress(&p, s_tile_scratch));
  const int slot = g_cache_n < kCacheEntries ? g_cache_n++ : g_cache_next;
  if (g_cache_n == kCacheEntries) g_cache_next = (slot + 1) % kCacheEntries;
  g_cache[slot] = CacheEntry{id, p};
  *out = static_cast<double*>(p);
  return DV_OK;
}

}  // namespace

extern "C" DV_API int dv_ccp_violation_noalloc(int32_t nc, int32_t nb, const double* gamma,
                                               const double* nP, const uint32_t* ida,
                                               const uint32_t* idb, const double* v, double mu,
                                               double h, double* out4, void* stream) {
  if (nc < 0 || nb < 0 || !out4 || !(h > 0)) return DV_ERR_ARG;
  if (nc > DV_NOALLOC_MAX_CONTACTS) {
    dv_set_error_text("dv_ccp_violation_noalloc: more contacts than DV_NOALLOC_MAX_CONTACTS "
                      "(16777216); split the call or use dv_ccp_violation");
    return DV_ERR_ARG;
  }
  if (nc > 0 && (!gamma || !nP || !ida || !idb || !v || nb <= 0)) return DV_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* tiles = nullptr;
  int rc = scratch_address(&tiles);
  if (rc != DV_OK) return rc;
  if (nc == 0) {
    k_violation_zero<<<1, 1, 0, st>>>(out4);
    DV_CUDA_TRY(cudaGetLastError());
    return DV_OK;
  }
  int nt = (nc + dv::kTileItems - 1) / dv::kTileItems;
  k_violation_tiles<<<nt, dv::kThreads, 0, st>>>(nc, nb, gamma, nP, ida, idb, v, mu, h, tiles);
  DV_CUDA_TRY(cudaGetLastError());
  k_violation_final<<<1, dv::kThreads, 0, st>>>(nc, nb, nt, tiles, gamma, nP, ida, idb, v, mu, h,
                                                out4);
  DV_CUDA_TRY(cudaGetLastError());
  return DV_OK;
}
