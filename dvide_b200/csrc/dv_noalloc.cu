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
// per device for the lifetime of the process.
//
// Scratch: s_tile_scratch holds 4 partial results per reduction tile of 512
// contacts, so one call handles at most DV_NOALLOC_MAX_CONTACTS contacts
// (16,777,216, i.e. 32,768 tiles; 1 MiB of device memory per device).
// Every slot a call reads is written earlier in the same call, so no state
// carries over between calls and nothing needs clearing; but all calls share
// the one array, so two calls whose kernels overlap on the GPU (different
// streams, no ordering between them) race and give wrong results.
//
// Set-up: host code may not use the array's name as a device address (it is a
// host-side stand-in).  The first call on each device, with that device
// current, looks the address up once with cudaGetSymbolAddress and caches it;
// make that first call before any stream capture begins.
#include <mutex>

#include "dv_internal.cuh"

namespace {

constexpr int kMaxTiles = DV_NOALLOC_MAX_CONTACTS / dv::kTileItems;
constexpr int kSlots = 4;  // sum gamma_n v_n, sum cone^2, min gamma_n, min v_n
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double s_tile_scratch[kSlots * kMaxTiles];

// Per-contact items of System::getCCPViolation (System.cu:1605-1643), with
// the stored normal n (B -> A) and the gap taken from normalsAndPenetrations
// (4 doubles per contact) and gamma / v in the reference's 3-per-item layout.
__device__ inline void violation_items(int c, const double* __restrict__ gamma,
                                       const double* __restrict__ nP,
                                       const uint32_t* __restrict__ ida,
                                       const uint32_t* __restrict__ idb,
                                       const double* __restrict__ v, double mu, double h,
                                       double* gn, double* vn, double* cv2) {
  double g0 = gamma[3 * (size_t)c], g1 = gamma[3 * (size_t)c + 1], g2 = gamma[3 * (size_t)c + 2];
  size_t a = ida[c], b = idb[c];
  double d0 = v[3 * a] - v[3 * b], d1 = v[3 * a + 1] - v[3 * b + 1], d2 = v[3 * a + 2] - v[3 * b + 2];
  const double* n = nP + 4 * (size_t)c;
  double dv = (n[0] * d0 + n[1] * d1) + n[2] * d2;
  *gn = g0;
  *vn = n[3] / h + dv;
  double gt = sqrt(g1 * g1 + g2 * g2);
  double cv = mu * g0 - gt;
  if (cv > 0) cv = 0;
  *cv2 = cv * cv;
}

__global__ void __launch_bounds__(dv::kThreads) k_violation_tiles(
    int nc, int nt, const double* __restrict__ gamma, const double* __restrict__ nP,
    const uint32_t* __restrict__ ida, const uint32_t* __restrict__ idb,
    const double* __restrict__ v, double mu, double h, double* __restrict__ tiles) {
  __shared__ double scratch[8];
  const int tile = blockIdx.x;
  double s_gv = 0.0, s_cv = 0.0, m_gn = INFINITY, m_vn = INFINITY;
  for (int m = 0; m < dv::kItemsPerThread; ++m) {
    int c = tile * dv::kTileItems + m * dv::kThreads + threadIdx.x;
    if (c < nc) {
      double gn, vn, cv2;
      violation_items(c, gamma, nP, ida, idb, v, mu, h, &gn, &vn, &cv2);
      s_gv = s_gv + gn * vn;
      s_cv = s_cv + cv2;
      m_gn = fmin(m_gn, gn);
      m_vn = fmin(m_vn, vn);
    }
  }
  double a = dv::block_fold256(s_gv, scratch);
  __syncthreads();
  double b = dv::block_fold256(s_cv, scratch);
  __syncthreads();
  double c = -dv::block_max256(-m_gn, scratch);
  __syncthreads();
  double d = -dv::block_max256(-m_vn, scratch);
  if (threadIdx.x == 0) {
    tiles[0 * kMaxTiles + tile] = a;
    tiles[1 * kMaxTiles + tile] = b;
    tiles[2 * kMaxTiles + tile] = c;
    tiles[3 * kMaxTiles + tile] = d;
  }
}

__global__ void __launch_bounds__(dv::kThreads) k_violation_final(int nt, const double* tiles,
                                                                  double* __restrict__ out4) {
  __shared__ double scratch[8];
  double s_gv = 0.0, s_cv = 0.0, m_gn = INFINITY, m_vn = INFINITY;
  for (int t = threadIdx.x; t < nt; t += dv::kThreads) {
    s_gv = s_gv + tiles[0 * kMaxTiles + t];
    s_cv = s_cv + tiles[1 * kMaxTiles + t];
    m_gn = fmin(m_gn, tiles[2 * kMaxTiles + t]);
    m_vn = fmin(m_vn, tiles[3 * kMaxTiles + t]);
  }
  double a = dv::block_fold256(s_gv, scratch);
  __syncthreads();
  double b = dv::block_fold256(s_cv, scratch);
  __syncthreads();
  double c = -dv::block_max256(-m_gn, scratch);
  __syncthreads();
  double d = -dv::block_max256(-m_vn, scratch);
  if (threadIdx.x == 0) {
    double x = c, y = d;
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

std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of s_tile_scratch on the current device (looked up once).
int scratch_address(double** out) {
  int dev = 0;
  DV_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return DV_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    DV_CUDA_TRY(cudaGetSymbolAddress(&p, s_tile_scratch));
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<double*>(g_scratch_addr[dev]);
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
  k_violation_tiles<<<nt, dv::kThreads, 0, st>>>(nc, nt, gamma, nP, ida, idb, v, mu, h, tiles);
  DV_CUDA_TRY(cudaGetLastError());
  k_violation_final<<<1, dv::kThreads, 0, st>>>(nt, tiles, out4);
  DV_CUDA_TRY(cudaGetLastError());
  return DV_OK;
}
