// dv_diag.cu -- diagnostics of one segment: System::getCCPViolation
// (System.cu:1590-1643) and the kinetic / potential energies
// (System.cu:1645-1658).  Sums use the solver's ordered reduction (tiles of
// 512 items, fixed fold order), so the CPU oracle reproduces them bit for bit.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "dv_engine.h"

namespace dv {

namespace {

__global__ void __launch_bounds__(kThreads) k_items_partials(const double* __restrict__ items, int n,
                                                             double* __restrict__ part) {
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
    int nc, int c0, size_t S, int w0, size_t WS, const double* __restrict__ gamma,
    const double* __restrict__ F, const double* __restrict__ gap, const uint32_t* __restrict__ ida,
    const uint32_t* __restrict__ idb, const double4* __restrict__ v4, double h, double mu,
    double* __restrict__ items) {
  int k = blockIdx.x * kThreads + threadIdx.x;
  if (k >= nc) return;
  int c = c0 + k;
  double g0 = gamma[w0 + k], g1 = gamma[WS + w0 + k], g2 = gamma[2 * WS + w0 + k];
  double4 va = v4[ida[c]], vb = v4[idb[c]];
  double d0 = va.x - vb.x, d1 = va.y - vb.y, d2 = va.z - vb.z;
  double dv = (F[c] * d0 + F[S + c] * d1) + F[2 * S + c] * d2;
  double vn = gap[c] / h + dv;
  double gt = sqrt(g1 * g1 + g2 * g2);
  double cv = mu * g0 - gt;
  if (cv > 0) cv = 0;
  items[k] = g0;
  items[(size_t)nc + k] = vn;
  items[2 * (size_t)nc + k] = g0 * vn;
  items[3 * (size_t)nc + k] = cv * cv;
}

// The same items with bilateral rows.  The reference reads entries 3 c,
// 3 c + 1, 3 c + 2 of gamma and of D v + b, vectors whose first nbil entries
// are the bilateral rows, with no offset (getNormalComponent,
// calculateConeViolation, System.cu:1590-1603): flat entry j < nbil is row j,
// entry j >= nbil component (j - nbil) % 3 of contact (j - nbil) / 3.
__global__ void __launch_bounds__(kThreads) k_violation_items_flat(
    int nc, int nbil, int c0, size_t S, int w0, size_t WS, const double* __restrict__ gamma,
    const double* __restrict__ bil_gam, const double* __restrict__ bil_b,
    const int2* __restrict__ bil_off, const double* __restrict__ F, const double* __restrict__ gap,
    const uint32_t* __restrict__ ida, const uint32_t* __restrict__ idb,
    const double4* __restrict__ v4, double h, double mu, double* __restrict__ items) {
  int k = blockIdx.x * kThreads + threadIdx.x;
  if (k >= nc) return;
  const double* vd = reinterpret_cast<const double*>(v4);
  auto gam = [&](long long j) -> double {
    if (j < nbil) return bil_gam[j];
    const long long q = j - nbil;
    return gamma[(q % 3) * WS + w0 + q / 3];
  };
  // entry j of D v + b (b: the last step's)
  auto dvb = [&](long long j) -> double {
    if (j < nbil) {
      const int2 o = bil_off[j];
      const double dv = o.y >= 0 ? vd[o.x] - vd[o.y] : vd[o.x];
      return bil_b[j] + dv;
    }
    const long long q = j - nbil;
    const int row = (int)(q % 3);
    const int c = c0 + (int)(q / 3);
    const double4 va = v4[ida[c]], vb = v4[idb[c]];
    const double d0 = va.x - vb.x, d1 = va.y - vb.y, d2 = va.z - vb.z;
    const double* f = F + (size_t)(3 * row) * S + c;
    const double dv = (f[0] * d0 + f[S] * d1) + f[2 * S] * d2;
    return (row == 0 ? gap[c] / h : 0.0) + dv;
  };
  const long long j = 3LL * k;
  const double g0 = gam(j), g1 = gam(j + 1), g2 = gam(j + 2);
  const double vn = dvb(j);
  double gt = sqrt(g1 * g1 + g2 * g2);
  double cv = mu * g0 - gt;
  if (cv > 0) cv = 0;
  items[k] = g0;
  items[(size_t)nc + k] = vn;
  items[2 * (size_t)nc + k] = g0 * vn;
  items[3 * (size_t)nc + k] = cv * cv;
}

__global__ void __launch_bounds__(kThreads) k_energy_items(int nb, int b0,
                                                           const double4* __restrict__ p4,
                                                           const double4* __restrict__ v4,
                                                           const double4* __restrict__ f4,
                                                           const double* __restrict__ minv,
                                                           double* __restrict__ items) {
  int i = blockIdx.x * kThreads + threadIdx.x;
  if (i >= nb) return;
  int b = b0 + i;
  double m = minv[b];
  if (m) m = 1.0 / m;
  double4 v = v4[b], p = p4[b], f = f4[b];
  items[i] = (v.x * (m * v.x) + v.y * (m * v.y)) + v.z * (m * v.z);
  items[(size_t)nb + i] = (f.x * p.x + f.y * p.y) + f.z * p.z;
}

}  // namespace

int Engine::ensure_red(size_t n) {
  if (!h_red_) {
    if (cudaMallocHost(&h_red_, 16 * sizeof(double)) != cudaSuccess)
      return dv_record_cuda_error(cudaErrorMemoryAllocation, "cudaMallocHost", __FILE__, __LINE__);
  }
  if (n <= d_red_cap_) return DV_OK;
  dfree(d_red_);
  d_red_cap_ = n;
  return dalloc(&d_red_, n);
}

// Ordered sum of `n` device items; the result lands in h_red_[slot] after a sync.
void Engine::ordered_sum_dev(const double* items, int n, double* part, int slot) {
  int nt = std::max(1, (n + kTileItems - 1) / kTileItems);
  k_items_partials<<<nt, kThreads, 0, st_>>>(items, n, part);
  k_items_final<<<1, kThreads, 0, st_>>>(part, nt, part + nt);
  cudaMemcpyAsync(h_red_ + slot, part + nt, sizeof(double), cudaMemcpyDeviceToHost, st_);
  launches_ += 2;
}

int Engine::ccp_violation(int s, double* out4) {
  out4[0] = out4[1] = out4[2] = out4[3] = 0.0;
  if (sync_words() != DV_OK) return DV_ERR_CUDA;
  const SegState& X = h_sst_[s];
  const int nc = X.nc;
  if (nc == 0) return DV_OK;
  const int nt = (nc + kTileItems - 1) / kTileItems;
  if (ensure_red(4 * (size_t)nc + 2 * (size_t)(nt + 2)) != DV_OK) return DV_ERR_OOM;
  double* items = d_red_;
  double* part = d_red_ + 4 * (size_t)nc;
  if (hseg_[s].nbil > 0)
    k_violation_items_flat<<<(nc + kThreads - 1) / kThreads, kThreads, 0, st_>>>(
        nc, hseg_[s].nbil, X.c0, d.ccap, hseg_[s].wbase, d.wtotal, d.gamma,
        d.bil_gam + hseg_[s].bil0, d.bil_b + hseg_[s].bil0, d.bil_off + hseg_[s].bil0, d.F, d.gap,
        d.ida, d.idb, d.v4, P_[s].h, P_[s].mu, items);
  else
    k_violation_items<<<(nc + kThreads - 1) / kThreads, kThreads, 0, st_>>>(
        nc, X.c0, d.ccap, hseg_[s].wbase, d.wtotal, d.gamma, d.F, d.gap, d.ida, d.idb, d.v4,
        P_[s].h, P_[s].mu, items);
  ++launches_;
  ordered_sum_dev(items + 2 * (size_t)nc, nc, part, 0);
  ordered_sum_dev(items + 3 * (size_t)nc, nc, part + nt + 2, 1);
  std::vector<double> gn(nc), vn(nc);
  DV_CUDA_TRY(cudaMemcpyAsync(gn.data(), items, sizeof(double) * nc, cudaMemcpyDeviceToHost, st_));
  DV_CUDA_TRY(cudaMemcpyAsync(vn.data(), items + nc, sizeof(double) * nc, cudaMemcpyDeviceToHost, st_));
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
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
  out4[2] = h_red_[0];
  out4[3] = sqrt(h_red_[1]);
  return DV_OK;
}

int Engine::energies(int s, double* kinetic, double* potential) {
  const int nb = hseg_[s].b1 - hseg_[s].b0;
  if (nb == 0) {
    if (kinetic) *kinetic = 0;
    if (potential) *potential = 0;
    return DV_OK;
  }
  const int nt = (nb + kTileItems - 1) / kTileItems;
  if (ensure_red(2 * (size_t)nb + 2 * (size_t)(nt + 2)) != DV_OK) return DV_ERR_OOM;
  double* items = d_red_;
  double* part = d_red_ + 2 * (size_t)nb;
  k_energy_items<<<(nb + kThreads - 1) / kThreads, kThreads, 0, st_>>>(nb, hseg_[s].b0, d.p4, d.v4,
                                                                       d.f4, d.minv, items);
  ++launches_;
  ordered_sum_dev(items, nb, part, 2);
  ordered_sum_dev(items + nb, nb, part + nt + 2, 3);
  DV_CUDA_TRY(cudaStreamSynchronize(st_));
  DV_CUDA_TRY(cudaGetLastError());
  if (kinetic) *kinetic = 0.5 * h_red_[2];
  if (potential) *potential = -h_red_[3];
  return DV_OK;
}

}  // namespace dv
