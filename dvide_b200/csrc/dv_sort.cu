// dv_sort.cu -- hand-written stable LSD radix sort of (uint32 key, uint32
// value) pairs and an int32 exclusive scan.  These replace the Thrust
// sort_by_key / reduce_by_key / inclusive_scan calls of the reference
// collision detector (CollisionDetector.cu:284-312, include.cuh:84-96).
//
// Radix pass (8-bit digit): each CTA owns a tile of 2048 items and counts its
// digits; a scan of the digit-major count table gives every (digit, tile) its
// output base; the scatter recomputes each item's rank among equal digits in
// index order with warp match masks, so equal keys keep their input order.
#include <algorithm>

#include "dv_internal.cuh"

namespace dv {

namespace {

constexpr int kRadixTile = 2048;
constexpr int kRadixRounds = kRadixTile / kThreads;  // 8
constexpr int kScanBlock = 1024;

__global__ void __launch_bounds__(kThreads) k_radix_count(const uint32_t* __restrict__ keys,
                                                          const int* __restrict__ n_dev, int shift,
                                                          uint32_t* __restrict__ hist, int ntiles) {
  __shared__ unsigned cnt[256];
  const int n = *n_dev;
  cnt[threadIdx.x] = 0;
  __syncthreads();
  int base = blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixRounds; ++r) {
    int i = base + r * kThreads + threadIdx.x;
    if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void __launch_bounds__(kThreads) k_radix_scatter(
    const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
    uint32_t* __restrict__ vout, const int* __restrict__ n_dev, int shift,
    const int* __restrict__ offs, int ntiles) {
  __shared__ int run[256];
  const int n = *n_dev;
  if (blockIdx.x * kRadixTile >= n) return;
  __shared__ int wcnt[kThreads / 32][256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  run[threadIdx.x] = offs[(size_t)threadIdx.x * ntiles + blockIdx.x];
  const unsigned lt_mask = (1u << lane) - 1u;
  int base = blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixRounds; ++r) {
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) wcnt[w][threadIdx.x] = 0;
    __syncthreads();
    int i = base + r * kThreads + threadIdx.x;
    bool valid = i < n;
    uint32_t key = valid ? kin[i] : 0u;
    uint32_t val = valid ? vin[i] : 0u;
    int d = valid ? (int)((key >> shift) & 255u) : 256;
    unsigned peers = __match_any_sync(0xffffffffu, d);
    int rank = __popc(peers & lt_mask);
    if (valid && rank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      int pre = 0;
      for (int w = 0; w < warp; ++w) pre += wcnt[w][d];
      int pos = run[d] + pre + rank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
    {
      int tot = 0;
#pragma unroll
      for (int w = 0; w < kThreads / 32; ++w) tot += wcnt[w][threadIdx.x];
      run[threadIdx.x] += tot;
    }
    __syncthreads();
  }
}

// Exclusive scan of one block of up to 1024 ints (4 per thread, contiguous).
__global__ void __launch_bounds__(kThreads) k_scan_block(const int* __restrict__ in,
                                                         int* __restrict__ out, int n,
                                                         int* __restrict__ block_sums,
                                                         int write_total) {
  __shared__ int wsum[kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int base = blockIdx.x * kScanBlock + threadIdx.x * 4;
  int v[4];
  int s = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    v[j] = (base + j < n) ? in[base + j] : 0;
    s += v[j];
  }
  // inclusive warp scan of thread sums
  int x = s;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = (lane < kThreads / 32) ? wsum[lane] : 0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, off);
      if (lane >= off) w += y;
    }
    if (lane < kThreads / 32) wsum[lane] = w;
  }
  __syncthreads();
  int excl = x - s + (warp > 0 ? wsum[warp - 1] : 0);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (base + j < n) out[base + j] = excl;
    excl += v[j];
  }
  if (threadIdx.x == kThreads - 1) {
    int total = wsum[kThreads / 32 - 1];
    if (block_sums) block_sums[blockIdx.x] = total;
    if (write_total) out[n] = total;
  }
}

__global__ void __launch_bounds__(kThreads) k_scan_add(int* __restrict__ out, int n,
                                                       const int* __restrict__ block_offs,
                                                       int nblk) {
  int add = block_offs[blockIdx.x];
  int base = blockIdx.x * kScanBlock + threadIdx.x * 4;
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (base + j < n) out[base + j] += add;
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = block_offs[nblk];
}

__global__ void k_set_zero_total(int* out) { out[0] = 0; }

__global__ void __launch_bounds__(kThreads) k_copy_pairs(const uint32_t* __restrict__ ks,
                                                         const uint32_t* __restrict__ vs,
                                                         uint32_t* __restrict__ kd,
                                                         uint32_t* __restrict__ vd,
                                                         const int* __restrict__ n_dev) {
  const int n = *n_dev;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
    kd[i] = ks[i];
    vd[i] = vs[i];
  }
}

}  // namespace

size_t scan_tmp_size(size_t n);

size_t radix_hist_size(size_t n) {
  size_t ntiles = (n + kRadixTile - 1) / kRadixTile;
  if (ntiles == 0) ntiles = 1;
  // counts, their scan (+ total), then the scan's own temporary space
  return 256 * ntiles * 2 + 1 + scan_tmp_size(256 * ntiles);
}

size_t scan_tmp_size(size_t n) {
  size_t total = 0;
  while (n > (size_t)kScanBlock) {
    size_t nblk = (n + kScanBlock - 1) / kScanBlock;
    total += nblk + (nblk + 1);
    n = nblk;
  }
  return total + 4;
}

void exclusive_scan_i32(const int* in, int* out, int n, int* tmp, cudaStream_t st,
                        int64_t* launches) {
  if (n <= 0) {
    k_set_zero_total<<<1, 1, 0, st>>>(out);
    ++*launches;
    return;
  }
  int nblk = (n + kScanBlock - 1) / kScanBlock;
  if (nblk == 1) {
    k_scan_block<<<1, kThreads, 0, st>>>(in, out, n, nullptr, 1);
    ++*launches;
    return;
  }
  int* sums = tmp;
  int* offs = tmp + nblk;
  int* rest = offs + nblk + 1;
  k_scan_block<<<nblk, kThreads, 0, st>>>(in, out, n, sums, 0);
  ++*launches;
  exclusive_scan_i32(sums, offs, nblk, rest, st, launches);
  k_scan_add<<<nblk, kThreads, 0, st>>>(out, n, offs, nblk);
  ++*launches;
}

void radix_sort_pairs(uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1, uint32_t* hist,
                      const int* n_dev, int n_cap, int bits, cudaStream_t st, int64_t* launches) {
  if (n_cap <= 1 || bits <= 0) return;
  int ntiles = (n_cap + kRadixTile - 1) / kRadixTile;
  int passes = (bits + 7) / 8;
  uint32_t* cnt = hist;
  int* offs = reinterpret_cast<int*>(hist + 256 * (size_t)ntiles);
  // the scan's temporary space sits after the count table and its scan
  int* scan_tmp = offs + 256 * (size_t)ntiles + 1;
  uint32_t *ki = k0, *vi = v0, *ko = k1, *vo = v1;
  for (int p = 0; p < passes; ++p) {
    int shift = 8 * p;
    k_radix_count<<<ntiles, kThreads, 0, st>>>(ki, n_dev, shift, cnt, ntiles);
    ++*launches;
    exclusive_scan_i32(reinterpret_cast<const int*>(cnt), offs, 256 * ntiles, scan_tmp, st,
                       launches);
    k_radix_scatter<<<ntiles, kThreads, 0, st>>>(ki, vi, ko, vo, n_dev, shift, offs, ntiles);
    ++*launches;
    uint32_t* t;
    t = ki; ki = ko; ko = t;
    t = vi; vi = vo; vo = t;
  }
  if (passes & 1) {  // the sorted data is in (k1, v1): move it back
    int g = std::min(ntiles * (kRadixTile / kThreads), 4 * 148 * 8);
    k_copy_pairs<<<g, kThreads, 0, st>>>(k1, v1, k0, v0, n_dev);
    ++*launches;
  }
}

}  // namespace dv
