// dv_collide.cu -- collision detection for spheres and boxes.
//
// Replaces CollisionDetector::generateAxisAlignedBoundingBoxes,
// detectPossibleCollisions_spatialSubdivision and detectCollisions
// (CollisionDetector.cu:24-501, 547-665) for rigid bodies.
//
// Candidate pairs are exactly the reference's: AABBs (extent + envelope)
// shifted by the global origin (AABB union min - 0.01), inclusive overlap on
// all three axes, same-family pairs (family != -1) excluded.  That set does not
// depend on the binning, so the reference's 20^3 global bins are replaced by:
//   * spheres in a uniform grid whose cell is wider than any sphere AABB,
//     keyed on the shifted AABB min corner; (cell, body) keys are radix
//     sorted; one warp per sphere scans the 27 neighbour cells (one lane per
//     cell) and lanes 27..31 scan the box list;
//   * boxes tested against every body by a block-parallel compaction.
// Each body's partners with larger id are sorted, so contacts come out in
// lexicographic (A, B) order, the order of the reference's sorted unique
// 64-bit pair keys (CollisionDetector.cu:319-325).  The narrowphase
// (sphere-sphere, sphere-box; box-box is never a contact) also emits the
// tangent frame of System.cu:753-762, so no separate Jacobian is built.
#include <stdio.h>

#include <algorithm>

#include "dv_internal.cuh"

namespace dv {

namespace {

constexpr int kWarpsPerCta = kThreads / 32;
constexpr int kMaxPerBody = 128;  // partners with larger id per sphere

__device__ inline unsigned long long ordered_bits(double x) {
  unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ inline double from_ordered(unsigned long long u) {
  u = (u >> 63) ? (u & 0x7fffffffffffffffull) : ~u;
  return __longlong_as_double((long long)u);
}

__device__ inline void aabb_of(double4 p, double4 g, double env, double4* mn, double4* mx) {
  double ex = g.x, ey = g.y, ez = g.z;
  if (g.y == 0) { ex = g.x; ey = g.x; ez = g.x; }
  ex = ex + env; ey = ey + env; ez = ez + env;
  *mn = make_double4(p.x - ex, p.y - ey, p.z - ez, 0.0);
  *mx = make_double4(p.x + ex, p.y + ey, p.z + ez, 0.0);
}

__global__ void k_bounds_init(GridInfo* g) {
  for (int d = 0; d < 3; ++d) {
    g->lo[d] = ~0ull;
    g->hi[d] = 0ull;
  }
}

// CollisionDetector.cu:24-79 (rigid-body branch): aabb = pos -+ (extent + envelope).
__global__ void __launch_bounds__(kThreads) k_aabb(const double4* __restrict__ p4,
                                                  const double4* __restrict__ g4, int nb,
                                                  double env, double4* __restrict__ amin,
                                                  double4* __restrict__ amax, GridInfo* grid) {
  __shared__ unsigned long long s_lo[3][kWarpsPerCta], s_hi[3][kWarpsPerCta];
  int i = blockIdx.x * kThreads + threadIdx.x;
  unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0ull, 0ull, 0ull};
  if (i < nb) {
    double4 mn, mx;
    aabb_of(p4[i], g4[i], env, &mn, &mx);
    amin[i] = mn;
    amax[i] = mx;
    lo[0] = ordered_bits(mn.x); lo[1] = ordered_bits(mn.y); lo[2] = ordered_bits(mn.z);
    hi[0] = ordered_bits(mx.x); hi[1] = ordered_bits(mx.y); hi[2] = ordered_bits(mx.z);
  }
  for (int d = 0; d < 3; ++d) {
    unsigned long long a = lo[d], b = hi[d];
    for (int off = 16; off >= 1; off >>= 1) {
      unsigned long long oa = __shfl_down_sync(0xffffffffu, a, off);
      unsigned long long ob = __shfl_down_sync(0xffffffffu, b, off);
      a = oa < a ? oa : a;
      b = ob > b ? ob : b;
    }
    if ((threadIdx.x & 31) == 0) {
      s_lo[d][threadIdx.x >> 5] = a;
      s_hi[d][threadIdx.x >> 5] = b;
    }
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    int d = threadIdx.x;
    unsigned long long a = s_lo[d][0], b = s_hi[d][0];
    for (int w = 1; w < kWarpsPerCta; ++w) {
      a = s_lo[d][w] < a ? s_lo[d][w] : a;
      b = s_hi[d][w] > b ? s_hi[d][w] : b;
    }
    atomicMin(&grid->lo[d], a);
    atomicMax(&grid->hi[d], b);
  }
}

// CollisionDetector.cu:566-568: origin = union min - 0.01; grid sized for the
// widest sphere AABB, capped at `cap` cells (a wider cell only adds candidates).
__global__ void k_grid_setup(GridInfo* g, double W, int cap) {
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = from_ordered(g->lo[d]);
    hi[d] = from_ordered(g->hi[d]);
  }
  g->ox = lo[0] - 0.01;
  g->oy = lo[1] - 0.01;
  g->oz = lo[2] - 0.01;
  double ext[3] = {hi[0] + 0.01 - g->ox, hi[1] + 0.01 - g->oy, hi[2] + 0.01 - g->oz};
  double w = W * (1.0 + 1e-6) + 1e-300;
  int dims[3];
  for (int it = 0; it < 64; ++it) {
    double total = 1.0;
    for (int d = 0; d < 3; ++d) {
      double c = floor(ext[d] / w) + 1.0;
      if (!(c < 1e9)) c = 1e9;
      dims[d] = (int)c;
      total *= c;
    }
    if (total <= (double)cap) break;
    w *= 1.26;
  }
  double total = (double)dims[0] * (double)dims[1] * (double)dims[2];
  if (!(total <= (double)cap) || !(w > 0)) {
    // non-finite or absurd extents: one cell holds every sphere (slow, still exact)
    dims[0] = dims[1] = dims[2] = 1;
    w = 1.0;
  }
  g->inv_w = 1.0 / w;
  g->dx = dims[0];
  g->dy = dims[1];
  g->dz = dims[2];
  g->ncells = dims[0] * dims[1] * dims[2];
}

__device__ inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// CollisionDetector.cu:574: aabb -= origin.  Spheres also get their cell key.
__global__ void __launch_bounds__(kThreads) k_shift_and_bin(
    int nb, const int* __restrict__ small_ids, int n_small, const double4* __restrict__ p4,
    const double4* __restrict__ g4, double env, double4* __restrict__ amin,
    double4* __restrict__ amax, const GridInfo* __restrict__ g, int4* __restrict__ cell,
    uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  int i = blockIdx.x * kThreads + threadIdx.x;
  double ox = g->ox, oy = g->oy, oz = g->oz;
  if (i < nb) {
    double4 a = amin[i], b = amax[i];
    amin[i] = make_double4(a.x - ox, a.y - oy, a.z - oz, 0.0);
    amax[i] = make_double4(b.x - ox, b.y - oy, b.z - oz, 0.0);
  }
  if (i < n_small) {
    int body = small_ids[i];
    double4 a, b;
    aabb_of(p4[body], g4[body], env, &a, &b);
    a = make_double4(a.x - ox, a.y - oy, a.z - oz, 0.0);
    double iw = g->inv_w;
    int cx = clampi((int)floor(a.x * iw), 0, g->dx - 1);
    int cy = clampi((int)floor(a.y * iw), 0, g->dy - 1);
    int cz = clampi((int)floor(a.z * iw), 0, g->dz - 1);
    int id = cx + g->dx * (cy + g->dy * cz);
    cell[body] = make_int4(cx, cy, cz, id);
    keys[i] = (uint32_t)id;
    vals[i] = (uint32_t)body;
  }
}

__global__ void __launch_bounds__(kThreads) k_cell_ranges(const uint32_t* __restrict__ keys,
                                                         int n, int* __restrict__ cstart,
                                                         int* __restrict__ cend, int ncap) {
  int j = blockIdx.x * kThreads + threadIdx.x;
  if (j >= n) return;
  uint32_t k = keys[j];
  if (k >= (uint32_t)ncap) return;
  if (j == 0 || keys[j - 1] != k) cstart[k] = j;
  if (j == n - 1 || keys[j + 1] != k) cend[k] = j + 1;
}

// CollisionDetector.cu:124-130 / 161-167.
__device__ inline bool is_candidate(const double4* __restrict__ amin,
                                    const double4* __restrict__ amax,
                                    const int* __restrict__ fam, int i, int j) {
  double4 A0 = amin[i], A1 = amax[i], B0 = amin[j], B1 = amax[j];
  bool in = (A0.x <= B1.x && B0.x <= A1.x) && (A0.y <= B1.y && B0.y <= A1.y) &&
            (A0.z <= B1.z && B0.z <= A1.z);
  if (i == j) in = false;
  int fa = fam[i], fb = fam[j];
  if (fa == fb && fa != -1) in = false;
  return in;
}

struct NpOut {
  d3 n;       // stored normal (B -> A)
  double gap; // -penetration
  d3 loc;
};

// CollisionDetector.cu:187-331 (test) and 333-501 (store), rigid bodies only.
__device__ inline bool narrowphase(const double4* __restrict__ p4, const double4* __restrict__ g4,
                                   int ia, int ib, double env, NpOut* o) {
  double4 pa = p4[ia], pb = p4[ib], ga = g4[ia], gb = g4[ib];
  d3 posA = mk3(pa.x, pa.y, pa.z), posB = mk3(pb.x, pb.y, pb.z);
  d3 gA = mk3(ga.x, ga.y, ga.z), gB = mk3(gb.x, gb.y, gb.z);
  double pen;
  d3 normal, location;
  if (gA.y == 0 && gB.y == 0) {
    d3 d = sub3(posB, posA);
    pen = (gA.x + gB.x) - length3(d);
    if (!(pen >= -env)) return false;
    normal = normalize3(d);
    location = add3(posA, scale3(normal, gA.x));
  } else if ((gA.y != 0 && gB.y == 0) || (gA.y == 0 && gB.y != 0)) {
    double dmin = 0;
    double r = gB.x;
    d3 center = posB;
    d3 bmin = sub3(posA, gA);
    d3 bmax = add3(posA, gA);
    bool sphereA = (gA.y == 0 && gB.y != 0);
    if (sphereA) {
      r = gA.x;
      center = posA;
      bmin = sub3(posB, gB);
      bmax = add3(posB, gB);
    }
    d3 nrm = mk3(0, 0, 0);
    double t;
    if (center.x < bmin.x) { t = center.x - bmin.x; dmin += t * t; nrm.x = nrm.x + t; }
    else if (center.x > bmax.x) { t = center.x - bmax.x; dmin += t * t; nrm.x = nrm.x + t; }
    if (center.y < bmin.y) { t = center.y - bmin.y; dmin += t * t; nrm.y = nrm.y + t; }
    else if (center.y > bmax.y) { t = center.y - bmax.y; dmin += t * t; nrm.y = nrm.y + t; }
    if (center.z < bmin.z) { t = center.z - bmin.z; dmin += t * t; nrm.z = nrm.z + t; }
    else if (center.z > bmax.z) { t = center.z - bmax.z; dmin += t * t; nrm.z = nrm.z + t; }
    pen = r - sqrt(dmin);
    if (!(pen >= -env)) return false;
    normal = normalize3(nrm);
    location = sub3(center, scale3(normal, r));
    if (sphereA) normal = neg3(normal);
  } else {
    return false;
  }
  o->n = neg3(normal);
  o->gap = -pen;
  o->loc = location;
  return true;
}

struct CollideArgs {
  int nb, n_small, n_large;
  const double4* p4;
  const double4* g4;
  const int* fam;
  const double4* amin;
  const double4* amax;
  const int4* cell;
  const int* small_ids;
  const int* large_ids;
  const uint32_t* sorted_bodies;  // small bodies sorted by cell
  const int* cstart;
  const int* cend;
  const GridInfo* grid;
  double env;
  int* cnt_cont;
  int* cnt_cand;
  int* counters;
  const int* cbase;
  // contact outputs
  size_t ccap;
  uint32_t* ida;
  uint32_t* idb;
  double* F;
  double* gap;
  double* loc;
  unsigned* err;
};

__device__ inline void write_contact(const CollideArgs& a, size_t c, int ia, int ib,
                                     const NpOut& o) {
  a.ida[c] = (uint32_t)ia;
  a.idb[c] = (uint32_t)ib;
  d3 u, v;
  frame_from_normal(o.n, &u, &v);
  size_t S = a.ccap;
  a.F[0 * S + c] = o.n.x; a.F[1 * S + c] = o.n.y; a.F[2 * S + c] = o.n.z;
  a.F[3 * S + c] = u.x;   a.F[4 * S + c] = u.y;   a.F[5 * S + c] = u.z;
  a.F[6 * S + c] = v.x;   a.F[7 * S + c] = v.y;   a.F[8 * S + c] = v.z;
  a.gap[c] = o.gap;
  a.loc[0 * S + c] = o.loc.x;
  a.loc[1 * S + c] = o.loc.y;
  a.loc[2 * S + c] = o.loc.z;
}

// One warp per sphere A: partners B > A from the 27 neighbour cells (lane =
// cell) and from the box list (lanes 27..31).  kWrite = false counts,
// kWrite = true emits the sorted partner list at cbase[A].
template <bool kWrite>
__global__ void __launch_bounds__(kThreads) k_sphere_pairs(CollideArgs a) {
  __shared__ int s_buf[kWarpsPerCta][kMaxPerBody];
  __shared__ int s_cnt[kWarpsPerCta];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int j = blockIdx.x * kWarpsPerCta + warp;
  if (j >= a.n_small) return;
  const int A = a.small_ids[j];
  if (lane == 0) s_cnt[warp] = 0;
  __syncwarp();
  int ncand = 0, ncont = 0;
  if (lane < 27) {
    int4 cA = a.cell[A];
    int x = cA.x + (lane % 3) - 1, y = cA.y + ((lane / 3) % 3) - 1, z = cA.z + (lane / 9) - 1;
    const GridInfo* g = a.grid;
    if (x >= 0 && y >= 0 && z >= 0 && x < g->dx && y < g->dy && z < g->dz) {
      int id = x + g->dx * (y + g->dy * z);
      int s = a.cstart[id];
      if (s >= 0) {
        int e = a.cend[id];
        for (; s < e; ++s) {
          int B = (int)a.sorted_bodies[s];
          if (B <= A) continue;
          if (!is_candidate(a.amin, a.amax, a.fam, A, B)) continue;
          ++ncand;
          NpOut o;
          if (narrowphase(a.p4, a.g4, A, B, a.env, &o)) {
            ++ncont;
            if (kWrite) {
              int slot = atomicAdd(&s_cnt[warp], 1);
              if (slot < kMaxPerBody) s_buf[warp][slot] = B;
            }
          }
        }
      }
    }
  } else {
    for (int m = lane - 27; m < a.n_large; m += 5) {
      int B = a.large_ids[m];
      if (B <= A) continue;
      if (!is_candidate(a.amin, a.amax, a.fam, A, B)) continue;
      ++ncand;
      NpOut o;
      if (narrowphase(a.p4, a.g4, A, B, a.env, &o)) {
        ++ncont;
        if (kWrite) {
          int slot = atomicAdd(&s_cnt[warp], 1);
          if (slot < kMaxPerBody) s_buf[warp][slot] = B;
        }
      }
    }
  }
  if (!kWrite) {
    for (int off = 16; off >= 1; off >>= 1) {
      ncand += __shfl_down_sync(0xffffffffu, ncand, off);
      ncont += __shfl_down_sync(0xffffffffu, ncont, off);
    }
    if (lane == 0) {
      a.cnt_cand[A] = ncand;
      a.cnt_cont[A] = ncont;
      if (ncont > kMaxPerBody) atomicOr(a.err, kErrCapacity);
      if (ncand) atomicAdd(&a.counters[1], ncand);
    }
    return;
  }
  __syncwarp();
  int n = s_cnt[warp];
  if (n > kMaxPerBody) n = kMaxPerBody;
  // rank sort of the (distinct) partner ids, then emit in ascending order
  int mine[kMaxPerBody / 32];
  int rk[kMaxPerBody / 32];
#pragma unroll
  for (int t = 0; t < kMaxPerBody / 32; ++t) {
    int e = lane + 32 * t;
    mine[t] = (e < n) ? s_buf[warp][e] : 0x7fffffff;
    rk[t] = 0;
  }
  for (int e = 0; e < n; ++e) {
    int other = s_buf[warp][e];
#pragma unroll
    for (int t = 0; t < kMaxPerBody / 32; ++t) rk[t] += (other < mine[t]) ? 1 : 0;
  }
  __syncwarp();
  size_t base = (size_t)a.cbase[A];
#pragma unroll
  for (int t = 0; t < kMaxPerBody / 32; ++t) {
    int e = lane + 32 * t;
    if (e < n) {
      NpOut o;
      narrowphase(a.p4, a.g4, A, mine[t], a.env, &o);
      write_contact(a, base + rk[t], A, mine[t], o);
    }
  }
}

// Boxes: body L = large_ids[blockIdx.y] against the 256 bodies of chunk
// blockIdx.x, keeping B > L; ranks within the chunk by warp ballots.
template <bool kWrite>
__global__ void __launch_bounds__(kThreads) k_box_pairs(CollideArgs a, int* __restrict__ chunk_cnt,
                                                        const int* __restrict__ chunk_off,
                                                        int nchunks) {
  __shared__ int s_w[kWarpsPerCta];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int m = blockIdx.y;
  const int L = a.large_ids[m];
  const int B = blockIdx.x * kThreads + threadIdx.x;
  bool cand = false, cont = false;
  NpOut o;
  if (B < a.nb && B > L && is_candidate(a.amin, a.amax, a.fam, L, B)) {
    cand = true;
    cont = narrowphase(a.p4, a.g4, L, B, a.env, &o);
  }
  unsigned bal = __ballot_sync(0xffffffffu, cont);
  if (!kWrite) {
    unsigned balc = __ballot_sync(0xffffffffu, cand);
    if (lane == 0) s_w[warp] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int w = 0; w < kWarpsPerCta; ++w) tot += s_w[w];
      chunk_cnt[(size_t)m * nchunks + blockIdx.x] = tot;
      if (tot) atomicAdd(&a.cnt_cont[L], tot);
    }
    if (lane == 0 && balc) {
      atomicAdd(&a.cnt_cand[L], __popc(balc));
      atomicAdd(&a.counters[1], __popc(balc));
    }
    return;
  }
  if (lane == 0) s_w[warp] = __popc(bal);
  __syncthreads();
  if (!cont) return;
  int pre = 0;
  for (int w = 0; w < warp; ++w) pre += s_w[w];
  pre += __popc(bal & ((1u << lane) - 1u));
  size_t pos = (size_t)a.cbase[L] + (size_t)(chunk_off[(size_t)m * nchunks + blockIdx.x] -
                                             chunk_off[(size_t)m * nchunks]) + pre;
  write_contact(a, pos, L, B, o);
}

__global__ void __launch_bounds__(kThreads) k_count_b(const uint32_t* __restrict__ idb, int nc,
                                                     int* __restrict__ cnt, uint32_t* __restrict__ keys,
                                                     uint32_t* __restrict__ vals) {
  int c = blockIdx.x * kThreads + threadIdx.x;
  if (c >= nc) return;
  uint32_t b = idb[c];
  atomicAdd(&cnt[b], 1);
  keys[c] = b;
  vals[c] = (uint32_t)c;
}

// Per-body incidence length: contacts where the body is B plus where it is A.
__global__ void __launch_bounds__(kThreads) k_inc_count(int nb, const int* __restrict__ bstart,
                                                       const int* __restrict__ abase,
                                                       int* __restrict__ cnt) {
  int b = blockIdx.x * kThreads + threadIdx.x;
  if (b >= nb) return;
  cnt[b] = (bstart[b + 1] - bstart[b]) + (abase[b + 1] - abase[b]);
}

// B-side contacts (flagged, ascending) then the A-side range: the ascending
// contact order of the body's column of D.
__global__ void __launch_bounds__(kThreads) k_inc_fill(int nb, const int* __restrict__ bstart,
                                                      const uint32_t* __restrict__ binc,
                                                      const int* __restrict__ abase,
                                                      const int* __restrict__ istart,
                                                      uint32_t* __restrict__ inc) {
  int b = blockIdx.x * kThreads + threadIdx.x;
  if (b >= nb) return;
  int o = istart[b];
  for (int i = bstart[b]; i < bstart[b + 1]; ++i) inc[o++] = binc[i] | 0x80000000u;
  for (int c = abase[b]; c < abase[b + 1]; ++c) inc[o++] = (uint32_t)c;
}

CollideArgs make_args(SceneDev& sd, double env) {
  CollideArgs a;
  a.nb = sd.nb;
  a.n_small = sd.n_small;
  a.n_large = sd.n_large;
  a.p4 = sd.p4;
  a.g4 = sd.geom4;
  a.fam = sd.family;
  a.amin = sd.amin;
  a.amax = sd.amax;
  a.cell = sd.cell;
  a.small_ids = sd.small_ids;
  a.large_ids = sd.large_ids;
  a.sorted_bodies = sd.valA;
  a.cstart = sd.cell_start;
  a.cend = sd.cell_end;
  a.grid = sd.grid;
  a.env = env;
  a.cnt_cont = sd.cnt_cont;
  a.cnt_cand = sd.cnt_cand;
  a.counters = sd.counters;
  a.cbase = sd.cbase;
  a.ccap = sd.ccap;
  a.ida = sd.ida;
  a.idb = sd.idb;
  a.F = sd.F;
  a.gap = sd.gap;
  a.loc = sd.loc;
  a.err = reinterpret_cast<unsigned*>(sd.counters + 2);
  return a;
}

int bits_for(int n) {
  int b = 0;
  while (b < 31 && (1 << b) < n) ++b;
  return b;
}

}  // namespace

void collide_count(SceneDev& sd, double env, cudaStream_t st, int64_t* launches) {
  int nb = sd.nb;
  cudaMemsetAsync(sd.counters, 0, 4 * sizeof(int), st);
  cudaMemsetAsync(sd.cnt_cont, 0, sizeof(int) * (size_t)nb, st);
  cudaMemsetAsync(sd.cnt_cand, 0, sizeof(int) * (size_t)nb, st);
  k_bounds_init<<<1, 1, 0, st>>>(sd.grid);
  int gb = (nb + kThreads - 1) / kThreads;
  k_aabb<<<gb, kThreads, 0, st>>>(sd.p4, sd.geom4, nb, env, sd.amin, sd.amax, sd.grid);
  k_grid_setup<<<1, 1, 0, st>>>(sd.grid, sd.W, sd.ncell_cap);
  int gs = (std::max(nb, sd.n_small) + kThreads - 1) / kThreads;
  k_shift_and_bin<<<gs, kThreads, 0, st>>>(nb, sd.small_ids, sd.n_small, sd.p4, sd.geom4, env,
                                           sd.amin, sd.amax, sd.grid, sd.cell, sd.keyA, sd.valA);
  *launches += 4;
  if (sd.n_small > 0) {
    radix_sort_pairs(sd.keyA, sd.valA, sd.keyB, sd.valB, sd.radix_hist, sd.n_small,
                     bits_for(sd.ncell_cap), st, launches);
    cudaMemsetAsync(sd.cell_start, 0xff, sizeof(int) * (size_t)sd.ncell_cap, st);
    k_cell_ranges<<<(sd.n_small + kThreads - 1) / kThreads, kThreads, 0, st>>>(
        sd.keyA, sd.n_small, sd.cell_start, sd.cell_end, sd.ncell_cap);
    ++*launches;
  }
  CollideArgs a = make_args(sd, env);
  if (sd.n_small > 0) {
    k_sphere_pairs<false><<<(sd.n_small + kWarpsPerCta - 1) / kWarpsPerCta, kThreads, 0, st>>>(a);
    ++*launches;
  }
  if (sd.n_large > 0) {
    int nchunks = (nb + kThreads - 1) / kThreads;
    dim3 grid(nchunks, sd.n_large);
    k_box_pairs<false><<<grid, kThreads, 0, st>>>(a, sd.large_chunk, nullptr, nchunks);
    ++*launches;
  }
  exclusive_scan_i32(sd.cnt_cont, sd.cbase, nb, sd.scan_tmp, st, launches);
  cudaMemcpyAsync(sd.counters, sd.cbase + nb, sizeof(int), cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(sd.h_counters, sd.counters, 4 * sizeof(int), cudaMemcpyDeviceToHost, st);
}

void collide_write(SceneDev& sd, double env, cudaStream_t st, int64_t* launches) {
  int nb = sd.nb;
  CollideArgs a = make_args(sd, env);
  if (sd.n_small > 0) {
    k_sphere_pairs<true><<<(sd.n_small + kWarpsPerCta - 1) / kWarpsPerCta, kThreads, 0, st>>>(a);
    ++*launches;
  }
  if (sd.n_large > 0) {
    int nchunks = (nb + kThreads - 1) / kThreads;
    exclusive_scan_i32(sd.large_chunk, sd.large_chunk_off, nchunks * sd.n_large, sd.scan_tmp, st,
                       launches);
    dim3 grid(nchunks, sd.n_large);
    k_box_pairs<true><<<grid, kThreads, 0, st>>>(a, nullptr, sd.large_chunk_off, nchunks);
    ++*launches;
  }
  int nc = sd.nc;
  // B-side incidence: stable radix sort of (B, contact) keeps ascending contact order.
  cudaMemsetAsync(sd.cnt_cand, 0, sizeof(int) * (size_t)nb, st);
  if (nc > 0) {
    k_count_b<<<(nc + kThreads - 1) / kThreads, kThreads, 0, st>>>(sd.idb, nc, sd.cnt_cand,
                                                                   sd.keyA, sd.valA);
    ++*launches;
    radix_sort_pairs(sd.keyA, sd.valA, sd.keyB, sd.valB, sd.radix_hist, nc, bits_for(nb), st,
                     launches);
  }
  exclusive_scan_i32(sd.cnt_cand, sd.binc_start, nb, sd.scan_tmp, st, launches);
  if (nc > 0)
    cudaMemcpyAsync(sd.binc, sd.valA, sizeof(uint32_t) * (size_t)nc, cudaMemcpyDeviceToDevice, st);
  int gb = (nb + kThreads - 1) / kThreads;
  if (nb > 0) {
    k_inc_count<<<gb, kThreads, 0, st>>>(nb, sd.binc_start, sd.cbase, sd.cnt_cand);
    ++*launches;
  }
  exclusive_scan_i32(sd.cnt_cand, sd.inc_start, nb, sd.scan_tmp, st, launches);
  if (nb > 0 && nc > 0) {
    k_inc_fill<<<gb, kThreads, 0, st>>>(nb, sd.binc_start, sd.binc, sd.cbase, sd.inc_start,
                                        sd.inc);
    ++*launches;
  }
}

}  // namespace dv
