// dv_collide.cu -- collision detection for spheres and boxes, for every
// segment (scene) of an engine at once.
//
// Replaces CollisionDetector::generateAxisAlignedBoundingBoxes,
// detectPossibleCollisions_spatialSubdivision and detectCollisions
// (CollisionDetector.cu:24-501, 547-665) for rigid bodies.
//
// Candidate pairs are exactly the reference's: AABBs (extent + envelope)
// shifted by the segment's origin (AABB union min - 0.01), inclusive overlap
// on all three axes, same-family pairs (family != -1) excluded.  That set does
// not depend on the binning, so the reference's 20^3 global bins are replaced
// by:
//   * spheres in a uniform grid per segment whose cell is wider than any
//     sphere AABB of the segment, keyed on the shifted AABB min corner; the
//     segments' cells are numbered consecutively and (cell, body) keys of all
//     segments are radix sorted together; one warp per sphere scans the 27
//     neighbour cells (one lane per cell) and lanes 27..31 scan the
//     segment's box list;
//   * boxes tested against every body of their segment by a block-parallel
//     compaction.
// Each body's partners with larger id are sorted, so a segment's contacts come
// out in lexicographic (A, B) order, the order of the reference's sorted unique
// 64-bit pair keys (CollisionDetector.cu:319-325).  The narrowphase
// (sphere-sphere, sphere-box; box-box is never a contact) also emits the
// tangent frame of System.cu:753-762, so no separate Jacobian is built.
//
// Sizes that change every step (contacts, tiles) are read on the device, so
// the whole pipeline runs without a host round trip and can be captured in a
// CUDA graph.  EngineWords::err is sticky: once set, every later kernel of the
// step returns at once.
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

__global__ void k_seg_reset(int nseg, GridInfo* __restrict__ grid, SegState* __restrict__ sst,
                            EngineWords* __restrict__ ew) {
  if (ew->err) return;
  int s = blockIdx.x * kThreads + threadIdx.x;
  if (s == 0) {
    ew->npossible = 0;
    ew->n_wide = 0;
  }
  if (s >= nseg) return;
  for (int d = 0; d < 3; ++d) {
    grid[s].lo[d] = ~0ull;
    grid[s].hi[d] = 0ull;
  }
  sst[s].nc = 0;
  sst[s].npossible = 0;
}

// CollisionDetector.cu:24-79 (rigid-body branch): aabb = pos -+ (extent +
// envelope); per-segment AABB union by warp folds when the warp's bodies share
// a segment, per-body atomics otherwise.
__global__ void __launch_bounds__(kThreads) k_aabb(const double4* __restrict__ p4,
                                                  const double4* __restrict__ g4,
                                                  const int* __restrict__ bseg,
                                                  const SegParams* __restrict__ seg, int nb,
                                                  double4* __restrict__ amin,
                                                  double4* __restrict__ amax,
                                                  GridInfo* __restrict__ grid,
                                                  const EngineWords* __restrict__ ew) {
  if (ew->err) return;
  const int i = blockIdx.x * kThreads + threadIdx.x;
  const int lane = threadIdx.x & 31;
  int s = -1;
  unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0ull, 0ull, 0ull};
  if (i < nb) {
    s = bseg[i];
    if (seg[s].active) {
      double4 mn, mx;
      aabb_of(p4[i], g4[i], seg[s].env, &mn, &mx);
      amin[i] = mn;
      amax[i] = mx;
      lo[0] = ordered_bits(mn.x); lo[1] = ordered_bits(mn.y); lo[2] = ordered_bits(mn.z);
      hi[0] = ordered_bits(mx.x); hi[1] = ordered_bits(mx.y); hi[2] = ordered_bits(mx.z);
    } else {
      s = -1;
    }
  }
  const int s0 = __shfl_sync(0xffffffffu, s, 0);
  const bool uniform = __all_sync(0xffffffffu, s == s0);
  if (uniform) {
    if (s0 < 0) return;
    for (int d = 0; d < 3; ++d) {
      unsigned long long a = lo[d], b = hi[d];
      for (int off = 16; off >= 1; off >>= 1) {
        unsigned long long oa = __shfl_down_sync(0xffffffffu, a, off);
        unsigned long long ob = __shfl_down_sync(0xffffffffu, b, off);
        a = oa < a ? oa : a;
        b = ob > b ? ob : b;
      }
      if (lane == 0) {
        atomicMin(&grid[s0].lo[d], a);
        atomicMax(&grid[s0].hi[d], b);
      }
    }
  } else if (s >= 0) {
    for (int d = 0; d < 3; ++d) {
      atomicMin(&grid[s].lo[d], lo[d]);
      atomicMax(&grid[s].hi[d], hi[d]);
    }
  }
}

// CollisionDetector.cu:566-568: origin = union min - 0.01; grid sized for the
// widest sphere AABB of the segment, capped at its `cell_cap` cells (a wider
// cell only adds candidates).
__global__ void k_grid_setup(int nseg, const SegParams* __restrict__ seg,
                             GridInfo* __restrict__ grid, const EngineWords* __restrict__ ew) {
  if (ew->err) return;
  int s = blockIdx.x * kThreads + threadIdx.x;
  if (s >= nseg || !seg[s].active) return;
  GridInfo* g = grid + s;
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = from_ordered(g->lo[d]);
    hi[d] = from_ordered(g->hi[d]);
  }
  g->ox = lo[0] - 0.01;
  g->oy = lo[1] - 0.01;
  g->oz = lo[2] - 0.01;
  double ext[3] = {hi[0] + 0.01 - g->ox, hi[1] + 0.01 - g->oy, hi[2] + 0.01 - g->oz};
  double w = seg[s].W * (1.0 + 1e-6) + 1e-300;
  const int cap = seg[s].cell_cap;
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

// CollisionDetector.cu:574: aabb -= origin.  Spheres also get their cell key;
// spheres of inactive segments go to the parking cell `park`.
__global__ void __launch_bounds__(kThreads) k_shift_and_bin(
    int nb, const int* __restrict__ small_ids, int n_small, const int* __restrict__ bseg,
    const SegParams* __restrict__ seg, const double4* __restrict__ p4,
    const double4* __restrict__ g4, double4* __restrict__ amin, double4* __restrict__ amax,
    const GridInfo* __restrict__ grid, int4* __restrict__ cell, uint32_t* __restrict__ keys,
    uint32_t* __restrict__ vals, int park, const EngineWords* __restrict__ ew) {
  if (ew->err) return;
  int i = blockIdx.x * kThreads + threadIdx.x;
  if (i < nb) {
    int s = bseg[i];
    if (seg[s].active) {
      const GridInfo* g = grid + s;
      double ox = g->ox, oy = g->oy, oz = g->oz;
      double4 a = amin[i], b = amax[i];
      amin[i] = make_double4(a.x - ox, a.y - oy, a.z - oz, 0.0);
      amax[i] = make_double4(b.x - ox, b.y - oy, b.z - oz, 0.0);
    }
  }
  if (i < n_small) {
    int body = small_ids[i];
    int s = bseg[body];
    uint32_t key = (uint32_t)park;
    if (seg[s].active) {
      const GridInfo* g = grid + s;
      double4 a, b;
      aabb_of(p4[body], g4[body], seg[s].env, &a, &b);
      a = make_double4(a.x - g->ox, a.y - g->oy, a.z - g->oz, 0.0);
      double iw = g->inv_w;
      int cx = clampi((int)floor(a.x * iw), 0, g->dx - 1);
      int cy = clampi((int)floor(a.y * iw), 0, g->dy - 1);
      int cz = clampi((int)floor(a.z * iw), 0, g->dz - 1);
      int id = seg[s].cell_base + cx + g->dx * (cy + g->dy * cz);
      cell[body] = make_int4(cx, cy, cz, id);
      key = (uint32_t)id;
    }
    keys[i] = key;
    vals[i] = (uint32_t)body;
  }
}

__global__ void __launch_bounds__(kThreads) k_cell_ranges(const uint32_t* __restrict__ keys,
                                                         int n, int* __restrict__ cstart,
                                                         int* __restrict__ cend, int ncap,
                                                         const EngineWords* __restrict__ ew) {
  if (ew->err) return;
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
                                   int ia, int ib, double env, bool exact, NpOut* o) {
  double4 pa = p4[ia], pb = p4[ib], ga = g4[ia], gb = g4[ib];
  d3 posA = mk3(pa.x, pa.y, pa.z), posB = mk3(pb.x, pb.y, pb.z);
  d3 gA = mk3(ga.x, ga.y, ga.z), gB = mk3(gb.x, gb.y, gb.z);
  double pen;
  d3 normal, location;
  if (gA.y == 0 && gB.y == 0) {
    d3 d = sub3(posB, posA);
    pen = (gA.x + gB.x) - length3x(d, exact);
    if (!(pen >= -env)) return false;
    normal = normalize3x(d, exact);
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
    normal = normalize3x(nrm, exact);
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
  int nb, n_small, n_large, max_seg_chunks;
  const double4* p4;
  const double4* g4;
  const int* fam;
  const int* bseg;
  const SegParams* seg;
  SegState* sst;
  const double4* amin;
  const double4* amax;
  const int4* cell;
  const int* small_ids;
  const int* large_ids;
  const uint32_t* sorted_bodies;  // small bodies sorted by cell
  const int* cstart;
  const int* cend;
  const GridInfo* grid;
  int* cnt_cont;
  int* cnt_cand;
  int* wide_ids;
  const int* cbase;
  EngineWords* ew;
  // contact outputs
  size_t ccap;
  uint32_t* ida;
  uint32_t* idb;
  double* F;
  float* nf;
  double* gap;
  double* loc;
};

__device__ inline void write_contact(const CollideArgs& a, size_t c, int ia, int ib,
                                     const NpOut& o, bool exact) {
  a.ida[c] = (uint32_t)ia;
  a.idb[c] = (uint32_t)ib;
  d3 u, v;
  frame_from_normal(o.n, &u, &v, exact);
  size_t S = a.ccap;
  a.F[0 * S + c] = o.n.x; a.F[1 * S + c] = o.n.y; a.F[2 * S + c] = o.n.z;
  a.F[3 * S + c] = u.x;   a.F[4 * S + c] = u.y;   a.F[5 * S + c] = u.z;
  a.F[6 * S + c] = v.x;   a.F[7 * S + c] = v.y;   a.F[8 * S + c] = v.z;
  a.nf[0 * S + c] = (float)o.n.x;
  a.nf[1 * S + c] = (float)o.n.y;
  a.nf[2 * S + c] = (float)o.n.z;
  a.gap[c] = o.gap;
  a.loc[0 * S + c] = o.loc.x;
  a.loc[1 * S + c] = o.loc.y;
  a.loc[2 * S + c] = o.loc.z;
}

// One warp per sphere A: partners B > A from the 27 neighbour cells (lane =
// cell) and from the segment's box list (lanes 27..31).  kWrite = false
// counts, kWrite = true emits the sorted partner list at the body's slot.
template <bool kWrite>
__global__ void __launch_bounds__(kThreads) k_sphere_pairs(CollideArgs a) {
  __shared__ int s_buf[kWarpsPerCta][kMaxPerBody];
  __shared__ int s_cnt[kWarpsPerCta];
  if (a.ew->err) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int j = blockIdx.x * kWarpsPerCta + warp;
  if (j >= a.n_small) return;
  const int A = a.small_ids[j];
  const int sg = a.bseg[A];
  const SegParams& P = a.seg[sg];
  if (!P.active) return;
  if (kWrite && a.cnt_cont[A] > kMaxPerBody) return;  // k_sphere_pairs_wide's
  const double env = P.env;
  const bool exact = P.exact != 0;
  if (lane == 0) s_cnt[warp] = 0;
  __syncwarp();
  int ncand = 0, ncont = 0;
  if (lane < 27) {
    int4 cA = a.cell[A];
    int x = cA.x + (lane % 3) - 1, y = cA.y + ((lane / 3) % 3) - 1, z = cA.z + (lane / 9) - 1;
    const GridInfo* g = a.grid + sg;
    if (x >= 0 && y >= 0 && z >= 0 && x < g->dx && y < g->dy && z < g->dz) {
      int id = P.cell_base + x + g->dx * (y + g->dy * z);
      int s = a.cstart[id];
      if (s >= 0) {
        int e = a.cend[id];
        for (; s < e; ++s) {
          int B = (int)a.sorted_bodies[s];
          if (B <= A) continue;
          if (!is_candidate(a.amin, a.amax, a.fam, A, B)) continue;
          ++ncand;
          NpOut o;
          if (narrowphase(a.p4, a.g4, A, B, env, exact, &o)) {
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
    for (int m = P.l0 + lane - 27; m < P.l1; m += 5) {
      int B = a.large_ids[m];
      if (B <= A) continue;
      if (!is_candidate(a.amin, a.amax, a.fam, A, B)) continue;
      ++ncand;
      NpOut o;
      if (narrowphase(a.p4, a.g4, A, B, env, exact, &o)) {
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
      // more partners than this kernel lists: k_sphere_pairs_wide writes them
      if (ncont > kMaxPerBody) {
        const int k = atomicAdd(&a.ew->n_wide, 1);
        if (k < kWideSpheres && ncont <= kWidePartners) {
          a.wide_ids[k] = A;
        } else {
          atomicOr(&a.ew->err, kErrPartners);
          atomicOr(&a.sst[sg].err, kErrPartners);  // whose scene (a server retires it)
        }
      }
      if (ncand) {
        atomicAdd(&a.sst[sg].npossible, ncand);
        atomicAdd(&a.ew->npossible, ncand);
      }
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
  size_t base = (size_t)(a.cbase[A] + a.sst[sg].delta);
#pragma unroll
  for (int t = 0; t < kMaxPerBody / 32; ++t) {
    int e = lane + 32 * t;
    if (e < n) {
      NpOut o;
      narrowphase(a.p4, a.g4, A, mine[t], env, exact, &o);
      write_contact(a, base + rk[t], A, mine[t], o, exact);
    }
  }
}

// The write pass for the spheres the count pass listed in wide_ids (more than
// kMaxPerBody partners with larger ids): each CTA takes listed spheres in turn;
// for each it scans the same 27 cells and box list, keeps the partners in
// shared memory (at most kWidePartners), sorts them by id (bitonic) and writes
// the contacts at the sphere's slot in (A, B) order -- the same contacts, in
// the same order, as the warp kernel writes for a sphere with fewer partners.
__global__ void __launch_bounds__(kThreads) k_sphere_pairs_wide(CollideArgs a) {
  __shared__ int s_ids[kWidePartners];
  __shared__ int s_beg[28], s_off[29];
  __shared__ int s_n;
  if (a.ew->err) return;
  const int nw = min(a.ew->n_wide, kWideSpheres);
  for (int w = blockIdx.x; w < nw; w += gridDim.x) {
    __syncthreads();  // the previous sphere's reads of the shared arrays are done
    const int A = a.wide_ids[w];
    const int sg = a.bseg[A];
    const SegParams& P = a.seg[sg];
    const double env = P.env;
    const bool exact = P.exact != 0;
    // ranges 0..26: the neighbour cells (as the warp kernel's lanes); 27: boxes
    if (threadIdx.x < 28) {
      const int r = threadIdx.x;
      int beg = 0, len = 0;
      if (r < 27) {
        const int4 cA = a.cell[A];
        const int x = cA.x + (r % 3) - 1, y = cA.y + ((r / 3) % 3) - 1, z = cA.z + (r / 9) - 1;
        const GridInfo* g = a.grid + sg;
        if (x >= 0 && y >= 0 && z >= 0 && x < g->dx && y < g->dy && z < g->dz) {
          const int id = P.cell_base + x + g->dx * (y + g->dy * z);
          const int cs = a.cstart[id];
          if (cs >= 0) {
            beg = cs;
            len = a.cend[id] - cs;
          }
        }
      } else {
        beg = P.l0;
        len = P.l1 - P.l0;
      }
      s_beg[r] = beg;
      s_off[r + 1] = len;
    }
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
      s_off[0] = 0;
      for (int r = 0; r < 28; ++r) s_off[r + 1] += s_off[r];
    }
    __syncthreads();
    const int total = s_off[28];
    for (int f = threadIdx.x; f < total; f += kThreads) {
      int r = 0;
      while (r < 27 && s_off[r + 1] <= f) ++r;
      const int at = s_beg[r] + (f - s_off[r]);
      const int B = r < 27 ? (int)a.sorted_bodies[at] : a.large_ids[at];
      if (B <= A) continue;
      if (!is_candidate(a.amin, a.amax, a.fam, A, B)) continue;
      NpOut o;
      if (narrowphase(a.p4, a.g4, A, B, env, exact, &o)) {
        const int slot = atomicAdd(&s_n, 1);
        if (slot < kWidePartners) s_ids[slot] = B;
      }
    }
    __syncthreads();
    const int n = s_n;
    if (n != a.cnt_cont[A] || n > kWidePartners) {
      // not the count pass's partners (cannot happen: same tests, same order)
      if (threadIdx.x == 0) {
        atomicOr(&a.ew->err, kErrPartners);
        atomicOr(&a.sst[sg].err, kErrPartners);
      }
      return;
    }
    int m = 1;
    while (m < n) m <<= 1;
    for (int i = n + threadIdx.x; i < m; i += kThreads) s_ids[i] = 0x7fffffff;
    __syncthreads();
    for (int k = 2; k <= m; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = threadIdx.x; i < m; i += kThreads) {
          const int l = i ^ j;
          if (l > i) {
            const int x = s_ids[i], y = s_ids[l];
            if ((x > y) == ((i & k) == 0)) {
              s_ids[i] = y;
              s_ids[l] = x;
            }
          }
        }
        __syncthreads();
      }
    }
    const size_t base = (size_t)(a.cbase[A] + a.sst[sg].delta);
    for (int e = threadIdx.x; e < n; e += kThreads) {
      const int B = s_ids[e];
      NpOut o;
      narrowphase(a.p4, a.g4, A, B, env, exact, &o);
      write_contact(a, base + e, A, B, o, exact);
    }
  }
}

// Boxes: body L = large_ids[blockIdx.y] against the 256 bodies of chunk
// blockIdx.x of its segment, keeping B > L; ranks within the chunk by warp
// ballots.
template <bool kWrite>
__global__ void __launch_bounds__(kThreads) k_box_pairs(CollideArgs a, int* __restrict__ chunk_cnt,
                                                        const int* __restrict__ chunk_off) {
  __shared__ int s_w[kWarpsPerCta];
  if (a.ew->err) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int m = blockIdx.y;
  const int L = a.large_ids[m];
  const int sg = a.bseg[L];
  const SegParams& P = a.seg[sg];
  const size_t crow = (size_t)m * a.max_seg_chunks;
  if (!P.active || P.b0 + (int)blockIdx.x * kThreads >= P.b1) {
    if (!kWrite && threadIdx.x == 0) chunk_cnt[crow + blockIdx.x] = 0;
    return;
  }
  const int B = P.b0 + blockIdx.x * kThreads + threadIdx.x;
  bool cand = false, cont = false;
  NpOut o;
  if (B < P.b1 && B > L && is_candidate(a.amin, a.amax, a.fam, L, B)) {
    cand = true;
    cont = narrowphase(a.p4, a.g4, L, B, P.env, P.exact != 0, &o);
  }
  unsigned bal = __ballot_sync(0xffffffffu, cont);
  if (!kWrite) {
    unsigned balc = __ballot_sync(0xffffffffu, cand);
    if (lane == 0) s_w[warp] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int w = 0; w < kWarpsPerCta; ++w) tot += s_w[w];
      chunk_cnt[crow + blockIdx.x] = tot;
      if (tot) atomicAdd(&a.cnt_cont[L], tot);
    }
    if (lane == 0 && balc) {
      atomicAdd(&a.cnt_cand[L], __popc(balc));
      atomicAdd(&a.sst[sg].npossible, __popc(balc));
      atomicAdd(&a.ew->npossible, __popc(balc));
    }
    return;
  }
  if (lane == 0) s_w[warp] = __popc(bal);
  __syncthreads();
  if (!cont) return;
  int pre = 0;
  for (int w = 0; w < warp; ++w) pre += s_w[w];
  pre += __popc(bal & ((1u << lane) - 1u));
  size_t pos = (size_t)(a.cbase[L] + a.sst[sg].delta) +
               (size_t)(chunk_off[crow + blockIdx.x] - chunk_off[crow]) + pre;
  write_contact(a, pos, L, B, o, P.exact != 0);
}

// Contact layout: segment s gets nc_s = contacts of its bodies, slots
// [c0, c0 + nc_s) with c0 a multiple of kContactAlign, tiles [t0, t0 + nt).
// One CTA scans the segments in order.
__global__ void __launch_bounds__(1024) k_seg_layout(int nseg, int nb,
                                                     const SegParams* __restrict__ seg,
                                                     SegState* __restrict__ sst,
                                                     const int* __restrict__ cbase,
                                                     int* __restrict__ seg_tstart, size_t ccap,
                                                     int tcap, EngineWords* __restrict__ ew) {
  __shared__ long long s_c[32], s_t[32];
  __shared__ long long s_carry_c, s_carry_t;
  if (ew->err) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    s_carry_c = 0;
    s_carry_t = 0;
  }
  __syncthreads();
  for (int base = 0; base < nseg; base += 1024) {
    int s = base + threadIdx.x;
    long long nc = 0, pad = 0, nt = 0;
    if (s < nseg && seg[s].active) {
      nc = cbase[seg[s].b1] - cbase[seg[s].b0];
      pad = (nc + kContactAlign - 1) / kContactAlign * kContactAlign;
      // contact tiles, then the tiles of the bilateral rows
      nt = (nc + kTileItems - 1) / kTileItems + (seg[s].nbil + kTileItems - 1) / kTileItems;
      if (nc > seg[s].wcap) atomicOr(&ew->err, kErrCapacity);  // warm-start region too small
    }
    long long xc = pad, xt = nt;
    for (int off = 1; off < 32; off <<= 1) {
      long long yc = __shfl_up_sync(0xffffffffu, xc, off);
      long long yt = __shfl_up_sync(0xffffffffu, xt, off);
      if (lane >= off) { xc += yc; xt += yt; }
    }
    if (lane == 31) { s_c[warp] = xc; s_t[warp] = xt; }
    __syncthreads();
    if (warp == 0) {
      long long wc = s_c[lane], wt = s_t[lane];
      for (int off = 1; off < 32; off <<= 1) {
        long long yc = __shfl_up_sync(0xffffffffu, wc, off);
        long long yt = __shfl_up_sync(0xffffffffu, wt, off);
        if (lane >= off) { wc += yc; wt += yt; }
      }
      s_c[lane] = wc;
      s_t[lane] = wt;
    }
    __syncthreads();
    long long ec = s_carry_c + xc - pad + (warp ? s_c[warp - 1] : 0);
    long long et = s_carry_t + xt - nt + (warp ? s_t[warp - 1] : 0);
    if (s < nseg) {
      SegState& S = sst[s];
      S.nc = (int)nc;
      S.c0 = (int)ec;
      S.t0 = (int)et;
      S.nt = (int)nt;
      S.delta = (int)(ec - (seg[s].active ? cbase[seg[s].b0] : 0));
      seg_tstart[s] = (int)et;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      s_carry_c += s_c[31];
      s_carry_t += s_t[31];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    seg_tstart[nseg] = (int)s_carry_t;
    ew->nc_total = cbase[nb];
    ew->nc_pad = (int)s_carry_c;
    ew->ntiles = (int)s_carry_t;
    if (s_carry_c > (long long)ccap || s_carry_t > (long long)tcap) atomicOr(&ew->err, kErrCapacity);
  }
}

// tile -> segment (binary search of the tile starts)
__global__ void __launch_bounds__(kThreads) k_tile_table(int nseg, const int* __restrict__ seg_tstart,
                                                        int* __restrict__ tseg, int tcap,
                                                        const EngineWords* __restrict__ ew) {
  if (ew->err) return;
  const int nt = ew->ntiles;
  for (int t = blockIdx.x * kThreads + threadIdx.x; t < nt; t += gridDim.x * kThreads) {
    int lo = 0, hi = nseg - 1;  // last segment with tstart <= t and tiles
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (seg_tstart[mid] <= t) lo = mid; else hi = mid - 1;
    }
    tseg[t] = lo;
  }
}

// Contacts in (B, contact) key form for the B-side incidence; the radix input
// index is the contact's unpadded position.
__global__ void __launch_bounds__(kThreads) k_count_b(const uint32_t* __restrict__ idb,
                                                     const int* __restrict__ tseg,
                                                     const SegState* __restrict__ sst,
                                                     int* __restrict__ cnt, uint32_t* __restrict__ keys,
                                                     uint32_t* __restrict__ vals,
                                                     const EngineWords* __restrict__ ew) {
  if (ew->err) return;
  const int nt = ew->ntiles;
  for (int t = blockIdx.x; t < nt; t += gridDim.x) {
    const SegState& S = sst[tseg[t]];
    const int k0 = (t - S.t0) * kTileItems;
    for (int m = 0; m < kItemsPerThread; ++m) {
      int k = k0 + m * kThreads + threadIdx.x;
      if (k < S.nc) {
        int c = S.c0 + k;
        uint32_t b = idb[c];
        atomicAdd(&cnt[b], 1);
        keys[c - S.delta] = b;
        vals[c - S.delta] = (uint32_t)c;
      }
    }
  }
}

// Per-body incidence length: contacts where the body is B plus where it is A.
__global__ void __launch_bounds__(kThreads) k_inc_count(int nb, const int* __restrict__ bstart,
                                                       const int* __restrict__ acnt,
                                                       int* __restrict__ cnt,
                                                       const EngineWords* __restrict__ ew) {
  if (ew->err) return;
  int b = blockIdx.x * kThreads + threadIdx.x;
  if (b >= nb) return;
  cnt[b] = (bstart[b + 1] - bstart[b]) + acnt[b];
}

// B-side contacts (flagged, ascending) then the A-side range: the ascending
// contact order of the body's column of D.
__global__ void __launch_bounds__(kThreads) k_inc_fill(int nb, const int* __restrict__ bstart,
                                                      const uint32_t* __restrict__ binc,
                                                      const int* __restrict__ abase,
                                                      const int* __restrict__ acnt,
                                                      const int* __restrict__ bseg,
                                                      const SegState* __restrict__ sst,
                                                      const int* __restrict__ istart,
                                                      uint32_t* __restrict__ inc,
                                                      const EngineWords* __restrict__ ew) {
  if (ew->err) return;
  int b = blockIdx.x * kThreads + threadIdx.x;
  if (b >= nb) return;
  int o = istart[b];
  for (int i = bstart[b]; i < bstart[b + 1]; ++i) inc[o++] = binc[i] | 0x80000000u;
  const int n = acnt[b];
  if (n) {
    const int c0 = abase[b] + sst[bseg[b]].delta;
    for (int j = 0; j < n; ++j) inc[o++] = (uint32_t)(c0 + j);
  }
}

CollideArgs make_args(SceneDev& sd) {
  CollideArgs a;
  a.nb = sd.nb;
  a.n_small = sd.n_small;
  a.n_large = sd.n_large;
  a.max_seg_chunks = sd.max_seg_chunks;
  a.p4 = sd.p4;
  a.g4 = sd.geom4;
  a.fam = sd.family;
  a.bseg = sd.bseg;
  a.seg = sd.seg;
  a.sst = sd.sst;
  a.amin = sd.amin;
  a.amax = sd.amax;
  a.cell = sd.cell;
  a.small_ids = sd.small_ids;
  a.large_ids = sd.large_ids;
  a.sorted_bodies = sd.valA;
  a.cstart = sd.cell_start;
  a.cend = sd.cell_end;
  a.grid = sd.grid;
  a.cnt_cont = sd.cnt_cont;
  a.cnt_cand = sd.cnt_cand;
  a.wide_ids = sd.wide_ids;
  a.cbase = sd.cbase;
  a.ew = sd.ew;
  a.ccap = sd.ccap;
  a.ida = sd.ida;
  a.idb = sd.idb;
  a.F = sd.F;
  a.nf = sd.nf;
  a.gap = sd.gap;
  a.loc = sd.loc;
  return a;
}

int bits_for(int n) {
  int b = 0;
  while (b < 31 && (1 << b) < n) ++b;
  return b;
}

int blocks_for(long long n) { return (int)std::max(1LL, (n + kThreads - 1) / kThreads); }

}  // namespace

void collide(SceneDev& sd, cudaStream_t st, int64_t* launches) {
  const int nb = sd.nb;
  if (nb == 0) return;
  const int park = sd.ncell_cap - 1;  // cell of spheres in inactive segments
  cudaMemsetAsync(sd.cnt_cont, 0, sizeof(int) * (size_t)nb, st);
  cudaMemsetAsync(sd.cnt_cand, 0, sizeof(int) * (size_t)nb, st);
  k_seg_reset<<<blocks_for(sd.nseg), kThreads, 0, st>>>(sd.nseg, sd.grid, sd.sst, sd.ew);
  k_aabb<<<blocks_for(nb), kThreads, 0, st>>>(sd.p4, sd.geom4, sd.bseg, sd.seg, nb, sd.amin,
                                              sd.amax, sd.grid, sd.ew);
  k_grid_setup<<<blocks_for(sd.nseg), kThreads, 0, st>>>(sd.nseg, sd.seg, sd.grid, sd.ew);
  k_shift_and_bin<<<blocks_for(std::max(nb, sd.n_small)), kThreads, 0, st>>>(
      nb, sd.small_ids, sd.n_small, sd.bseg, sd.seg, sd.p4, sd.geom4, sd.amin, sd.amax, sd.grid,
      sd.cell, sd.keyA, sd.valA, park, sd.ew);
  *launches += 4;
  if (sd.n_small > 0) {
    radix_sort_pairs(sd.keyA, sd.valA, sd.keyB, sd.valB, sd.radix_hist, &sd.ew->n_small,
                     sd.n_small, bits_for(sd.ncell_cap), st, launches);
    cudaMemsetAsync(sd.cell_start, 0xff, sizeof(int) * (size_t)sd.ncell_cap, st);
    k_cell_ranges<<<blocks_for(sd.n_small), kThreads, 0, st>>>(sd.keyA, sd.n_small, sd.cell_start,
                                                               sd.cell_end, park, sd.ew);
    ++*launches;
  }
  CollideArgs a = make_args(sd);
  const int pair_blocks = (sd.n_small + kWarpsPerCta - 1) / kWarpsPerCta;
  dim3 box_grid(sd.max_seg_chunks, sd.n_large);
  if (sd.n_small > 0) {
    k_sphere_pairs<false><<<pair_blocks, kThreads, 0, st>>>(a);
    ++*launches;
  }
  if (sd.n_large > 0) {
    k_box_pairs<false><<<box_grid, kThreads, 0, st>>>(a, sd.large_chunk, nullptr);
    ++*launches;
  }
  exclusive_scan_i32(sd.cnt_cont, sd.cbase, nb, sd.scan_tmp, st, launches);
  k_seg_layout<<<1, 1024, 0, st>>>(sd.nseg, nb, sd.seg, sd.sst, sd.cbase, sd.seg_tstart, sd.ccap,
                                   sd.tcap, sd.ew);
  k_tile_table<<<std::max(1, std::min(sd.tcap / kThreads + 1, 1184)), kThreads, 0, st>>>(
      sd.nseg, sd.seg_tstart, sd.tseg, sd.tcap, sd.ew);
  *launches += 2;
  if (sd.n_small > 0) {
    k_sphere_pairs<true><<<pair_blocks, kThreads, 0, st>>>(a);
    k_sphere_pairs_wide<<<kWideGrid, kThreads, 0, st>>>(a);
    *launches += 2;
  }
  if (sd.n_large > 0) {
    exclusive_scan_i32(sd.large_chunk, sd.large_chunk_off, sd.max_seg_chunks * sd.n_large,
                       sd.scan_tmp, st, launches);
    k_box_pairs<true><<<box_grid, kThreads, 0, st>>>(a, nullptr, sd.large_chunk_off);
    ++*launches;
  }
  // B-side incidence: stable radix sort of (B, contact) keeps ascending contact order.
  cudaMemsetAsync(sd.cnt_cand, 0, sizeof(int) * (size_t)nb, st);
  const int tile_blocks = std::max(1, std::min(sd.tcap, 4 * 148 * 4));
  k_count_b<<<tile_blocks, kThreads, 0, st>>>(sd.idb, sd.tseg, sd.sst, sd.cnt_cand, sd.keyA,
                                              sd.valA, sd.ew);
  ++*launches;
  radix_sort_pairs(sd.keyA, sd.valA, sd.keyB, sd.valB, sd.radix_hist, &sd.ew->nc_total,
                   (int)sd.ccap, bits_for(nb), st, launches);
  exclusive_scan_i32(sd.cnt_cand, sd.binc_start, nb, sd.scan_tmp, st, launches);
  k_inc_count<<<blocks_for(nb), kThreads, 0, st>>>(nb, sd.binc_start, sd.cnt_cont, sd.cnt_cand,
                                                   sd.ew);
  ++*launches;
  exclusive_scan_i32(sd.cnt_cand, sd.inc_start, nb, sd.scan_tmp, st, launches);
  k_inc_fill<<<blocks_for(nb), kThreads, 0, st>>>(nb, sd.binc_start, sd.valA, sd.cbase,
                                                  sd.cnt_cont, sd.bseg, sd.sst, sd.inc_start,
                                                  sd.inc, sd.ew);
  ++*launches;
}

}  // namespace dv
