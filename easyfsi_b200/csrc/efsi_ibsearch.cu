// Immersed-boundary node search and in/out classification of the fluid
// nodes against the marker surface (HibmMpmIbNodeSearch, hibm_mpm.py:5385-6220).
//
// The reference visits every projection triangle (or, with none, every
// marker) from every node: O(nodes x triangles).  Here the triangles are
// binned once per call into a uniform grid of cells no smaller than the
// search radius, each triangle into every cell its bounding box, widened by
// the radius, overlaps.  A node then visits only the triangles of its own
// cell, which include every triangle closer than the radius.  The reference
// keeps the first candidate (in index order) whose distance is strictly the
// smallest; that is the lexicographic minimum of (distance, index), which
// each node computes here independently of the visiting order.  Far nodes
// (classify_far_internal_nodes) still need every triangle: they stop at the
// first triangle that sees them outside, since that alone makes the node
// "none" whatever the remaining triangles give.
//
// The same file holds the consumers of the search: the boundary-condition
// targets of the external IB nodes and the velocity-Dirichlet row assemblies
// (HibmMpmIbBoundaryConditions, hibm_mpm.py:6222-7800).
//
// Geometry runs in f32 with the reference's order of operations.  This file
// is compiled with -fmad=false, so no product is fused into a sum and the
// results round exactly as the expressions read.
#include <algorithm>
#include <cmath>

#include "efsi_common.cuh"

struct efsi_ib_search_plan {
  int32_t* count = nullptr;   // per bin
  int32_t* offset = nullptr;  // per bin + 1
  int32_t* cursor = nullptr;  // per bin
  int32_t* tile_sums = nullptr;
  int64_t bin_cap = 0;
  int32_t* entries = nullptr;  // triangle / marker indices by bin
  int64_t entry_cap = 0;
  unsigned long long* total = nullptr;       // entry total (device)
  unsigned long long* host_total = nullptr;  // and its pinned readback
  int32_t* claim = nullptr;  // per fluid cell: relocation claims, then region writers
  int64_t claim_cap = 0;
};

namespace efsi {
namespace {

constexpr int kNodeNone = 0, kNodeExternal = 1, kNodeInternal = 2;  // hibm_mpm.py:5387-5389
constexpr int kMaxBinsPerAxis = 128;
constexpr int64_t kMaxEntries = int64_t(1) << 27;  // beyond this the nodes scan every item
constexpr int kScanThreads = 1024, kScanPer = 4, kScanTile = kScanThreads * kScanPer;
constexpr int kRelocationWalkSteps = 24;  // HIBM_OWNER_RELOCATION_WALK_STEPS (hibm_mpm.py:23)

struct F3 {
  float x, y, z;
};
__device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ F3 sub(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ F3 add(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ F3 scale(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ F3 divide(F3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 cross(F3 a, F3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float norm(F3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ F3 ld3(const float* p, int64_t i) {
  return f3(__ldg(p + 3 * i), __ldg(p + 3 * i + 1), __ldg(p + 3 * i + 2));
}
__device__ __forceinline__ void st3(float* p, int64_t i, F3 v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}

// hibm_mpm.py:5494-5549: closest point of triangle abc to p (Voronoi-region
// walk); false for a degenerate triangle.
__device__ bool closest_point(F3 p, F3 a, F3 b, F3 c, F3& closest, F3& fn) {
  const F3 ab = sub(b, a), ac = sub(c, a);
  fn = cross(ab, ac);
  const float nn = norm(fn);
  closest = a;
  if (!(nn > 1.0e-12f)) return false;
  fn = divide(fn, nn);
  const F3 ap = sub(p, a);
  const float d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.0f && d2 <= 0.0f) return true;
  const F3 bp = sub(p, b);
  const float d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.0f && d4 <= d3) {
    closest = b;
    return true;
  }
  const float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
    closest = add(a, scale(ab, d1 / fmaxf(d1 - d3, 1.0e-30f)));
    return true;
  }
  const F3 cp = sub(p, c);
  const float d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0f && d5 <= d6) {
    closest = c;
    return true;
  }
  const float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
    closest = add(a, scale(ac, d2 / fmaxf(d2 - d6, 1.0e-30f)));
    return true;
  }
  const float va = d3 * d6 - d5 * d4;
  if (va <= 0.0f && d4 - d3 >= 0.0f && d5 - d6 >= 0.0f) {
    closest = add(b, scale(sub(c, b), (d4 - d3) / fmaxf(d4 - d3 + d5 - d6, 1.0e-30f)));
    return true;
  }
  const float denom = fmaxf(va + vb + vc, 1.0e-30f);
  const float v = vb / denom, w = vc / denom;
  closest = add(add(a, scale(ab, v)), scale(ac, w));
  return true;
}

struct SearchArgs {
  int nx, ny, nz;
  int64_t n;
  const float *cx, *cy, *cz;  // node centres per axis, or null: bmin + (i + 0.5) * sp
  float bmin[3], sp[3];
  const float* mx;  // marker positions (3 per marker)
  const float* mn;  // marker normals
  int marker_count;
  const int32_t* tri;  // projection triangles (3 marker indices each)
  int tri_count;
  float radius, probe, tol;
  int classify_far;
  // bins over the node box: cell of x on axis a = clamp(floor((x - lo) * inv), 0, nb - 1)
  float lo[3], inv[3], pad;
  int nb[3];
  const int32_t* offset;   // null: every node visits every item
  const int32_t* entries;
  // per-node fields (hibm_mpm.py:5418-5436) and the four report counts
  int32_t* kind;
  int32_t* nearest;
  float* sd;
  float* bp;
  float* ip;
  int32_t* pidx;
  float* pw;
  int32_t* report;
};

__device__ __forceinline__ int items(const SearchArgs& A) { return A.tri_count > 0 ? A.tri_count : A.marker_count; }

// Monotone in x, so a point inside an interval lands in a cell between the
// interval ends' cells.  NaN goes to cell 0.
__device__ __forceinline__ int bin_of(float x, float lo, float inv, int nb) {
  const float f = floorf((x - lo) * inv);
  if (!(f >= 0.0f)) return 0;
  if (f >= (float)(nb - 1)) return nb - 1;
  return (int)f;
}

__device__ __forceinline__ bool tri_indices(const SearchArgs& A, int t, int& ia, int& ib, int& ic) {
  ia = __ldg(A.tri + 3 * t);
  ib = __ldg(A.tri + 3 * t + 1);
  ic = __ldg(A.tri + 3 * t + 2);
  return ia >= 0 && ib >= 0 && ic >= 0 && ia < A.marker_count && ib < A.marker_count && ic < A.marker_count;
}

// hibm_mpm.py:5551-5560
__device__ __forceinline__ F3 oriented_normal(const SearchArgs& A, F3 fn, int ia, int ib, int ic) {
  F3 normal = fn;
  F3 avg = add(add(ld3(A.mn, ia), ld3(A.mn, ib)), ld3(A.mn, ic));
  const float an = norm(avg);
  if (an > 1.0e-12f) {
    avg = divide(avg, an);
    if (dot(normal, avg) < 0.0f) normal = f3(-normal.x, -normal.y, -normal.z);
  }
  return normal;
}

// Distance and signed distance of node p to item t (hibm_mpm.py:5900-5920 /
// 5967-5970); false for a degenerate triangle, which the node skips.
__device__ bool item_eval(const SearchArgs& A, int t, F3 p, float& distance, float& sdist) {
  if (A.tri_count > 0) {
    int ia, ib, ic;
    if (!tri_indices(A, t, ia, ib, ic)) return false;
    F3 closest, fn;
    if (!closest_point(p, ld3(A.mx, ia), ld3(A.mx, ib), ld3(A.mx, ic), closest, fn)) return false;
    const F3 normal = oriented_normal(A, fn, ia, ib, ic);
    const F3 off = sub(p, closest);
    distance = norm(off);
    sdist = dot(off, normal);
    return true;
  }
  const F3 off = sub(p, ld3(A.mx, t));
  distance = norm(off);
  sdist = dot(off, ld3(A.mn, t));
  return true;
}

__device__ __forceinline__ float clamp01(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

// Everything the node stores about its selected item t: the nearest marker,
// boundary point, normal, projection indices and barycentric weights
// (hibm_mpm.py:5562-5600, 5921-5935, 5971-6010).
__device__ void item_detail(const SearchArgs& A, int t, F3 p, int& marker, F3& boundary, F3& normal, int ix[3],
                            float w[3]) {
  if (A.tri_count > 0) {
    int ia, ib, ic;
    tri_indices(A, t, ia, ib, ic);
    const F3 a = ld3(A.mx, ia), b = ld3(A.mx, ib), c = ld3(A.mx, ic);
    F3 fn;
    closest_point(p, a, b, c, boundary, fn);
    normal = oriented_normal(A, fn, ia, ib, ic);
    // barycentric weights of the closest point, clamped and renormalised
    const F3 ab = sub(b, a), ac = sub(c, a), ap = sub(boundary, a);
    const float d00 = dot(ab, ab), d01 = dot(ab, ac), d11 = dot(ac, ac), d20 = dot(ap, ab), d21 = dot(ap, ac);
    const float denom = d00 * d11 - d01 * d01;
    w[0] = 1.0f;
    w[1] = 0.0f;
    w[2] = 0.0f;
    if (fabsf(denom) > 1.0e-30f) {
      float v = (d11 * d20 - d01 * d21) / denom;
      float ww = (d00 * d21 - d01 * d20) / denom;
      float u = 1.0f - v - ww;
      u = clamp01(u);
      v = clamp01(v);
      ww = clamp01(ww);
      const float total = fmaxf(u + v + ww, 1.0e-30f);
      w[0] = u / total;
      w[1] = v / total;
      w[2] = ww / total;
    }
    // the triangle's marker nearest to the node, first on ties
    marker = ia;
    const F3 oa = sub(p, a), ob = sub(p, b), oc = sub(p, c);
    float best = dot(oa, oa);
    const float db = dot(ob, ob);
    if (db < best) {
      best = db;
      marker = ib;
    }
    if (dot(oc, oc) < best) marker = ic;
    ix[0] = ia;
    ix[1] = ib;
    ix[2] = ic;
    return;
  }
  marker = t;
  boundary = ld3(A.mx, t);
  normal = ld3(A.mn, t);
  ix[0] = t;
  ix[1] = -1;
  ix[2] = -1;
  w[0] = 1.0f;
  w[1] = 0.0f;
  w[2] = 0.0f;
}

// The reference's strict "<" over items in index order keeps the smallest
// index among those at the smallest distance, and only distances below its
// 1e30 start value.
struct Best {
  float d = 1.0e30f;
  int t = -1;
  __device__ __forceinline__ void offer(float dist, int item) {
    const bool take = t < 0 ? dist < 1.0e30f : (dist < d || (dist == d && item < t));
    if (take) {
      d = dist;
      t = item;
    }
  }
};

__device__ __forceinline__ F3 node_position(const SearchArgs& A, int i, int j, int k) {
  if (A.cx != nullptr) return f3(__ldg(A.cx + i), __ldg(A.cy + j), __ldg(A.cz + k));
  return f3(A.bmin[0] + ((float)i + 0.5f) * A.sp[0], A.bmin[1] + ((float)j + 0.5f) * A.sp[1],
            A.bmin[2] + ((float)k + 0.5f) * A.sp[2]);
}

// Bin range of item t: its bounding box widened by the pad.
__device__ __forceinline__ void item_bins(const SearchArgs& A, int t, int b0[3], int b1[3]) {
  F3 lo, hi;
  if (A.tri_count > 0) {
    int ia, ib, ic;
    if (!tri_indices(A, t, ia, ib, ic)) {
      for (int a = 0; a < 3; ++a) b0[a] = 1, b1[a] = 0;  // empty range: never visited
      return;
    }
    const F3 a = ld3(A.mx, ia), b = ld3(A.mx, ib), c = ld3(A.mx, ic);
    lo = f3(fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z));
    hi = f3(fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z));
  } else {
    lo = hi = ld3(A.mx, t);
  }
  const float l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
  for (int a = 0; a < 3; ++a) {
    b0[a] = bin_of(l[a] - A.pad, A.lo[a], A.inv[a], A.nb[a]);
    b1[a] = bin_of(h[a] + A.pad, A.lo[a], A.inv[a], A.nb[a]);
  }
}

__global__ void k_ibs_bin_count(SearchArgs A, int32_t* count, unsigned long long* total) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= items(A)) return;
  int b0[3], b1[3];
  item_bins(A, t, b0, b1);
  if (b1[0] < b0[0]) return;
  atomicAdd(total, (unsigned long long)(b1[0] - b0[0] + 1) * (unsigned long long)(b1[1] - b0[1] + 1) *
                       (unsigned long long)(b1[2] - b0[2] + 1));
  for (int bx = b0[0]; bx <= b1[0]; ++bx)
    for (int by = b0[1]; by <= b1[1]; ++by)
      for (int bz = b0[2]; bz <= b1[2]; ++bz) atomicAdd(count + ((int64_t)bx * A.nb[1] + by) * A.nb[2] + bz, 1);
}

__global__ void k_ibs_bin_fill(SearchArgs A, const int32_t* offset, int32_t* cursor, int32_t* entries) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= items(A)) return;
  int b0[3], b1[3];
  item_bins(A, t, b0, b1);
  for (int bx = b0[0]; bx <= b1[0]; ++bx)
    for (int by = b0[1]; by <= b1[1]; ++by)
      for (int bz = b0[2]; bz <= b1[2]; ++bz) {
        const int64_t b = ((int64_t)bx * A.nb[1] + by) * A.nb[2] + bz;
        entries[offset[b] + atomicAdd(cursor + b, 1)] = t;
      }
}

// Exclusive block scan of one value per thread (kScanThreads threads).
__device__ __forceinline__ int32_t block_scan(int32_t v, int32_t* warp_tot, int32_t& total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    int32_t t = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;
  }
  __syncthreads();
  total = warp_tot[31];
  return (w > 0 ? warp_tot[w - 1] : 0) + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_ibs_tile_sums(const int32_t* count, int64_t n, int32_t* tile_sums) {
  __shared__ int32_t warp_tot[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanPer;
  int32_t s = 0;
#pragma unroll
  for (int q = 0; q < kScanPer; ++q) s += base + q < n ? count[base + q] : 0;
  int32_t total;
  block_scan(s, warp_tot, total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// One block: exclusive prefix of the tile sums, in place.
__global__ void __launch_bounds__(kScanThreads) k_ibs_tile_prefix(int32_t* tile_sums, int tiles) {
  __shared__ int32_t warp_tot[32];
  int32_t carry = 0;
  for (int base = 0; base < tiles; base += kScanThreads) {
    const int t = base + threadIdx.x;
    const int32_t v = t < tiles ? tile_sums[t] : 0;
    int32_t total;
    const int32_t ex = block_scan(v, warp_tot, total);
    if (t < tiles) tile_sums[t] = carry + ex;
    carry += total;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kScanThreads) k_ibs_offsets(const int32_t* count, int64_t n, const int32_t* tile_prefix,
                                                              int32_t* offset, int32_t* cursor) {
  __shared__ int32_t warp_tot[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanPer;
  int32_t v[kScanPer], s = 0;
#pragma unroll
  for (int q = 0; q < kScanPer; ++q) {
    v[q] = base + q < n ? count[base + q] : 0;
    s += v[q];
  }
  int32_t total;
  int32_t run = block_scan(s, warp_tot, total) + tile_prefix[blockIdx.x];
#pragma unroll
  for (int q = 0; q < kScanPer; ++q) {
    if (base + q < n) {
      offset[base + q] = run;
      cursor[base + q] = 0;
    }
    run += v[q];
  }
  if (base <= n - 1 && n - 1 < base + kScanPer) offset[n] = run;  // the entry total
}

// One thread per node (hibm_mpm.py:5837-6068 / 5603-5835).
__global__ void __launch_bounds__(256) k_ibs_search(SearchArgs A) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.n) return;
  const int k = (int)(c % A.nz), j = (int)((c / A.nz) % A.ny), i = (int)(c / ((int64_t)A.ny * A.nz));
  const F3 p = node_position(A, i, j, k);
  Best nearest, external;
  bool external_seen = false;
  int lo_e = 0, hi_e = items(A);
  const int32_t* list = nullptr;
  if (A.offset != nullptr) {
    const int64_t b = ((int64_t)bin_of(p.x, A.lo[0], A.inv[0], A.nb[0]) * A.nb[1] +
                       bin_of(p.y, A.lo[1], A.inv[1], A.nb[1])) * A.nb[2] +
                      bin_of(p.z, A.lo[2], A.inv[2], A.nb[2]);
    lo_e = __ldg(A.offset + b);
    hi_e = __ldg(A.offset + b + 1);
    list = A.entries;
  }
  for (int e = lo_e; e < hi_e; ++e) {
    const int t = list != nullptr ? __ldg(list + e) : e;
    float d, s;
    if (!item_eval(A, t, p, d, s)) continue;
    if (d < A.radius) {
      if (s > A.tol) {
        external_seen = true;
        external.offer(d, t);
      }
      nearest.offer(d, t);
    }
  }
  int kind = kNodeNone, marker = -1, ix[3] = {-1, -1, -1};
  float sd = 0.0f, w[3] = {0.0f, 0.0f, 0.0f};
  F3 boundary = f3(0.0f, 0.0f, 0.0f), interior = f3(0.0f, 0.0f, 0.0f);
  if (nearest.t >= 0) {
    atomicAdd(A.report + 0, 1);
    const int sel = (external_seen && external.t >= 0) ? external.t : nearest.t;
    F3 normal;
    item_detail(A, sel, p, marker, boundary, normal, ix, w);
    float dsel;
    item_eval(A, sel, p, dsel, sd);
    const float normal_distance = dot(sub(p, boundary), normal);
    float interior_distance = A.probe;
    if (normal_distance > A.tol) interior_distance = normal_distance + A.probe;
    interior = add(boundary, scale(normal, interior_distance));
    if (fabsf(sd) <= A.tol) atomicAdd(A.report + 3, 1);
    if (external_seen) {
      kind = kNodeExternal;
      atomicAdd(A.report + 1, 1);
    } else {
      kind = kNodeInternal;
      atomicAdd(A.report + 2, 1);
    }
  } else if (A.classify_far) {
    Best global;
    bool global_external_seen = false;
    const int nitems = items(A);
    for (int t = 0; t < nitems; ++t) {
      float d, s;
      if (!item_eval(A, t, p, d, s)) continue;
      if (s > A.tol) {
        global_external_seen = true;  // the node stays "none"
        break;
      }
      global.offer(d, t);
    }
    if (!global_external_seen && global.t >= 0) {
      kind = kNodeInternal;
      F3 normal;
      item_detail(A, global.t, p, marker, boundary, normal, ix, w);
      float dsel;
      item_eval(A, global.t, p, dsel, sd);
      interior = add(boundary, scale(normal, A.probe));
      atomicAdd(A.report + 2, 1);
    }
  }
  A.kind[c] = kind;
  A.nearest[c] = marker;
  A.sd[c] = sd;
  st3(A.bp, c, boundary);
  st3(A.ip, c, interior);
  for (int q = 0; q < 3; ++q) {
    A.pidx[3 * c + q] = ix[q];
    A.pw[3 * c + q] = w[q];
  }
}

__global__ void k_ibs_fill_anchor(int32_t* anchor, int64_t n3) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n3) anchor[q] = -1;
}

// ---------------------------------------------------------------------------
// Boundary-condition targets (hibm_mpm.py:6499-6577)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float max_abs3(F3 v) { return fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fabsf(v.z)); }

// atomic max / min of non-negative floats through their ordered bit patterns
__device__ __forceinline__ void atomic_max_nonneg(float* a, float v) { atomicMax((int*)a, __float_as_int(v)); }
__device__ __forceinline__ void atomic_min_nonneg(float* a, float v) { atomicMin((int*)a, __float_as_int(v)); }

__global__ void __launch_bounds__(256) k_ib_build_bc(int64_t n, const int32_t* __restrict__ kind,
                                                     const int32_t* __restrict__ nearest,
                                                     const int32_t* __restrict__ pidx, const float* __restrict__ pw,
                                                     const float* __restrict__ mv, const float* __restrict__ mn,
                                                     const float* __restrict__ mg, int marker_count,
                                                     int32_t* __restrict__ active, float* __restrict__ vel,
                                                     float* __restrict__ nrm, float* __restrict__ grad,
                                                     efsi_ib_bc_report* rep) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  int act = 0;
  F3 tv = f3(0.0f, 0.0f, 0.0f), tn = f3(0.0f, 0.0f, 0.0f);
  float tg = 0.0f;
  const int k = kind[c];
  if (k == kNodeExternal) {
    const int marker = nearest[c];
    if (0 <= marker && marker < marker_count) {
      float total = 0.0f;
      for (int q = 0; q < 3; ++q) {
        const int pm = pidx[3 * c + q];
        const float w = pw[3 * c + q];
        if (0 <= pm && pm < marker_count && w > 0.0f) {
          tv = add(tv, scale(ld3(mv, pm), w));
          tn = add(tn, scale(ld3(mn, pm), w));
          tg = tg + w * __ldg(mg + pm);
          total = total + w;
        }
      }
      if (total > 1.0e-12f) {
        const float inv = 1.0f / total;
        tv = scale(tv, inv);
        tn = scale(tn, inv);
        tg = tg * inv;
        const float nn = norm(tn);
        tn = nn > 1.0e-12f ? divide(tn, nn) : ld3(mn, marker);
      } else {
        tv = ld3(mv, marker);
        tn = ld3(mn, marker);
        tg = __ldg(mg + marker);
      }
      act = 1;
      atomicAdd(&rep->no_slip_dirichlet_count, 1);
      atomicAdd(&rep->pressure_neumann_count, 1);
      atomic_max_nonneg(&rep->max_abs_velocity_mps, max_abs3(tv));
    }
  } else if (k == kNodeInternal) {
    atomicAdd(&rep->inactive_internal_node_count, 1);
  }
  active[c] = act;
  st3(vel, c, tv);
  st3(nrm, c, tn);
  grad[c] = tg;
}

// ---------------------------------------------------------------------------
// Velocity-Dirichlet rows (hibm_mpm.py:6649-7800)
// ---------------------------------------------------------------------------
struct VdArgs {
  int n[3];
  int64_t ncell;
  const float* f[3];  // faces, n + 1
  const float* c[3];  // centres
  const int32_t* act;
  const float* bv;
  const float* bn;
  const float* bp;
  const float* ip;
  const int32_t* nearest;
  const int32_t* obs;
  const float* vel;
  const int32_t* mreg;
  int mcount;
  int32_t* vd_active;
  float* vd_value;
  float* vd_weight;
  int32_t* anchor;
  int32_t* region;
  efsi_ib_vd_report* rep;
  int32_t* claim;
};

__device__ __forceinline__ int64_t vidx(const VdArgs& A, int i, int j, int k) {
  return ((int64_t)i * A.n[1] + j) * A.n[2] + k;
}

// hibm_mpm.py:6714-6743
__device__ float axis_coordinate(float value, const float* faces, const float* centers, int count) {
  if (value <= centers[0]) {
    const float half = fmaxf(centers[0] - faces[0], 1.0e-18f);
    return -0.5f * (centers[0] - value) / half;
  }
  if (value >= centers[count - 1]) {
    const float half = fmaxf(faces[count] - centers[count - 1], 1.0e-18f);
    return (float)(count - 1) + 0.5f * (value - centers[count - 1]) / half;
  }
  int lower = 0, upper = count - 1;
  while (upper - lower > 1) {
    const int middle = (lower + upper) / 2;
    if (value >= centers[middle])
      lower = middle;
    else
      upper = middle;
  }
  upper = min(lower + 1, count - 1);
  const float distance = fmaxf(centers[upper] - centers[lower], 1.0e-18f);
  return (float)lower + (value - centers[lower]) / distance;
}

__device__ __forceinline__ F3 grid_coordinate(const VdArgs& A, F3 p) {
  return f3(axis_coordinate(p.x, A.f[0], A.c[0], A.n[0]), axis_coordinate(p.y, A.f[1], A.c[1], A.n[1]),
            axis_coordinate(p.z, A.f[2], A.c[2], A.n[2]));
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }

__device__ __forceinline__ void nearest_cell(const VdArgs& A, F3 g, int& i, int& j, int& k) {
  i = clampi((int)floorf(g.x + 0.5f), 0, A.n[0] - 1);
  j = clampi((int)floorf(g.y + 0.5f), 0, A.n[1] - 1);
  k = clampi((int)floorf(g.z + 0.5f), 0, A.n[2] - 1);
}

// hibm_mpm.py:6782-6812
__device__ F3 sample_velocity(const VdArgs& A, F3 g, float& fluid_weight) {
  const int i0 = clampi((int)floorf(g.x), 0, A.n[0] - 2);
  const int j0 = clampi((int)floorf(g.y), 0, A.n[1] - 2);
  const int k0 = clampi((int)floorf(g.z), 0, A.n[2] - 2);
  const float tx = fminf(fmaxf(g.x - (float)i0, 0.0f), 1.0f);
  const float ty = fminf(fmaxf(g.y - (float)j0, 0.0f), 1.0f);
  const float tz = fminf(fmaxf(g.z - (float)k0, 0.0f), 1.0f);
  F3 value = f3(0.0f, 0.0f, 0.0f);
  fluid_weight = 0.0f;
  for (int oi = 0; oi < 2; ++oi)
    for (int oj = 0; oj < 2; ++oj)
      for (int ok = 0; ok < 2; ++ok) {
        const float wx = oi == 0 ? 1.0f - tx : tx, wy = oj == 0 ? 1.0f - ty : ty, wz = ok == 0 ? 1.0f - tz : tz;
        const float w = wx * wy * wz;
        const int64_t c = vidx(A, i0 + oi, j0 + oj, k0 + ok);
        if (__ldg(A.obs + c) == 0) {
          value = add(value, scale(ld3(A.vel, c), w));
          fluid_weight = fluid_weight + w;
        }
      }
  if (fluid_weight > 1.0e-12f) value = divide(value, fluid_weight);
  return value;
}

// hibm_mpm.py:6846-6902
__device__ F3 walk_sample(const VdArgs& A, F3 bp, F3 normal, float base, float step, float& weight, float& distance) {
  weight = 0.0f;
  distance = base;
  for (int s = 0; s < 5; ++s) {
    const float cd = base + step * (float)s;
    float w;
    const F3 v = sample_velocity(A, grid_coordinate(A, add(bp, scale(normal, cd))), w);
    if (w > 1.0e-12f) {
      weight = w;
      distance = cd;
      return v;
    }
  }
  return f3(0.0f, 0.0f, 0.0f);
}

__device__ __forceinline__ float walk_step(F3 n, float wx, float wy, float wz) {
  const float s = fabsf(n.x) / fmaxf(wx, 1.0e-12f) + fabsf(n.y) / fmaxf(wy, 1.0e-12f) + fabsf(n.z) / fmaxf(wz, 1.0e-12f);
  return 0.5f / fmaxf(s, 1.0e-12f);
}

__device__ __forceinline__ void decode(const VdArgs& A, int64_t c, int& i, int& j, int& k) {
  k = (int)(c % A.n[2]);
  j = (int)((c / A.n[2]) % A.n[1]);
  i = (int)(c / ((int64_t)A.n[1] * A.n[2]));
}

__device__ __forceinline__ void report_row(const VdArgs& A, float alpha, F3 v, bool max_weight) {
  atomicAdd(&A.rep->active_rows, 1);
  atomic_min_nonneg(&A.rep->min_projection_weight, alpha);
  if (max_weight) atomic_max_nonneg(&A.rep->max_projection_weight, alpha);
  atomic_max_nonneg(&A.rep->max_abs_velocity_mps, max_abs3(v));
}

__global__ void k_vd_report_init(efsi_ib_vd_report* rep) {
  efsi_ib_vd_report r{};
  r.min_projection_weight = 1.0e30f;
  *rep = r;
}

__global__ void k_vd_fill(int32_t* a, int64_t n, int32_t v) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) a[q] = v;
}

// anchor reset and prefill from the interior probe point (hibm_mpm.py:7551-7616)
__global__ void __launch_bounds__(256) k_vd_prefill(VdArgs A) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.ncell) return;
  int ai = -1, aj = -1, ak = -1;
  if (A.act[c] == 1) {
    int i, j, k;
    nearest_cell(A, grid_coordinate(A, ld3(A.ip, c)), i, j, k);
    if (__ldg(A.obs + vidx(A, i, j, k)) == 0) ai = i, aj = j, ak = k;
  }
  A.anchor[3 * c] = ai;
  A.anchor[3 * c + 1] = aj;
  A.anchor[3 * c + 2] = ak;
}

// row reconstruction (hibm_mpm.py:6904-7335)
__global__ void __launch_bounds__(256) k_vd_reconstruct(VdArgs A) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.ncell) return;
  int act = 0;
  F3 value = f3(0.0f, 0.0f, 0.0f);
  float weight = 0.0f;
  if (A.act[c] == 1 && __ldg(A.obs + c) == 0) {
    int i, j, k;
    decode(A, c, i, j, k);
    const F3 bv = ld3(A.bv, c), normal = ld3(A.bn, c), bp = ld3(A.bp, c), ip = ld3(A.ip, c);
    const F3 node = f3(__ldg(A.c[0] + i), __ldg(A.c[1] + j), __ldg(A.c[2] + k));
    const float normal_den = dot(sub(ip, bp), normal);
    const float normal_dist = dot(sub(node, bp), normal);
    const float wx = __ldg(A.f[0] + i + 1) - __ldg(A.f[0] + i);
    const float wy = __ldg(A.f[1] + j + 1) - __ldg(A.f[1] + j);
    const float wz = __ldg(A.f[2] + k + 1) - __ldg(A.f[2] + k);
    float fw, sample_den;
    const F3 iv = walk_sample(A, bp, normal, normal_den, walk_step(normal, wx, wy, wz), fw, sample_den);
    F3 fb_vel = iv;
    float fb_alpha = 0.0f;
    int fai = -1, faj = -1, fak = -1;
    const bool segment = fw > 1.0e-12f && sample_den > 1.0e-12f && normal_dist >= 0.0f && normal_dist <= sample_den;
    bool fallback = false;
    if (!segment && fw > 1.0e-12f && sample_den > 1.0e-12f && normal_den > 1.0e-12f) {
      const F3 off = sub(node, bp);
      const float line = sqrtf(fmaxf(dot(off, off), 0.0f));
      if (line > 1.0e-12f) {
        const F3 fn = divide(off, line);
        const float fstep = walk_step(fn, wx, wy, wz);
        float fbw, fb_den;
        fb_vel = walk_sample(A, bp, fn, line + fstep, fstep, fbw, fb_den);
        if (fbw > 1.0e-12f && fb_den > line + 1.0e-12f) {
          fb_alpha = fminf(fmaxf(line / fmaxf(fb_den, 1.0e-12f), 0.0f), 1.0f);
          nearest_cell(A, grid_coordinate(A, add(bp, scale(fn, fb_den))), fai, faj, fak);
          fallback = __ldg(A.obs + vidx(A, fai, faj, fak)) == 0;
        }
      }
    }
    act = 1;
    if (segment) {
      const float alpha = fminf(fmaxf(normal_dist / sample_den, 0.0f), 1.0f);
      value = add(bv, scale(sub(iv, bv), alpha));
      weight = alpha;
      int ai, aj, ak;
      nearest_cell(A, grid_coordinate(A, add(bp, scale(normal, sample_den))), ai, aj, ak);
      if (__ldg(A.obs + vidx(A, ai, aj, ak)) == 0) {
        A.anchor[3 * c] = ai;
        A.anchor[3 * c + 1] = aj;
        A.anchor[3 * c + 2] = ak;
      }
      report_row(A, alpha, value, true);
    } else if (fallback) {
      value = add(bv, scale(sub(fb_vel, bv), fb_alpha));
      weight = fb_alpha;
      A.anchor[3 * c] = fai;
      A.anchor[3 * c + 1] = faj;
      A.anchor[3 * c + 2] = fak;
      report_row(A, fb_alpha, value, true);
    } else {
      value = bv;
      if (fw <= 1.0e-12f && normal_den > 1.0e-12f && normal_dist >= 0.0f) {
        atomicAdd(&A.rep->narrow_gap_rows, 1);
      } else {
        atomicAdd(&A.rep->invalid_rows, 1);
        if (fw <= 1.0e-12f)
          atomicAdd(&A.rep->invalid_no_fluid_sample_rows, 1);
        else if (normal_den <= 1.0e-12f)
          atomicAdd(&A.rep->invalid_nonpositive_gap_rows, 1);
        else if (normal_dist < 0.0f)
          atomicAdd(&A.rep->invalid_node_behind_boundary_rows, 1);
        else if (normal_dist > normal_den)
          atomicAdd(&A.rep->invalid_node_beyond_interior_rows, 1);
      }
      report_row(A, 0.0f, bv, false);
    }
  }
  A.vd_active[c] = act;
  st3(A.vd_value, c, value);
  A.vd_weight[c] = weight;
}

// The first fluid cell along the walk from a masked node's boundary point
// (its own side first, then the other; hibm_mpm.py:7359-7438); false if none.
__device__ bool relocation_target(const VdArgs& A, int64_t c, int& ti, int& tj, int& tk, float& tdist, F3& twn,
                                  float& tstep) {
  int i, j, k;
  decode(A, c, i, j, k);
  const F3 normal = ld3(A.bn, c), bp = ld3(A.bp, c);
  const F3 node = f3(__ldg(A.c[0] + i), __ldg(A.c[1] + j), __ldg(A.c[2] + k));
  const float side = dot(sub(node, bp), normal);
  const F3 primary = side < 0.0f ? f3(-normal.x, -normal.y, -normal.z) : normal;
  const float node_dist = fabsf(side);
  const float wx = __ldg(A.f[0] + i + 1) - __ldg(A.f[0] + i);
  const float wy = __ldg(A.f[1] + j + 1) - __ldg(A.f[1] + j);
  const float wz = __ldg(A.f[2] + k + 1) - __ldg(A.f[2] + k);
  for (int s = 0; s < 2; ++s) {
    const F3 wn = s == 0 ? primary : f3(-primary.x, -primary.y, -primary.z);
    const float start = s == 0 ? node_dist : 0.0f;
    const float step = walk_step(wn, wx, wy, wz);
    for (int q = 0; q < kRelocationWalkSteps; ++q) {
      const float cd = start + step * (float)(q + 1);
      int ci, cj, ck;
      nearest_cell(A, grid_coordinate(A, add(bp, scale(wn, cd))), ci, cj, ck);
      if (__ldg(A.obs + vidx(A, ci, cj, ck)) != 0) continue;
      const float ccd = dot(sub(f3(__ldg(A.c[0] + ci), __ldg(A.c[1] + cj), __ldg(A.c[2] + ck)), bp), wn);
      if (ccd > 1.0e-12f) {
        ti = ci;
        tj = cj;
        tk = ck;
        tdist = ccd;
        twn = wn;
        tstep = step;
        return true;
      }
    }
  }
  return false;
}

// Relocation, pass 1: every masked node claims its target cell unless a row
// sits there already; the lowest node index wins, as the first claim of the
// nodes visited in order.
__global__ void __launch_bounds__(256) k_vd_relocate_claim(VdArgs A) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.ncell || !(A.act[c] == 1 && __ldg(A.obs + c) != 0)) return;
  int ti, tj, tk;
  float tdist, tstep;
  F3 twn;
  if (!relocation_target(A, c, ti, tj, tk, tdist, twn, tstep)) return;
  const int64_t t = vidx(A, ti, tj, tk);
  if (A.vd_active[t] == 0) atomicMin(A.claim + t, (int32_t)c);
}

// Relocation, pass 2 (hibm_mpm.py:7439-7549): the winner writes the row.
__global__ void __launch_bounds__(256) k_vd_relocate_apply(VdArgs A) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.ncell || !(A.act[c] == 1 && __ldg(A.obs + c) != 0)) return;
  int ti, tj, tk;
  float tdist, tstep;
  F3 twn;
  if (!relocation_target(A, c, ti, tj, tk, tdist, twn, tstep)) {
    atomicAdd(&A.rep->blocked_rows, 1);
    return;
  }
  const int64_t t = vidx(A, ti, tj, tk);
  if (A.claim[t] != (int32_t)c) {
    atomicAdd(&A.rep->merged_rows, 1);
    return;
  }
  const F3 bp = ld3(A.bp, c), bv = ld3(A.bv, c);
  float sw, sd;
  const F3 sv = walk_sample(A, bp, twn, tdist + 2.0f * tstep, tstep, sw, sd);
  F3 tv = bv;
  float alpha = 0.0f;
  if (sw > 1.0e-12f && sd > tdist) {
    alpha = fminf(fmaxf(tdist / sd, 0.0f), 1.0f);
    tv = add(bv, scale(sub(sv, bv), alpha));
  }
  A.vd_active[t] = 1;
  st3(A.vd_value, t, tv);
  A.vd_weight[t] = alpha;
  A.anchor[3 * c] = ti;
  A.anchor[3 * c + 1] = tj;
  A.anchor[3 * c + 2] = tk;
  atomicAdd(&A.rep->relocated_rows, 1);
  report_row(A, alpha, tv, true);
}

// Region stamp (hibm_mpm.py:7618-7653): a cell written by several nodes
// keeps the region of the highest node index, as the last write of the nodes
// visited in order.  pass 0: record writers, pass 1: the writers write.
__device__ __forceinline__ bool stamp_anchor(const VdArgs& A, int64_t c, int64_t& a) {
  const int ai = A.anchor[3 * c], aj = A.anchor[3 * c + 1], ak = A.anchor[3 * c + 2];
  if (!(ai >= 0 && ai < A.n[0] && aj >= 0 && aj < A.n[1] && ak >= 0 && ak < A.n[2])) return false;
  a = vidx(A, ai, aj, ak);
  return A.vd_active[a] != 0;
}

__global__ void __launch_bounds__(256) k_vd_stamp(VdArgs A, int pass) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.ncell || A.act[c] != 1) return;
  const int marker = A.nearest[c];
  if (marker < 0 || marker >= A.mcount) return;
  const int32_t region = __ldg(A.mreg + marker);
  int64_t a;
  const bool own = A.vd_active[c] != 0, anc = stamp_anchor(A, c, a);
  if (pass == 0) {
    if (own) atomicMax(A.claim + c, (int32_t)c);
    if (anc) atomicMax(A.claim + a, (int32_t)c);
  } else {
    if (own && A.claim[c] == (int32_t)c) A.region[c] = region;
    if (anc && A.claim[a] == (int32_t)c) A.region[a] = region;
  }
}

// hibm_mpm.py:6649-6688 _assemble_velocity_dirichlet_boundary_rows_kernel:
// the target velocity itself on every active IB node that is not masked.
__global__ void __launch_bounds__(256) k_vd_direct(VdArgs A) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.ncell) return;
  int act = 0;
  F3 value = f3(0.0f, 0.0f, 0.0f);
  if (A.act[c] == 1) {
    if (__ldg(A.obs + c) == 0) {
      act = 1;
      value = ld3(A.bv, c);
      atomicAdd(&A.rep->active_rows, 1);
      atomic_max_nonneg(&A.rep->max_abs_velocity_mps, max_abs3(value));
    } else {
      atomicAdd(&A.rep->blocked_rows, 1);
    }
  }
  A.vd_active[c] = act;
  st3(A.vd_value, c, value);
}

template <typename T>
int grow(T*& buf, int64_t& cap, int64_t need) {
  if (need <= cap) return EFSI_OK;
  cudaFree(buf);
  buf = nullptr;
  cap = 0;
  EFSI_CUDA_CHECK(cudaMalloc(&buf, (size_t)need * sizeof(T)));
  cap = need;
  return EFSI_OK;
}

}  // namespace
}  // namespace efsi

using namespace efsi;

extern "C" {

int efsi_ib_search_plan_create(efsi_ib_search_plan** out) {
  EFSI_ARG_CHECK(out != nullptr, "null plan pointer");
  efsi_ib_search_plan* P = new efsi_ib_search_plan();
  if (cudaMalloc(&P->total, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMallocHost(&P->host_total, sizeof(unsigned long long)) != cudaSuccess) {
    cudaFree(P->total);
    delete P;
    set_error("cudaMallocHost failed for the node-search readback");
    return EFSI_ERR_CUDA;
  }
  *out = P;
  return EFSI_OK;
}

int efsi_ib_search_plan_destroy(efsi_ib_search_plan* P) {
  if (P == nullptr) return EFSI_OK;
  cudaFree(P->count);
  cudaFree(P->offset);
  cudaFree(P->cursor);
  cudaFree(P->tile_sums);
  cudaFree(P->entries);
  cudaFree(P->claim);
  cudaFree(P->total);
  cudaFreeHost(P->host_total);
  delete P;
  return EFSI_OK;
}

int efsi_ib_reset_anchor_cells(int32_t* anchor_cells, int64_t node_count, void* stream) {
  EFSI_ARG_CHECK(anchor_cells != nullptr && node_count >= 0, "bad anchor-cell arguments");
  if (node_count == 0) return EFSI_OK;
  const int64_t n3 = 3 * node_count;
  EFSI_COUNTED k_ibs_fill_anchor<<<(unsigned)((n3 + 255) / 256), 256, 0, as_stream(stream)>>>(anchor_cells, n3);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_ib_node_search(efsi_ib_search_plan* P, const efsi_ib_search_params* prm, const efsi_ib_search_fields* out,
                        void* stream) {
  EFSI_ARG_CHECK(P != nullptr && prm != nullptr && out != nullptr, "null argument");
  EFSI_ARG_CHECK(prm->nx > 0 && prm->ny > 0 && prm->nz > 0, "grid_nodes must be positive");
  EFSI_ARG_CHECK(prm->marker_count >= 0 && prm->triangle_count >= 0, "negative marker or triangle count");
  EFSI_ARG_CHECK(prm->marker_count == 0 || (prm->marker_x != nullptr && prm->marker_n != nullptr),
                 "marker arrays missing");
  EFSI_ARG_CHECK(prm->triangle_count == 0 || prm->triangles != nullptr, "triangle array missing");
  EFSI_ARG_CHECK(std::isfinite(prm->search_radius_m) && prm->search_radius_m > 0.0f,
                 "search_radius_m must be a finite positive number");
  EFSI_ARG_CHECK(std::isfinite(prm->interior_probe_distance_m) && prm->interior_probe_distance_m > 0.0f,
                 "interior_probe_distance_m must be a finite positive number");
  EFSI_ARG_CHECK(std::isfinite(prm->sign_tolerance_m) && prm->sign_tolerance_m >= 0.0f,
                 "sign_tolerance_m must be a finite non-negative number");
  const bool centres = prm->cell_center_x_m != nullptr;
  EFSI_ARG_CHECK(!centres || (prm->cell_center_y_m != nullptr && prm->cell_center_z_m != nullptr),
                 "cell centre arrays must be given for all three axes");
  EFSI_ARG_CHECK(out->node_kind && out->nearest_marker && out->signed_distance_m && out->boundary_point_m &&
                     out->interior_fluid_point_m && out->projection_marker_indices &&
                     out->projection_marker_weights && out->report,
                 "output field missing");
  for (int a = 0; a < 3; ++a)
    EFSI_ARG_CHECK(std::isfinite(prm->box_min_m[a]) && std::isfinite(prm->box_max_m[a]) &&
                       prm->box_max_m[a] > prm->box_min_m[a],
                   "box_max_m must be greater than box_min_m");
  cudaStream_t s = as_stream(stream);

  SearchArgs A{};
  A.nx = prm->nx;
  A.ny = prm->ny;
  A.nz = prm->nz;
  A.n = (int64_t)prm->nx * prm->ny * prm->nz;
  A.cx = prm->cell_center_x_m;
  A.cy = prm->cell_center_y_m;
  A.cz = prm->cell_center_z_m;
  for (int a = 0; a < 3; ++a) {
    A.bmin[a] = prm->bounds_min_m[a];
    A.sp[a] = prm->spacing_m[a];
  }
  A.mx = prm->marker_x;
  A.mn = prm->marker_n;
  A.marker_count = prm->marker_count;
  A.tri = prm->triangles;
  A.tri_count = prm->triangle_count;
  A.radius = prm->search_radius_m;
  A.probe = prm->interior_probe_distance_m;
  A.tol = prm->sign_tolerance_m;
  A.classify_far = prm->classify_far_internal_nodes ? 1 : 0;
  A.kind = out->node_kind;
  A.nearest = out->nearest_marker;
  A.sd = out->signed_distance_m;
  A.bp = out->boundary_point_m;
  A.ip = out->interior_fluid_point_m;
  A.pidx = out->projection_marker_indices;
  A.pw = out->projection_marker_weights;
  A.report = out->report;
  EFSI_CUDA_CHECK(cudaMemsetAsync(out->report, 0, 4 * sizeof(int32_t), s));

  // Bins over the node box, cells no smaller than the radius.  The pad widens
  // every item's box by the radius plus a margin far above f32 rounding of
  // the distances and coordinates.
  float scale_m = 0.0f;
  int64_t nbins = 1;
  for (int a = 0; a < 3; ++a) {
    const float ext = prm->box_max_m[a] - prm->box_min_m[a];
    const double cells = std::floor((double)ext / (double)prm->search_radius_m);
    A.nb[a] = (int)std::max(1.0, std::min((double)kMaxBinsPerAxis, cells));
    A.lo[a] = prm->box_min_m[a];
    A.inv[a] = (float)A.nb[a] / ext;
    nbins *= A.nb[a];
    scale_m = std::max({scale_m, ext, std::fabs(prm->box_min_m[a]), std::fabs(prm->box_max_m[a])});
  }
  A.pad = prm->search_radius_m * 1.001f + 1.0e-5f * scale_m;
  const int nitems = prm->triangle_count > 0 ? prm->triangle_count : prm->marker_count;
  A.offset = nullptr;
  A.entries = nullptr;
  if (nitems > 0) {
    const int64_t tiles = (nbins + kScanTile - 1) / kScanTile;
    if (nbins > P->bin_cap) {
      cudaFree(P->count);
      cudaFree(P->offset);
      cudaFree(P->cursor);
      cudaFree(P->tile_sums);
      P->count = P->offset = P->cursor = P->tile_sums = nullptr;
      P->bin_cap = 0;
      EFSI_CUDA_CHECK(cudaMalloc(&P->count, (size_t)nbins * sizeof(int32_t)));
      EFSI_CUDA_CHECK(cudaMalloc(&P->offset, (size_t)(nbins + 1) * sizeof(int32_t)));
      EFSI_CUDA_CHECK(cudaMalloc(&P->cursor, (size_t)nbins * sizeof(int32_t)));
      EFSI_CUDA_CHECK(cudaMalloc(&P->tile_sums, (size_t)tiles * sizeof(int32_t)));
      P->bin_cap = nbins;
    }
    // per-bin counts and, in 64 bits, the entry total: the int32 scan runs
    // only when that total is small enough for it
    EFSI_CUDA_CHECK(cudaMemsetAsync(P->count, 0, (size_t)nbins * sizeof(int32_t), s));
    EFSI_CUDA_CHECK(cudaMemsetAsync(P->total, 0, sizeof(unsigned long long), s));
    const unsigned ig = (unsigned)((nitems + 255) / 256);
    EFSI_COUNTED k_ibs_bin_count<<<ig, 256, 0, s>>>(A, P->count, P->total);
    EFSI_LAUNCH_CHECK();
    EFSI_CUDA_CHECK(
        cudaMemcpyAsync(P->host_total, P->total, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
    const unsigned long long total = *P->host_total;
    if (total <= (unsigned long long)kMaxEntries) {
      EFSI_COUNTED k_ibs_tile_sums<<<(unsigned)tiles, kScanThreads, 0, s>>>(P->count, nbins, P->tile_sums);
      EFSI_COUNTED k_ibs_tile_prefix<<<1, kScanThreads, 0, s>>>(P->tile_sums, (int)tiles);
      EFSI_COUNTED k_ibs_offsets<<<(unsigned)tiles, kScanThreads, 0, s>>>(P->count, nbins, P->tile_sums, P->offset,
                                                                        P->cursor);
      EFSI_TRY(grow(P->entries, P->entry_cap, std::max<int64_t>((int64_t)total, 1)));
      EFSI_COUNTED k_ibs_bin_fill<<<ig, 256, 0, s>>>(A, P->offset, P->cursor, P->entries);
      EFSI_LAUNCH_CHECK();
      A.offset = P->offset;
      A.entries = P->entries;
    }
  }
  EFSI_COUNTED k_ibs_search<<<(unsigned)((A.n + 255) / 256), 256, 0, s>>>(A);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_ib_build_boundary_conditions(int64_t node_count, const int32_t* node_kind, const int32_t* nearest_marker,
                                      const int32_t* projection_marker_indices,
                                      const float* projection_marker_weights, const float* marker_velocity,
                                      const float* marker_normal, const float* marker_gradient, int32_t marker_count,
                                      int32_t* active, float* velocity, float* normal, float* gradient,
                                      efsi_ib_bc_report* report_device, void* stream) {
  EFSI_ARG_CHECK(node_count >= 0 && marker_count >= 0, "negative node or marker count");
  EFSI_ARG_CHECK(node_kind && nearest_marker && projection_marker_indices && projection_marker_weights && active &&
                     velocity && normal && gradient && report_device,
                 "null argument");
  EFSI_ARG_CHECK(marker_count == 0 || (marker_velocity && marker_normal && marker_gradient), "marker arrays missing");
  cudaStream_t s = as_stream(stream);
  EFSI_CUDA_CHECK(cudaMemsetAsync(report_device, 0, sizeof(efsi_ib_bc_report), s));
  if (node_count == 0) return EFSI_OK;
  EFSI_COUNTED k_ib_build_bc<<<(unsigned)((node_count + 255) / 256), 256, 0, s>>>(
      node_count, node_kind, nearest_marker, projection_marker_indices, projection_marker_weights, marker_velocity,
      marker_normal, marker_gradient, marker_count, active, velocity, normal, gradient, report_device);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_ib_velocity_dirichlet_rows(efsi_ib_search_plan* P, const efsi_ib_vd_params* prm,
                                    const efsi_ib_vd_fields* out, int32_t reconstruct, void* stream) {
  EFSI_ARG_CHECK(P != nullptr && prm != nullptr && out != nullptr, "null argument");
  EFSI_ARG_CHECK(prm->nx >= 2 && prm->ny >= 2 && prm->nz >= 2, "grid_nodes must contain three values >= 2");
  EFSI_ARG_CHECK(prm->active_ib_node && prm->target_velocity && prm->obstacle && out->active && out->value_mps &&
                     out->report,
                 "null argument");
  if (reconstruct) {
    EFSI_ARG_CHECK(prm->face_x_m && prm->face_y_m && prm->face_z_m && prm->center_x_m && prm->center_y_m &&
                       prm->center_z_m && prm->target_normal && prm->boundary_point_m &&
                       prm->interior_fluid_point_m && prm->velocity && out->projection_weight && out->anchor_cell,
                   "reconstructed rows need the grid axes, targets, node points, velocity and anchor fields");
    EFSI_ARG_CHECK(prm->marker_region_id == nullptr || (out->marker_region_id && prm->nearest_marker),
                   "the region stamp needs the nearest markers and the region output");
  }
  cudaStream_t s = as_stream(stream);
  VdArgs A{};
  A.n[0] = prm->nx;
  A.n[1] = prm->ny;
  A.n[2] = prm->nz;
  A.ncell = (int64_t)prm->nx * prm->ny * prm->nz;
  A.f[0] = prm->face_x_m;
  A.f[1] = prm->face_y_m;
  A.f[2] = prm->face_z_m;
  A.c[0] = prm->center_x_m;
  A.c[1] = prm->center_y_m;
  A.c[2] = prm->center_z_m;
  A.act = prm->active_ib_node;
  A.bv = prm->target_velocity;
  A.bn = prm->target_normal;
  A.bp = prm->boundary_point_m;
  A.ip = prm->interior_fluid_point_m;
  A.nearest = prm->nearest_marker;
  A.obs = prm->obstacle;
  A.vel = prm->velocity;
  A.mreg = prm->marker_region_id;
  A.mcount = prm->marker_count;
  A.vd_active = out->active;
  A.vd_value = out->value_mps;
  A.vd_weight = out->projection_weight;
  A.anchor = out->anchor_cell;
  A.region = out->marker_region_id;
  A.rep = out->report;
  const unsigned grid = (unsigned)((A.ncell + 255) / 256);
  EFSI_COUNTED k_vd_report_init<<<1, 1, 0, s>>>(out->report);
  if (!reconstruct) {
    EFSI_COUNTED k_vd_direct<<<grid, 256, 0, s>>>(A);
    EFSI_LAUNCH_CHECK();
    return EFSI_OK;
  }
  EFSI_TRY(grow(P->claim, P->claim_cap, A.ncell));
  A.claim = P->claim;
  EFSI_COUNTED k_vd_prefill<<<grid, 256, 0, s>>>(A);
  EFSI_COUNTED k_vd_reconstruct<<<grid, 256, 0, s>>>(A);
  EFSI_COUNTED k_vd_fill<<<grid, 256, 0, s>>>(A.claim, A.ncell, INT32_MAX);
  EFSI_COUNTED k_vd_relocate_claim<<<grid, 256, 0, s>>>(A);
  EFSI_COUNTED k_vd_relocate_apply<<<grid, 256, 0, s>>>(A);
  if (A.mreg != nullptr) {
    EFSI_COUNTED k_vd_fill<<<grid, 256, 0, s>>>(A.claim, A.ncell, -1);
    EFSI_COUNTED k_vd_stamp<<<grid, 256, 0, s>>>(A, 0);
    EFSI_COUNTED k_vd_stamp<<<grid, 256, 0, s>>>(A, 1);
  }
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

}  // extern "C"
