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
};

namespace efsi {
namespace {

constexpr int kNodeNone = 0, kNodeExternal = 1, kNodeInternal = 2;  // hibm_mpm.py:5387-5389
constexpr int kMaxBinsPerAxis = 128;
constexpr int64_t kMaxEntries = int64_t(1) << 27;  // beyond this the nodes scan every item
constexpr int kScanThreads = 1024, kScanPer = 4, kScanTile = kScanThreads * kScanPer;

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
__device__ __forceinline__ F3 ld3(const float* p, int i) {
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

}  // extern "C"
