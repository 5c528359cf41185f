// HIBM surface-marker kernels, B200 path (simulation_core/hibm_mpm.py):
// pressure traction sampling at the markers, marker forces, clearing the MPM
// external forces, marker -> particle force spreading and particle -> marker
// surface feedback.
//
// The reference's spreading and feedback loop, for every marker, serially over
// ALL particles (twice for the spreading): O(markers x particles).  The tent
// kernel w = prod_d max(1 - |dx_d| / R, 0) vanishes outside a cube of half-edge
// R, so here particles are first sorted into bins of edge R (counting sort,
// particle order kept inside a bin) and a marker only visits the 3x3x3 bins
// around it.  Particles outside the bin box are clamped into the edge bins,
// which keeps every particle within R of a marker inside the visited bins.
#include <cuda_runtime.h>

#include <cmath>
#include <utility>

#include "efsi_common.cuh"

struct efsi_bin_plan {
  int capacity = 0;
  float bmin[3] = {0, 0, 0};
  float R = 1.0f;
  float invR = 1.0f;
  int nb[3] = {1, 1, 1};
  int nbins = 1;  // + 1 bucket for non-finite particles
  int count_last = 0;
  int32_t* key = nullptr;
  int32_t* sorted = nullptr;
  int32_t* count = nullptr;
  int32_t* offset = nullptr;
  int32_t* cursor = nullptr;
  int32_t* tile_sums = nullptr;  // per-tile bin counts of the offset scan
};

namespace efsi {

__device__ __forceinline__ bool finite3(const float* v) {
  return isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]);
}

__device__ __forceinline__ void atomic_max_nonneg_d(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// hibm_mpm.py:911-939 _axis_grid_coordinate_device (f32).
__device__ __forceinline__ float axis_coord_m(float v, const float* faces, const float* centers, int count) {
  float coord;
  const float c0 = centers[0], cl = centers[count - 1];
  if (v <= c0) {
    float hw = fmaxf(__fsub_rn(c0, faces[0]), 1.0e-18f);
    coord = __fdiv_rn(__fmul_rn(-0.5f, __fsub_rn(c0, v)), hw);
  } else if (v >= cl) {
    float hw = fmaxf(__fsub_rn(faces[count], cl), 1.0e-18f);
    coord = __fadd_rn((float)(count - 1), __fdiv_rn(__fmul_rn(0.5f, __fsub_rn(v, cl)), hw));
  } else {
    int lo = 0, hi = count - 1;
    while (hi - lo > 1) {
      int mid = (lo + hi) / 2;
      if (v >= centers[mid])
        lo = mid;
      else
        hi = mid;
    }
    hi = min(lo + 1, count - 1);
    float dist = fmaxf(__fsub_rn(centers[hi], centers[lo]), 1.0e-18f);
    coord = __fadd_rn((float)lo, __fdiv_rn(__fsub_rn(v, centers[lo]), dist));
  }
  return coord;
}

// hibm_mpm.py:981-1009 obstacle-masked trilinear pressure sample (f64 value,
// f32 weights).
__device__ __forceinline__ double sample_p(int nx, int ny, int nz, const int32_t* obs, const double* p, float gx,
                                           float gy, float gz, double& fw) {
  int i0 = min(max((int)floorf(gx), 0), nx - 2);
  int j0 = min(max((int)floorf(gy), 0), ny - 2);
  int k0 = min(max((int)floorf(gz), 0), nz - 2);
  float tx = fminf(fmaxf(gx - (float)i0, 0.0f), 1.0f);
  float ty = fminf(fmaxf(gy - (float)j0, 0.0f), 1.0f);
  float tz = fminf(fmaxf(gz - (float)k0, 0.0f), 1.0f);
  double val = 0.0;
  fw = 0.0;
  for (int oi = 0; oi < 2; ++oi)
    for (int oj = 0; oj < 2; ++oj)
      for (int ok = 0; ok < 2; ++ok) {
        float w = __fmul_rn(__fmul_rn(oi == 0 ? 1.0f - tx : tx, oj == 0 ? 1.0f - ty : ty), ok == 0 ? 1.0f - tz : tz);
        int64_t c = ((int64_t)(i0 + oi) * ny + (j0 + oj)) * nz + (k0 + ok);
        if (obs[c] == 0) {
          val += (double)w * p[c];
          fw += (double)w;
        }
      }
  if (fw > 1.0e-12) val /= fw;
  return val;
}

// hibm_mpm.py:2253-2432 _sample_pressure_only_marker_tractions_kernel.
__global__ void k_tractions(int nx, int ny, int nz, efsi_grid_axes A, const float* wx, const float* wy,
                            const float* wz, const int32_t* obs, const double* p, int M, const float* xg,
                            const float* ng, const int32_t* region, int two_sided, int one_sided_region,
                            float one_sided_ref, double* t, int32_t* valid, double* rep) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  const float x[3] = {xg[3 * m], xg[3 * m + 1], xg[3 * m + 2]};
  const float n[3] = {ng[3 * m], ng[3 * m + 1], ng[3 * m + 2]};
  const float g0 = axis_coord_m(x[0], A.fx, A.cx, nx), g1 = axis_coord_m(x[1], A.fy, A.cy, ny),
              g2 = axis_coord_m(x[2], A.fz, A.cz, nz);
  double pw;
  double pr = sample_p(nx, ny, nz, obs, p, g0, g1, g2, pw);
  double tr[3] = {-pr * (double)n[0], -pr * (double)n[1], -pr * (double)n[2]};
  bool ok = pw > 1.0e-12;
  if (two_sided) {
    int in = min(max((int)floorf(g0), 0), nx - 1), jn = min(max((int)floorf(g1), 0), ny - 1),
        kn = min(max((int)floorf(g2), 0), nz - 1);
    float nsi = __fadd_rn(__fadd_rn(__fdiv_rn(fabsf(n[0]), wx[in]), __fdiv_rn(fabsf(n[1]), wy[jn])),
                          __fdiv_rn(fabsf(n[2]), wz[kn]));
    float h = __fdiv_rn(1.0f, fmaxf(nsi, 1.0e-12f));
    double outside = 0.0, inside = 0.0;
    int of = 0, inf_ = 0;
    for (int pi = 0; pi < 3; ++pi) {
      const float mul = (float)(pi + 1);
      float op[3], ip[3];
      for (int a = 0; a < 3; ++a) {
        float step = __fmul_rn(__fmul_rn(mul, h), n[a]);
        op[a] = __fadd_rn(x[a], step);
        ip[a] = __fsub_rn(x[a], step);
      }
      double w;
      double so = sample_p(nx, ny, nz, obs, p, axis_coord_m(op[0], A.fx, A.cx, nx), axis_coord_m(op[1], A.fy, A.cy, ny),
                           axis_coord_m(op[2], A.fz, A.cz, nz), w);
      if (of == 0 && w > 1.0e-12) {
        outside = so;
        of = 1;
      }
      double si = sample_p(nx, ny, nz, obs, p, axis_coord_m(ip[0], A.fx, A.cx, nx), axis_coord_m(ip[1], A.fy, A.cy, ny),
                           axis_coord_m(ip[2], A.fz, A.cz, nz), w);
      if (inf_ == 0 && w > 1.0e-12) {
        inside = si;
        inf_ = 1;
      }
    }
    const double ref = (double)one_sided_ref;
    if (one_sided_region != -1 && region[m] == one_sided_region && inf_) {
      for (int a = 0; a < 3; ++a) tr[a] = (inside - ref) * (double)n[a];
      ok = true;
      atomicAdd(rep + 3, 1.0);
    } else if (one_sided_region != -1 && region[m] == one_sided_region && of) {
      for (int a = 0; a < 3; ++a) tr[a] = (ref - outside) * (double)n[a];
      ok = true;
      atomicAdd(rep + 3, 1.0);
    } else if (of && inf_) {
      for (int a = 0; a < 3; ++a) tr[a] = (inside - outside) * (double)n[a];
      ok = true;
      atomicAdd(rep + 2, 1.0);
    } else {
      ok = false;
    }
  }
  if (ok) {
    for (int a = 0; a < 3; ++a) t[3 * m + a] = tr[a];
    valid[m] = 1;
    atomicAdd(rep + 0, 1.0);
    atomic_max_nonneg_d(rep + 4, sqrt(tr[0] * tr[0] + tr[1] * tr[1] + tr[2] * tr[2]));
  } else {
    t[3 * m] = t[3 * m + 1] = t[3 * m + 2] = 0.0;
    valid[m] = 0;
    atomicAdd(rep + 1, 1.0);
  }
}

// hibm_mpm.py:903-909 _compute_marker_forces_kernel.
__global__ void k_marker_forces(int M, const double* t, const float* A, double* F) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  const double a = (double)A[m];
  F[3 * m] = t[3 * m] * a;
  F[3 * m + 1] = t[3 * m + 1] * a;
  F[3 * m + 2] = t[3 * m + 2] * a;
}

// hibm_mpm.py:4861-4878 _clear_mpm_external_forces_kernel.
__global__ void k_clear_fext(int P, float* f, double* rep) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  float* q = f + 3 * p;
  float nn = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
  if (rep != nullptr && nn > 0.0f) {
    atomicAdd(rep + 0, 1.0);
    atomic_max_nonneg_d(rep + 1, (double)nn);
  }
  q[0] = q[1] = q[2] = 0.0f;
}

struct BinView {
  float bmin[3];
  float invR;
  float R;
  int nb[3];
  int nbins;
  const int32_t* sorted;
  const int32_t* offset;
};

__device__ __forceinline__ int bin_axis(float v, float lo, float invR, int n) {
  int b = (int)floorf((v - lo) * invR);
  return min(max(b, 0), n - 1);
}

__global__ void k_bin_count(BinView B, const float* x, int P, int32_t* key, int32_t* count) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  int kk = B.nbins;
  const float* xp = x + 3 * p;
  if (finite3(xp)) {
    int b0 = bin_axis(xp[0], B.bmin[0], B.invR, B.nb[0]);
    int b1 = bin_axis(xp[1], B.bmin[1], B.invR, B.nb[1]);
    int b2 = bin_axis(xp[2], B.bmin[2], B.invR, B.nb[2]);
    kk = (b0 * B.nb[1] + b1) * B.nb[2] + b2;
  }
  key[p] = kk;
  unsigned peers = __match_any_sync(__activemask(), kk);
  int leader = __ffs(peers) - 1;
  if ((threadIdx.x & 31) == leader) atomicAdd(count + kk, __popc(peers));
}

// Bin offsets by a two-pass scan over tiles of kScanTile counts: per-tile
// totals, then every tile scans itself after summing the totals before it.
constexpr int kScanThreads = 1024, kScanPer = 4, kScanTile = kScanThreads * kScanPer;

__device__ __forceinline__ int32_t block_exclusive_scan(int32_t v, int32_t* warp_tot, int32_t& total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    int32_t t = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;  // inclusive over warps
  }
  __syncthreads();
  total = warp_tot[31];
  const int32_t before = w > 0 ? warp_tot[w - 1] : 0;
  return before + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_bin_tile_sums(const int32_t* count, int n, int32_t* tile_sums) {
  __shared__ int32_t warp_tot[32];
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanPer;
  int32_t s = 0;
#pragma unroll
  for (int q = 0; q < kScanPer; ++q) s += base + q < n ? count[base + q] : 0;
  int32_t total;
  block_exclusive_scan(s, warp_tot, total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_bin_offsets(const int32_t* count, int n, const int32_t* tile_sums,
                                                              int32_t* offset, int32_t* cursor) {
  __shared__ int32_t warp_tot[32];
  __shared__ int32_t carry;
  if (threadIdx.x < 32) {
    int32_t c = 0;
    for (int t = threadIdx.x; t < (int)blockIdx.x; t += 32) c += tile_sums[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (threadIdx.x == 0) carry = c;
  }
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanPer;
  int32_t v[kScanPer], s = 0;
#pragma unroll
  for (int q = 0; q < kScanPer; ++q) {
    v[q] = base + q < n ? count[base + q] : 0;
    s += v[q];
  }
  int32_t total;
  int32_t run = block_exclusive_scan(s, warp_tot, total) + carry;
#pragma unroll
  for (int q = 0; q < kScanPer; ++q) {
    if (base + q < n) {
      offset[base + q] = run;
      cursor[base + q] = 0;
    }
    run += v[q];
  }
  if (base <= n - 1 && n - 1 < base + kScanPer) offset[n] = run;  // the grand total
}

__global__ void k_bin_fill(int P, const int32_t* key, const int32_t* offset, int32_t* cursor, int32_t* sorted) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const int kk = key[p];
  const int slot = atomicAdd(cursor + kk, 1);
  sorted[offset[kk] + slot] = p;
}

// Restores particle order inside every bin, so the spreading sums are
// reproducible run to run: one warp per bin places each entry at its rank
// (the number of smaller particle indices in the bin).
__global__ void k_bin_rank(int nbins, const int32_t* offset, const int32_t* in, int32_t* out) {
  const int b = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = (int)(threadIdx.x & 31);
  if (b >= nbins) return;
  const int lo = offset[b], hi = offset[b + 1];
  for (int q = lo + lane; q < hi; q += 32) {
    const int32_t v = in[q];
    int rank = 0;
    for (int r = lo; r < hi; ++r) rank += in[r] < v;
    out[lo + rank] = v;
  }
}

// hibm_mpm.py:4838-4848 tent weight.
__device__ __forceinline__ float tent(const float* xm, const float* xp, float R) {
  float w = 1.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) w *= fmaxf(1.0f - fabsf(xm[a] - xp[a]) / R, 0.0f);
  return w;
}

// Visits the particles of the 3 x 3 x 3 bins around xm with the whole warp
// (every lane must call it): lane b < 27 fetches the offsets of neighbour bin
// b = (d0 + 1) * 9 + (d1 + 1) * 3 + (d2 + 1), a warp scan of the bin sizes
// numbers the visits 0 .. total-1 in bin order, and the lanes take visits
// lane, lane + 32, ..., each finding its bin by a binary search over the
// scan.  The 27 bins are fetched in parallel and every lane has work.
template <class Fn>
__device__ __forceinline__ void for_near(const BinView& B, const float* xm, int lane, Fn fn) {
  int lo = 0, cnt = 0;
  if (lane < 27) {
    const int d0 = lane / 9 - 1, d1 = (lane / 3) % 3 - 1, d2 = lane % 3 - 1;
    const int b0 = bin_axis(xm[0], B.bmin[0], B.invR, B.nb[0]) + d0;
    const int b1 = bin_axis(xm[1], B.bmin[1], B.invR, B.nb[1]) + d1;
    const int b2 = bin_axis(xm[2], B.bmin[2], B.invR, B.nb[2]) + d2;
    if (b0 >= 0 && b0 < B.nb[0] && b1 >= 0 && b1 < B.nb[1] && b2 >= 0 && b2 < B.nb[2]) {
      const int bin = (b0 * B.nb[1] + b1) * B.nb[2] + b2;
      lo = __ldg(B.offset + bin);
      cnt = __ldg(B.offset + bin + 1) - lo;
    }
  }
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const int excl = incl - cnt;
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  for (int base = 0; base < total; base += 32) {
    const int idx = base + lane;
    // the last lane j with excl_j <= idx owns visit idx (excl is non-decreasing)
    int j = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const int e = __shfl_sync(0xffffffffu, excl, j + step);
      if (e <= idx) j += step;
    }
    const int lo_j = __shfl_sync(0xffffffffu, lo, j);
    const int ex_j = __shfl_sync(0xffffffffu, excl, j);
    if (idx < total) fn(__ldg(B.sorted + lo_j + (idx - ex_j)));
  }
}

// Butterfly sums over the warp: every lane gets the same total, summed in a
// fixed order (reproducible run to run).
__device__ __forceinline__ float warp_allsum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_allsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// hibm_mpm.py:4899-4959 _scatter_marker_forces_to_mpm_particles_kernel: one
// warp per marker; the tent-weight sum over the marker's neighbourhood is a
// warp reduction, then the lanes spread F * w / wsum to the particles.
__global__ void k_scatter(BinView B, int M, const float* xg, const double* Fg, const float* xp, float* fext,
                          double* rep) {
  const int m = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = (int)(threadIdx.x & 31);
  if (m >= M) return;  // uniform over the warp
  const float xm[3] = {__ldg(xg + 3 * m), __ldg(xg + 3 * m + 1), __ldg(xg + 3 * m + 2)};
  const double Fm[3] = {__ldg(Fg + 3 * m), __ldg(Fg + 3 * m + 1), __ldg(Fg + 3 * m + 2)};
  const bool valid = finite3(xm) && isfinite(Fm[0]) && isfinite(Fm[1]) && isfinite(Fm[2]);
  const float R = B.R;
  float wl = 0.0f;
  if (valid) for_near(B, xm, lane, [&](int p) { wl += tent(xm, xp + 3 * p, R); });
  const float wsum = warp_allsum(wl);
  if (valid && wsum > 1.0e-12f) {
    double e0 = 0, e1 = 0, e2 = 0, contrib = 0;
    for_near(B, xm, lane, [&](int p) {
      float w = tent(xm, xp + 3 * p, R);
      if (w > 0.0f) {
        const double ratio = (double)(w / wsum);
        float f0 = (float)(Fm[0] * ratio), f1 = (float)(Fm[1] * ratio), f2 = (float)(Fm[2] * ratio);
        atomicAdd(fext + 3 * p, f0);
        atomicAdd(fext + 3 * p + 1, f1);
        atomicAdd(fext + 3 * p + 2, f2);
        e0 += f0;
        e1 += f1;
        e2 += f2;
        contrib += 1.0;
      }
    });
    e0 = warp_allsum(e0);
    e1 = warp_allsum(e1);
    e2 = warp_allsum(e2);
    contrib = warp_allsum(contrib);
    if (lane == 0) {
      atomicAdd(rep + 0, 1.0);
      atomicAdd(rep + 3, Fm[0]);
      atomicAdd(rep + 4, Fm[1]);
      atomicAdd(rep + 5, Fm[2]);
      atomicAdd(rep + 2, contrib);
      atomicAdd(rep + 6, e0);
      atomicAdd(rep + 7, e1);
      atomicAdd(rep + 8, e2);
    }
  } else if (lane == 0) {
    atomicAdd(rep + 1, 1.0);
  }
}

// hibm_mpm.py:5097-5180 / 5012-5053 surface feedback: one warp per marker,
// tent-weighted sums of particle velocity (and normal / area) as warp
// reductions.
__global__ void k_feedback(BinView B, int M, float* xg, float* vg, float* ng, float* Ag, const float* xp,
                           const float* vp, const float* np_, const float* ap, float dt, double* rep) {
  const int m = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = (int)(threadIdx.x & 31);
  if (m >= M) return;  // uniform over the warp
  const bool geometry = np_ != nullptr && ap != nullptr;
  const float xo[3] = {xg[3 * m], xg[3 * m + 1], xg[3 * m + 2]};
  const float no[3] = {ng[3 * m], ng[3 * m + 1], ng[3 * m + 2]};
  const float ao = Ag[m];
  float vs[3] = {0, 0, 0}, ns[3] = {0, 0, 0}, as = 0.0f, ws = 0.0f, gs = 0.0f;
  const float R = B.R;
  for_near(B, xo, lane, [&](int p) {
    float w = tent(xo, xp + 3 * p, R);
    if (w > 0.0f) {
      vs[0] += w * __ldg(vp + 3 * p);
      vs[1] += w * __ldg(vp + 3 * p + 1);
      vs[2] += w * __ldg(vp + 3 * p + 2);
      ws += w;
      if (geometry) {
        const float* pn = np_ + 3 * p;
        if (sqrtf(pn[0] * pn[0] + pn[1] * pn[1] + pn[2] * pn[2]) > 1.0e-12f && ap[p] > 0.0f) {
          ns[0] += w * pn[0];
          ns[1] += w * pn[1];
          ns[2] += w * pn[2];
          as += w * ap[p];
          gs += w;
        }
      }
    }
  });
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    vs[a] = warp_allsum(vs[a]);
    ns[a] = warp_allsum(ns[a]);
  }
  as = warp_allsum(as);
  ws = warp_allsum(ws);
  gs = warp_allsum(gs);
  if (lane != 0) return;
  if (ws > 1.0e-12f) {
    float nv[3], nx[3];
    for (int a = 0; a < 3; ++a) {
      nv[a] = vs[a] / ws;
      nx[a] = xo[a] + dt * nv[a];
      xg[3 * m + a] = nx[a];
      vg[3 * m + a] = nv[a];
    }
    atomicAdd(rep + 0, 1.0);
    double dd = 0, sp = 0;
    for (int a = 0; a < 3; ++a) {
      dd += (double)(nx[a] - xo[a]) * (nx[a] - xo[a]);
      sp += (double)nv[a] * nv[a];
    }
    atomic_max_nonneg_d(rep + 4, sqrt(dd));
    atomic_max_nonneg_d(rep + 5, sqrt(sp));
    if (geometry) {
      float nn = sqrtf(ns[0] * ns[0] + ns[1] * ns[1] + ns[2] * ns[2]);
      if (gs > 1.0e-12f && nn > 1.0e-12f) {
        double dn = 0;
        for (int a = 0; a < 3; ++a) {
          float v = ns[a] / nn;
          ng[3 * m + a] = v;
          dn += (double)(v - no[a]) * (v - no[a]);
        }
        float na = as / gs;
        Ag[m] = na;
        atomicAdd(rep + 2, 1.0);
        atomic_max_nonneg_d(rep + 6, sqrt(dn));
        atomic_max_nonneg_d(rep + 7, (double)fabsf(na - ao));
      } else {
        atomicAdd(rep + 3, 1.0);
      }
    }
  } else {
    atomicAdd(rep + 1, 1.0);
    if (geometry) atomicAdd(rep + 3, 1.0);
  }
}

static BinView bin_view(const efsi_bin_plan* P) {
  BinView B;
  for (int a = 0; a < 3; ++a) {
    B.bmin[a] = P->bmin[a];
    B.nb[a] = P->nb[a];
  }
  B.invR = P->invR;
  B.R = P->R;
  B.nbins = P->nbins;
  B.sorted = P->sorted;
  B.offset = P->offset;
  return B;
}

}  // namespace efsi

using namespace efsi;

extern "C" {

int efsi_sample_pressure_tractions(int32_t nx, int32_t ny, int32_t nz, const efsi_grid_axes* axes, const float* wx,
                                   const float* wy, const float* wz, const int32_t* obstacle, const double* pressure,
                                   int32_t marker_count, const float* x_gamma, const float* n_gamma,
                                   const int32_t* region, int32_t two_sided, int32_t one_sided_region,
                                   float one_sided_reference, double* t_gamma, int32_t* valid, double* report_device,
                                   void* stream) {
  EFSI_ARG_CHECK(nx >= 2 && ny >= 2 && nz >= 2 && axes != nullptr && report_device != nullptr,
                 "invalid traction sampling arguments");
  cudaStream_t s = as_stream(stream);
  EFSI_CUDA_CHECK(cudaMemsetAsync(report_device, 0, 5 * sizeof(double), s));
  if (marker_count <= 0) return EFSI_OK;
  EFSI_COUNTED k_tractions<<<(marker_count + 127) / 128, 128, 0, s>>>(nx, ny, nz, *axes, wx, wy, wz, obstacle, pressure,
                                                         marker_count, x_gamma, n_gamma, region, two_sided,
                                                         one_sided_region, one_sided_reference, t_gamma, valid,
                                                         report_device);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_compute_marker_forces(int32_t marker_count, const double* t_gamma, const float* area, double* f_gamma,
                               void* stream) {
  if (marker_count <= 0) return EFSI_OK;
  EFSI_COUNTED k_marker_forces<<<(marker_count + 255) / 256, 256, 0, as_stream(stream)>>>(marker_count, t_gamma, area, f_gamma);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_clear_external_forces(int32_t particle_count, float* external_force, double* report_device, void* stream) {
  EFSI_ARG_CHECK(particle_count > 0, "particle_count must be positive");
  cudaStream_t s = as_stream(stream);
  if (report_device) EFSI_CUDA_CHECK(cudaMemsetAsync(report_device, 0, 2 * sizeof(double), s));
  EFSI_COUNTED k_clear_fext<<<(particle_count + 255) / 256, 256, 0, s>>>(particle_count, external_force, report_device);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_bin_plan_create(int32_t capacity, const float* box_min, const float* box_max, float support_radius,
                         efsi_bin_plan** out) {
  EFSI_ARG_CHECK(capacity > 0 && box_min && box_max && out, "invalid bin plan arguments");
  EFSI_ARG_CHECK(std::isfinite(support_radius) && support_radius > 0.0f, "support radius must be finite positive");
  efsi_bin_plan* P = new efsi_bin_plan();
  P->capacity = capacity;
  P->R = support_radius;
  P->invR = 1.0f / support_radius;
  int64_t nb = 1;
  for (int a = 0; a < 3; ++a) {
    EFSI_ARG_CHECK(box_max[a] > box_min[a], "bin box must have positive extent");
    P->bmin[a] = box_min[a];
    double n = std::ceil(((double)box_max[a] - (double)box_min[a]) / (double)support_radius);
    if (n < 1.0) n = 1.0;
    if (n > 1024.0) n = 1024.0;  // bounds the bin table; far bins merge at the edges
    P->nb[a] = (int)n;
    nb *= P->nb[a];
  }
  EFSI_ARG_CHECK(nb < (int64_t)1 << 28, "too many bins");
  P->nbins = (int)nb;
  if (cudaMalloc(&P->key, capacity * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&P->sorted, capacity * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&P->count, (P->nbins + 1) * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&P->offset, (P->nbins + 2) * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&P->cursor, (P->nbins + 1) * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&P->tile_sums, ((P->nbins + 1) / kScanTile + 1) * sizeof(int32_t)) != cudaSuccess) {
    efsi_bin_plan_destroy(P);
    set_error("cudaMalloc failed for the bin plan");
    return EFSI_ERR_CUDA;
  }
  *out = P;
  return EFSI_OK;
}

int efsi_bin_plan_destroy(efsi_bin_plan* P) {
  if (!P) return EFSI_OK;
  cudaFree(P->key);
  cudaFree(P->sorted);
  cudaFree(P->count);
  cudaFree(P->offset);
  cudaFree(P->cursor);
  cudaFree(P->tile_sums);
  delete P;
  return EFSI_OK;
}

int efsi_bin_particles(efsi_bin_plan* P, const float* particle_x, int32_t particle_count, void* stream) {
  EFSI_ARG_CHECK(P != nullptr && particle_x != nullptr, "null bin plan or positions");
  EFSI_ARG_CHECK(particle_count > 0 && particle_count <= P->capacity, "particle_count out of range");
  cudaStream_t s = as_stream(stream);
  BinView B = bin_view(P);
  EFSI_CUDA_CHECK(cudaMemsetAsync(P->count, 0, (P->nbins + 1) * sizeof(int32_t), s));
  const unsigned pb = (particle_count + 255) / 256;
  EFSI_COUNTED k_bin_count<<<pb, 256, 0, s>>>(B, particle_x, particle_count, P->key, P->count);
  const int nc = P->nbins + 1;
  const unsigned tiles = (unsigned)((nc + kScanTile - 1) / kScanTile);
  EFSI_COUNTED k_bin_tile_sums<<<tiles, kScanThreads, 0, s>>>(P->count, nc, P->tile_sums);
  EFSI_COUNTED k_bin_offsets<<<tiles, kScanThreads, 0, s>>>(P->count, nc, P->tile_sums, P->offset, P->cursor);
  // unordered fill into the key buffer (no longer needed), ordered copy into `sorted`
  EFSI_COUNTED k_bin_fill<<<pb, 256, 0, s>>>(particle_count, P->key, P->offset, P->cursor, P->sorted);
  std::swap(P->key, P->sorted);
  EFSI_COUNTED k_bin_rank<<<(unsigned)(((int64_t)P->nbins * 32 + 255) / 256), 256, 0, s>>>(P->nbins, P->offset,
                                                                                          P->key, P->sorted);
  EFSI_LAUNCH_CHECK();
  P->count_last = particle_count;
  return EFSI_OK;
}

int efsi_scatter_marker_forces(efsi_bin_plan* P, int32_t marker_count, const float* x_gamma, const double* f_gamma,
                               const float* particle_x, float* external_force, double* report_device, void* stream) {
  EFSI_ARG_CHECK(P != nullptr && report_device != nullptr, "null bin plan or report");
  EFSI_ARG_CHECK(P->count_last > 0, "bin the particles first (efsi_bin_particles)");
  cudaStream_t s = as_stream(stream);
  EFSI_CUDA_CHECK(cudaMemsetAsync(report_device, 0, 9 * sizeof(double), s));
  if (marker_count <= 0) return EFSI_OK;
  // 36 bytes per marker (x, F) and 12 per binned particle position read
  EFSI_TIMED(KF_SCATTER, 36.0 * marker_count + 12.0 * P->count_last, s,
             EFSI_COUNTED k_scatter<<<(marker_count + 7) / 8, 256, 0, s>>>(bin_view(P), marker_count, x_gamma, f_gamma,
                                                                             particle_x, external_force,
                                                                             report_device));
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_surface_feedback(efsi_bin_plan* P, int32_t marker_count, float* x_gamma, float* v_gamma, float* n_gamma,
                          float* area_gamma, const float* particle_x, const float* particle_v,
                          const float* particle_normal, const float* particle_area, float dt, double* report_device,
                          void* stream) {
  EFSI_ARG_CHECK(P != nullptr && report_device != nullptr, "null bin plan or report");
  EFSI_ARG_CHECK(P->count_last > 0, "bin the particles first (efsi_bin_particles)");
  cudaStream_t s = as_stream(stream);
  EFSI_CUDA_CHECK(cudaMemsetAsync(report_device, 0, 8 * sizeof(double), s));
  if (marker_count <= 0) return EFSI_OK;
  // 52 bytes per marker (read x; write x, v, n, A) and 40 per binned
  // particle (x, v, normal, area)
  EFSI_TIMED(KF_FEEDBACK, 52.0 * marker_count + 40.0 * P->count_last, s,
             EFSI_COUNTED k_feedback<<<(marker_count + 7) / 8, 256, 0, s>>>(
                 bin_view(P), marker_count, x_gamma, v_gamma, n_gamma, area_gamma, particle_x, particle_v,
                 particle_normal, particle_area, dt, report_device));
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

}  // extern "C"
