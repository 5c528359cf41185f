#include <algorithm>
// Fluid kernels around the pressure solve, B200 path: divergence, the level-0
// right-hand side, the pressure-gradient correction and wall conditions, the
// semi-Lagrangian predictor, divergence statistics and the point-force
// spreading / body-force update (simulation_core/fluid.py).  All of them are
// single-pass, one thread per cell (or per vertex), with the f32 / f64 mix of
// the reference kernels; they read the level-0 stencil mask built by
// efsi_fv_set_masks instead of the int32 obstacle field.
#include <cuda_runtime.h>

#include <cmath>

#include "efsi_fv_internal.cuh"

namespace efsi {

__device__ __forceinline__ int64_t cix(int i, int j, int k, int ny, int nz) { return ((int64_t)i * ny + j) * nz + k; }

#define EFSI_CELL(L)                                        \
  const int k = blockIdx.x * blockDim.x + threadIdx.x;     \
  const int j = blockIdx.y * blockDim.y + threadIdx.y;     \
  const int i = blockIdx.z * blockDim.z + threadIdx.z;     \
  if (i >= (L).nx || j >= (L).ny || k >= (L).nz) return;   \
  const int64_t c = cix(i, j, k, (L).ny, (L).nz);

// fluid.py:3451-3486 _compute_divergence_kernel.
__global__ void k_divergence(LevelDev L, const float* __restrict__ vel, int outlet, float* __restrict__ div) {
  EFSI_CELL(L)
  const unsigned m = L.mask[c];
  if (m & M_SOLID) {
    div[c] = 0.0f;
    return;
  }
  const int64_t sx = (int64_t)L.ny * L.nz, sy = L.nz;
  float lx = 0.f, rx = 0.f, by = 0.f, fy = 0.f, bz = 0.f, tz = 0.f;
  if (m & M_XM) lx = vel[3 * c + 0];
  if (m & M_XP) rx = vel[3 * (c + sx) + 0];
  if (m & M_YM) by = vel[3 * c + 1];
  if (m & M_YP) fy = vel[3 * (c + sy) + 1];
  if (outlet && k == 0)
    bz = vel[3 * c + 2];
  else if (m & M_ZM)
    bz = vel[3 * c + 2];
  if (m & M_ZP) tz = vel[3 * (c + 1) + 2];
  float a = __fdiv_rn(__fsub_rn(rx, lx), L.wx[i]);
  float b = __fdiv_rn(__fsub_rn(fy, by), L.wy[j]);
  float d = __fdiv_rn(__fsub_rn(tz, bz), L.wz[k]);
  div[c] = __fadd_rn(__fadd_rn(a, b), d);
}

// fluid.py:5228-5243 _mg_prepare_level0_kernel.
__global__ void k_prepare_level0(LevelDev L, const float* __restrict__ div, const float* __restrict__ src,
                                 const double* __restrict__ iface_rhs, float scale, double* __restrict__ rhs) {
  EFSI_CELL(L)
  const unsigned m = L.mask[c];
  if (m & M_SOLID) {
    rhs[c] = 0.0;
    return;
  }
  float v = __fmul_rn(scale, __fsub_rn(div[c], src[c]));
  rhs[c] = (double)v - (iface_rhs ? iface_rhs[c] : 0.0);
}

// fluid.py:3997-4054 _pressure_jacobi_kernel (legacy uniform-spacing Jacobi).
__global__ void k_legacy_jacobi(LevelDev L, const int32_t* __restrict__ obs, const double* __restrict__ p,
                                const float* __restrict__ div, const float* __restrict__ src, float scale, float ix2,
                                float iy2, float iz2, int outlet, double* __restrict__ tmp) {
  EFSI_CELL(L)
  const int im = max(i - 1, 0), ip = min(i + 1, L.nx - 1), jm = max(j - 1, 0), jp = min(j + 1, L.ny - 1),
            km = max(k - 1, 0), kp = min(k + 1, L.nz - 1);
  auto at = [&](int a, int b, int d) { return cix(a, b, d, L.ny, L.nz); };
  double ns = (double)ix2 * (p[at(im, j, k)] + p[at(ip, j, k)]) + (double)iy2 * (p[at(i, jm, k)] + p[at(i, jp, k)]) +
              (double)iz2 * (p[at(i, j, km)] + p[at(i, j, kp)]);
  float den = 2.0f * (ix2 + iy2 + iz2);
  const bool adj = obs[at(im, j, k)] == 1 || obs[at(ip, j, k)] == 1 || obs[at(i, jm, k)] == 1 ||
                   obs[at(i, jp, k)] == 1 || obs[at(i, j, km)] == 1 || obs[at(i, j, kp)] == 1;
  if (adj || (outlet && k == 0)) {
    ns = 0.0;
    den = 0.0f;
    if (i > 0 && obs[at(i - 1, j, k)] == 0) { ns += (double)ix2 * p[at(i - 1, j, k)]; den += ix2; }
    if (i < L.nx - 1 && obs[at(i + 1, j, k)] == 0) { ns += (double)ix2 * p[at(i + 1, j, k)]; den += ix2; }
    if (j > 0 && obs[at(i, j - 1, k)] == 0) { ns += (double)iy2 * p[at(i, j - 1, k)]; den += iy2; }
    if (j < L.ny - 1 && obs[at(i, j + 1, k)] == 0) { ns += (double)iy2 * p[at(i, j + 1, k)]; den += iy2; }
    if (k > 0 && obs[at(i, j, k - 1)] == 0) { ns += (double)iz2 * p[at(i, j, k - 1)]; den += iz2; }
    if (k < L.nz - 1 && obs[at(i, j, k + 1)] == 0) { ns += (double)iz2 * p[at(i, j, k + 1)]; den += iz2; }
    if (outlet && k == 0) den += 2.0f * iz2;
  }
  const float rhs = scale * (div[c] - src[c]);
  if (obs[c] == 1 || den <= 0.0f)
    tmp[c] = 0.0;
  else
    tmp[c] = (ns - (double)rhs) / (double)den;
}

// fluid.py:5538-5582 _subtract_pressure_gradient_kernel.
__global__ void k_gradient(LevelDev L, const double* __restrict__ p, const int32_t* __restrict__ va,
                           const float* __restrict__ vw, const float* __restrict__ vval, float dtr_f, int outlet,
                           float* __restrict__ vel) {
  EFSI_CELL(L)
  const unsigned m = L.mask[c];
  if (m & M_SOLID) {
    vel[3 * c] = vel[3 * c + 1] = vel[3 * c + 2] = 0.0f;
    return;
  }
  const int64_t sx = (int64_t)L.ny * L.nz, sy = L.nz;
  const double center = p[c];
  double g0 = 0.0, g1 = 0.0, g2 = 0.0;
  if (m & M_XM) g0 = __ddiv_rn(center - p[c - sx], (double)L.cdx_f[i]);
  if (m & M_YM) g1 = __ddiv_rn(center - p[c - sy], (double)L.cdy_f[j]);
  if (m & M_ZM)
    g2 = __ddiv_rn(center - p[c - 1], (double)L.cdz_f[k]);
  else if (outlet && k == 0)
    g2 = __ddiv_rn(2.0 * center, (double)L.wz[k]);
  double cw = 1.0;
  if (va != nullptr && va[c] != 0) {
    cw = (double)fminf(fmaxf(vw[c], 0.0f), 1.0f);
    if (cw <= 0.0) {
      vel[3 * c] = vval[3 * c];
      vel[3 * c + 1] = vval[3 * c + 1];
      vel[3 * c + 2] = vval[3 * c + 2];
    }
  }
  if (cw > 0.0) {
    const double s = __dmul_rn(cw, (double)dtr_f);
    vel[3 * c + 0] = __fsub_rn(vel[3 * c + 0], (float)__dmul_rn(s, g0));
    vel[3 * c + 1] = __fsub_rn(vel[3 * c + 1], (float)__dmul_rn(s, g1));
    vel[3 * c + 2] = __fsub_rn(vel[3 * c + 2], (float)__dmul_rn(s, g2));
  }
}

// fluid.py:5529-5536 _apply_closed_boundary_no_normal_flow_kernel.
__global__ void k_closed_boundary(int nx, int ny, int nz, int outlet, float* __restrict__ vel) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t a = (int64_t)ny * nz, b = (int64_t)nx * nz, cc = (int64_t)nx * ny;
  if (t < a) {
    int j = (int)(t / nz), k = (int)(t % nz);
    vel[3 * cix(0, j, k, ny, nz) + 0] = 0.0f;
  } else if (t < a + b) {
    int64_t u = t - a;
    int i = (int)(u / nz), k = (int)(u % nz);
    vel[3 * cix(i, 0, k, ny, nz) + 1] = 0.0f;
  } else if (t < a + b + cc && !outlet) {
    int64_t u = t - a - b;
    int i = (int)(u / ny), j = (int)(u % ny);
    vel[3 * cix(i, j, 0, ny, nz) + 2] = 0.0f;
  }
}

// fluid.py:5762-5766 _apply_zmin_no_backflow_kernel.
__global__ void k_zmin_no_backflow(LevelDev L, float* __restrict__ vel) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)L.nx * L.ny) return;
  int i = (int)(t / L.ny), j = (int)(t % L.ny);
  int64_t c = cix(i, j, 0, L.ny, L.nz);
  if ((L.mask[c] & M_FLUID) && vel[3 * c + 2] > 0.0f) vel[3 * c + 2] = 0.0f;
}

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  // Non-negative doubles order like their bit patterns.
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// fluid.py:2549-2593 _apply_velocity_dirichlet_boundary_rows_kernel.
__global__ void k_vdir_rows(LevelDev L, const int32_t* __restrict__ va, const float* __restrict__ vval, float rho,
                            float* __restrict__ vel, double* rep) {
  EFSI_CELL(L)
  if (va[c] == 0 || !(L.mask[c] & M_FLUID)) return;
  float d0 = vval[3 * c] - vel[3 * c], d1 = vval[3 * c + 1] - vel[3 * c + 1], d2 = vval[3 * c + 2] - vel[3 * c + 2];
  vel[3 * c] = vval[3 * c];
  vel[3 * c + 1] = vval[3 * c + 1];
  vel[3 * c + 2] = vval[3 * c + 2];
  if (rep != nullptr) {
    float dn = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
    float vol = L.wx[i] * L.wy[j] * L.wz[k];
    atomicAdd(rep + 0, 1.0);
    atomicAdd(rep + 1, (double)dn);
    atomic_max_nonneg(rep + 2, (double)dn);
    atomicAdd(rep + 3, (double)(rho * d0 * vol));
    atomicAdd(rep + 4, (double)(rho * d1 * vol));
    atomicAdd(rep + 5, (double)(rho * d2 * vol));
  }
}

// fluid.py:2407-2433 _axis_grid_coordinate_device (f32).  The bracketing
// centre interval is the one the reference's bisection finds (the largest lo
// with centers[lo] <= v); with a hint (the index of a cell near v, -1: none)
// it is found by walking from the hint, which takes a step or two for a
// semi-Lagrangian departure point instead of log2(count) dependent loads.
__device__ __forceinline__ float axis_coord(float v, const float* __restrict__ faces,
                                            const float* __restrict__ centers, int count, int hint = -1) {
  float coord;
  const float c0 = __ldg(centers), cl = __ldg(centers + count - 1);
  if (v <= c0) {
    float hw = fmaxf(__fsub_rn(c0, __ldg(faces)), 1.0e-18f);
    coord = __fdiv_rn(__fmul_rn(-0.5f, __fsub_rn(c0, v)), hw);
  } else if (v >= cl) {
    float hw = fmaxf(__fsub_rn(__ldg(faces + count), cl), 1.0e-18f);
    coord = __fadd_rn((float)(count - 1), __fdiv_rn(__fmul_rn(0.5f, __fsub_rn(v, cl)), hw));
  } else {
    int lo = 0, hi = count - 1;
    if (hint >= 0) {
      // c0 < v < cl: the bracket lo in [0, count - 2] exists and is unique
      lo = min(max(hint, 0), count - 2);
      while (lo < count - 2 && v >= __ldg(centers + lo + 1)) ++lo;
      while (lo > 0 && v < __ldg(centers + lo)) --lo;
    } else {
      while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (v >= __ldg(centers + mid))
          lo = mid;
        else
          hi = mid;
      }
    }
    hi = min(lo + 1, count - 1);
    const float clo = __ldg(centers + lo);
    float dist = fmaxf(__fsub_rn(__ldg(centers + hi), clo), 1.0e-18f);
    coord = __fadd_rn((float)lo, __fdiv_rn(__fsub_rn(v, clo), dist));
  }
  return coord;
}

// fluid.py:2383-2404 _sample_velocity_prev_trilinear (obstacle-masked).
__device__ __forceinline__ void sample_prev(const LevelDev& L, const float* __restrict__ vp, float gx, float gy,
                                            float gz, const float fb[3], float out[3]) {
  int i0 = min(max((int)floorf(gx), 0), L.nx - 2);
  int j0 = min(max((int)floorf(gy), 0), L.ny - 2);
  int k0 = min(max((int)floorf(gz), 0), L.nz - 2);
  float tx = fminf(fmaxf(__fsub_rn(gx, (float)i0), 0.0f), 1.0f);
  float ty = fminf(fmaxf(__fsub_rn(gy, (float)j0), 0.0f), 1.0f);
  float tz = fminf(fmaxf(__fsub_rn(gz, (float)k0), 0.0f), 1.0f);
  float v0 = 0.f, v1 = 0.f, v2 = 0.f, fw = 0.f;
#pragma unroll
  for (int oi = 0; oi < 2; ++oi)
#pragma unroll
    for (int oj = 0; oj < 2; ++oj)
#pragma unroll
      for (int ok = 0; ok < 2; ++ok) {
        float wx = oi == 0 ? __fsub_rn(1.0f, tx) : tx;
        float wy = oj == 0 ? __fsub_rn(1.0f, ty) : ty;
        float wz = ok == 0 ? __fsub_rn(1.0f, tz) : tz;
        float w = __fmul_rn(__fmul_rn(wx, wy), wz);
        int64_t cc = cix(i0 + oi, j0 + oj, k0 + ok, L.ny, L.nz);
        if (__ldg(L.mask + cc) & M_FLUID) {
          v0 = __fadd_rn(v0, __fmul_rn(w, __ldg(vp + 3 * cc)));
          v1 = __fadd_rn(v1, __fmul_rn(w, __ldg(vp + 3 * cc + 1)));
          v2 = __fadd_rn(v2, __fmul_rn(w, __ldg(vp + 3 * cc + 2)));
          fw = __fadd_rn(fw, w);
        }
      }
  if (fw > 1.0e-12f) {
    out[0] = __fdiv_rn(v0, fw);
    out[1] = __fdiv_rn(v1, fw);
    out[2] = __fdiv_rn(v2, fw);
  } else {
    out[0] = fb[0];
    out[1] = fb[1];
    out[2] = fb[2];
  }
}

// fluid.py:2447-2513 _predict_kernel.
__global__ void __launch_bounds__(256) k_predict(LevelDev L, efsi_grid_axes A, const float* __restrict__ vp,
                                                 float dt, float nu, int rk2, float* __restrict__ vel) {
  EFSI_CELL(L)
  const unsigned m = __ldg(L.mask + c);
  if (m & M_SOLID) {
    vel[3 * c] = vel[3 * c + 1] = vel[3 * c + 2] = 0.0f;
    return;
  }
  const int64_t sx = (int64_t)L.ny * L.nz, sy = L.nz;
  const float cen[3] = {__ldg(vp + 3 * c), __ldg(vp + 3 * c + 1), __ldg(vp + 3 * c + 2)};
  const float x = __ldg(A.cx + i), y = __ldg(A.cy + j), z = __ldg(A.cz + k);
  float tr[3] = {cen[0], cen[1], cen[2]};
  if (rk2) {
    float hd = __fmul_rn(0.5f, dt);
    float mx = __fsub_rn(x, __fmul_rn(hd, cen[0]));
    float my = __fsub_rn(y, __fmul_rn(hd, cen[1]));
    float mz = __fsub_rn(z, __fmul_rn(hd, cen[2]));
    sample_prev(L, vp, axis_coord(mx, A.fx, A.cx, L.nx, i), axis_coord(my, A.fy, A.cy, L.ny, j),
                axis_coord(mz, A.fz, A.cz, L.nz, k), cen, tr);
  }
  float bx = __fsub_rn(x, __fmul_rn(dt, tr[0]));
  float by = __fsub_rn(y, __fmul_rn(dt, tr[1]));
  float bz = __fsub_rn(z, __fmul_rn(dt, tr[2]));
  float adv[3];
  sample_prev(L, vp, axis_coord(bx, A.fx, A.cx, L.nx, i), axis_coord(by, A.fy, A.cy, L.ny, j),
              axis_coord(bz, A.fz, A.cz, L.nz, k), cen, adv);
  const float dtnu = __fmul_rn(dt, nu);
  const float icx = __ldg(L.cdx_f + i), icy = __ldg(L.cdy_f + j), icz = __ldg(L.cdz_f + k);
  const float icxp = (i < L.nx - 1) ? __ldg(L.cdx_f + i + 1) : 1.0f;
  const float icyp = (j < L.ny - 1) ? __ldg(L.cdy_f + j + 1) : 1.0f;
  const float iczp = (k < L.nz - 1) ? __ldg(L.cdz_f + k + 1) : 1.0f;
  const float wxi = __ldg(L.wx + i), wyj = __ldg(L.wy + j), wzk = __ldg(L.wz + k);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float fxb = 0.f, fxf = 0.f, fyb = 0.f, fyf = 0.f, fzb = 0.f, fzf = 0.f;
    if (m & M_XM) fxb = __fdiv_rn(__fsub_rn(cen[a], __ldg(vp + 3 * (c - sx) + a)), icx);
    if (m & M_XP) fxf = __fdiv_rn(__fsub_rn(__ldg(vp + 3 * (c + sx) + a), cen[a]), icxp);
    if (m & M_YM) fyb = __fdiv_rn(__fsub_rn(cen[a], __ldg(vp + 3 * (c - sy) + a)), icy);
    if (m & M_YP) fyf = __fdiv_rn(__fsub_rn(__ldg(vp + 3 * (c + sy) + a), cen[a]), icyp);
    if (m & M_ZM) fzb = __fdiv_rn(__fsub_rn(cen[a], __ldg(vp + 3 * (c - 1) + a)), icz);
    if (m & M_ZP) fzf = __fdiv_rn(__fsub_rn(__ldg(vp + 3 * (c + 1) + a), cen[a]), iczp);
    float lap = __fadd_rn(__fadd_rn(__fdiv_rn(__fsub_rn(fxf, fxb), wxi), __fdiv_rn(__fsub_rn(fyf, fyb), wyj)),
                          __fdiv_rn(__fsub_rn(fzf, fzb), wzk));
    vel[3 * c + a] = __fadd_rn(adv[a], __fmul_rn(dtnu, lap));
  }
}

// fluid.py:3494-3565 divergence statistics: max |v|, sum v^2, count.
__global__ void k_div_stats(LevelDev L, const float* __restrict__ div, const double* __restrict__ idiv,
                            const float* __restrict__ src, int mode, int interior_only, double* partials,
                            unsigned* ticket, double* out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z * blockDim.z + threadIdx.z;
  double sq = 0.0, cnt = 0.0, mx = 0.0;
  if (i < L.nx && j < L.ny && k < L.nz) {
    const int64_t c = cix(i, j, k, L.ny, L.nz);
    bool interior = i > 0 && i < L.nx - 1 && j > 0 && j < L.ny - 1 && k > 0 && k < L.nz - 1;
    if ((L.mask[c] & M_FLUID) && (!interior_only || interior)) {
      double total = (double)div[c] + (idiv ? idiv[c] : 0.0);
      // Taichi adds the f32 divergence to the f64 interface term in f64.
      double v = mode == 1 ? fabs(total - (double)src[c]) : fabs(total);
      sq = v * v;
      cnt = 1.0;
      mx = v;
    }
  }
  // block max
  __shared__ double smax[32];
  double wm = mx;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) wm = fmax(wm, __shfl_down_sync(0xffffffffu, wm, o));
  const unsigned tid = flat_tid();
  if ((tid & 31u) == 0) smax[tid >> 5] = wm;
  __syncthreads();
  if (tid == 0) {
    double b = 0.0;
    for (unsigned w = 0; w < (flat_nthreads() + 31u) / 32u; ++w) b = fmax(b, smax[w]);
    atomic_max_nonneg(out + 0, b);
  }
  double v[2] = {sq, cnt}, t[2];
  if (grid_sum<2>(v, partials, ticket, t)) {
    if (tid == 0) {
      out[1] = t[0];
      out[2] = t[1];
    }
  }
}

// fluid.py:3574-3663 _divergence_final_report_kernel with the stencil tests
// of fluid.py:3665-3768: per fluid cell the raw |div| and residual
// |div - source| into 18 slots (max, sum of squares, count each):
//   0/1 all, 2/3 interior, 4/5 near a velocity-Dirichlet row, 6/7 far from
//   one, 8/9 with a pressure-correctable face, 10/11 without (12-15 the
//   interior ones of those two), 16/17 outlet-unreached cells (reach given),
//   which are kept out of all other slots.
// Block sums in shared memory, then one global atomic per slot (the
// reference's own reductions are atomic).
__global__ void __launch_bounds__(256) k_div_final_report(LevelDev L, const float* __restrict__ div,
                                                          const double* __restrict__ idiv,
                                                          const float* __restrict__ src,
                                                          const int32_t* __restrict__ vda,
                                                          const int32_t* __restrict__ reach, int outlet,
                                                          double* out) {
  __shared__ double s_sum[18], s_cnt[18];
  __shared__ unsigned long long s_max[18];
  const unsigned tid = flat_tid();
  if (tid < 18) {
    s_sum[tid] = 0.0;
    s_cnt[tid] = 0.0;
    s_max[tid] = 0ull;
  }
  __syncthreads();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z * blockDim.z + threadIdx.z;
  if (i < L.nx && j < L.ny && k < L.nz) {
    const int64_t c = cix(i, j, k, L.ny, L.nz);
    const unsigned m = L.mask[c];
    if (m & M_FLUID) {
      const int64_t sx = (int64_t)L.ny * L.nz, sy = L.nz;
      const double total = (double)div[c] + (idiv ? idiv[c] : 0.0);
      const double raw = fabs(total), res = fabs(total - (double)src[c]);
      auto put = [&](int slot, double v) {
        atomicAdd(&s_sum[slot], v * v);
        atomicAdd(&s_cnt[slot], 1.0);
        atomicMax(&s_max[slot], (unsigned long long)__double_as_longlong(v));
      };
      if (reach != nullptr && reach[c] == 0) {
        put(16, raw);
        put(17, res);
      } else {
        const bool interior = i > 0 && i < L.nx - 1 && j > 0 && j < L.ny - 1 && k > 0 && k < L.nz - 1;
        auto va = [&](int64_t q) { return vda != nullptr && vda[q] != 0; };
        const bool near = va(c) || (i < L.nx - 1 && va(c + sx)) || (j < L.ny - 1 && va(c + sy)) ||
                          (k < L.nz - 1 && va(c + 1));
        const bool corr = ((m & M_XM) && !va(c)) || ((m & M_XP) && !va(c + sx)) || ((m & M_YM) && !va(c)) ||
                          ((m & M_YP) && !va(c + sy)) || ((m & M_ZM) && !va(c)) || ((m & M_ZP) && !va(c + 1)) ||
                          (outlet && k == 0 && !va(c));
        put(0, raw);
        put(1, res);
        if (interior) {
          put(2, raw);
          put(3, res);
        }
        put(near ? 4 : 6, raw);
        put(near ? 5 : 7, res);
        put(corr ? 8 : 10, raw);
        put(corr ? 9 : 11, res);
        if (interior) {
          put(corr ? 12 : 14, raw);
          put(corr ? 13 : 15, res);
        }
      }
    }
  }
  __syncthreads();
  if (tid < 18 && s_cnt[tid] > 0.0) {
    atomicAdd(out + 3 * tid + 1, s_sum[tid]);
    atomicAdd(out + 3 * tid + 2, s_cnt[tid]);
    atomic_max_nonneg(out + 3 * tid, __longlong_as_double((long long)s_max[tid]));
  }
}

// fluid.py:3196-3273 _spread_surface_forces_kernel (force density, per vertex).
__global__ void k_spread(LevelDev L, efsi_grid_axes A, const float* __restrict__ pos, const float* __restrict__ fs,
                         int nv, float cx, float cy, float cz, float sign, float* __restrict__ force, double* rep) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  float p0 = pos[3 * v] + cx, p1 = pos[3 * v + 1] + cy, p2 = pos[3 * v + 2] + cz;
  float f[3] = {fs[3 * v], fs[3 * v + 1], fs[3 * v + 2]};
  float ff[3] = {sign * f[0], sign * f[1], sign * f[2]};
  atomicAdd(rep + 0, (double)f[0]);
  atomicAdd(rep + 1, (double)f[1]);
  atomicAdd(rep + 2, (double)f[2]);
  float gx = axis_coord(p0, A.fx, A.cx, L.nx), gy = axis_coord(p1, A.fy, A.cy, L.ny),
        gz = axis_coord(p2, A.fz, A.cz, L.nz);
  int bi = (int)floorf(gx), bj = (int)floorf(gy), bk = (int)floorf(gz);
  float tx = gx - (float)bi, ty = gy - (float)bj, tz = gz - (float)bk;
  float wsum = 0.0f;
  for (int pass = 0; pass < 2; ++pass)
    for (int oi = 0; oi < 2; ++oi)
      for (int oj = 0; oj < 2; ++oj)
        for (int ok = 0; ok < 2; ++ok) {
          int ii = bi + oi, jj = bj + oj, kk = bk + ok;
          if (ii < 0 || ii >= L.nx || jj < 0 || jj >= L.ny || kk < 0 || kk >= L.nz) continue;
          float w = (oi == 0 ? 1.0f - tx : tx) * (oj == 0 ? 1.0f - ty : ty) * (ok == 0 ? 1.0f - tz : tz);
          int64_t c = cix(ii, jj, kk, L.ny, L.nz);
          if (!(L.mask[c] & M_FLUID)) continue;
          if (pass == 0) {
            wsum += w;
          } else if (wsum > 0.0f) {
            float wn = w / wsum;
            float vol = L.wx[ii] * L.wy[jj] * L.wz[kk];
            for (int a = 0; a < 3; ++a) {
              float cf = ff[a] * wn;
              atomicAdd(force + 3 * c + a, cf / vol);
              atomicAdd(rep + 3 + a, (double)cf);
            }
          }
        }
}

// fluid.py:3301-3328 _apply_body_force_kernel.
__global__ void k_body_force(LevelDev L, const float* __restrict__ force, float dt, float rho, float* __restrict__ vel,
                             double* rep) {
  EFSI_CELL(L)
  if (!(L.mask[c] & M_FLUID)) return;
  const float vol = L.wx[i] * L.wy[j] * L.wz[k];
  const float s = dt / rho;
  float dv[3];
  for (int a = 0; a < 3; ++a) {
    float fd = force[3 * c + a];
    dv[a] = fd * s;
    vel[3 * c + a] += dv[a];
    if (rep != nullptr) {
      atomicAdd(rep + a, (double)(fd * vol * dt));
      atomicAdd(rep + 3 + a, (double)(rho * dv[a] * vol));
    }
  }
  if (rep != nullptr && sqrtf(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]) > 0.0f) atomicAdd(rep + 6, 1.0);
}

}  // namespace efsi

namespace efsi {
constexpr int kZeroListMax = 64;
struct ZeroList {
  int n;
  uint32_t* p[kZeroListMax];
  int64_t words[kZeroListMax];
};
__global__ void k_zero_list(ZeroList Z) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int b = 0; b < Z.n; ++b)
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < Z.words[b]; q += stride) Z.p[b][q] = 0u;
}
}  // namespace efsi

using namespace efsi;

extern "C" {

int efsi_compute_divergence(efsi_fv_plan* P, const float* velocity, int32_t outlet, float* divergence, void* stream) {
  EFSI_TRY(level_zero_check(P));
  LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  EFSI_COUNTED k_divergence<<<S.grid, S.block, 0, as_stream(stream)>>>(L, velocity, outlet, divergence);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_mg_prepare_level0(efsi_fv_plan* P, const float* divergence, const float* volume_source,
                           const double* iface_rhs, float rhs_scale, double* rhs, void* stream) {
  EFSI_TRY(level_zero_check(P));
  LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  EFSI_COUNTED k_prepare_level0<<<S.grid, S.block, 0, as_stream(stream)>>>(L, divergence, volume_source, iface_rhs, rhs_scale,
                                                              rhs);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_legacy_jacobi_solve(efsi_fv_plan* P, const float* divergence, const float* volume_source, float rhs_scale,
                             float inv_dx2, float inv_dy2, float inv_dz2, int32_t outlet, int32_t iterations,
                             double* pressure, double* tmp, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(P->obstacle0 != nullptr, "masks were built without an obstacle field");
  LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  cudaStream_t s = as_stream(stream);
  for (int it = 0; it < iterations; ++it) {
    EFSI_COUNTED k_legacy_jacobi<<<S.grid, S.block, 0, s>>>(L, P->obstacle0, pressure, divergence, volume_source, rhs_scale,
                                               inv_dx2, inv_dy2, inv_dz2, outlet, tmp);
    EFSI_CUDA_CHECK(cudaMemcpyAsync(pressure, tmp, P->lv[0].n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  }
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_subtract_pressure_gradient(efsi_fv_plan* P, const double* pressure, const int32_t* vdir_active,
                                    const float* vdir_weight, const float* vdir_value, float dt_over_rho,
                                    int32_t outlet, float* velocity, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(vdir_active == nullptr || (vdir_weight != nullptr && vdir_value != nullptr),
                 "vdir arrays must be given together");
  LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  EFSI_COUNTED k_gradient<<<S.grid, S.block, 0, as_stream(stream)>>>(L, pressure, vdir_active, vdir_weight, vdir_value,
                                                        dt_over_rho, outlet, velocity);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_apply_closed_boundary(efsi_fv_plan* P, int32_t outlet, float* velocity, void* stream) {
  EFSI_TRY(level_zero_check(P));
  const LevelBuf& B = P->lv[0];
  int64_t total = (int64_t)B.ny * B.nz + (int64_t)B.nx * B.nz + (int64_t)B.nx * B.ny;
  EFSI_COUNTED k_closed_boundary<<<(unsigned)((total + 255) / 256), 256, 0, as_stream(stream)>>>(B.nx, B.ny, B.nz, outlet,
                                                                                     velocity);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_apply_zmin_no_backflow(efsi_fv_plan* P, float* velocity, void* stream) {
  EFSI_TRY(level_zero_check(P));
  LevelDev L = level_dev(P, 0);
  int64_t total = (int64_t)L.nx * L.ny;
  EFSI_COUNTED k_zmin_no_backflow<<<(unsigned)((total + 255) / 256), 256, 0, as_stream(stream)>>>(L, velocity);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_apply_velocity_dirichlet_rows(efsi_fv_plan* P, const int32_t* vdir_active, const float* vdir_value,
                                       float density, float* velocity, double* report_device, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(vdir_active != nullptr && vdir_value != nullptr, "null Dirichlet arrays");
  LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  cudaStream_t s = as_stream(stream);
  if (report_device) EFSI_CUDA_CHECK(cudaMemsetAsync(report_device, 0, 6 * sizeof(double), s));
  EFSI_COUNTED k_vdir_rows<<<S.grid, S.block, 0, s>>>(L, vdir_active, vdir_value, density, velocity, report_device);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_predict(efsi_fv_plan* P, const efsi_grid_axes* axes, const float* velocity_prev, float dt, float nu,
                 int32_t rk2, float* velocity, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(axes != nullptr && velocity_prev != nullptr && velocity != nullptr && velocity != velocity_prev,
                 "predict needs distinct velocity and velocity_prev buffers");
  LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  EFSI_TIMED(KF_PREDICT, 25.0 * P->lv[0].n, as_stream(stream),
             EFSI_COUNTED k_predict<<<S.grid, S.block, 0, as_stream(stream)>>>(L, *axes, velocity_prev, dt, nu, rk2, velocity));
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_divergence_stats(efsi_fv_plan* P, const float* divergence, const double* iface_div,
                          const float* volume_source, int32_t mode, int32_t interior_only, double* out_host,
                          void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(mode == 0 || volume_source != nullptr, "residual statistics need the volume source");
  LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  cudaStream_t s = as_stream(stream);
  double* tmp = P->aux;
  EFSI_CUDA_CHECK(cudaMemsetAsync(tmp, 0, 3 * sizeof(double), s));
  EFSI_COUNTED k_div_stats<<<S.grid, S.block, 0, s>>>(L, divergence, iface_div, volume_source, mode, interior_only, P->partials,
                                         &P->sc->ticket, tmp);
  EFSI_LAUNCH_CHECK();
  EFSI_CUDA_CHECK(cudaMemcpyAsync(out_host, tmp, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
  EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  return EFSI_OK;
}

int efsi_divergence_final_report(efsi_fv_plan* P, const float* divergence, const double* iface_div,
                                 const float* volume_source, const int32_t* velocity_dirichlet_active,
                                 const int32_t* outlet_reachable, int32_t outlet, double* out_host, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(divergence != nullptr && volume_source != nullptr && out_host != nullptr, "null argument");
  LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  cudaStream_t s = as_stream(stream);
  if (P->report_buf == nullptr) EFSI_CUDA_CHECK(cudaMalloc(&P->report_buf, 54 * sizeof(double)));
  EFSI_CUDA_CHECK(cudaMemsetAsync(P->report_buf, 0, 54 * sizeof(double), s));
  EFSI_COUNTED k_div_final_report<<<S.grid, S.block, 0, s>>>(L, divergence, iface_div, volume_source,
                                                             velocity_dirichlet_active, outlet_reachable,
                                                             outlet ? 1 : 0, P->report_buf);
  EFSI_LAUNCH_CHECK();
  EFSI_CUDA_CHECK(cudaMemcpyAsync(out_host, P->report_buf, 54 * sizeof(double), cudaMemcpyDeviceToHost, s));
  EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  return EFSI_OK;
}

int efsi_spread_surface_forces(efsi_fv_plan* P, const efsi_grid_axes* axes, const float* position, const float* force,
                               int32_t vertex_count, float cx, float cy, float cz, float force_sign,
                               float* grid_force_density, double* report_device, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(vertex_count > 0 && axes != nullptr && report_device != nullptr, "invalid spreading arguments");
  LevelDev L = level_dev(P, 0);
  cudaStream_t s = as_stream(stream);
  EFSI_CUDA_CHECK(cudaMemsetAsync(grid_force_density, 0, P->lv[0].n * 3 * sizeof(float), s));
  EFSI_CUDA_CHECK(cudaMemsetAsync(report_device, 0, 6 * sizeof(double), s));
  EFSI_COUNTED k_spread<<<(vertex_count + 127) / 128, 128, 0, s>>>(L, *axes, position, force, vertex_count, cx, cy, cz, force_sign,
                                                      grid_force_density, report_device);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_apply_body_force(efsi_fv_plan* P, const float* grid_force_density, float dt, float density, float* velocity,
                          double* report_device, void* stream) {
  EFSI_TRY(level_zero_check(P));
  LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  cudaStream_t s = as_stream(stream);
  if (report_device) EFSI_CUDA_CHECK(cudaMemsetAsync(report_device, 0, 7 * sizeof(double), s));
  EFSI_COUNTED k_body_force<<<S.grid, S.block, 0, s>>>(L, grid_force_density, dt, density, velocity, report_device);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}


// Zeroes up to 64 buffers (4-byte multiples) in one launch: the per-solve
// clears of the reference's multigrid work fields (fluid.py:5228-5260
// _prepare_fv_multigrid_rhs) as one kernel instead of one fill per field.
int efsi_zero_buffers(int32_t count, void* const* ptrs, const int64_t* bytes, void* stream) {
  EFSI_ARG_CHECK(count >= 0 && count <= efsi::kZeroListMax, "at most 64 buffers per call");
  if (count == 0) return EFSI_OK;
  EFSI_ARG_CHECK(ptrs != nullptr && bytes != nullptr, "null argument");
  efsi::ZeroList Z{};
  Z.n = count;
  int64_t total = 0;
  for (int q = 0; q < count; ++q) {
    EFSI_ARG_CHECK(ptrs[q] != nullptr && bytes[q] >= 0 && bytes[q] % 4 == 0, "buffers must be 4-byte multiples");
    Z.p[q] = static_cast<uint32_t*>(ptrs[q]);
    Z.words[q] = bytes[q] / 4;
    total += Z.words[q];
  }
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 8));
  EFSI_COUNTED efsi::k_zero_list<<<grid, 256, 0, as_stream(stream)>>>(Z);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

}  // extern "C"
