// Finite-volume pressure projection on a graded Cartesian grid, B200 path.
//
// Replaces the Taichi kernels of simulation_core/fluid.py that sit on the
// pressure-projection hot path: the variable-spacing 7-point operator
// (fluid.py:4080-4456), its damped-Jacobi smoother (fluid.py:4224-4273), the
// multigrid residual / restriction / prolongation (fluid.py:5262-5406), the
// weighted CG inner products and updates (fluid.py:4459-4726) and the flexible
// PCG driver (fluid.py:6535-6811).
//
// Layout in HBM: every cell field is C order (nx, ny, nz), k fastest; level 0
// keeps the reference's f64 pressure / CG vectors, coarse levels are f32.  The
// obstacle / Dirichlet / outlet structure of a level is folded once per
// projection into one byte per cell (six "face open" bits, fluid bit, solid
// bit), and the f32 axis metrics into per-axis f64 face-coefficient tables, so
// a stencil evaluation reads 1 byte of structure per cell instead of seven
// 4-byte obstacle values.
//
// Fusions relative to the reference's kernel sequence (each keeps the
// reference's per-element arithmetic):
//   * SpMV + <d, Ad>_V + alpha, and the direction update d = z + beta d is
//     evaluated inside the SpMV (d ping-pongs between two buffers);
//   * the CG update also forms delta = r_new - r_old for the flexible beta;
//   * z's zero-mean projection is applied on the fly by its consumers;
//   * the V-cycle's level residual is formed inside the restriction, the
//     prolongation inside the first post-smoothing sweep, and the first
//     pre-smoothing sweep uses the zero initial guess;
//   * every scalar reduction is a deterministic two-stage block reduction whose
//     last block also evaluates alpha / beta / means (no extra launches).
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "efsi_fv_internal.cuh"
#include "efsi_unet_internal.cuh"
#include <cuda_bf16.h>
#include "efsi_march.cuh"

namespace efsi {

#define EFSI_CELL_PROLOGUE(L)                                 \
  const int k = blockIdx.x * blockDim.x + threadIdx.x;       \
  const int j = blockIdx.y * blockDim.y + threadIdx.y;       \
  const int i = blockIdx.z * blockDim.z + threadIdx.z;       \
  const bool active = (i < (L).nx && j < (L).ny && k < (L).nz); \
  const int64_t c = active ? cidx(i, j, k, (L).ny, (L).nz) : 0;

// ---------------------------------------------------------------------------
// Setup kernels
// ---------------------------------------------------------------------------

// f64 face coefficient tables: c-[i] = 1/(w[i] cd[i]), c+[i] = 1/(w[i] cd[i+1]).
__global__ void k_axis_coef(const float* w, const float* cd, int n, double* cm, double* cp) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  cm[i] = i > 0 ? 1.0 / ((double)w[i] * (double)cd[i]) : 0.0;
  cp[i] = i < n - 1 ? 1.0 / ((double)w[i] * (double)cd[i + 1]) : 0.0;
}

__global__ void k_mask_from_obstacle(int nx, int ny, int nz, const int32_t* obs, const int32_t* va,
                                     const float* vw, uint8_t* mask, float* fw) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= nx || j >= ny || k >= nz) return;
  const int64_t c = cidx(i, j, k, ny, nz);
  const int64_t sx = (int64_t)ny * nz, sy = nz;
  unsigned m = 0;
  if (i > 0 && obs[c - sx] == 0) m |= M_XM;
  if (i < nx - 1 && obs[c + sx] == 0) m |= M_XP;
  if (j > 0 && obs[c - sy] == 0) m |= M_YM;
  if (j < ny - 1 && obs[c + sy] == 0) m |= M_YP;
  if (k > 0 && obs[c - 1] == 0) m |= M_ZM;
  if (k < nz - 1 && obs[c + 1] == 0) m |= M_ZP;
  if (obs[c] == 0) m |= M_FLUID;
  if (obs[c] == 1) m |= M_SOLID;
  mask[c] = (uint8_t)m;
  if (fw != nullptr) {
    float w = 1.0f;
    if (va != nullptr && va[c] != 0) w = fminf(fmaxf(vw[c], 0.0f), 1.0f);
    fw[c] = w;
  }
}

// Coarse obstacle / Dirichlet flag and weight / interface diagonal of level
// l+1 from level l (fluid.py:5331-5382).  The f32 locals of the reference
// round every accumulation to f32; a product of an f64 fine value with the f32
// cell volume is formed in f64 first.
template <typename TF>
__global__ void k_coarsen_structure(int fnx, int fny, int fnz, const int32_t* fobs, const int32_t* fva,
                                    const float* fvw, const TF* fiface, const float* fwx, const float* fwy,
                                    const float* fwz, int cnx, int cny, int cnz, int32_t* cobs, int32_t* cva,
                                    float* cvw, float* ciface) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= cnx || j >= cny || k >= cnz) return;
  float wdiag = 0.0f, free_vol = 0.0f, vdw = 0.0f;
  int ocount = 0, vcount = 0;
  for (int oi = 0; oi < 2; ++oi)
    for (int oj = 0; oj < 2; ++oj)
      for (int ok = 0; ok < 2; ++ok) {
        int fi = 2 * i + oi, fj = 2 * j + oj, fk = 2 * k + ok;
        if (fi < fnx && fj < fny && fk < fnz) {
          int64_t f = cidx(fi, fj, fk, fny, fnz);
          if (fva != nullptr && fva[f] != 0) {
            vcount += 1;
            vdw = fmaxf(vdw, fvw[f]);
          }
          if (fobs[f] == 1) {
            ocount += 1;
          } else {
            float vol = __fmul_rn(__fmul_rn(fwx[fi], fwy[fj]), fwz[fk]);
            if (fiface != nullptr) {
              if (sizeof(TF) == 8)
                wdiag = (float)__dadd_rn((double)wdiag, __dmul_rn((double)fiface[f], (double)vol));
              else
                wdiag = __fadd_rn(wdiag, __fmul_rn((float)fiface[f], vol));
            }
            free_vol = __fadd_rn(free_vol, vol);
          }
        }
      }
  int64_t cc = cidx(i, j, k, cny, cnz);
  cobs[cc] = ocount > 0 ? 1 : 0;
  if (ciface != nullptr) ciface[cc] = ocount > 0 ? 0.0f : __fdiv_rn(wdiag, fmaxf(free_vol, 1.0e-30f));
  if (cva != nullptr) {
    cva[cc] = vcount > 0 ? 1 : 0;
    cvw[cc] = vcount > 0 ? vdw : 0.0f;
  }
}

// ---------------------------------------------------------------------------
// Level kernels (smoother, residual, restriction, prolongation)
// ---------------------------------------------------------------------------

// Right-hand side of a level row: the level's rhs array, or -r at level 0 of
// the PCG's V-cycle (legacy_rhs = -positive_rhs, fluid.py:4485-4500).
template <typename TP, bool kNegR>
__device__ __forceinline__ double rhs_at(const void* rhs, int64_t c, unsigned m) {
  if (kNegR) {
    if (m & M_SOLID) return 0.0;
    return -__ldg(reinterpret_cast<const double*>(rhs) + c);
  }
  return (double)__ldg(reinterpret_cast<const TP*>(rhs) + c);
}


template <typename TP>
__device__ __forceinline__ double fused_iterate(const TP* __restrict__ p, const ProlongSrc& pr, int64_t cell, int ii,
                                                int jj, int kk, bool fluid) {
  if (pr.pc == nullptr) return (double)__ldg(p + cell);
  TP v = __ldg(p + cell);
  if (fluid) {
    int ci = min(ii / 2, pr.cnx - 1), cj = min(jj / 2, pr.cny - 1), ck = min(kk / 2, pr.cnz - 1);
    float corr = __fmul_rn(pr.scale, __ldg(pr.pc + cidx(ci, cj, ck, pr.cny, pr.cnz)));
    if (sizeof(TP) == 8)
      v = (TP)__dadd_rn((double)v, (double)corr);
    else
      v = (TP)__fadd_rn((float)v, corr);
  }
  return (double)v;
}

// One damped-Jacobi sweep (fluid.py:4224-4273), out of place.
//   kZero   : the input iterate is identically zero (first sweep of a
//             V-cycle level), so p is not read.
//   pr.pc   : fuse the prolongation p += s * p_coarse (fluid.py:5391-5406).
//   partials: when not null, also reduce sum_fluid out * V (z mean, level 0).
template <typename TP, bool kNegR, bool kZero>
__global__ void __launch_bounds__(256) k_sweep(LevelDev L, const TP* __restrict__ p, const void* rhs,
                                               TP* __restrict__ out, int outlet, double omega, ProlongSrc pr,
                                               double* partials, CgScalars* sc) {
  pdl_wait();
  EFSI_CELL_PROLOGUE(L)
  double zv = 0.0;
  if (active) {
    const unsigned m = __ldg(L.mask + c);
    if (m & M_SOLID) {
      out[c] = (TP)0;
    } else {
      double ns, den;
      if (kZero) {
        den = 0.0;
        ns = 0.0;
        // denominator only (neighbour values are zero)
        auto zero = [](int64_t, int, int, int) { return 0.0; };
        stencil(L, zero, i, j, k, c, m, outlet, ns, den);
      } else {
        auto val = [&](int64_t cell, int ii, int jj, int kk) { return fused_iterate(p, pr, cell, ii, jj, kk, true); };
        stencil(L, val, i, j, k, c, m, outlet, ns, den);
      }
      den += iface_at<TP>(L, c);
      TP res;
      if (den <= 0.0) {
        res = (TP)0;
      } else {
        double jv = (ns - rhs_at<TP, kNegR>(rhs, c, m)) / den;
        double pc = kZero ? 0.0 : fused_iterate(p, pr, c, i, j, k, (m & M_FLUID) != 0);
        res = (TP)(pc + omega * (jv - pc));
      }
      out[c] = res;
      if (partials != nullptr && (m & M_FLUID)) zv = (double)res * vol64(L, i, j, k);
    }
  }
  if (partials != nullptr) {
    double v[1] = {zv}, t[1];
    if (grid_sum<1>(v, partials, &sc->ticket, t)) {
      if (flat_tid() == 0) {
        sc->mean_z = sc->free_vol > 0.0 ? 1.0 * t[0] / sc->free_vol : 0.0;
        sc->zproj = 1;
      }
    }
  }
}

// fluid.py:5262-5307 residual of one row (level storage precision).
template <typename TP, bool kNegR>
__device__ __forceinline__ TP row_residual(const LevelDev& L, const TP* __restrict__ p, const void* rhs, int i, int j,
                                           int k, int64_t c, unsigned m, int outlet) {
  if (m & M_SOLID) return (TP)0;
  double ns, den;
  auto val = [&](int64_t cell, int, int, int) { return (double)__ldg(p + cell); };
  stencil(L, val, i, j, k, c, m, outlet, ns, den);
  den += iface_at<TP>(L, c);
  double applied = ns - den * (double)__ldg(p + c);
  return (TP)(rhs_at<TP, kNegR>(rhs, c, m) - applied);
}

template <typename TP, bool kNegR>
__global__ void __launch_bounds__(256) k_residual(LevelDev L, const TP* __restrict__ p, const void* rhs,
                                                  TP* __restrict__ res, int outlet) {
  EFSI_CELL_PROLOGUE(L)
  if (!active) return;
  const unsigned m = __ldg(L.mask + c);
  res[c] = row_residual<TP, kNegR>(L, p, rhs, i, j, k, c, m, outlet);
}

// fluid.py:5310-5388 volume-weighted restriction of the residual, with the
// fine residual formed on the fly (kFromP) or read from an array.
template <typename TP, bool kNegR, bool kFromP>
__global__ void __launch_bounds__(256) k_restrict(LevelDev F, const TP* __restrict__ p_or_res, const void* rhs,
                                                  int outlet, int cnx, int cny, int cnz, float* __restrict__ crhs) {
  pdl_wait();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= cnx || j >= cny || k >= cnz) return;
  float wres = 0.0f, free_vol = 0.0f;
  int ocount = 0;
#pragma unroll
  for (int oi = 0; oi < 2; ++oi)
#pragma unroll
    for (int oj = 0; oj < 2; ++oj)
#pragma unroll
      for (int ok = 0; ok < 2; ++ok) {
        int fi = 2 * i + oi, fj = 2 * j + oj, fk = 2 * k + ok;
        if (fi < F.nx && fj < F.ny && fk < F.nz) {
          int64_t f = cidx(fi, fj, fk, F.ny, F.nz);
          unsigned m = __ldg(F.mask + f);
          if (m & M_SOLID) {
            ocount += 1;
          } else {
            float vol = __fmul_rn(__fmul_rn(__ldg(F.wx + fi), __ldg(F.wy + fj)), __ldg(F.wz + fk));
            TP r = kFromP ? row_residual<TP, kNegR>(F, p_or_res, rhs, fi, fj, fk, f, m, outlet) : __ldg(p_or_res + f);
            if (sizeof(TP) == 8)
              wres = (float)__dadd_rn((double)wres, __dmul_rn((double)r, (double)vol));
            else
              wres = __fadd_rn(wres, __fmul_rn((float)r, vol));
            free_vol = __fadd_rn(free_vol, vol);
          }
        }
      }
  crhs[cidx(i, j, k, cny, cnz)] = ocount > 0 ? 0.0f : __fdiv_rn(wres, fmaxf(free_vol, 1.0e-30f));
}

template <typename TP>
__global__ void __launch_bounds__(256) k_prolong(LevelDev L, TP* __restrict__ p, ProlongSrc pr) {
  EFSI_CELL_PROLOGUE(L)
  if (!active) return;
  const unsigned m = __ldg(L.mask + c);
  if (m & M_FLUID) p[c] = (TP)fused_iterate(p, pr, c, i, j, k, true);
}

// ---------------------------------------------------------------------------
// Tiled level kernels.  A block of 32 (k) x 8 (j) threads walks tiles of
// 32 x 8 x kCI cells (grid-stride over tiles, about four resident blocks per
// SM); each thread marches kCI consecutive cells along i.  All stencil inputs
// of the kCI cells -- the i-column from i0-1 to i0+kCI and the four lateral
// neighbours of every cell -- are loaded before any arithmetic, which keeps
// ~25 independent loads per thread in flight.  Reductions keep one partial per
// block, so the last-block finisher handles a few hundred partials.
// ---------------------------------------------------------------------------
constexpr int kTK = 32, kTJ = 8, kCI = 4;

__host__ __device__ __forceinline__ int tiles_of(int nx, int ny, int nz) {
  return ((nz + kTK - 1) / kTK) * ((ny + kTJ - 1) / kTJ) * ((nx + kCI - 1) / kCI);
}

__device__ __forceinline__ bool tile_coords(const LevelDev& L, int tile, int& i0, int& j, int& k) {
  const int ntk = (L.nz + kTK - 1) / kTK, ntj = (L.ny + kTJ - 1) / kTJ;
  const int tk = tile % ntk, rest = tile / ntk;
  const int tj = rest % ntj, ti = rest / ntj;
  k = tk * kTK + (int)threadIdx.x;
  j = tj * kTJ + (int)threadIdx.y;
  i0 = ti * kCI;
  return j < L.ny && k < L.nz;
}

// Neighbour sum / denominator from pre-loaded neighbour values (same order
// and arithmetic as `stencil`).
__device__ __forceinline__ void stencil_vals(const LevelDev& L, int i, int j, int k, int64_t c, unsigned m, int outlet,
                                             double vxm, double vxp, double vym, double vyp, double vzm, double vzp,
                                             double& ns, double& den) {
  double kxm = __ldg(L.cxm + i), kxp = __ldg(L.cxp + i);
  double kym = __ldg(L.cym + j), kyp = __ldg(L.cyp + j);
  double kzm = __ldg(L.czm + k), kzp = __ldg(L.czp + k);
  if (L.fw != nullptr) {
    const int64_t sx = (int64_t)L.ny * L.nz, sy = L.nz;
    const double fc = (double)__ldg(L.fw + c);
    kxm *= fc;
    kxp *= (double)__ldg(L.fw + (i < L.nx - 1 ? c + sx : c));
    kym *= fc;
    kyp *= (double)__ldg(L.fw + (j < L.ny - 1 ? c + sy : c));
    kzm *= fc;
    kzp *= (double)__ldg(L.fw + (k < L.nz - 1 ? c + 1 : c));
  }
  ns = 0.0;
  den = 0.0;
  if (m & M_XM) {
    ns += kxm * vxm;
    den += kxm;
  }
  if (m & M_XP) {
    ns += kxp * vxp;
    den += kxp;
  }
  if (m & M_YM) {
    ns += kym * vym;
    den += kym;
  }
  if (m & M_YP) {
    ns += kyp * vyp;
    den += kyp;
  }
  if (m & M_ZM) {
    ns += kzm * vzm;
    den += kzm;
  }
  if (m & M_ZP) {
    ns += kzp * vzp;
    den += kzp;
  }
  if (outlet && k == 0) den += L.oz;
}

// Loads the i-column (i0-1 .. i0+kCI) and the lateral neighbours of the kCI
// cells through `val(cell, i, j, k)`; out-of-domain positions read an
// in-domain cell (their faces are closed, the value is never used).
template <class VAL>
__device__ __forceinline__ void load_column(const LevelDev& L, const VAL& val, int i0, int j, int k,
                                            double (&col)[kCI + 2], double (&lat)[kCI][4]) {
  const int64_t sx = (int64_t)L.ny * L.nz, sy = L.nz;
  const int64_t base = (int64_t)j * L.nz + k;
  const int nx1 = L.nx - 1;
  const bool hym = j > 0, hyp = j < L.ny - 1, hzm = k > 0, hzp = k < L.nz - 1;
#pragma unroll
  for (int q = 0; q < kCI + 2; ++q) {
    const int ii = min(max(i0 - 1 + q, 0), nx1);
    col[q] = val(ii * sx + base, ii, j, k);
  }
#pragma unroll
  for (int q = 0; q < kCI; ++q) {
    const int ii = min(i0 + q, nx1);
    const int64_t c = ii * sx + base;
    lat[q][0] = val(hym ? c - sy : c, ii, hym ? j - 1 : j, k);
    lat[q][1] = val(hyp ? c + sy : c, ii, hyp ? j + 1 : j, k);
    lat[q][2] = val(hzm ? c - 1 : c, ii, j, hzm ? k - 1 : k);
    lat[q][3] = val(hzp ? c + 1 : c, ii, j, hzp ? k + 1 : k);
  }
}

// Tiled damped-Jacobi sweep (see k_sweep).
template <typename TP, bool kNegR, bool kZero>
__global__ void __launch_bounds__(256) kt_sweep(LevelDev L, const TP* __restrict__ p, const void* rhs,
                                                TP* __restrict__ out, int outlet, double omega, ProlongSrc pr,
                                                double* partials, CgScalars* sc) {
  pdl_wait();
  const int nt = tiles_of(L.nx, L.ny, L.nz);
  const int64_t sx = (int64_t)L.ny * L.nz;
  double zsum = 0.0;
  for (int tile = blockIdx.x; tile < nt; tile += gridDim.x) {
    int i0, j, k;
    if (!tile_coords(L, tile, i0, j, k)) continue;
    const int64_t base = (int64_t)j * L.nz + k;
    unsigned msk[kCI];
    double rv[kCI];
#pragma unroll
    for (int q = 0; q < kCI; ++q) {
      const int64_t c = (int64_t)min(i0 + q, L.nx - 1) * sx + base;
      msk[q] = __ldg(L.mask + c);
      rv[q] = rhs_at<TP, kNegR>(rhs, c, msk[q]);
    }
    double col[kCI + 2], lat[kCI][4];
    if (!kZero) {
      auto val = [&](int64_t cell, int ii, int jj, int kk) { return fused_iterate(p, pr, cell, ii, jj, kk, true); };
      load_column(L, val, i0, j, k, col, lat);
    } else {
#pragma unroll
      for (int q = 0; q < kCI + 2; ++q) col[q] = 0.0;
#pragma unroll
      for (int q = 0; q < kCI; ++q) lat[q][0] = lat[q][1] = lat[q][2] = lat[q][3] = 0.0;
    }
#pragma unroll
    for (int q = 0; q < kCI; ++q) {
      const int i = i0 + q;
      if (i >= L.nx) break;
      const int64_t c = (int64_t)i * sx + base;
      const unsigned m = msk[q];
      if (m & M_SOLID) {
        out[c] = (TP)0;
        continue;
      }
      double ns, den;
      stencil_vals(L, i, j, k, c, m, outlet, col[q], col[q + 2], lat[q][0], lat[q][1], lat[q][2], lat[q][3], ns, den);
      den += iface_at<TP>(L, c);
      TP res;
      if (den <= 0.0) {
        res = (TP)0;
      } else {
        const double jv = (ns - rv[q]) / den;
        double pc = 0.0;
        if (!kZero) pc = (m & M_FLUID) || pr.pc == nullptr ? col[q + 1] : (double)__ldg(p + c);
        res = (TP)(pc + omega * (jv - pc));
      }
      out[c] = res;
      if (partials != nullptr && (m & M_FLUID)) zsum += (double)res * vol64(L, i, j, k);
    }
  }
  if (partials != nullptr) {
    double v[1] = {zsum}, t[1];
    if (grid_sum<1>(v, partials, &sc->ticket, t)) {
      if (flat_tid() == 0) {
        sc->mean_z = sc->free_vol > 0.0 ? 1.0 * t[0] / sc->free_vol : 0.0;
        sc->zproj = 1;
      }
    }
  }
}

// Tiled d_new = z' (+ beta d_old), Ad = A d_new, <d, Ad>_V and alpha (see k_spmv_dir).
template <bool kCopy>
__global__ void __launch_bounds__(256) kt_spmv_dir(LevelDev L, const double* __restrict__ z,
                                                   const double* __restrict__ d_old, double* __restrict__ d_new,
                                                   double* __restrict__ Ad, int outlet, double* partials,
                                                   CgScalars* sc) {
  pdl_wait();
  const int nt = tiles_of(L.nx, L.ny, L.nz);
  const int64_t sx = (int64_t)L.ny * L.nz;
  const double beta = kCopy ? 0.0 : sc->beta;
  const int zproj = sc->zproj;
  const double mz = sc->mean_z;
  double part = 0.0;
  for (int tile = blockIdx.x; tile < nt; tile += gridDim.x) {
    int i0, j, k;
    if (!tile_coords(L, tile, i0, j, k)) continue;
    const int64_t base = (int64_t)j * L.nz + k;
    unsigned msk[kCI];
#pragma unroll
    for (int q = 0; q < kCI; ++q) msk[q] = __ldg(L.mask + (int64_t)min(i0 + q, L.nx - 1) * sx + base);
    // Neighbours in the stencil are open (obstacle == 0, hence fluid).
    auto dval = [&](int64_t cell, int, int, int) {
      double zz = __ldg(z + cell);
      if (zproj) zz = zz - mz;
      return kCopy ? zz : zz + beta * __ldg(d_old + cell);
    };
    double col[kCI + 2], lat[kCI][4];
    load_column(L, dval, i0, j, k, col, lat);
#pragma unroll
    for (int q = 0; q < kCI; ++q) {
      const int i = i0 + q;
      if (i >= L.nx) break;
      const int64_t c = (int64_t)i * sx + base;
      const unsigned m = msk[q];
      double dc;
      if (m & M_SOLID) {
        dc = 0.0;
      } else if (!(m & M_FLUID) && zproj) {
        dc = kCopy ? 0.0 : 0.0 + beta * __ldg(d_old + c);  // z' = 0 off the fluid set
      } else {
        dc = col[q + 1];
      }
      d_new[c] = dc;
      double o;
      if (m & M_SOLID) {
        o = 0.0;
      } else {
        double ns, den;
        stencil_vals(L, i, j, k, c, m, outlet, col[q], col[q + 2], lat[q][0], lat[q][1], lat[q][2], lat[q][3], ns,
                     den);
        o = (den + iface_at<double>(L, c)) * dc - ns;
      }
      Ad[c] = o;
      if (m & M_FLUID) part += dc * o * vol64(L, i, j, k);
    }
  }
  double v[1] = {part}, t[1];
  if (grid_sum<1>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) {
      spmv_alpha(sc, t[0]);
    }
  }
}

// Tiled CG update (see k_cg_update).  kPart 0 updates x and r (and delta);
// 1 only x, 2 only r (and delta): the two halves of one update, which the
// PCG runs on two streams when no sums are wanted (x is needed by nothing
// but the next update, so its half overlaps the preconditioner).
template <bool kDelta, int kPart = 0>
__global__ void __launch_bounds__(256) kt_cg_update(LevelDev L, double* __restrict__ x, const double* __restrict__ d,
                                                    double* __restrict__ r, const double* __restrict__ Ad,
                                                    double* __restrict__ delta, int want_means, int want_rr,
                                                    double* partials, CgScalars* sc) {
  pdl_wait();
  constexpr bool kX = kPart != 2, kR = kPart != 1;
  const int nt = tiles_of(L.nx, L.ny, L.nz);
  const int64_t sx = (int64_t)L.ny * L.nz;
  const double alpha = sc->alpha;
  double px = 0.0, pr = 0.0, prr = 0.0;
  for (int tile = blockIdx.x; tile < nt; tile += gridDim.x) {
    int i0, j, k;
    if (!tile_coords(L, tile, i0, j, k)) continue;
    const int64_t base = (int64_t)j * L.nz + k;
    const int qn = min(kCI, L.nx - i0);
    unsigned msk[kCI];
    double xv[kCI], dv[kCI], rv[kCI], av[kCI];
#pragma unroll
    for (int q = 0; q < kCI; ++q) {
      if (q >= qn) break;
      const int64_t c = (int64_t)(i0 + q) * sx + base;
      msk[q] = __ldg(L.mask + c);
      if (kX) {
        xv[q] = x[c];
        dv[q] = __ldg(d + c);
      }
      if (kR) {
        rv[q] = r[c];
        av[q] = __ldg(Ad + c);
      }
    }
#pragma unroll
    for (int q = 0; q < kCI; ++q) {
      if (q >= qn) break;
      const int i = i0 + q;
      const int64_t c = (int64_t)i * sx + base;
      if (msk[q] & M_SOLID) {
        if (kX) x[c] = 0.0;
        if (kR) r[c] = 0.0;
        if (kR && kDelta) delta[c] = 0.0;
      } else if (kPart == 1) {
        x[c] = xv[q] + alpha * dv[q];
      } else if (kPart == 2) {
        const double rn = rv[q] - alpha * av[q];
        r[c] = rn;
        if (kDelta) delta[c] = 1.0 * rn + -1.0 * rv[q];
      } else {
        const double xn = xv[q] + alpha * dv[q];
        const double rn = rv[q] - alpha * av[q];
        x[c] = xn;
        r[c] = rn;
        if (kDelta) delta[c] = 1.0 * rn + -1.0 * rv[q];
        if (msk[q] & M_FLUID) {
          const double V = vol64(L, i, j, k);
          px += xn * V;
          pr += rn * V;
          prr += rn * rn * V;
        }
      }
    }
  }
  if (want_means) {
    double v[2] = {px, pr}, t[2];
    if (grid_sum<2>(v, partials, &sc->ticket, t)) {
      if (flat_tid() == 0) {
        sc->mean_x = sc->free_vol > 0.0 ? 1.0 * t[0] / sc->free_vol : 0.0;
        sc->mean_r = sc->free_vol > 0.0 ? 1.0 * t[1] / sc->free_vol : 0.0;
      }
    }
  } else if (want_rr) {
    double v[1] = {prr}, t[1];
    if (grid_sum<1>(v, partials, &sc->ticket, t)) {
      if (flat_tid() == 0) sc->rr = t[0];
    }
  }
}

// The r half of a split update (kt_cg_update<true, 2>) that also forms the
// V-cycle's first level-0 sweep from a zero iterate, which reads only its own
// row: z0 = 0 + omega ((0 - (-r)) / den - 0), 0 on solid rows and where
// den <= 0, as km_sweep0 forms it: f64 z0 with the precomputed reciprocal of
// den; f32 z0 (the FP32 V-cycle, which runs without an interface diagonal)
// dividing by den formed from the row's open faces.
template <typename TZ>
__global__ void __launch_bounds__(256) kt_cg_update_r_zero(LevelDev L, double* __restrict__ r,
                                                           const double* __restrict__ Ad,
                                                           double* __restrict__ delta,
                                                           const double* __restrict__ rden,
                                                           TZ* __restrict__ z0, double omega, int outlet,
                                                           CgScalars* sc) {
  pdl_wait();
  const int nt = tiles_of(L.nx, L.ny, L.nz);
  const int64_t sx = (int64_t)L.ny * L.nz;
  const double alpha = sc->alpha;
  for (int tile = blockIdx.x; tile < nt; tile += gridDim.x) {
    int i0, j, k;
    if (!tile_coords(L, tile, i0, j, k)) continue;
    const int64_t base = (int64_t)j * L.nz + k;
    const int qn = min(kCI, L.nx - i0);
    unsigned msk[kCI];
    double rv[kCI], av[kCI], rd[kCI];
#pragma unroll
    for (int q = 0; q < kCI; ++q) {
      if (q >= qn) break;
      const int64_t c = (int64_t)(i0 + q) * sx + base;
      msk[q] = __ldg(L.mask + c);
      rv[q] = r[c];
      av[q] = __ldg(Ad + c);
      if (sizeof(TZ) == 8) rd[q] = __ldg(rden + c);
    }
    const RowCoef rc = row_coef(L, j, k);
#pragma unroll
    for (int q = 0; q < kCI; ++q) {
      if (q >= qn) break;
      const int i = i0 + q;
      const int64_t c = (int64_t)i * sx + base;
      if (msk[q] & M_SOLID) {
        r[c] = 0.0;
        delta[c] = 0.0;
        z0[c] = (TZ)0;
      } else {
        const double rn = rv[q] - alpha * av[q];
        r[c] = rn;
        delta[c] = 1.0 * rn + -1.0 * rv[q];
        const double rvn = -rn;
        TZ res = (TZ)0;
        if (sizeof(TZ) == 8) {
          if (rd[q] > 0.0) res = (TZ)(0.0 + omega * ((0.0 - rvn) * rd[q] - 0.0));
        } else {
          double ns, den;
          stencil_sel<true>(L, rc, __ldg(L.cxm + i), __ldg(L.cxp + i), i, j, k, c, msk[q], outlet, 0.0, 0.0, 0.0, 0.0,
                            0.0, 0.0, ns, den);
          if (den > 0.0) {
            const double jv = (ns - rvn) / den;
            res = (TZ)(0.0 + omega * (jv - 0.0));
          }
        }
        z0[c] = res;
      }
    }
  }
}

// Tiled rz_new / beta numerator / beta (see k_cg_dots).
template <bool kMG, bool kRestart>
__global__ void __launch_bounds__(256) kt_cg_dots(LevelDev L, const double* __restrict__ r,
                                                  const double* __restrict__ z, const double* __restrict__ delta,
                                                  double* partials, CgScalars* sc) {
  pdl_wait();
  const int nt = tiles_of(L.nx, L.ny, L.nz);
  const int64_t sx = (int64_t)L.ny * L.nz;
  CgScalars s;
  s.mean_z = sc->mean_z;
  const int zproj = sc->zproj;
  double a = 0.0, b = 0.0;
  for (int tile = blockIdx.x; tile < nt; tile += gridDim.x) {
    int i0, j, k;
    if (!tile_coords(L, tile, i0, j, k)) continue;
    const int64_t base = (int64_t)j * L.nz + k;
    const int qn = min(kCI, L.nx - i0);
    unsigned msk[kCI];
    double rv[kCI], zv[kCI], dv[kCI];
#pragma unroll
    for (int q = 0; q < kCI; ++q) {
      if (q >= qn) break;
      const int64_t c = (int64_t)(i0 + q) * sx + base;
      msk[q] = __ldg(L.mask + c);
      rv[q] = __ldg(r + c);
      zv[q] = __ldg(z + c);
      dv[q] = (kMG && !kRestart) ? __ldg(delta + c) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < kCI; ++q) {
      if (q >= qn) break;
      if (!(msk[q] & M_FLUID)) continue;
      const double V = vol64(L, i0 + q, j, k);
      const double zz = zproj ? zv[q] - s.mean_z : zv[q];
      a += rv[q] * zz * V;
      if (kMG && !kRestart) b += zz * dv[q] * V;
    }
  }
  double v[2] = {a, b}, t[2];
  if (grid_sum<2>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) {
      if (kRestart) {
        sc->rz = t[0];
      } else {
        cg_beta_step(sc, t[0], t[1], kMG);
        sc->rz = t[0];
      }
    }
  }
}

// Tiled x -= mean_x, r -= mean_r and <r, r>_V (see k_sub_mean_xr).
__global__ void __launch_bounds__(256) kt_sub_mean_xr(LevelDev L, double* __restrict__ x, double* __restrict__ r,
                                                      double* partials, CgScalars* sc) {
  pdl_wait();
  const int nt = tiles_of(L.nx, L.ny, L.nz);
  const int64_t sx = (int64_t)L.ny * L.nz;
  const double mx = sc->mean_x, mr = sc->mean_r;
  double prr = 0.0;
  for (int tile = blockIdx.x; tile < nt; tile += gridDim.x) {
    int i0, j, k;
    if (!tile_coords(L, tile, i0, j, k)) continue;
    const int64_t base = (int64_t)j * L.nz + k;
    const int qn = min(kCI, L.nx - i0);
#pragma unroll
    for (int q = 0; q < kCI; ++q) {
      if (q >= qn) break;
      const int64_t c = (int64_t)(i0 + q) * sx + base;
      if (__ldg(L.mask + c) & M_FLUID) {
        x[c] = x[c] - mx;
        const double rn = r[c] - mr;
        r[c] = rn;
        prr += rn * rn * vol64(L, i0 + q, j, k);
      } else {
        x[c] = 0.0;
        r[c] = 0.0;
      }
    }
  }
  double v[1] = {prr}, t[1];
  if (grid_sum<1>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) sc->rr = t[0];
  }
}

// ---------------------------------------------------------------------------
// V-cycle tail: all coarse levels from `lt` down to the coarsest run inside one
// CTA, iterates / rhs / masks in shared memory, with the same per-row
// arithmetic as k_sweep / k_restrict (f32 storage, f64 row arithmetic).  One
// launch replaces the per-level launches of the small levels.
// ---------------------------------------------------------------------------
constexpr int kTailMaxLevels = 12;
constexpr int kTailThreads = 512;

struct TailDesc {
  int lt, nl;
  int outlet, pre, coarse, post;
  float scale;
  double omega;
  LevelDev L[kTailMaxLevels];
  int foff[kTailMaxLevels];  // float offset of level l's block (pA, pB, rhs) in shared memory
  int moff[kTailMaxLevels];  // byte offset of level l's mask copy
  int coff[kTailMaxLevels];  // byte offset of level l's row table: 6 face coefficients + denominator (f64, SoA)
  int noff[kTailMaxLevels];  // byte offset of level l's neighbour table: 6 cell indices (int, SoA)
  const float* rhs_in;       // rhs of level lt (written by the restriction from lt - 1)
  float* p_out;              // final iterate of level lt
};

__device__ __forceinline__ void tail_ijk(const LevelDev& L, int t, int& i, int& j, int& k) {
  k = t % L.nz;
  const int ij = t / L.nz;
  j = ij % L.ny;
  i = ij / L.ny;
}

// Row tables of a tail level, built once per launch: for every cell the six
// face coefficients behind open faces (0 behind closed ones; Dirichlet face
// weights applied), the denominator (fluid.py:4080-4221, summed in the order
// x-, x+, y-, y+, z-, z+, then the outlet term and the interface diagonal)
// and the six neighbour indices (the cell itself behind a closed face).  The
// sweeps and residuals then read only shared memory; the arithmetic is that of
// `stencil`, with closed faces contributing exact zeros.
struct TailTables {
  const double* a;  // [6][n]
  const double* den;  // [n]
  const int* nb;  // [6][n]
  int n;
};

__device__ __forceinline__ TailTables tail_tables(const TailDesc& T, int l, unsigned char* smem) {
  const LevelDev& L = T.L[l];
  TailTables tb;
  tb.n = L.nx * L.ny * L.nz;
  tb.a = reinterpret_cast<const double*>(smem + T.coff[l]);
  tb.den = tb.a + 6 * tb.n;
  tb.nb = reinterpret_cast<const int*>(smem + T.noff[l]);
  return tb;
}

__device__ void tail_build_tables(const TailDesc& T, int l, unsigned char* smem, uint8_t* ms) {
  const LevelDev& L = T.L[l];
  const int n = L.nx * L.ny * L.nz;
  double* a = reinterpret_cast<double*>(smem + T.coff[l]);
  double* den = a + 6 * n;
  int* nb = reinterpret_cast<int*>(smem + T.noff[l]);
  const int sx = L.ny * L.nz, sy = L.nz;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    int i, j, k;
    tail_ijk(L, t, i, j, k);
    const unsigned m = L.mask[t];
    ms[t] = (uint8_t)m;
    const int c[6] = {i > 0 ? t - sx : t, i < L.nx - 1 ? t + sx : t, j > 0 ? t - sy : t,
                      j < L.ny - 1 ? t + sy : t, k > 0 ? t - 1 : t, k < L.nz - 1 ? t + 1 : t};
    double kf[6] = {__ldg(L.cxm + i), __ldg(L.cxp + i), __ldg(L.cym + j),
                    __ldg(L.cyp + j), __ldg(L.czm + k), __ldg(L.czp + k)};
    if (L.fw != nullptr) {
      const double fc = (double)__ldg(L.fw + t);
      kf[0] *= fc;
      kf[1] *= (double)__ldg(L.fw + c[1]);
      kf[2] *= fc;
      kf[3] *= (double)__ldg(L.fw + c[3]);
      kf[4] *= fc;
      kf[5] *= (double)__ldg(L.fw + c[5]);
    }
    const unsigned bit[6] = {M_XM, M_XP, M_YM, M_YP, M_ZM, M_ZP};
    double d = 0.0;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const double af = (m & bit[f]) ? kf[f] : 0.0;
      a[f * n + t] = af;
      nb[f * n + t] = c[f];
      d = d + af;
    }
    if (T.outlet && k == 0) d += L.oz;
    d += iface_at<float>(L, t);
    den[t] = d;
  }
}

// Neighbour sum of row t from the tables (same order and fused multiply-adds
// as `stencil`).
__device__ __forceinline__ double tail_ns(const TailTables& tb, const float* p, int t) {
  double ns = fma(tb.a[t], (double)p[tb.nb[t]], 0.0);
#pragma unroll
  for (int f = 1; f < 6; ++f) ns = fma(tb.a[f * tb.n + t], (double)p[tb.nb[f * tb.n + t]], ns);
  return ns;
}

// One Jacobi sweep of level l: src -> dst (src null: zero initial guess).
__device__ void tail_sweep(const TailTables& tb, const float* src, float* dst, const float* rhs, const uint8_t* mask,
                           double omega) {
  for (int t = threadIdx.x; t < tb.n; t += blockDim.x) {
    const unsigned m = mask[t];
    float res = 0.0f;
    if (!(m & M_SOLID)) {
      const double den = tb.den[t];
      if (den > 0.0) {
        const double ns = src != nullptr ? tail_ns(tb, src, t) : 0.0;
        const double jv = (ns - (double)rhs[t]) / den;
        const double pcur = src != nullptr ? (double)src[t] : 0.0;
        res = (float)(pcur + omega * (jv - pcur));
      }
    }
    dst[t] = res;
  }
  __syncthreads();
}

// p += s * p_coarse on the fluid cells of level l (fluid.py:5391-5406).
__device__ void tail_prolong(const TailDesc& T, int l, float* p, const uint8_t* mask, const float* pc) {
  const LevelDev& L = T.L[l];
  const LevelDev& C = T.L[l + 1];
  const int n = L.nx * L.ny * L.nz;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    if (!(mask[t] & M_FLUID)) continue;
    int i, j, k;
    tail_ijk(L, t, i, j, k);
    const int ci = min(i / 2, C.nx - 1), cj = min(j / 2, C.ny - 1), ck = min(k / 2, C.nz - 1);
    p[t] = __fadd_rn(p[t], __fmul_rn(T.scale, pc[(ci * C.ny + cj) * C.nz + ck]));
  }
  __syncthreads();
}

// Residual of level l formed from the tables and volume-weighted into the
// rhs of l+1 (fluid.py:5262-5388).
__device__ void tail_restrict(const TailDesc& T, int l, const TailTables& tb, const float* p, const float* rhs,
                              const uint8_t* mask, float* crhs) {
  const LevelDev& F = T.L[l];
  const LevelDev& C = T.L[l + 1];
  const int nc = C.nx * C.ny * C.nz;
  for (int t = threadIdx.x; t < nc; t += blockDim.x) {
    int i, j, k;
    tail_ijk(C, t, i, j, k);
    float wres = 0.0f, free_vol = 0.0f;
    int ocount = 0;
    for (int oi = 0; oi < 2; ++oi)
      for (int oj = 0; oj < 2; ++oj)
        for (int ok = 0; ok < 2; ++ok) {
          const int fi = 2 * i + oi, fj = 2 * j + oj, fk = 2 * k + ok;
          if (fi < F.nx && fj < F.ny && fk < F.nz) {
            const int f = (fi * F.ny + fj) * F.nz + fk;
            if (mask[f] & M_SOLID) {
              ocount += 1;
            } else {
              const float vol = __fmul_rn(__fmul_rn(__ldg(F.wx + fi), __ldg(F.wy + fj)), __ldg(F.wz + fk));
              const double ns = tail_ns(tb, p, f);
              const float r = (float)((double)rhs[f] - (ns - tb.den[f] * (double)p[f]));
              wres = __fadd_rn(wres, __fmul_rn(r, vol));
              free_vol = __fadd_rn(free_vol, vol);
            }
          }
        }
    crhs[t] = ocount > 0 ? 0.0f : __fdiv_rn(wres, fmaxf(free_vol, 1.0e-30f));
  }
  __syncthreads();
}

// The whole tail V-cycle by one CTA (all threads of the block take part).
__device__ void tail_body(const TailDesc& T, unsigned char* tail_smem) {
  float* fpool = reinterpret_cast<float*>(tail_smem);
  // row tables and masks of every tail level, the rhs of level lt
  for (int l = T.lt; l < T.nl; ++l) tail_build_tables(T, l, tail_smem, tail_smem + T.moff[l]);
  {
    const LevelDev& L = T.L[T.lt];
    const int n = L.nx * L.ny * L.nz;
    float* rhs = fpool + T.foff[T.lt] + 2 * n;
    for (int t = threadIdx.x; t < n; t += blockDim.x) rhs[t] = T.rhs_in[t];
  }
  __syncthreads();
  int cur[kTailMaxLevels];  // 0: pA holds the iterate, 1: pB
  for (int l = T.lt; l < T.nl; ++l) {
    const LevelDev& L = T.L[l];
    const int n = L.nx * L.ny * L.nz;
    float* pa = fpool + T.foff[l];
    float* buf[2] = {pa, pa + n};
    const float* rhs = pa + 2 * n;
    const uint8_t* ms = tail_smem + T.moff[l];
    const TailTables tb = tail_tables(T, l, tail_smem);
    const bool coarsest = (l == T.nl - 1);
    const int sweeps = coarsest ? T.coarse : T.pre;
    int c = -1;
    for (int it = 0; it < sweeps; ++it) {
      const int d = (it & 1);
      tail_sweep(tb, c < 0 ? nullptr : buf[c], buf[d], rhs, ms, T.omega);
      c = d;
    }
    cur[l] = c;
    if (!coarsest) {
      const LevelDev& C = T.L[l + 1];
      float* crhs = fpool + T.foff[l + 1] + 2 * (C.nx * C.ny * C.nz);
      tail_restrict(T, l, tb, buf[c], rhs, ms, crhs);
    }
  }
  for (int l = T.nl - 2; l >= T.lt; --l) {
    const LevelDev& L = T.L[l];
    const int n = L.nx * L.ny * L.nz;
    float* pa = fpool + T.foff[l];
    float* buf[2] = {pa, pa + n};
    const float* rhs = pa + 2 * n;
    const uint8_t* ms = tail_smem + T.moff[l];
    const TailTables tb = tail_tables(T, l, tail_smem);
    const LevelDev& C = T.L[l + 1];
    const float* pc = fpool + T.foff[l + 1] + cur[l + 1] * (C.nx * C.ny * C.nz);
    int c = cur[l];
    tail_prolong(T, l, buf[c], ms, pc);
    for (int it = 0; it < T.post; ++it) {
      const int d = 1 - c;
      tail_sweep(tb, buf[c], buf[d], rhs, ms, T.omega);
      c = d;
    }
    cur[l] = c;
  }
  {
    const LevelDev& L = T.L[T.lt];
    const int n = L.nx * L.ny * L.nz;
    const float* res = fpool + T.foff[T.lt] + cur[T.lt] * n;
    for (int t = threadIdx.x; t < n; t += blockDim.x) T.p_out[t] = res[t];
  }
}

__global__ void __launch_bounds__(kTailThreads) k_mg_tail(TailDesc T) {
  pdl_wait();
  extern __shared__ __align__(16) unsigned char tail_smem[];
  tail_body(T, tail_smem);
}

// ---------------------------------------------------------------------------
// Coarse levels first .. lt-1 and the tail in one launch.  The blocks of the
// grid share the cells of each phase (grid-stride); a barrier separates the
// phases.  Per V-cycle this replaces the per-level launches (3 + 2 per level:
// the pre-sweeps, the restriction and the post-sweeps) and the tail launch by
// one launch and its barriers.  The arithmetic is that of k_sweep /
// k_restrict / k_prolong (and so of the plane-marching kernels): the same
// `stencil` rows in the same order.  Fields written inside the launch are
// read with plain (coherent) loads, never through the read-only path.
// Two forms:
//   - cooperative (first = 1): as many blocks as fit on the GPU, a software
//     grid barrier; every barrier wait is bounded, a block that gives up
//     sets the fault flag, and every block returns at the next barrier that
//     sees the flag;
//   - one thread-block cluster (first = 2, level 1 stays on the
//     plane-marching kernels): the cluster's hardware barrier
//     (barrier.cluster arrive.release / wait.acquire), which every thread of
//     every CTA reaches at the same phase boundaries.
// Phases:
//   level first: the zero-guess sweep, the other pre-sweeps;
//   level l: the restriction into l+1 fused with the zero-guess sweep of
//            l+1 (it only needs the cell's own rhs), the other pre-sweeps;
//   the tail (block 0);
//   level l = lt-1 .. first: the prolongation-fused first post-sweep, the
//            others.
// ---------------------------------------------------------------------------
struct CoarseDesc {
  TailDesc T;  // T.L[l] for every level l >= first; the tail of levels lt..nl-1
  float* pa[kTailMaxLevels];
  float* pb[kTailMaxLevels];
  float* rhs[kTailMaxLevels];
  unsigned* bar;  // [0] arrivals, [1] generation
  int* fault;
  unsigned spin_ns;  // back-off between polls of the generation (0: none)
  int first;         // first level run here (its rhs is already restricted)
  int cluster;       // 1: the grid is one thread-block cluster (hardware barrier)
};

constexpr long long kCoarseWaitLimit = 4000000000LL;  // ~2 s of clock64

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ bool coarse_barrier(const CoarseDesc& D) {
  if (D.cluster) {
    // every thread of every CTA of the cluster arrives (release) and waits
    // (acquire): the phase's global writes are visible to the whole cluster
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
    return true;
  }
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned* count = D.bar;
    unsigned* gen = D.bar + 1;
    const unsigned g = ld_acquire_u32(gen);
    __threadfence();
    if (atomicAdd(count, 1u) == gridDim.x - 1) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      const long long t0 = clock64();
      while (ld_acquire_u32(gen) == g) {
        if (D.spin_ns > 0) __nanosleep(D.spin_ns);
        if (clock64() - t0 > kCoarseWaitLimit) {
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
    if (!ok) atomicExch(D.fault, 1);
    if (*reinterpret_cast<volatile int*>(D.fault) != 0) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// fused_iterate<float> with plain loads
__device__ __forceinline__ double pk_iterate(const float* p, const ProlongSrc& pr, int64_t cell, int ii, int jj, int kk,
                                             bool fluid) {
  float v = p[cell];
  if (pr.pc != nullptr && fluid) {
    const int ci = min(ii / 2, pr.cnx - 1), cj = min(jj / 2, pr.cny - 1), ck = min(kk / 2, pr.cnz - 1);
    v = __fadd_rn(v, __fmul_rn(pr.scale, pr.pc[cidx(ci, cj, ck, pr.cny, pr.cnz)]));
  }
  return (double)v;
}

// One cell of the damped-Jacobi sweep of k_sweep<float, false, kZero>.
template <bool kZero>
__device__ __forceinline__ float pk_sweep_cell(const LevelDev& L, const float* p, double rhs_v, int outlet,
                                               double omega, const ProlongSrc& pr, int i, int j, int k, int64_t c,
                                               unsigned m) {
  if (m & M_SOLID) return 0.0f;
  double ns, den;
  if (kZero) {
    auto zero = [](int64_t, int, int, int) { return 0.0; };
    stencil(L, zero, i, j, k, c, m, outlet, ns, den);
  } else {
    auto val = [&](int64_t cell, int ii, int jj, int kk) { return pk_iterate(p, pr, cell, ii, jj, kk, true); };
    stencil(L, val, i, j, k, c, m, outlet, ns, den);
  }
  den += iface_at<float>(L, c);
  if (den <= 0.0) return 0.0f;
  const double jv = (ns - rhs_v) / den;
  const double pc = kZero ? 0.0 : pk_iterate(p, pr, c, i, j, k, (m & M_FLUID) != 0);
  return (float)(pc + omega * (jv - pc));
}

// row_residual<float, false> with plain loads
__device__ __forceinline__ float pk_residual(const LevelDev& L, const float* p, const float* rhs, int i, int j, int k,
                                             int64_t c, unsigned m, int outlet) {
  if (m & M_SOLID) return 0.0f;
  double ns, den;
  auto val = [&](int64_t cell, int, int, int) { return (double)p[cell]; };
  stencil(L, val, i, j, k, c, m, outlet, ns, den);
  den += iface_at<float>(L, c);
  const double applied = ns - den * (double)p[c];
  return (float)((double)rhs[c] - applied);
}

// k_restrict<float, false, true> of coarse cell (i, j, k)
__device__ __forceinline__ float pk_restrict_cell(const LevelDev& F, const float* p, const float* rhs, int outlet,
                                                  int i, int j, int k) {
  float wres = 0.0f, free_vol = 0.0f;
  int ocount = 0;
#pragma unroll
  for (int oi = 0; oi < 2; ++oi)
#pragma unroll
    for (int oj = 0; oj < 2; ++oj)
#pragma unroll
      for (int ok = 0; ok < 2; ++ok) {
        const int fi = 2 * i + oi, fj = 2 * j + oj, fk = 2 * k + ok;
        if (fi < F.nx && fj < F.ny && fk < F.nz) {
          const int64_t f = cidx(fi, fj, fk, F.ny, F.nz);
          const unsigned m = __ldg(F.mask + f);
          if (m & M_SOLID) {
            ocount += 1;
          } else {
            const float vol = __fmul_rn(__fmul_rn(__ldg(F.wx + fi), __ldg(F.wy + fj)), __ldg(F.wz + fk));
            const float r = pk_residual(F, p, rhs, fi, fj, fk, f, m, outlet);
            wres = __fadd_rn(wres, __fmul_rn(r, vol));
            free_vol = __fadd_rn(free_vol, vol);
          }
        }
      }
  return ocount > 0 ? 0.0f : __fdiv_rn(wres, fmaxf(free_vol, 1.0e-30f));
}

// (coarse levels hold fewer than 2^31 cells: 32-bit division)
__device__ __forceinline__ void pk_ijk(const LevelDev& L, int64_t t, int& i, int& j, int& k) {
  const unsigned u = (unsigned)t, nz = (unsigned)L.nz, ny = (unsigned)L.ny;
  const unsigned ij = u / nz;
  k = (int)(u - ij * nz);
  i = (int)(ij / ny);
  j = (int)(ij - (unsigned)i * ny);
}

#define PK_CELLS(L, t)                                                                    \
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x,                        \
               t##_n = (int64_t)(L).nx * (L).ny * (L).nz;                                 \
       t < t##_n; t += (int64_t)gridDim.x * blockDim.x)

// One sweep of level l from `src` (null: zero guess) into `dst`.
__device__ void pk_sweep(const LevelDev& L, const float* src, const float* rhs, float* dst, int outlet, double omega,
                         const ProlongSrc& pr) {
  PK_CELLS(L, t) {
    int i, j, k;
    pk_ijk(L, t, i, j, k);
    const unsigned m = __ldg(L.mask + t);
    dst[t] = src == nullptr ? pk_sweep_cell<true>(L, nullptr, (double)rhs[t], outlet, omega, pr, i, j, k, t, m)
                            : pk_sweep_cell<false>(L, src, (double)rhs[t], outlet, omega, pr, i, j, k, t, m);
  }
}

__global__ void __launch_bounds__(kTailThreads) k_mg_coarse(const __grid_constant__ CoarseDesc D) {
  extern __shared__ __align__(16) unsigned char tail_smem[];
  const TailDesc& T = D.T;
  const int lt = T.lt;
  const ProlongSrc none{nullptr, 0, 0, 0, 0.0f};
  int cur[kTailMaxLevels];
  // down
  for (int l = D.first; l < lt; ++l) {
    const LevelDev& L = T.L[l];
    float* buf[2] = {D.pa[l], D.pb[l]};
    if (l == D.first) pk_sweep(L, nullptr, D.rhs[l], buf[0], T.outlet, T.omega, none);
    int c = 0;
    for (int it = 1; it < T.pre; ++it) {
      if (!coarse_barrier(D)) return;
      pk_sweep(L, buf[c], D.rhs[l], buf[1 - c], T.outlet, T.omega, none);
      c = 1 - c;
    }
    cur[l] = c;
    if (!coarse_barrier(D)) return;
    const LevelDev& C = T.L[l + 1];
    const bool fuse0 = l + 1 < lt;
    PK_CELLS(C, t) {
      int i, j, k;
      pk_ijk(C, t, i, j, k);
      const float v = pk_restrict_cell(L, buf[c], D.rhs[l], T.outlet, i, j, k);
      D.rhs[l + 1][t] = v;
      if (fuse0)
        D.pa[l + 1][t] = pk_sweep_cell<true>(C, nullptr, (double)v, T.outlet, T.omega, none, i, j, k, t,
                                             __ldg(C.mask + t));
    }
  }
  if (!coarse_barrier(D)) return;
  if (blockIdx.x == 0) tail_body(T, tail_smem);
  if (!coarse_barrier(D)) return;
  // up
  const float* fin = T.p_out;  // final iterate of level l + 1
  for (int l = lt - 1; l >= D.first; --l) {
    const LevelDev& L = T.L[l];
    const LevelDev& C = T.L[l + 1];
    const ProlongSrc pr{fin, C.nx, C.ny, C.nz, T.scale};
    float* buf[2] = {D.pa[l], D.pb[l]};
    const int c = cur[l];
    float* seq[2] = {buf[1 - c], buf[c]};
    const float* src = buf[c];
    for (int it = 0; it < T.post; ++it) {
      if (it > 0 && !coarse_barrier(D)) return;
      pk_sweep(L, src, D.rhs[l], seq[it & 1], T.outlet, T.omega, it == 0 ? pr : none);
      src = seq[it & 1];
    }
    fin = src;
    if (l > D.first && !coarse_barrier(D)) return;
  }
}
#undef PK_CELLS

// ---------------------------------------------------------------------------
// Level-0 CG kernels (f64)
// ---------------------------------------------------------------------------

// z' : the zero-mean projected preconditioned residual (fluid.py:4716-4722),
// evaluated where it is consumed.
__device__ __forceinline__ double zp_at(const double* __restrict__ z, const CgScalars& s, int64_t c, unsigned m,
                                        int zproj) {
  double zv = __ldg(z + c);
  if (!zproj) return zv;
  return (m & M_FLUID) ? zv - s.mean_z : 0.0;
}

// d_new = z' (copy) or z' + beta d_old (fluid.py:4604-4611, masked), then
// Ad = A d_new (fluid.py:4312-4345), <d, Ad>_V and alpha (fluid.py:4567-4574).
template <bool kCopy>
__global__ void __launch_bounds__(256) k_spmv_dir(LevelDev L, const double* __restrict__ z,
                                                  const double* __restrict__ d_old, double* __restrict__ d_new,
                                                  double* __restrict__ Ad, int outlet, double* partials,
                                                  CgScalars* sc) {
  pdl_wait();
  EFSI_CELL_PROLOGUE(L)
  const double beta = kCopy ? 0.0 : sc->beta;
  const int zproj = sc->zproj;
  const double mz = sc->mean_z;
  CgScalars s;
  s.mean_z = mz;
  double part = 0.0;
  if (active) {
    const unsigned m = __ldg(L.mask + c);
    // Neighbours in the stencil are open (obstacle == 0, hence fluid).
    auto dval = [&](int64_t cell, int, int, int) {
      double zz = __ldg(z + cell);
      if (zproj) zz = zz - mz;
      return kCopy ? zz : zz + beta * __ldg(d_old + cell);
    };
    double dc;
    if (m & M_SOLID) {
      dc = 0.0;
    } else {
      double zz = zp_at(z, s, c, m, zproj);
      dc = kCopy ? zz : zz + beta * __ldg(d_old + c);
    }
    d_new[c] = dc;
    double out;
    if (m & M_SOLID) {
      out = 0.0;
    } else {
      double ns, den;
      stencil(L, dval, i, j, k, c, m, outlet, ns, den);
      out = (den + iface_at<double>(L, c)) * dc - ns;
    }
    Ad[c] = out;
    if (m & M_FLUID) part = dc * out * vol64(L, i, j, k);
  }
  double v[1] = {part}, t[1];
  if (grid_sum<1>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) {
      spmv_alpha(sc, t[0]);
    }
  }
}

// fluid.py:4577-4587 _cg_apply_alpha_kernel with delta = r_new - r_old
// (fluid.py:6794) and optional partial sums of x V, r V (mean projection) and
// r r V (residual check).
template <bool kDelta>
__global__ void __launch_bounds__(256) k_cg_update(LevelDev L, double* __restrict__ x, const double* __restrict__ d,
                                                   double* __restrict__ r, const double* __restrict__ Ad,
                                                   double* __restrict__ delta, int want_means, int want_rr,
                                                   double* partials, CgScalars* sc) {
  pdl_wait();
  EFSI_CELL_PROLOGUE(L)
  const double alpha = sc->alpha;
  double px = 0.0, pr = 0.0, prr = 0.0;
  if (active) {
    const unsigned m = __ldg(L.mask + c);
    if (m & M_SOLID) {
      x[c] = 0.0;
      r[c] = 0.0;
      if (kDelta) delta[c] = 0.0;
    } else {
      double r_old = r[c];
      double xn = x[c] + alpha * __ldg(d + c);
      double rn = r_old - alpha * __ldg(Ad + c);
      x[c] = xn;
      r[c] = rn;
      if (kDelta) delta[c] = 1.0 * rn + -1.0 * r_old;
      if (m & M_FLUID) {
        double V = vol64(L, i, j, k);
        px = xn * V;
        pr = rn * V;
        prr = rn * rn * V;
      }
    }
  }
  if (want_means) {
    double v[2] = {px, pr}, t[2];
    if (grid_sum<2>(v, partials, &sc->ticket, t)) {
      if (flat_tid() == 0) {
        sc->mean_x = sc->free_vol > 0.0 ? 1.0 * t[0] / sc->free_vol : 0.0;
        sc->mean_r = sc->free_vol > 0.0 ? 1.0 * t[1] / sc->free_vol : 0.0;
      }
    }
  } else if (want_rr) {
    double v[1] = {prr}, t[1];
    if (grid_sum<1>(v, partials, &sc->ticket, t)) {
      if (flat_tid() == 0) sc->rr = t[0];
    }
  }
}

// Subtract the means found by k_cg_update from x and r (fluid.py:6685-6689),
// then reduce r r V for the residual check.
__global__ void __launch_bounds__(256) k_sub_mean_xr(LevelDev L, double* __restrict__ x, double* __restrict__ r,
                                                     double* partials, CgScalars* sc) {
  pdl_wait();
  EFSI_CELL_PROLOGUE(L)
  const double mx = sc->mean_x, mr = sc->mean_r;
  double prr = 0.0;
  if (active) {
    const unsigned m = __ldg(L.mask + c);
    if (m & M_FLUID) {
      x[c] = x[c] - mx;
      double rn = r[c] - mr;
      r[c] = rn;
      prr = rn * rn * vol64(L, i, j, k);
    } else {
      x[c] = 0.0;
      r[c] = 0.0;
    }
  }
  double v[1] = {prr}, t[1];
  if (grid_sum<1>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) sc->rr = t[0];
  }
}

// rz_new = <r, z'>_V and (flexible) beta numerator <z', delta>_V, then beta
// (fluid.py:4590-4601) and rz <- rz_new; kRestart instead stores rz (initial
// and restarted directions, fluid.py:6662, 6780).
template <bool kMG, bool kRestart>
__global__ void __launch_bounds__(256) k_cg_dots(LevelDev L, const double* __restrict__ r,
                                                 const double* __restrict__ z, const double* __restrict__ delta,
                                                 double* partials, CgScalars* sc) {
  pdl_wait();
  EFSI_CELL_PROLOGUE(L)
  CgScalars s;
  s.mean_z = sc->mean_z;
  const int zproj = sc->zproj;
  double a = 0.0, b = 0.0;
  if (active) {
    const unsigned m = __ldg(L.mask + c);
    if (m & M_FLUID) {
      double V = vol64(L, i, j, k);
      double zz = zp_at(z, s, c, m, zproj);
      a = __ldg(r + c) * zz * V;
      if (kMG && !kRestart) b = zz * __ldg(delta + c) * V;
    }
  }
  double v[2] = {a, b}, t[2];
  if (grid_sum<2>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) {
      if (kRestart) {
        sc->rz = t[0];
      } else {
        cg_beta_step(sc, t[0], t[1], kMG);
        sc->rz = t[0];
      }
    }
  }
}

// fluid.py:4503-4516 Jacobi preconditioner, optionally with the z mean sums.
__global__ void __launch_bounds__(256) k_jacobi_precond(LevelDev L, const double* __restrict__ diag,
                                                        const double* __restrict__ r, double* __restrict__ z,
                                                        int want_mean, double* partials, CgScalars* sc) {
  pdl_wait();
  EFSI_CELL_PROLOGUE(L)
  double pz = 0.0;
  if (active) {
    const unsigned m = __ldg(L.mask + c);
    double zv;
    if (m & M_SOLID) {
      zv = 0.0;
    } else {
      double dg = __ldg(diag + c);
      zv = dg > 0.0 ? __ldg(r + c) / dg : 0.0;
    }
    z[c] = zv;
    if (m & M_FLUID) pz = zv * vol64(L, i, j, k);
  }
  if (want_mean) {
    double v[1] = {pz}, t[1];
    if (grid_sum<1>(v, partials, &sc->ticket, t)) {
      if (flat_tid() == 0) {
        sc->mean_z = sc->free_vol > 0.0 ? 1.0 * t[0] / sc->free_vol : 0.0;
        sc->zproj = 1;
      }
    }
  }
}

// fluid.py:4345-4456: the interface-coupling terms of the level-0 operator,
// held as rows of (source cell, coefficient = T / V_receiver) entries per
// receiving cell in the order the reference's coupling list visits them:
// out[c] += -(coef * p[src]) entry by entry (with `residual`, the terms are
// subtracted from a residual b - A p instead).  Rows are distinct cells, so
// the result does not depend on thread order.  The row count is read from the
// device, which keeps captured graphs valid when the couplings change.
__global__ void __launch_bounds__(256) k_couple(const int32_t* __restrict__ rows, const int32_t* __restrict__ ptr,
                                                const int32_t* __restrict__ src, const double* __restrict__ coef,
                                                const int32_t* __restrict__ nrows, const double* __restrict__ p,
                                                double* __restrict__ out, int residual) {
  pdl_wait();
  const int n = *nrows;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int c = rows[r];
    double acc = out[c];
    for (int e = ptr[r]; e < ptr[r + 1]; ++e) {
      const double term = -(coef[e] * __ldg(p + src[e]));
      acc = residual ? acc - term : acc + term;
    }
    out[c] = acc;
  }
}

// <d, Ad>_V after the coupling terms, and alpha (fluid.py:4567-4574).
__global__ void __launch_bounds__(256) k_dot_alpha(LevelDev L, const double* __restrict__ d,
                                                   const double* __restrict__ Ad, double* partials, CgScalars* sc) {
  pdl_wait();
  EFSI_CELL_PROLOGUE(L)
  double a = 0.0;
  if (active && (__ldg(L.mask + c) & M_FLUID)) a = __ldg(d + c) * __ldg(Ad + c) * vol64(L, i, j, k);
  double v[1] = {a}, t[1];
  if (grid_sum<1>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) cg_alpha_step(sc, t[0]);
  }
}

// The residual's V-weighted mean (mean) or <r, r>_V, after the couplings.
__global__ void __launch_bounds__(256) k_residual_reduce(LevelDev L, const double* __restrict__ r, int mean,
                                                         double* partials, CgScalars* sc) {
  pdl_wait();
  EFSI_CELL_PROLOGUE(L)
  double a = 0.0;
  if (active && (__ldg(L.mask + c) & M_FLUID)) {
    const double rv = __ldg(r + c), V = vol64(L, i, j, k);
    a = mean ? rv * V : rv * rv * V;
  }
  double v[1] = {a}, t[1];
  if (grid_sum<1>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) {
      if (mean)
        sc->mean_r = sc->free_vol > 0.0 ? 1.0 * t[0] / sc->free_vol : 0.0;
      else
        sc->rr = t[0];
    }
  }
}

__global__ void k_set_defer(CgScalars* sc, int v) {
  if (threadIdx.x == 0) sc->defer_alpha = v;
}

// Learned preconditioner (codes 4 and 5): a two-level preconditioner whose
// coarse correction is the network.  With r' = r - A z_pre after the
// pre-smoothing sweeps, k_learned_sumsq reduces sum_fluid r'^2 V into
// sc->dot; k_learned_pack forms the network input (r' over its
// volume-weighted RMS, fluid mask, log2 cell widths over the finest width);
// k_learned_unpack writes n = RMS * output channel 0 on the fluid cells and
// reduces <r', n>_V; k_learned_combine adds s n to z_pre with the energy-
// minimising scale s = <r', n>_V / <n, A n>_V (sc->dot holds the denominator).
// az == nullptr means A z_pre = 0 (the network input of r itself).
__global__ void __launch_bounds__(256) k_learned_sumsq(LevelDev L, const double* __restrict__ r,
                                                       const double* __restrict__ az, double* partials, CgScalars* sc) {
  pdl_wait();
  EFSI_CELL_PROLOGUE(L)
  double a = 0.0;
  if (active && (__ldg(L.mask + c) & M_FLUID)) {
    const double rv = __ldg(r + c) - (az != nullptr ? __ldg(az + c) : 0.0);
    a = rv * rv * vol64(L, i, j, k);
  }
  double v[1] = {a}, t[1];
  if (grid_sum<1>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) sc->dot = t[0];
  }
}

__device__ __forceinline__ double learned_rms(const CgScalars* sc) {
  const double ms = sc->free_vol > 0.0 ? sc->dot / sc->free_vol : 0.0;
  return ms > 0.0 ? sqrt(ms) : 1.0;
}

__global__ void __launch_bounds__(256) k_learned_pack(LevelDev L, const double* __restrict__ r,
                                                      const double* __restrict__ az, __nv_bfloat16* __restrict__ in,
                                                      float wx0, float wy0, float wz0, const CgScalars* sc) {
  pdl_wait();
  EFSI_CELL_PROLOGUE(L)
  if (!active) return;
  const bool fluid = (__ldg(L.mask + c) & M_FLUID) != 0;
  const float inv = (float)(1.0 / learned_rms(sc));
  const double rv = fluid ? __ldg(r + c) - (az != nullptr ? __ldg(az + c) : 0.0) : 0.0;
  float ch[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) ch[q] = 0.0f;
  ch[0] = (float)rv * inv;
  ch[1] = fluid ? 1.0f : 0.0f;
  ch[2] = log2f(__ldg(L.wx + i) / wx0);
  ch[3] = log2f(__ldg(L.wy + j) / wy0);
  ch[4] = log2f(__ldg(L.wz + k) / wz0);
  __align__(16) __nv_bfloat16 hb[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) hb[q] = __float2bfloat16_rn(ch[q]);
  uint4* dst = reinterpret_cast<uint4*>(in + c * 16);
  dst[0] = reinterpret_cast<const uint4*>(hb)[0];
  dst[1] = reinterpret_cast<const uint4*>(hb)[1];
}

__global__ void __launch_bounds__(256) k_learned_unpack(LevelDev L, const float* __restrict__ out,
                                                        const double* __restrict__ r, const double* __restrict__ az,
                                                        double* __restrict__ n_out, double* partials, CgScalars* sc) {
  pdl_wait();
  EFSI_CELL_PROLOGUE(L)
  double pn = 0.0;
  if (active) {
    const unsigned m = __ldg(L.mask + c);
    double nv = 0.0;
    if (m & M_FLUID) {
      nv = (double)__ldg(out + c * 16) * learned_rms(sc);
      pn = (__ldg(r + c) - __ldg(az + c)) * nv * vol64(L, i, j, k);
    }
    n_out[c] = nv;
  }
  double v[1] = {pn}, t[1];
  if (grid_sum<1>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) sc->learned_num = t[0];
  }
}

__global__ void __launch_bounds__(256) k_learned_combine(LevelDev L, const double* __restrict__ zpre,
                                                         double* __restrict__ n_io, const CgScalars* sc) {
  pdl_wait();
  EFSI_CELL_PROLOGUE(L)
  if (!active) return;
  const double den = sc->dot, num = sc->learned_num;
  const double s = (den > 0.0 && isfinite(den) && isfinite(num)) ? num / den : 0.0;
  n_io[c] = __ldg(zpre + c) + s * n_io[c];
}

// Unreached-component anchoring of outlet solves (fluid.py:4905-4981):
// per component c, the volume-weighted sum and volume of a field over its
// cells (shared-memory sums per block, then one global atomic per block and
// component, as the reference's atomic sums), then field -= sum / volume on
// the component's cells.
constexpr int kMaxUnreachedComponents = 256;

__global__ void k_comp_zero(double* acc) {
  pdl_wait();
  for (int q = threadIdx.x; q < 2 * kMaxUnreachedComponents; q += blockDim.x) acc[q] = 0.0;
}

__global__ void __launch_bounds__(256) k_comp_accumulate(LevelDev L, const double* __restrict__ f,
                                                         const int32_t* __restrict__ comp, int ncomp, double* acc) {
  pdl_wait();
  __shared__ double s_sum[kMaxUnreachedComponents], s_vol[kMaxUnreachedComponents];
  __shared__ int s_any;
  const int tid = flat_tid(), nthr = blockDim.x * blockDim.y * blockDim.z;
  for (int q = tid; q < ncomp; q += nthr) {
    s_sum[q] = 0.0;
    s_vol[q] = 0.0;
  }
  if (tid == 0) s_any = 0;
  __syncthreads();
  EFSI_CELL_PROLOGUE(L)
  if (active) {
    const int cc = __ldg(comp + c);
    if (cc >= 0 && cc < ncomp) {
      const double vol = vol64(L, i, j, k);
      atomicAdd(&s_sum[cc], __ldg(f + c) * vol);
      atomicAdd(&s_vol[cc], vol);
      s_any = 1;
    }
  }
  __syncthreads();
  if (!s_any) return;
  for (int q = tid; q < ncomp; q += nthr)
    if (s_vol[q] != 0.0) {
      atomicAdd(acc + q, s_sum[q]);
      atomicAdd(acc + kMaxUnreachedComponents + q, s_vol[q]);
    }
}

__global__ void __launch_bounds__(256) k_comp_subtract(LevelDev L, double* __restrict__ f,
                                                       const int32_t* __restrict__ comp, const double* acc) {
  pdl_wait();
  EFSI_CELL_PROLOGUE(L)
  if (!active) return;
  const int cc = __ldg(comp + c);
  if (cc < 0) return;
  const double vol = acc[kMaxUnreachedComponents + cc];
  if (vol > 0.0) f[c] -= acc[cc] / vol;
}

// Device-side PCG loop (efsi_pcg_params::device_loop).  k_dl_init runs
// after the initial residual and preconditioner: b_norm, the initial
// relative residual, beta = 0 (the first direction is z), and whether the
// loop body runs at all; k_dl_check ends every 16-iteration body: the
// relative residual of the last update, and whether to go on (not
// converged, no breakdown or fault, and another 16 iterations within
// max_iters).
__global__ void k_dl_init(CgScalars* sc, double tol, cudaGraphConditionalHandle h) {
  pdl_wait();
  if (threadIdx.x != 0) return;
  const double bn = sqrt(fmax(sc->bnorm2, 0.0));
  sc->dl_bnorm = bn;
  sc->dl_iter = 0;
  sc->dl_converged = 0;
  unsigned go = 0;
  if (bn <= 1.0e-30) {
    sc->dl_converged = 1;
    sc->dl_rel0 = sc->dl_rel = 0.0;
  } else {
    const double rel = sqrt(fmax(sc->rr, 0.0)) / bn;
    sc->dl_rel0 = sc->dl_rel = rel;
    if (rel <= tol)
      sc->dl_converged = 1;
    else if (!(isfinite(sc->rz) && sc->rz > 0.0))
      sc->code = 2;
    else
      go = 1;
  }
  sc->beta = 0.0;
  cudaGraphSetConditional(h, go);
}

__global__ void k_dl_zero_if_tiny(LevelDev L, double* __restrict__ pressure, const CgScalars* sc) {
  pdl_wait();
  EFSI_CELL_PROLOGUE(L)
  if (active && !(sqrt(fmax(sc->bnorm2, 0.0)) > 1.0e-30)) pressure[c] = 0.0;
}

__global__ void k_dl_check(CgScalars* sc, double tol, int max_iters, cudaGraphConditionalHandle h) {
  pdl_wait();
  if (threadIdx.x != 0) return;
  const int it = sc->dl_iter + 16;
  sc->dl_iter = it;
  const double rel = sqrt(fmax(sc->rr, 0.0)) / sc->dl_bnorm;
  sc->dl_rel = rel;
  unsigned go = 1;
  if (rel <= tol) {
    sc->dl_converged = 1;
    go = 0;
  } else if (sc->code != 0 || sc->fault != 0 || !isfinite(rel) || it + 16 > max_iters) {
    go = 0;
  }
  cudaGraphSetConditional(h, go);
}

// Reciprocal of the level-0 row denominator (fluid.py:4080-4221: the open
// faces' coefficients in the order x-, x+, y-, y+, z-, z+, the outlet term,
// the interface diagonal), 0 where the denominator is not positive or the
// cell is solid.  The plane-marching sweeps multiply by it instead of
// forming the denominator and dividing.
__global__ void __launch_bounds__(256) k_rden(LevelDev L, int outlet, double* __restrict__ rden) {
  EFSI_CELL_PROLOGUE(L)
  if (!active) return;
  const unsigned m = __ldg(L.mask + c);
  double rd = 0.0;
  if (!(m & M_SOLID)) {
    double ns, den;
    stencil_sel<true>(L, row_coef(L, j, k), __ldg(L.cxm + i), __ldg(L.cxp + i), i, j, k, c, m, outlet, 0.0, 0.0,
                      0.0, 0.0, 0.0, 0.0, ns, den);
    den += iface_at<double>(L, c);
    if (den > 0.0) rd = 1.0 / den;
  }
  rden[c] = rd;
}

// fluid.py:4677-4693 with multiplier -1 on the level-0 rhs, plus the free
// volume (computed in the same pass as the reference does).
__global__ void __launch_bounds__(256) k_rhs_mean(LevelDev L, const double* __restrict__ rhs, double multiplier,
                                                  double* partials, CgScalars* sc) {
  EFSI_CELL_PROLOGUE(L)
  double a = 0.0, b = 0.0;
  if (active) {
    const unsigned m = __ldg(L.mask + c);
    if (m & M_FLUID) {
      double V = vol64(L, i, j, k);
      a = __ldg(rhs + c) * V;
      b = V;
    }
  }
  double v[2] = {a, b}, t[2];
  if (grid_sum<2>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) {
      sc->free_vol = t[1];
      sc->mean_b = t[1] > 0.0 ? multiplier * t[0] / t[1] : 0.0;
    }
  }
}

// b = -rhs - mean (fluid.py:4472-4482), <b, b>_V.
__global__ void __launch_bounds__(256) k_build_b(LevelDev L, const double* __restrict__ rhs, int use_mean,
                                                 double* __restrict__ b, double* partials, CgScalars* sc) {
  EFSI_CELL_PROLOGUE(L)
  const double mean = use_mean ? sc->mean_b : 0.0;
  double pb = 0.0;
  if (active) {
    const unsigned m = __ldg(L.mask + c);
    double bv = (m & M_SOLID) ? 0.0 : -__ldg(rhs + c) - mean;
    b[c] = bv;
    if (m & M_FLUID) pb = bv * bv * vol64(L, i, j, k);
  }
  double v[1] = {pb}, t[1];
  if (grid_sum<1>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) sc->bnorm2 = t[0];
  }
}

// r = b - A x (fluid.py:6613-6614 / 6744-6754), optionally with r V sums
// (mean) or r r V (no mean projection).
__global__ void __launch_bounds__(256) k_true_residual(LevelDev L, const double* __restrict__ x,
                                                       const double* __restrict__ b, double* __restrict__ r,
                                                       int outlet, int want_mean, double* partials, CgScalars* sc) {
  EFSI_CELL_PROLOGUE(L)
  double pa = 0.0;
  if (active) {
    const unsigned m = __ldg(L.mask + c);
    double rv;
    if (m & M_SOLID) {
      rv = 0.0;
    } else {
      double ns, den;
      auto val = [&](int64_t cell, int, int, int) { return __ldg(x + cell); };
      stencil(L, val, i, j, k, c, m, outlet, ns, den);
      double ax = (den + iface_at<double>(L, c)) * __ldg(x + c) - ns;
      rv = 1.0 * __ldg(b + c) + -1.0 * ax;
    }
    r[c] = rv;
    if (m & M_FLUID) pa = want_mean ? rv * vol64(L, i, j, k) : rv * rv * vol64(L, i, j, k);
  }
  double v[1] = {pa}, t[1];
  if (grid_sum<1>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) {
      if (want_mean)
        sc->mean_r = sc->free_vol > 0.0 ? 1.0 * t[0] / sc->free_vol : 0.0;
      else
        sc->rr = t[0];
    }
  }
}

// r -= mean_r (fluid), then r r V.
__global__ void __launch_bounds__(256) k_sub_mean_r(LevelDev L, double* __restrict__ r, double* partials,
                                                    CgScalars* sc) {
  EFSI_CELL_PROLOGUE(L)
  const double mr = sc->mean_r;
  double prr = 0.0;
  if (active) {
    const unsigned m = __ldg(L.mask + c);
    if (m & M_FLUID) {
      double rn = r[c] - mr;
      r[c] = rn;
      prr = rn * rn * vol64(L, i, j, k);
    } else {
      r[c] = 0.0;
    }
  }
  double v[1] = {prr}, t[1];
  if (grid_sum<1>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) sc->rr = t[0];
  }
}

__global__ void __launch_bounds__(256) k_fv_apply(LevelDev L, const double* __restrict__ p, double* __restrict__ out,
                                                  int outlet) {
  EFSI_CELL_PROLOGUE(L)
  if (!active) return;
  const unsigned m = __ldg(L.mask + c);
  if (m & M_SOLID) {
    out[c] = 0.0;
    return;
  }
  double ns, den;
  auto val = [&](int64_t cell, int, int, int) { return __ldg(p + cell); };
  stencil(L, val, i, j, k, c, m, outlet, ns, den);
  out[c] = (den + iface_at<double>(L, c)) * __ldg(p + c) - ns;
}

__global__ void __launch_bounds__(256) k_fv_diag(LevelDev L, double* __restrict__ diag, int outlet) {
  EFSI_CELL_PROLOGUE(L)
  if (!active) return;
  const unsigned m = __ldg(L.mask + c);
  if (m & M_SOLID) {
    diag[c] = 0.0;
    return;
  }
  double ns, den;
  auto zero = [](int64_t, int, int, int) { return 0.0; };
  stencil(L, zero, i, j, k, c, m, outlet, ns, den);
  diag[c] = den + iface_at<double>(L, c);
}

__global__ void __launch_bounds__(256) k_weighted_dot(LevelDev L, const double* __restrict__ a,
                                                      const double* __restrict__ b, double* partials, CgScalars* sc) {
  EFSI_CELL_PROLOGUE(L)
  double pa = 0.0;
  if (active) {
    const unsigned m = __ldg(L.mask + c);
    if (m & M_FLUID) pa = __ldg(a + c) * __ldg(b + c) * vol64(L, i, j, k);
  }
  double v[1] = {pa}, t[1];
  if (grid_sum<1>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) sc->dot = t[0];
  }
}

__global__ void k_set_zproj(CgScalars* sc, int v) {
  pdl_wait();
  if (threadIdx.x == 0) {
    sc->zproj = v;
    if (!v) sc->mean_z = 0.0;
  }
}

__global__ void k_reset_scalars(CgScalars* sc) {
  if (threadIdx.x == 0) {
    CgScalars z;
    memset(&z, 0, sizeof(z));
    *sc = z;
  }
}

// Clears the breakdown code after the initial direction: a V-cycle whose last
// sweep finished the dots ran the beta test against rz = 0 (no previous
// direction yet) and flagged a breakdown that the first direction does not
// have (fluid.py:6662-6673 computes only rz there).
__global__ void k_clear_code(CgScalars* sc) {
  pdl_wait();
  if (threadIdx.x == 0) {
    sc->code = 0;
    sc->code_dAd = 0.0;
  }
}

}  // namespace efsi

namespace efsi {

namespace {
thread_local std::string g_err;
std::atomic<unsigned long long> g_launches{0};
}  // namespace

void set_error(const std::string& msg) { g_err = msg; }
thread_local unsigned long long g_capture_count = 0;
extern thread_local bool g_capturing;
void count_launch() {
  if (g_capturing)
    ++g_capture_count;  // a captured launch runs once per graph replay
  else
    g_launches.fetch_add(1, std::memory_order_relaxed);
}
void count_graph_launch(unsigned long long nodes) { g_launches.fetch_add(nodes, std::memory_order_relaxed); }
unsigned long long take_capture_count() {
  unsigned long long v = g_capture_count;
  g_capture_count = 0;
  return v;
}
bool pdl_enabled() {
  static const bool on = std::getenv("EFSI_NO_PDL") == nullptr;
  return on;
}

namespace {
struct FamilyTimer {
  bool on = false;
  std::vector<cudaEvent_t> start, stop;
  std::vector<double> bytes;
  size_t used = 0;
};
FamilyTimer g_timers[KF_COUNT];
std::mutex g_timer_mutex;
}  // namespace

thread_local bool g_capturing = false;  // defined here, declared above
void set_capturing(bool on) { g_capturing = on; }
bool timing_enabled(int family) { return !g_capturing && family >= 0 && family < KF_COUNT && g_timers[family].on; }

void timing_begin(int family, cudaStream_t s) {
  std::lock_guard<std::mutex> lock(g_timer_mutex);
  FamilyTimer& T = g_timers[family];
  if (T.used == T.start.size()) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    T.start.push_back(a);
    T.stop.push_back(b);
    T.bytes.push_back(0.0);
  }
  cudaEventRecord(T.start[T.used], s);
}

void timing_end(int family, cudaStream_t s, double bytes) {
  std::lock_guard<std::mutex> lock(g_timer_mutex);
  FamilyTimer& T = g_timers[family];
  cudaEventRecord(T.stop[T.used], s);
  T.bytes[T.used] = bytes;
  T.used += 1;
}

LevelDev level_dev(const efsi_fv_plan* P, int l) {
  const LevelBuf& B = P->lv[l];
  LevelDev L;
  L.nx = B.nx;
  L.ny = B.ny;
  L.nz = B.nz;
  L.cxm = B.coef;
  L.cxp = B.coef + B.nx;
  L.cym = B.coef + 2 * B.nx;
  L.cyp = B.coef + 2 * B.nx + B.ny;
  L.czm = B.coef + 2 * B.nx + 2 * B.ny;
  L.czp = B.coef + 2 * B.nx + 2 * B.ny + B.nz;
  L.oz = B.oz;
  L.wx = B.wx;
  L.wy = B.wy;
  L.wz = B.wz;
  L.cdx_f = B.cdx;
  L.cdy_f = B.cdy;
  L.cdz_f = B.cdz;
  L.mask = B.mask;
  L.fw = P->has_vdir ? B.fw : nullptr;
  if (l == 0)
    L.iface = P->has_iface ? (const void*)P->iface0 : nullptr;
  else
    L.iface = P->has_iface ? (const void*)B.iface : nullptr;
  return L;
}

int level_zero_check(const efsi_fv_plan* P) {
  EFSI_ARG_CHECK(P != nullptr, "null plan");
  EFSI_ARG_CHECK(P->lv.size() > 0 && P->lv[0].mask != nullptr, "plan has no masks; call efsi_fv_set_masks first");
  return EFSI_OK;
}

}  // namespace efsi

namespace efsi {
// Load every kernel of the solver into the context up front: with lazy module
// loading a kernel's first launch would otherwise happen inside a stream
// capture (16-iteration PCG blocks are captured into CUDA graphs).
static void preload_kernels() {
  cudaFuncAttributes a;
  const void* fns[] = {
      (const void*)k_sweep<double, true, true>,   (const void*)k_sweep<double, true, false>,
      (const void*)k_sweep<double, false, false>, (const void*)k_sweep<float, false, true>,
      (const void*)k_sweep<float, false, false>,  (const void*)k_restrict<double, true, true>,
      (const void*)k_restrict<float, false, true>, (const void*)k_restrict<double, false, true>,
      (const void*)k_spmv_dir<true>,              (const void*)k_spmv_dir<false>,
      (const void*)k_cg_update<true>,             (const void*)k_cg_update<false>,
      (const void*)k_cg_dots<true, false>,        (const void*)k_cg_dots<false, false>,
      (const void*)k_cg_dots<false, true>,        (const void*)k_sub_mean_xr,
      (const void*)k_jacobi_precond,              (const void*)k_set_zproj,
      (const void*)k_true_residual,               (const void*)k_sub_mean_r,
      (const void*)k_rhs_mean,                    (const void*)k_build_b,
      (const void*)k_fv_diag,                     (const void*)k_reset_scalars,
      (const void*)k_clear_code,
      (const void*)kt_sweep<double, true, true>,  (const void*)kt_sweep<double, true, false>,
      (const void*)kt_sweep<float, false, true>,  (const void*)kt_sweep<float, false, false>,
      (const void*)kt_spmv_dir<true>,             (const void*)kt_spmv_dir<false>,
      (const void*)kt_cg_update<true>,            (const void*)kt_cg_update<false>,
      (const void*)kt_cg_update<true, 1>,         (const void*)kt_cg_update<true, 2>,
      (const void*)kt_cg_update_r_zero<double>,   (const void*)kt_cg_update_r_zero<float>,
      (const void*)kt_cg_dots<true, false>,       (const void*)kt_cg_dots<false, false>,
      (const void*)kt_sub_mean_xr,                (const void*)k_mg_tail,
#define EFSI_MARCH_FNS(A)                                                                              \
      (const void*)km_sweep<double, true, false, A, false>, (const void*)km_sweep<double, true, true, A, false>, \
      (const void*)km_sweep<double, true, false, A, true>, (const void*)km_sweep<double, true, true, A, true>,   \
      (const void*)km_sweep<double, false, false, A, false>, (const void*)km_sweep<float, false, false, A, false>, \
      (const void*)km_sweep<float, false, true, A, false>, (const void*)km_sweep0<double, true, A>,        \
      (const void*)km_sweep0<double, false, A>, (const void*)km_sweep0<float, false, A>,                   \
      (const void*)km_restrict<double, true, A>, (const void*)km_restrict<double, false, A>,               \
      (const void*)km_restrict<float, false, A>, (const void*)km_spmv_dir<true, A>,                        \
      (const void*)km_spmv_dir<false, A>, (const void*)km_sweep<double, true, false, A, true, true>,       \
      (const void*)km_sweep<double, true, true, A, true, true>
      EFSI_MARCH_FNS(false), EFSI_MARCH_FNS(true),
#undef EFSI_MARCH_FNS
#define EFSI_MIXED_FNS(A)                                                                                       \
  (const void*)km_sweep32<false, A, false>, (const void*)km_sweep32<false, A, true>,                           \
      (const void*)km_sweep32<true, A, false>, (const void*)km_sweep32<true, A, true>,                         \
      (const void*)km_sweep0<float, true, A>, (const void*)km_restrict<float, true, A>
      EFSI_MIXED_FNS(false), EFSI_MIXED_FNS(true),
#undef EFSI_MIXED_FNS
  };
  for (const void* f : fns) cudaFuncGetAttributes(&a, f);
  // the plane-marching kernels take up to ~70 KB of dynamic shared memory
#define EFSI_MARCH_SMEM(A)                                                                                        \
  {(const void*)km_sweep<double, true, false, A, false>, march_smem<double, 1, double, true>()},                  \
      {(const void*)km_sweep<double, true, true, A, false>, march_smem<double, 1, double, true>()},               \
      {(const void*)km_sweep<double, true, false, A, true>, march_smem<double, 1, double, true>()},               \
      {(const void*)km_sweep<double, true, true, A, true>, march_smem<double, 1, double, true>()},                \
      {(const void*)km_sweep<double, false, false, A, false>, march_smem<double, 1, double, true>()},             \
      {(const void*)km_sweep<float, false, false, A, false>, march_smem<float, 1, float, true>()},                \
      {(const void*)km_sweep<float, false, true, A, false>, march_smem<float, 1, float, true>()},                 \
      {(const void*)km_restrict<double, true, A>, march_smem<double, 1, double, true>()},                         \
      {(const void*)km_restrict<double, false, A>, march_smem<double, 1, double, true>()},                        \
      {(const void*)km_restrict<float, false, A>, march_smem<float, 1, float, true>()},                           \
      {(const void*)km_spmv_dir<true, A>, march_smem<double, 1, double, false>()},                                \
      {(const void*)km_spmv_dir<false, A>, march_smem<double, 2, double, false>()},                               \
      {(const void*)km_sweep<double, true, false, A, true, true>, march_smem<double, 1, double, true>()},         \
      {(const void*)km_sweep<double, true, true, A, true, true>, march_smem<double, 1, double, true>()}
#define EFSI_MIXED_SMEM(A)                                                                                        \
  {(const void*)km_sweep32<false, A, false>, march_smem<float, 1, double, true>()},                              \
      {(const void*)km_sweep32<false, A, true>, march_smem<float, 1, double, true>()},                           \
      {(const void*)km_sweep32<true, A, false>, march_smem<float, 1, double, true>()},                           \
      {(const void*)km_sweep32<true, A, true>, march_smem<float, 1, double, true>()},                            \
      {(const void*)km_restrict<float, true, A>, march_smem<float, 1, double, true>()}
  const std::pair<const void*, int> dyn[] = {EFSI_MARCH_SMEM(false), EFSI_MARCH_SMEM(true), EFSI_MIXED_SMEM(false),
                                             EFSI_MIXED_SMEM(true)};
#undef EFSI_MARCH_SMEM
#undef EFSI_MIXED_SMEM
  for (const auto& d : dyn) cudaFuncSetAttribute(d.first, cudaFuncAttributeMaxDynamicSharedMemorySize, d.second);
  cudaGetLastError();
}
}  // namespace efsi


namespace efsi {
// Picks the first coarse level from which every level fits the tail kernel's
// shared memory (13 bytes per cell) and has at most EFSI_TAIL_MAX_CELLS cells
// (default 4096; 0 disables the tail).
static void configure_tail(efsi_fv_plan* P) {
  P->tail_level = P->n_levels;
  int max_cells = 4096;
  if (const char* env = std::getenv("EFSI_TAIL_MAX_CELLS")) max_cells = std::atoi(env);
  if (max_cells <= 0 || P->n_levels < 2 || P->n_levels > kTailMaxLevels) return;
  int dev = 0;
  cudaGetDevice(&dev);
  int smem_optin = 0;
  cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  for (int lt = 1; lt < P->n_levels; ++lt) {
    if (P->lv[lt].n > max_cells) continue;
    // layout: row tables (7 f64 per cell), iterates + rhs (3 f32 per cell),
    // neighbour tables (6 int per cell), masks (1 byte per cell, 16-aligned)
    size_t cells = 0, bytes_mask = 0;
    for (int l = lt; l < P->n_levels; ++l) {
      cells += (size_t)P->lv[l].n;
      bytes_mask += ((size_t)P->lv[l].n + 15) / 16 * 16;
    }
    const size_t total = cells * (7 * sizeof(double) + 3 * sizeof(float) + 6 * sizeof(int)) + bytes_mask;
    if ((int64_t)total > (int64_t)smem_optin) continue;
    size_t co = 0, fo = cells * 7 * sizeof(double), no = fo + cells * 3 * sizeof(float), mo = no + cells * 6 * sizeof(int);
    for (int l = lt; l < P->n_levels; ++l) {
      const size_t n = (size_t)P->lv[l].n;
      P->tail_coff[l] = (int)co;
      co += n * 7 * sizeof(double);
      P->tail_foff[l] = (int)(fo / sizeof(float));
      fo += n * 3 * sizeof(float);
      P->tail_noff[l] = (int)no;
      no += n * 6 * sizeof(int);
      P->tail_moff[l] = (int)mo;
      mo += (n + 15) / 16 * 16;
    }
    if (cudaFuncSetAttribute(k_mg_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    P->tail_level = lt;
    P->tail_smem_bytes = total;
    return;
  }
}

// The cooperative coarse-level kernel runs levels 1 .. lt-1 and the tail when
// the tail exists and starts at level 2 or deeper, cooperative launches are
// supported, and EFSI_NO_COARSE_KERNEL is unset: as many blocks as fit on the
// GPU at once (at most two per SM), each with the tail's shared memory.
// Sets up the cluster form of the coarse-level kernel: levels 2 .. lt-1 and
// the tail on one cluster of `ctas` CTAs (one per SM).  Returns false with a
// note when the device cannot run it.
static bool configure_coarse_cluster(efsi_fv_plan* P, int ctas) {
  if (P->tail_level < 3 || P->tail_level >= P->n_levels) {
    P->coarse_note = "no level between 1 and the tail (tail level " + std::to_string(P->tail_level) + " of " +
                     std::to_string(P->n_levels) + " levels)";
    return false;
  }
  if (ctas < 2 || ctas > 16) {
    P->coarse_note = "EFSI_COARSE_CLUSTER must be 2 .. 16";
    return false;
  }
  static std::mutex attr_mutex;
  static int attr_bytes = 0;
  static bool nonportable = false;
  cudaError_t e = cudaSuccess;
  {
    std::lock_guard<std::mutex> lock(attr_mutex);
    if ((int)P->tail_smem_bytes > attr_bytes) {
      e = cudaFuncSetAttribute(k_mg_coarse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P->tail_smem_bytes);
      if (e == cudaSuccess) attr_bytes = (int)P->tail_smem_bytes;
    }
    if (e == cudaSuccess && ctas > 8 && !nonportable) {
      e = cudaFuncSetAttribute(k_mg_coarse, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
      if (e == cudaSuccess) nonportable = true;
    }
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    P->coarse_note = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return false;
  }
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)ctas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)ctas);
  cfg.blockDim = dim3(kTailThreads);
  cfg.dynamicSmemBytes = P->tail_smem_bytes;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  e = cudaOccupancyMaxActiveClusters(&clusters, k_mg_coarse, &cfg);
  if (e != cudaSuccess || clusters < 1) {
    cudaGetLastError();
    P->coarse_note = std::string("cluster occupancy: ") + cudaGetErrorString(e) + ", clusters " +
                     std::to_string(clusters);
    return false;
  }
  P->coarse_blocks = ctas;
  P->coarse_first = 2;
  P->coarse_cluster = 1;
  P->coarse_note = "";
  return true;
}

static void configure_coarse(efsi_fv_plan* P) {
  P->coarse_blocks = 0;
  P->coarse_first = 1;
  P->coarse_cluster = 0;
  if (std::getenv("EFSI_NO_COARSE_KERNEL") != nullptr) {
    P->coarse_note = "the coarse-level kernel is off (EFSI_NO_COARSE_KERNEL)";
    return;
  }
  if (const char* cl = std::getenv("EFSI_COARSE_CLUSTER")) {
    if (std::atoi(cl) > 0) {
      configure_coarse_cluster(P, std::atoi(cl));
      return;
    }
  }
  // opt-in (EFSI_COARSE_KERNEL=1): on a B200 the per-level launches measured
  // faster (c2: 94 us against 143 us per V-cycle for levels 1-6)
  const char* on = std::getenv("EFSI_COARSE_KERNEL");
  if (on == nullptr || std::atoi(on) == 0) {
    P->coarse_note = "the cooperative coarse-level kernel is off (EFSI_COARSE_KERNEL=1 selects it)";
    return;
  }
  if (P->tail_level < 2 || P->tail_level >= P->n_levels) {
    P->coarse_note = "no tail below level 1 (tail level " + std::to_string(P->tail_level) + " of " +
                     std::to_string(P->n_levels) + " levels)";
    return;
  }
  int dev = 0, coop = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (!coop || sms <= 0) {
    P->coarse_note = "cooperative launches are not supported on this device";
    return;
  }
  // the largest tail of any plan so far (the kernel's own static shared
  // memory comes on top, so the opt-in maximum itself would be refused)
  static std::mutex attr_mutex;
  static int attr_bytes = 0;
  cudaError_t e = cudaSuccess;
  {
    std::lock_guard<std::mutex> lock(attr_mutex);
    if ((int)P->tail_smem_bytes > attr_bytes) {
      e = cudaFuncSetAttribute(k_mg_coarse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P->tail_smem_bytes);
      if (e == cudaSuccess) attr_bytes = (int)P->tail_smem_bytes;
    }
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    P->coarse_note = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return;
  }
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mg_coarse, kTailThreads, P->tail_smem_bytes);
  if (e != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    P->coarse_note = std::string("occupancy: ") + cudaGetErrorString(e) + ", blocks per SM " + std::to_string(per_sm);
    return;
  }
  if (cudaMalloc(&P->coarse_bar, 2 * sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(P->coarse_bar, 0, 2 * sizeof(unsigned)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(P->coarse_bar);
    P->coarse_bar = nullptr;
    P->coarse_note = "cannot allocate the grid barrier";
    return;
  }
  int want = 2;
  if (const char* env = std::getenv("EFSI_COARSE_BLOCKS_PER_SM")) want = std::max(1, std::atoi(env));
  P->coarse_blocks = std::min(per_sm, want) * sms;
  P->coarse_note = "";
}
}  // namespace efsi

using namespace efsi;

extern "C" {

const char* efsi_last_error(void) { return g_err.c_str(); }
const char* efsi_version(void) { return "easyfsi_b200 0.1 (sm_100a)"; }
uint64_t efsi_kernel_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int efsi_kernel_timing_enable(int32_t family, int32_t enable) {
  EFSI_ARG_CHECK(family >= 0 && family < KF_COUNT, "unknown kernel family");
  std::lock_guard<std::mutex> lock(g_timer_mutex);
  g_timers[family].on = enable != 0;
  g_timers[family].used = 0;
  return EFSI_OK;
}

int efsi_kernel_timing_read(int32_t family, int64_t* launches, double* total_ms, double* total_bytes) {
  EFSI_ARG_CHECK(family >= 0 && family < KF_COUNT && launches && total_ms && total_bytes, "invalid timing query");
  std::lock_guard<std::mutex> lock(g_timer_mutex);
  FamilyTimer& T = g_timers[family];
  double ms = 0.0, by = 0.0;
  for (size_t q = 0; q < T.used; ++q) {
    EFSI_CUDA_CHECK(cudaEventSynchronize(T.stop[q]));
    float e = 0.0f;
    EFSI_CUDA_CHECK(cudaEventElapsedTime(&e, T.start[q], T.stop[q]));
    ms += e;
    by += T.bytes[q];
  }
  *launches = (int64_t)T.used;
  *total_ms = ms;
  *total_bytes = by;
  return EFSI_OK;
}

int efsi_fv_plan_create(const efsi_level_desc* levels, int32_t n_levels, int32_t uniform_grid, efsi_fv_plan** out) {
  EFSI_ARG_CHECK(levels != nullptr && out != nullptr && n_levels >= 1, "invalid plan arguments");
  efsi_fv_plan* P = new efsi_fv_plan();
  P->n_levels = n_levels;
  P->uniform = uniform_grid;
  P->lv.resize(n_levels);
  size_t max_blocks = 1;
  auto fail = [&](int code) {
    efsi_fv_plan_destroy(P);
    return code;
  };
  for (int l = 0; l < n_levels; ++l) {
    const efsi_level_desc& D = levels[l];
    LevelBuf& B = P->lv[l];
    if (D.nx < 1 || D.ny < 1 || D.nz < 1 || !D.wx || !D.wy || !D.wz || !D.cdx || !D.cdy || !D.cdz) {
      set_error("invalid level descriptor");
      return fail(EFSI_ERR_ARG);
    }
    B.nx = D.nx;
    B.ny = D.ny;
    B.nz = D.nz;
    B.n = (int64_t)D.nx * D.ny * D.nz;
    B.wx = D.wx;
    B.wy = D.wy;
    B.wz = D.wz;
    B.cdx = D.cdx;
    B.cdy = D.cdy;
    B.cdz = D.cdz;
    B.shape = shape3(B.nx, B.ny, B.nz);
    max_blocks = std::max<size_t>(max_blocks, B.shape.nblocks());
    {
      const dim3 g0 = sweep0_grid(B.nx, B.ny, B.nz);
      max_blocks = std::max<size_t>(max_blocks, (size_t)g0.x * g0.y * g0.z);
    }
    {
      int dev = 0, nsm = 148;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      int per_sm = 4;
      if (const char* env = std::getenv("EFSI_TILED_BLOCKS_PER_SM")) per_sm = std::max(1, std::atoi(env));
      const int nt = tiles_of(B.nx, B.ny, B.nz);
      B.tiled = B.nz >= 16 && B.ny >= 8 && std::getenv("EFSI_NO_TILED") == nullptr;
      B.tgrid = (unsigned)std::max(1, std::min(nt, nsm * per_sm));
      const MarchCfg mc = march_cfg(B.nx, B.ny, B.nz, nsm * 3);
      // levels below EFSI_MARCH_MIN_CELLS (default 0) keep the per-cell kernels
      int64_t march_min = 0;
      if (const char* env = std::getenv("EFSI_MARCH_MIN_CELLS")) march_min = std::atoll(env);
      B.march = B.nz >= 16 && B.ny >= 8 && B.n >= march_min && std::getenv("EFSI_NO_MARCH") == nullptr;
      B.march_ok = B.march;
      B.mchunk = mc.chunk;
      B.mgrid = mc.grid;
      const MarchCfg ms = march_cfg(B.nx, B.ny, B.nz, nsm * 2);
      B.spchunk = ms.chunk;
      B.spgrid = ms.grid;
    }
    size_t ncoef = 2 * (size_t)(B.nx + B.ny + B.nz);
    if (cudaMalloc(&B.coef, ncoef * sizeof(double)) != cudaSuccess || cudaMalloc(&B.mask, B.n) != cudaSuccess) {
      set_error("cudaMalloc failed for level tables");
      return fail(EFSI_ERR_CUDA);
    }
    EFSI_COUNTED k_axis_coef<<<(B.nx + 127) / 128, 128>>>(D.wx, D.cdx, B.nx, B.coef, B.coef + B.nx);
    EFSI_COUNTED k_axis_coef<<<(B.ny + 127) / 128, 128>>>(D.wy, D.cdy, B.ny, B.coef + 2 * B.nx, B.coef + 2 * B.nx + B.ny);
    EFSI_COUNTED k_axis_coef<<<(B.nz + 127) / 128, 128>>>(D.wz, D.cdz, B.nz, B.coef + 2 * B.nx + 2 * B.ny,
                                             B.coef + 2 * B.nx + 2 * B.ny + B.nz);
    float wz0 = 0.0f;
    cudaMemcpy(&wz0, D.wz, sizeof(float), cudaMemcpyDeviceToHost);
    B.oz = 2.0 / ((double)wz0 * (double)wz0);
    size_t es = (l == 0) ? sizeof(double) : sizeof(float);
    if (cudaMalloc(&B.pa, B.n * es) != cudaSuccess || cudaMalloc(&B.pb, B.n * es) != cudaSuccess) {
      set_error("cudaMalloc failed for level iterates");
      return fail(EFSI_ERR_CUDA);
    }
    if (l == 0 && (cudaMalloc(&B.pa32, B.n * sizeof(float)) != cudaSuccess ||
                   cudaMalloc(&B.pb32, B.n * sizeof(float)) != cudaSuccess)) {
      set_error("cudaMalloc failed for the mixed-precision level-0 iterates");
      return fail(EFSI_ERR_CUDA);
    }
    if (l > 0) {
      if (cudaMalloc(&B.rhs, B.n * sizeof(float)) != cudaSuccess ||
          cudaMalloc(&B.obs, B.n * sizeof(int32_t)) != cudaSuccess) {
        set_error("cudaMalloc failed for coarse level");
        return fail(EFSI_ERR_CUDA);
      }
    }
  }
  const int64_t n0 = P->lv[0].n;
  double** vecs[] = {&P->r, &P->z, &P->d0, &P->d1, &P->Ad, &P->delta, &P->b, &P->diag};
  for (double** v : vecs) {
    if (cudaMalloc(v, n0 * sizeof(double)) != cudaSuccess) {
      set_error("cudaMalloc failed for CG vectors");
      return fail(EFSI_ERR_CUDA);
    }
  }
  P->partials_len = 4 * max_blocks;
  if (cudaMalloc(&P->partials, P->partials_len * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&P->sc, sizeof(CgScalars)) != cudaSuccess || cudaMalloc(&P->aux, 16 * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&P->host_sc, sizeof(CgScalars)) != cudaSuccess ||
      cudaMemset(P->sc, 0, sizeof(CgScalars)) != cudaSuccess) {
    set_error("cudaMalloc failed for reduction scratch");
    return fail(EFSI_ERR_CUDA);
  }
  preload_kernels();
  configure_tail(P);
  configure_coarse(P);
  if (cudaStreamCreateWithFlags(&P->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("cannot create the capture stream");
    return fail(EFSI_ERR_CUDA);
  }
  EFSI_COUNTED k_reset_scalars<<<1, 32>>>(P->sc);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    set_error(std::string("plan setup failed: ") + cudaGetErrorString(e));
    return fail(EFSI_ERR_CUDA);
  }
  *out = P;
  return EFSI_OK;
}

int efsi_fv_plan_destroy(efsi_fv_plan* P) {
  if (P == nullptr) return EFSI_OK;
  for (PcgGraph& g : P->graphs) cudaGraphExecDestroy(g.exec);
  P->graphs.clear();
  if (P->cap_stream) cudaStreamDestroy(P->cap_stream);
  if (P->body_stream) cudaStreamDestroy(P->body_stream);
  if (P->side_stream) cudaStreamDestroy(P->side_stream);
  if (P->ev_fork) cudaEventDestroy(P->ev_fork);
  if (P->ev_join) cudaEventDestroy(P->ev_join);
  for (LevelBuf& B : P->lv) {
    cudaFree(B.coef);
    cudaFree(B.mask);
    cudaFree(B.fw);
    cudaFree(B.obs);
    cudaFree(B.va);
    cudaFree(B.vw);
    cudaFree(B.iface);
    cudaFree(B.pa);
    cudaFree(B.pb);
    cudaFree(B.pa32);
    cudaFree(B.pb32);
    cudaFree(B.rhs);
  }
  double* vecs[] = {P->r, P->z, P->d0, P->d1, P->Ad, P->delta, P->b, P->diag, P->partials};
  for (double* v : vecs) cudaFree(v);
  cudaFree(P->sc);
  cudaFree(P->aux);
  cudaFree(P->bicg_work);
  cudaFree(P->unet_in);
  cudaFree(P->coarse_bar);
  cudaFree(P->ucomp);
  cudaFree(P->ucomp_acc);
  cudaFree(P->report_buf);
  cudaFree(P->rden[0]);
  cudaFree(P->rden[1]);
  cudaFree(P->cpl_rows);
  cudaFree(P->cpl_ptr);
  cudaFree(P->cpl_src);
  cudaFree(P->cpl_coef);
  cudaFree(P->cpl_n);
  if (P->host_sc) cudaFreeHost(P->host_sc);
  delete P;
  return EFSI_OK;
}

int efsi_fv_set_masks(efsi_fv_plan* P, const int32_t* obstacle, const int32_t* vdir_active, const float* vdir_weight,
                      const double* iface_diag, void* stream) {
  EFSI_ARG_CHECK(P != nullptr && obstacle != nullptr, "null plan or obstacle");
  EFSI_ARG_CHECK((vdir_active == nullptr) == (vdir_weight == nullptr), "vdir_active and vdir_weight go together");
  cudaStream_t s = as_stream(stream);
  P->rden_ok[0] = P->rden_ok[1] = false;
  P->has_vdir = vdir_active != nullptr;
  P->has_iface = iface_diag != nullptr;
  P->iface0 = iface_diag;
  P->obstacle0 = obstacle;
  for (int l = 0; l < P->n_levels; ++l) {
    LevelBuf& B = P->lv[l];
    if (P->has_vdir && B.fw == nullptr) EFSI_CUDA_CHECK(cudaMalloc(&B.fw, B.n * sizeof(float)));
    if (l > 0 && P->has_vdir && B.va == nullptr) {
      EFSI_CUDA_CHECK(cudaMalloc(&B.va, B.n * sizeof(int32_t)));
      EFSI_CUDA_CHECK(cudaMalloc(&B.vw, B.n * sizeof(float)));
    }
    if (l > 0 && P->has_iface && B.iface == nullptr) EFSI_CUDA_CHECK(cudaMalloc(&B.iface, B.n * sizeof(float)));
  }
  // level 0
  {
    LevelBuf& B = P->lv[0];
    EFSI_COUNTED k_mask_from_obstacle<<<B.shape.grid, B.shape.block, 0, s>>>(B.nx, B.ny, B.nz, obstacle, vdir_active, vdir_weight,
                                                                 B.mask, P->has_vdir ? B.fw : nullptr);
    EFSI_LAUNCH_CHECK();
  }
  for (int l = 1; l < P->n_levels; ++l) {
    LevelBuf& F = P->lv[l - 1];
    LevelBuf& C = P->lv[l];
    const int32_t* fobs = (l == 1) ? obstacle : F.obs;
    const int32_t* fva = P->has_vdir ? ((l == 1) ? vdir_active : F.va) : nullptr;
    const float* fvw = P->has_vdir ? ((l == 1) ? vdir_weight : F.vw) : nullptr;
    if (l == 1) {
      EFSI_COUNTED k_coarsen_structure<double><<<C.shape.grid, C.shape.block, 0, s>>>(
          F.nx, F.ny, F.nz, fobs, fva, fvw, P->has_iface ? iface_diag : nullptr, F.wx, F.wy, F.wz, C.nx, C.ny, C.nz,
          C.obs, P->has_vdir ? C.va : nullptr, P->has_vdir ? C.vw : nullptr,
          P->has_iface ? (float*)C.iface : nullptr);
    } else {
      EFSI_COUNTED k_coarsen_structure<float><<<C.shape.grid, C.shape.block, 0, s>>>(
          F.nx, F.ny, F.nz, fobs, fva, fvw, P->has_iface ? (const float*)F.iface : nullptr, F.wx, F.wy, F.wz, C.nx,
          C.ny, C.nz, C.obs, P->has_vdir ? C.va : nullptr, P->has_vdir ? C.vw : nullptr,
          P->has_iface ? (float*)C.iface : nullptr);
    }
    EFSI_LAUNCH_CHECK();
    EFSI_COUNTED k_mask_from_obstacle<<<C.shape.grid, C.shape.block, 0, s>>>(C.nx, C.ny, C.nz, C.obs, P->has_vdir ? C.va : nullptr,
                                                                 P->has_vdir ? C.vw : nullptr, C.mask,
                                                                 P->has_vdir ? C.fw : nullptr);
    EFSI_LAUNCH_CHECK();
  }
  return EFSI_OK;
}

int efsi_fv_apply(efsi_fv_plan* P, const double* p, double* out, int32_t outlet, void* stream) {
  EFSI_TRY(level_zero_check(P));
  LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  EFSI_COUNTED k_fv_apply<<<S.grid, S.block, 0, as_stream(stream)>>>(L, p, out, outlet);
  if (P->cpl_nrows > 0)
    EFSI_COUNTED k_couple<<<148, 256, 0, as_stream(stream)>>>(P->cpl_rows, P->cpl_ptr, P->cpl_src, P->cpl_coef, P->cpl_n,
                                                            p, out, 0);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_fv_diagonal(efsi_fv_plan* P, double* diag, int32_t outlet, void* stream) {
  EFSI_TRY(level_zero_check(P));
  LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  EFSI_COUNTED k_fv_diag<<<S.grid, S.block, 0, as_stream(stream)>>>(L, diag, outlet);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_apply_jacobi_preconditioner(efsi_fv_plan* P, const double* diag, const double* r, double* z, void* stream) {
  EFSI_TRY(level_zero_check(P));
  LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  EFSI_COUNTED k_jacobi_precond<<<S.grid, S.block, 0, as_stream(stream)>>>(L, diag, r, z, 0, P->partials, P->sc);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_weighted_dot(efsi_fv_plan* P, const double* a, const double* b, double* result_host, void* stream) {
  EFSI_TRY(level_zero_check(P));
  LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  cudaStream_t s = as_stream(stream);
  EFSI_COUNTED k_weighted_dot<<<S.grid, S.block, 0, s>>>(L, a, b, P->partials, P->sc);
  EFSI_LAUNCH_CHECK();
  EFSI_CUDA_CHECK(cudaMemcpyAsync(result_host, &P->sc->dot, sizeof(double), cudaMemcpyDeviceToHost, s));
  EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  return EFSI_OK;
}

int efsi_fv_jacobi_sweep(efsi_fv_plan* P, int32_t level, const void* p, const void* rhs, void* tmp, int32_t outlet,
                         double omega, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(level >= 0 && level < P->n_levels, "level out of range");
  LevelDev L = level_dev(P, level);
  const Shape3& S = P->lv[level].shape;
  ProlongSrc none{nullptr, 0, 0, 0, 0.0f};
  double om = (double)(float)omega;
  if (level == 0)
    EFSI_COUNTED k_sweep<double, false, false><<<S.grid, S.block, 0, as_stream(stream)>>>(
        L, (const double*)p, rhs, (double*)tmp, outlet, om, none, nullptr, P->sc);
  else
    EFSI_COUNTED k_sweep<float, false, false><<<S.grid, S.block, 0, as_stream(stream)>>>(L, (const float*)p, rhs, (float*)tmp,
                                                                            outlet, om, none, nullptr, P->sc);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_fv_residual(efsi_fv_plan* P, int32_t level, const void* p, const void* rhs, void* residual, int32_t outlet,
                     void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(level >= 0 && level < P->n_levels, "level out of range");
  LevelDev L = level_dev(P, level);
  const Shape3& S = P->lv[level].shape;
  if (level == 0)
    EFSI_COUNTED k_residual<double, false><<<S.grid, S.block, 0, as_stream(stream)>>>(L, (const double*)p, rhs, (double*)residual,
                                                                         outlet);
  else
    EFSI_COUNTED k_residual<float, false><<<S.grid, S.block, 0, as_stream(stream)>>>(L, (const float*)p, rhs, (float*)residual,
                                                                        outlet);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_mg_restrict(efsi_fv_plan* P, int32_t level, const void* fine_residual, float* coarse_rhs, float* coarse_iface,
                     int32_t* coarse_obstacle, int32_t* coarse_vdir_active, float* coarse_vdir_weight, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(level >= 0 && level + 1 < P->n_levels, "level out of range");
  LevelDev F = level_dev(P, level);
  const LevelBuf& C = P->lv[level + 1];
  cudaStream_t s = as_stream(stream);
  if (level == 0)
    EFSI_COUNTED k_restrict<double, false, false><<<C.shape.grid, C.shape.block, 0, s>>>(F, (const double*)fine_residual, nullptr,
                                                                             0, C.nx, C.ny, C.nz, coarse_rhs);
  else
    EFSI_COUNTED k_restrict<float, false, false><<<C.shape.grid, C.shape.block, 0, s>>>(F, (const float*)fine_residual, nullptr, 0,
                                                                            C.nx, C.ny, C.nz, coarse_rhs);
  EFSI_LAUNCH_CHECK();
  if (coarse_iface != nullptr) {
    if (P->has_iface)
      EFSI_CUDA_CHECK(cudaMemcpyAsync(coarse_iface, C.iface, C.n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    else
      EFSI_CUDA_CHECK(cudaMemsetAsync(coarse_iface, 0, C.n * sizeof(float), s));
  }
  if (coarse_obstacle != nullptr)
    EFSI_CUDA_CHECK(cudaMemcpyAsync(coarse_obstacle, C.obs, C.n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
  if (coarse_vdir_active != nullptr) {
    if (P->has_vdir)
      EFSI_CUDA_CHECK(cudaMemcpyAsync(coarse_vdir_active, C.va, C.n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    else
      EFSI_CUDA_CHECK(cudaMemsetAsync(coarse_vdir_active, 0, C.n * sizeof(int32_t), s));
  }
  if (coarse_vdir_weight != nullptr) {
    if (P->has_vdir)
      EFSI_CUDA_CHECK(cudaMemcpyAsync(coarse_vdir_weight, C.vw, C.n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    else
      EFSI_CUDA_CHECK(cudaMemsetAsync(coarse_vdir_weight, 0, C.n * sizeof(float), s));
  }
  return EFSI_OK;
}

int efsi_mg_prolong(efsi_fv_plan* P, int32_t level, void* fine_p, const float* coarse_p, double scale, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(level >= 0 && level + 1 < P->n_levels, "level out of range");
  LevelDev L = level_dev(P, level);
  const LevelBuf& C = P->lv[level + 1];
  ProlongSrc pr{coarse_p, C.nx, C.ny, C.nz, (float)scale};
  const Shape3& S = P->lv[level].shape;
  if (level == 0)
    EFSI_COUNTED k_prolong<double><<<S.grid, S.block, 0, as_stream(stream)>>>(L, (double*)fine_p, pr);
  else
    EFSI_COUNTED k_prolong<float><<<S.grid, S.block, 0, as_stream(stream)>>>(L, (float*)fine_p, pr);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

}  // extern "C"

namespace efsi {


// ---------------------------------------------------------------------------
// TMA descriptors of level fields for the plane-marching kernels
// ---------------------------------------------------------------------------
// MAP_VALUE32: an FP32 value tile on level 0 (the mixed-precision V-cycle)
enum : int { MAP_VALUE = 0, MAP_RHS = 1, MAP_MASK = 2, MAP_VALUE32 = 3 };

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    cudaGetLastError();
  });
  return fn;
}

// Descriptor of field `ptr` of level l (f64 at level 0, f32 on coarse levels;
// the mask is u8): value tiles are (8 + 2) rows x (32 + 2 x 16 bytes) with
// their origin 16 bytes left of and one row above the column tile, rhs and
// mask tiles are 8 x 32 at the tile origin.  Null when the field cannot be
// described (misaligned base or row pitch, or no encoder).
static const CUtensorMap* plane_map(efsi_fv_plan* P, int l, const void* ptr, int kind) {
  for (const PlaneMap& m : P->maps)
    if (m.ptr == ptr && m.level == l && m.kind == kind) return &m.map;
  auto enc = tensor_map_encoder();
  if (enc == nullptr || ptr == nullptr || (reinterpret_cast<uintptr_t>(ptr) & 15u) != 0) return nullptr;
  const LevelBuf& B = P->lv[l];
  const int es = kind == MAP_MASK ? 1 : (l == 0 && kind != MAP_VALUE32 ? 8 : 4);
  if (((size_t)B.nz * es) % 16 != 0) return nullptr;
  const CUtensorMapDataType dt = kind == MAP_MASK ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                 : es == 8        ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                                  : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint64_t dims[3] = {(cuuint64_t)B.nz, (cuuint64_t)B.ny, (cuuint64_t)B.nx};
  const cuuint64_t strides[2] = {(cuuint64_t)B.nz * es, (cuuint64_t)B.nz * B.ny * es};
  cuuint32_t box[3] = {(cuuint32_t)kMK, (cuuint32_t)kMJ, 1u};
  if (kind == MAP_VALUE || kind == MAP_VALUE32) {
    box[0] = (cuuint32_t)(kMK + 2 * (16 / es));
    box[1] = (cuuint32_t)(kMJ + 2);
  }
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  PlaneMap pm;
  pm.ptr = ptr;
  pm.level = l;
  pm.kind = kind;
  if (enc(&pm.map, dt, 3, const_cast<void*>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return nullptr;
  P->maps.push_back(pm);
  return &P->maps.back().map;
}

// d_new = z' (+ beta d_old), Ad = A d_new, <d, Ad>_V and alpha (marching
// kernel); false when the fields cannot be streamed with TMA.
static bool launch_march_spmv(efsi_fv_plan* P, const LevelDev& L, bool copy, const double* z, const double* d_old,
                              double* d_new, double* Ad, int outlet, double* partials, CgScalars* sc,
                              cudaStream_t s) {
  const LevelBuf& B = P->lv[0];
  const CUtensorMap* mz = plane_map(P, 0, z, MAP_VALUE);
  const CUtensorMap* mm = plane_map(P, 0, B.mask, MAP_MASK);
  const CUtensorMap* md = copy ? mz : plane_map(P, 0, d_old, MAP_VALUE);
  if (!mz || !mm || !md) return false;
  const dim3 blk(kMK, kTY);
  const bool aux = L.fw != nullptr || L.iface != nullptr;
  const int sm1 = march_smem<double, 1, double, false>(), sm2 = march_smem<double, 2, double, false>();
  if (copy && aux)
    EFSI_COUNTED launch_pdl(km_spmv_dir<true, true>, B.spgrid, blk, sm1, s, L, B.spchunk, *mz, *md, *mm, d_new, Ad, outlet,
                                                                    partials, sc);
  else if (copy)
    EFSI_COUNTED launch_pdl(km_spmv_dir<true, false>, B.spgrid, blk, sm1, s, L, B.spchunk, *mz, *md, *mm, d_new, Ad, outlet,
                                                                     partials, sc);
  else if (aux)
    EFSI_COUNTED launch_pdl(km_spmv_dir<false, true>, B.spgrid, blk, sm2, s, L, B.spchunk, *mz, *md, *mm, d_new, Ad, outlet,
                                                                     partials, sc);
  else
    EFSI_COUNTED launch_pdl(km_spmv_dir<false, false>, B.spgrid, blk, sm2, s, L, B.spchunk, *mz, *md, *mm, d_new, Ad, outlet,
                                                                      partials, sc);
  return true;
}

// One sweep with the marching kernels; false when the fields cannot be
// streamed with TMA (the caller then runs the per-cell kernel).
template <typename TP, bool kNegR, bool kZero, bool kAux>
static bool launch_march_sweep(efsi_fv_plan* P, int l, const LevelDev& L, const TP* p, const void* rhs, TP* out,
                               int outlet, double om, ProlongSrc pr, double* partials, cudaStream_t s,
                               const double* dots_delta) {
  using TR = typename std::conditional<kNegR, double, TP>::type;
  const LevelBuf& B = P->lv[l];
  const dim3 blk(kMK, kTY);
  // level 0 of the PCG's V-cycle: the precomputed reciprocal denominators
  // when they are current for this outlet mode
  const double* rden = (l == 0 && kNegR && std::is_same<TP, double>::value && P->rden_ok[outlet ? 1 : 0])
                           ? P->rden[outlet ? 1 : 0]
                           : nullptr;
  if (kZero) {
    EFSI_COUNTED launch_pdl(km_sweep0<TP, kNegR, kAux>, sweep0_grid(B.nx, B.ny, B.nz), blk, 0, s, L, rhs, out, outlet, om,
                                                                                           partials, P->sc, rden);
    return true;
  }
  const CUtensorMap* mp = plane_map(P, l, p, MAP_VALUE);
  const CUtensorMap* mr = plane_map(P, l, rhs, MAP_RHS);
  const CUtensorMap* mm = plane_map(P, l, B.mask, MAP_MASK);
  if (!mp || !mr || !mm) return false;
  const int sm = march_smem<TP, 1, TR, true>();
  if constexpr (std::is_same<TP, double>::value && kNegR && !kZero) {
    const double* dd = dots_delta;
    const bool pro = pr.pc != nullptr;
    // the reciprocal pays off in the dots-fused sweep (measured on c2: 49.4 ->
    // 44.4 us); the plain and prolongation-fused sweeps keep the division
    // (28.5 / 44.5 us against 30.4 / 46.0 us with the extra 8 bytes per cell)
    if (rden != nullptr && dd != nullptr) {
      if (pro)
        EFSI_COUNTED launch_pdl(km_sweep<TP, kNegR, true, kAux, true, true>, B.mgrid, blk, sm, s, L, B.mchunk, *mp, *mr,
                                *mm, out, outlet, om, pr, partials, P->sc, dd, rden);
      else
        EFSI_COUNTED launch_pdl(km_sweep<TP, kNegR, false, kAux, true, true>, B.mgrid, blk, sm, s, L, B.mchunk, *mp,
                                *mr, *mm, out, outlet, om, pr, partials, P->sc, dd, rden);
      return true;
    }
    if (dd != nullptr) {
      if (pro)
        EFSI_COUNTED launch_pdl(km_sweep<TP, kNegR, true, kAux, true>, B.mgrid, blk, sm, s, 
            L, B.mchunk, *mp, *mr, *mm, out, outlet, om, pr, partials, P->sc, dd, (const double*)nullptr);
      else
        EFSI_COUNTED launch_pdl(km_sweep<TP, kNegR, false, kAux, true>, B.mgrid, blk, sm, s, 
            L, B.mchunk, *mp, *mr, *mm, out, outlet, om, pr, partials, P->sc, dd, (const double*)nullptr);
      return true;
    }
  }
  if (pr.pc != nullptr)
    EFSI_COUNTED launch_pdl(km_sweep<TP, kNegR, true, kAux, false>, B.mgrid, blk, sm, s, 
        L, B.mchunk, *mp, *mr, *mm, out, outlet, om, pr, partials, P->sc, (const double*)nullptr, (const double*)nullptr);
  else
    EFSI_COUNTED launch_pdl(km_sweep<TP, kNegR, false, kAux, false>, B.mgrid, blk, sm, s, 
        L, B.mchunk, *mp, *mr, *mm, out, outlet, om, pr, partials, P->sc, (const double*)nullptr, (const double*)nullptr);
  return true;
}

// Level-0 sweep of the mixed-precision V-cycle (FP32 iterate and arithmetic);
// out64 (with partials, and dots_delta when the PCG dots are finished in it)
// receives the f64 result.  False when the fields cannot be streamed.
static bool launch_sweep32(efsi_fv_plan* P, const float* p, const double* r, float* out, double* out64, int outlet,
                           double om, ProlongSrc pr, double* partials, const double* dots_delta, cudaStream_t s) {
  LevelDev L = level_dev(P, 0);
  const LevelBuf& B = P->lv[0];
  const CUtensorMap* mp = plane_map(P, 0, p, MAP_VALUE32);
  const CUtensorMap* mr = plane_map(P, 0, r, MAP_RHS);
  const CUtensorMap* mm = plane_map(P, 0, B.mask, MAP_MASK);
  if (!B.march || !mp || !mr || !mm) return false;
  const dim3 blk(kMK, kTY);
  const int sm = march_smem<float, 1, double, true>();
  const bool aux = L.fw != nullptr || L.iface != nullptr, pro = pr.pc != nullptr, dots = dots_delta != nullptr;
#define EFSI_SWEEP32(PRO, AUX, DOTS)                                                                              \
  EFSI_COUNTED launch_pdl(km_sweep32<PRO, AUX, DOTS>, B.mgrid, blk, sm, s, L, B.mchunk, *mp, *mr, *mm, out, out64, \
                          outlet, om, pr, partials, P->sc, dots_delta)
  if (pro && aux && dots) EFSI_SWEEP32(true, true, true);
  else if (pro && aux) EFSI_SWEEP32(true, true, false);
  else if (pro && dots) EFSI_SWEEP32(true, false, true);
  else if (pro) EFSI_SWEEP32(true, false, false);
  else if (aux && dots) EFSI_SWEEP32(false, true, true);
  else if (aux) EFSI_SWEEP32(false, true, false);
  else if (dots) EFSI_SWEEP32(false, false, true);
  else EFSI_SWEEP32(false, false, false);
#undef EFSI_SWEEP32
  return true;
}

// One smoother sweep of level l (plane-marching kernel when the level is
// large enough, else the per-cell kernel).
// With dots_delta (level 0, the last sweep of the PCG's V-cycle, partials
// given) the march kernel also finishes the PCG dots and *dots_done is set;
// the per-cell fallback leaves them to the dots kernel.
template <typename TP, bool kNegR, bool kZero>
static void launch_sweep(efsi_fv_plan* P, int l, const TP* p, const void* rhs, TP* out, int outlet, double om,
                         ProlongSrc pr, double* partials, cudaStream_t s, const double* dots_delta = nullptr,
                         bool* dots_done = nullptr) {
  LevelDev L = level_dev(P, l);
  const LevelBuf& B = P->lv[l];
  if (B.march) {
    const bool done = (L.fw != nullptr || L.iface != nullptr)
                          ? launch_march_sweep<TP, kNegR, kZero, true>(P, l, L, p, rhs, out, outlet, om, pr, partials,
                                                                        s, dots_delta)
                          : launch_march_sweep<TP, kNegR, kZero, false>(P, l, L, p, rhs, out, outlet, om, pr,
                                                                         partials, s, dots_delta);
    if (done) {
      if (dots_done != nullptr && dots_delta != nullptr && !kZero) *dots_done = true;
      return;
    }
  }
  if (B.tiled)
    EFSI_COUNTED launch_pdl(kt_sweep<TP, kNegR, kZero>, B.tgrid, dim3(kTK, kTJ), 0, s, L, p, rhs, out, outlet, om, pr, partials,
                                                                              P->sc);
  else
    EFSI_COUNTED launch_pdl(k_sweep<TP, kNegR, kZero>, B.shape.grid, B.shape.block, 0, s, L, p, rhs, out, outlet, om, pr,
                                                                                   partials, P->sc);
}

// Residual of level l's iterate p restricted into level l+1's rhs.  With
// `czero` (level l+1's first iterate buffer) the plane-marching restriction
// also writes level l+1's zero-guess sweep there (damping omega); returns
// whether it did, so that the caller skips that sweep's own launch.
template <typename TP, bool kNegR>
static bool launch_restrict(efsi_fv_plan* P, int l, const TP* p, const void* rhs, int outlet, cudaStream_t s,
                            float* czero = nullptr, double omega = 0.0) {
  LevelDev L = level_dev(P, l);
  const LevelBuf& B = P->lv[l];
  const LevelBuf& C = P->lv[l + 1];
  if (B.march) {
    using TR = typename std::conditional<kNegR, double, TP>::type;
    const CUtensorMap* mp = plane_map(P, l, p, (l == 0 && sizeof(TP) == 4) ? MAP_VALUE32 : MAP_VALUE);
    const CUtensorMap* mr = plane_map(P, l, rhs, MAP_RHS);
    const CUtensorMap* mm = plane_map(P, l, B.mask, MAP_MASK);
    if (mp && mr && mm) {
      const int sm = march_smem<TP, 1, TR, true>();
      const LevelDev LC = level_dev(P, l + 1);
      if (L.fw != nullptr || L.iface != nullptr)
        EFSI_COUNTED launch_pdl(km_restrict<TP, kNegR, true>, B.mgrid, dim3(kMK, kTY), sm, s, L, B.mchunk, *mp, *mr,
                                *mm, outlet, C.nx, C.ny, C.nz, C.rhs, P->sc, LC, czero, omega);
      else
        EFSI_COUNTED launch_pdl(km_restrict<TP, kNegR, false>, B.mgrid, dim3(kMK, kTY), sm, s, L, B.mchunk, *mp, *mr,
                                *mm, outlet, C.nx, C.ny, C.nz, C.rhs, P->sc, LC, czero, omega);
      return czero != nullptr;
    }
  }
  EFSI_COUNTED launch_pdl(k_restrict<TP, kNegR, true>, C.shape.grid, C.shape.block, 0, s, L, p, rhs, outlet, C.nx, C.ny,
                                                                                 C.nz, C.rhs);
  return false;
}

// The level-0 reciprocal denominators for this outlet mode (recomputed after
// every efsi_fv_set_masks).  EFSI_NO_RDEN keeps the sweeps dividing.
static int ensure_rden(efsi_fv_plan* P, int outlet, cudaStream_t s) {
  static const bool off = std::getenv("EFSI_NO_RDEN") != nullptr;
  const int o = outlet ? 1 : 0;
  if (off || P->rden_ok[o] || !P->lv[0].march) return EFSI_OK;
  if (P->rden[o] == nullptr) EFSI_CUDA_CHECK(cudaMalloc(&P->rden[o], P->lv[0].n * sizeof(double)));
  const LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  EFSI_COUNTED k_rden<<<S.grid, S.block, 0, s>>>(L, o, P->rden[o]);
  EFSI_LAUNCH_CHECK();
  P->rden_ok[o] = true;
  return EFSI_OK;
}

// ---------------------------------------------------------------------------
// V-cycle (fluid.py:6085-6262), zero initial guess, level-0 rhs = -r.
// The result lands in z; when `want_mean` the last sweep also reduces the
// fluid z V sum so consumers can apply the zero-mean projection on the fly.
// ---------------------------------------------------------------------------
// mixed: level 0 runs in FP32 (fv_multigrid_mixed; the caller checks that
// level 0 has the plane-marching kernels and more than one level exists).
// Whether the V-cycle forms coarse level c's zero-guess sweep inside the
// restriction into it: c runs its own pre-sweeps (it lies above the tail and
// below the coarse-level kernel's first level), or it is the coarsest level
// of a hierarchy without a tail.  EFSI_NO_RESTRICT_SWEEP0 keeps the separate
// launch.
static bool vcycle_fuses_zero(const efsi_fv_plan* P, int c) {
  static const bool off = std::getenv("EFSI_NO_RESTRICT_SWEEP0") != nullptr;
  const int nl = P->n_levels, lt = P->tail_level;
  const bool coarse_kernel = P->coarse_blocks > 0 && lt >= P->coarse_first + 1 && lt < nl;
  const int down_end = coarse_kernel ? P->coarse_first : (lt < nl) ? lt : nl - 1;
  return !off && c >= 1 && (c < down_end || (!coarse_kernel && lt >= nl && c == nl - 1));
}

static int vcycle(efsi_fv_plan* P, const double* r, double* z, int outlet, int pre, int coarse, int post,
                  bool want_mean, cudaStream_t s, const double* dots_delta = nullptr, bool* dots_done = nullptr,
                  bool mixed = false, bool level0_zero_done = false) {
  pre = std::max(1, pre);
  coarse = std::max(1, coarse);
  post = std::max(1, post);
  const double om = (double)0.8f;
  const float scale = P->uniform ? 1.0f : 0.7f;
  const int nl = P->n_levels;
  const double n0 = (double)P->lv[0].n;
  ProlongSrc none{nullptr, 0, 0, 0, 0.0f};
  double* partials = want_mean ? P->partials : nullptr;
  if (nl <= 1) {
    const int n = std::max(pre + post, coarse);
    double* bufs[2] = {(double*)P->lv[0].pa, (double*)P->lv[0].pb};
    const double* cur = nullptr;
    for (int it = 0; it < n; ++it) {
      double* dst = (it == n - 1) ? z : bufs[it & 1];
      double* part = (it == n - 1) ? partials : nullptr;
      if (it == 0)
        launch_sweep<double, true, true>(P, 0, nullptr, r, dst, outlet, om, none, part, s);
      else
        launch_sweep<double, true, false>(P, 0, cur, r, dst, outlet, om, none, part, s,
                                          it == n - 1 ? dots_delta : nullptr, dots_done);
      cur = dst;
    }
    EFSI_LAUNCH_CHECK();
    return EFSI_OK;
  }
  // Down: the iterate after pre-smoothing of level l lives in cur[l].  Levels
  // from P->tail_level on run inside k_mg_tail.
  const int lt = P->tail_level;
  // levels 1 .. lt-1 and the tail in one cooperative launch (k_mg_coarse)
  const int cfirst = P->coarse_first;
  const bool coarse_kernel = P->coarse_blocks > 0 && lt >= cfirst + 1 && lt < nl;
  std::vector<const void*> cur(nl, nullptr);
  const int down_end = coarse_kernel ? cfirst : (lt < nl) ? lt : nl - 1;
  // zero_done[l]: level l's zero-guess sweep was formed by the restriction
  // into it (into lv[l].pa), so its own launch is skipped
  std::vector<char> zero_done(nl, 0);
  auto fuse_zero = [&](int c) { return vcycle_fuses_zero(P, c); };
  for (int l = 0; l < down_end; ++l) {
    LevelDev L = level_dev(P, l);
    LevelBuf& B = P->lv[l];
    void* bufs[2] = {B.pa, B.pb};
    if (l == 0 && mixed) {
      bufs[0] = B.pa32;
      bufs[1] = B.pb32;
    }
    const void* c = nullptr;
    for (int it = 0; it < pre; ++it) {
      void* dst = bufs[it & 1];
      if (l == 0 && mixed) {
        if (it == 0) {
          if (!level0_zero_done)  // else the CG update formed it in bufs[0]
            launch_sweep<float, true, true>(P, 0, nullptr, r, (float*)dst, outlet, om, none, nullptr, s);
        } else if (!launch_sweep32(P, (const float*)c, r, (float*)dst, nullptr, outlet, om, none, nullptr, nullptr, s)) {
          set_error("the mixed-precision V-cycle needs the plane-marching kernels on level 0");
          return EFSI_ERR_ARG;
        }
      } else if (l == 0) {
        if (it == 0) {
          if (!level0_zero_done)  // else the CG update formed it in bufs[0]
            EFSI_TIMED(KF_SWEEP_L0, 17.0 * n0, s,
                       (launch_sweep<double, true, true>(P, 0, nullptr, r, (double*)dst, outlet, om, none, nullptr, s)));
        } else
          EFSI_TIMED(KF_SWEEP_L0, 25.0 * n0, s,
                     (launch_sweep<double, true, false>(P, 0, (const double*)c, r, (double*)dst, outlet, om, none,
                                                        nullptr, s)));
      } else {
        if (it == 0) {
          if (!zero_done[l])
            launch_sweep<float, false, true>(P, l, nullptr, B.rhs, (float*)dst, outlet, om, none, nullptr, s);
        } else {
          launch_sweep<float, false, false>(P, l, (const float*)c, B.rhs, (float*)dst, outlet, om, none, nullptr, s);
        }
      }
      c = dst;
    }
    cur[l] = c;
    const LevelBuf& C = P->lv[l + 1];
    float* cz = fuse_zero(l + 1) ? (float*)C.pa : nullptr;
    bool fz = false;
    if (l == 0 && mixed)
      fz = launch_restrict<float, true>(P, 0, (const float*)c, r, outlet, s, cz, om);
    else if (l == 0)
      EFSI_TIMED(KF_RESTRICT_L0, 17.0 * B.n + (cz ? 9.0 : 4.0) * C.n, s,
                 (fz = launch_restrict<double, true>(P, 0, (const double*)c, r, outlet, s, cz, om)));
    else
      fz = launch_restrict<float, false>(P, l, (const float*)c, B.rhs, outlet, s, cz, om);
    zero_done[l + 1] = fz ? 1 : 0;
  }
  if (lt < nl) {
    CoarseDesc D;
    TailDesc& T = D.T;
    T.lt = lt;
    T.nl = nl;
    T.outlet = outlet;
    T.pre = pre;
    T.coarse = coarse;
    T.post = post;
    T.scale = scale;
    T.omega = om;
    for (int l = lt; l < nl; ++l) {
      T.L[l] = level_dev(P, l);
      T.foff[l] = P->tail_foff[l];
      T.moff[l] = P->tail_moff[l];
      T.coff[l] = P->tail_coff[l];
      T.noff[l] = P->tail_noff[l];
    }
    T.rhs_in = P->lv[lt].rhs;
    T.p_out = (float*)P->lv[lt].pa;
    if (coarse_kernel) {
      for (int l = cfirst; l < nl; ++l) {
        T.L[l] = level_dev(P, l);
        D.pa[l] = (float*)P->lv[l].pa;
        D.pb[l] = (float*)P->lv[l].pb;
        D.rhs[l] = P->lv[l].rhs;
      }
      D.bar = P->coarse_bar;
      D.fault = &P->sc->fault;
      static const unsigned spin_ns = std::getenv("EFSI_COARSE_SPIN_NS") ? (unsigned)std::atoi(std::getenv("EFSI_COARSE_SPIN_NS")) : 0u;
      D.spin_ns = spin_ns;
      D.first = cfirst;
      D.cluster = P->coarse_cluster;
      cudaLaunchAttribute attr[1];
      if (P->coarse_cluster) {
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)P->coarse_blocks;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
      } else {
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
      }
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)P->coarse_blocks);
      cfg.blockDim = dim3(kTailThreads);
      cfg.dynamicSmemBytes = P->tail_smem_bytes;
      cfg.stream = s;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      EFSI_COUNTED cudaLaunchKernelEx(&cfg, k_mg_coarse, D);
      // the kernel's final iterate of level cfirst: the pre-sweeps end in
      // buffer (pre - 1) & 1, the post-sweeps alternate from the other one
      const int c = (pre - 1) & 1;
      void* bufs1[2] = {P->lv[cfirst].pa, P->lv[cfirst].pb};
      void* seq1[2] = {bufs1[1 - c], bufs1[c]};
      cur[cfirst] = seq1[(post - 1) & 1];
    } else {
      EFSI_COUNTED launch_pdl(k_mg_tail, 1, kTailThreads, P->tail_smem_bytes, s, T);
      cur[lt] = P->lv[lt].pa;
    }
  } else {
    // Coarsest level: `coarse` sweeps from zero.
    const int l = nl - 1;
    LevelBuf& B = P->lv[l];
    void* bufs[2] = {B.pa, B.pb};
    const void* c = nullptr;
    for (int it = 0; it < coarse; ++it) {
      void* dst = bufs[it & 1];
      if (it == 0) {
        if (!zero_done[l])
          launch_sweep<float, false, true>(P, l, nullptr, B.rhs, (float*)dst, outlet, om, none, nullptr, s);
      } else
        launch_sweep<float, false, false>(P, l, (const float*)c, B.rhs, (float*)dst, outlet, om, none, nullptr, s);
      c = dst;
    }
    cur[l] = c;
  }
  // Up: prolongation fused into the first post sweep.
  const int up_start = coarse_kernel ? cfirst - 1 : (lt < nl) ? lt - 1 : nl - 2;
  for (int l = up_start; l >= 0; --l) {
    LevelBuf& B = P->lv[l];
    const LevelBuf& C = P->lv[l + 1];
    ProlongSrc pr{(const float*)cur[l + 1], C.nx, C.ny, C.nz, scale};
    const void* c = cur[l];
    void* other = (l == 0 && mixed) ? (void*)((c == B.pa32) ? B.pb32 : B.pa32) : ((c == B.pa) ? B.pb : B.pa);
    void* seq[2] = {other, const_cast<void*>(c)};
    for (int it = 0; it < post; ++it) {
      const bool last = (it == post - 1);
      void* dst = (l == 0 && last) ? (void*)z : seq[it & 1];
      ProlongSrc p_use = (it == 0) ? pr : none;
      double* part = (l == 0 && last) ? partials : nullptr;
      if (l == 0 && mixed) {
        const double* dd = last ? dots_delta : nullptr;
        if (!launch_sweep32(P, (const float*)c, r, last ? nullptr : (float*)dst, last ? z : nullptr, outlet, om,
                            p_use, part, dd, s)) {
          set_error("the mixed-precision V-cycle needs the plane-marching kernels on level 0");
          return EFSI_ERR_ARG;
        }
        if (dd != nullptr && dots_done != nullptr) *dots_done = true;
      } else if (l == 0)
        EFSI_TIMED(KF_SWEEP_L0, 25.0 * n0 + (it == 0 ? 4.0 * C.n : 0.0), s,
                   (launch_sweep<double, true, false>(P, 0, (const double*)c, r, (double*)dst, outlet, om, p_use, part,
                                                      s, last ? dots_delta : nullptr, dots_done)));
      else
        launch_sweep<float, false, false>(P, l, (const float*)c, B.rhs, (float*)dst, outlet, om, p_use, nullptr, s);
      c = dst;
    }
    cur[l] = c;
  }
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

}  // namespace efsi

extern "C" {

int efsi_mg_vcycle(efsi_fv_plan* P, const double* r, double* z, int32_t outlet, int32_t pre, int32_t coarse,
                   int32_t post, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_TRY(ensure_rden(P, outlet, as_stream(stream)));
  return vcycle(P, r, z, outlet, pre, coarse, post, false, as_stream(stream));
}

}  // extern "C"

namespace efsi {

// ---------------------------------------------------------------------------
// Flexible PCG driver (fluid.py:6535-6811).  All scalars stay on the device;
// the host reads them where the reference does (b_norm, the initial residual
// and preconditioner dot, and every 16th iteration's residual).
// ---------------------------------------------------------------------------
void set_capturing(bool on);
void count_graph_launch(unsigned long long nodes);
unsigned long long take_capture_count();

struct PcgRun {
  efsi_fv_plan* P;
  const efsi_pcg_params* prm;
  cudaStream_t s;
  LevelDev L;
  Shape3 S;
  bool use_mg;
  int pre, coarse, post;
  double* d_cur;
  double* d_nxt;
  bool copy_next;  // next SpMV starts a fresh direction d = z'
  bool dots_fused;  // the last preconditioner sweep also finished the PCG dots
  bool mixed;       // FP32 level-0 V-cycle
  bool learned;     // the attached network (code 4)
  bool anchor;      // outlet solve with unreached components: their means are subtracted
  bool zero0_ready = false;  // the last update formed the V-cycle's first level-0 sweep (in lv[0].pa)
};

// fluid.py:4965-4981 on a level-0 field: the unreached components' means
// subtracted (three launches, capturable).
static void subtract_unreached_means(efsi_fv_plan* P, double* f, cudaStream_t s) {
  const LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  EFSI_COUNTED launch_pdl(k_comp_zero, 1, 256, 0, s, P->ucomp_acc);
  EFSI_COUNTED launch_pdl(k_comp_accumulate, S.grid, S.block, 0, s, L, (const double*)f, (const int32_t*)P->ucomp,
                          P->ucomp_n, P->ucomp_acc);
  EFSI_COUNTED launch_pdl(k_comp_subtract, S.grid, S.block, 0, s, L, f, (const int32_t*)P->ucomp,
                          (const double*)P->ucomp_acc);
}

static int read_scalars(PcgRun& R) {
  EFSI_CUDA_CHECK(cudaMemcpyAsync(R.P->host_sc, R.P->sc, sizeof(CgScalars), cudaMemcpyDeviceToHost, R.s));
  EFSI_CUDA_CHECK(cudaStreamSynchronize(R.s));
  if (R.P->host_sc->fault) {
    set_error("a plane-marching kernel's TMA stage did not complete in time");
    return EFSI_ERR_CUDA;
  }
  return EFSI_OK;
}

// z = M^-1 r (+ z mean for the on-the-fly projection when remove_mean).
static int precondition(PcgRun& R) {
  const bool want_mean = R.prm->remove_mean != 0;
  R.dots_fused = false;
  if (R.learned) {
    // two-level: two damped-Jacobi sweeps (the V-cycle's level-0 smoother)
    // from zero, the network's correction of the remaining residual at its
    // energy-minimising scale, two more sweeps
    efsi_fv_plan* P = R.P;
    const int outlet = R.prm->outlet;
    const double om = (double)0.8f;
    const ProlongSrc none{nullptr, 0, 0, 0, 0.0f};
    double* za = static_cast<double*>(P->lv[0].pa);
    double* zb = static_cast<double*>(P->lv[0].pb);
    __nv_bfloat16* in = static_cast<__nv_bfloat16*>(P->unet_in);
    launch_sweep<double, true, true>(P, 0, nullptr, P->r, za, outlet, om, none, nullptr, R.s);
    launch_sweep<double, true, false>(P, 0, za, P->r, zb, outlet, om, none, nullptr, R.s);
    EFSI_COUNTED k_fv_apply<<<R.S.grid, R.S.block, 0, R.s>>>(R.L, zb, P->Ad, outlet);
    EFSI_COUNTED launch_pdl(k_learned_sumsq, R.S.grid, R.S.block, 0, R.s, R.L, (const double*)P->r,
                            (const double*)P->Ad, P->partials, P->sc);
    EFSI_COUNTED launch_pdl(k_learned_pack, R.S.grid, R.S.block, 0, R.s, R.L, (const double*)P->r,
                            (const double*)P->Ad, in, P->unet_wmin[0], P->unet_wmin[1], P->unet_wmin[2],
                            (const CgScalars*)P->sc);
    const float* out = nullptr;
    EFSI_TRY(unet_run(P->unet, P->lv[0].nx, P->lv[0].ny, P->lv[0].nz, in, &P->sc->fault, &out, R.s));
    EFSI_COUNTED launch_pdl(k_learned_unpack, R.S.grid, R.S.block, 0, R.s, R.L, out, (const double*)P->r,
                            (const double*)P->Ad, za, P->partials, P->sc);
    EFSI_COUNTED k_fv_apply<<<R.S.grid, R.S.block, 0, R.s>>>(R.L, za, P->Ad, outlet);
    EFSI_COUNTED k_weighted_dot<<<R.S.grid, R.S.block, 0, R.s>>>(R.L, za, P->Ad, P->partials, P->sc);
    EFSI_COUNTED launch_pdl(k_learned_combine, R.S.grid, R.S.block, 0, R.s, R.L, (const double*)zb, za,
                            (const CgScalars*)P->sc);
    launch_sweep<double, true, false>(P, 0, za, P->r, zb, outlet, om, none, nullptr, R.s);
    launch_sweep<double, true, false>(P, 0, zb, P->r, P->z, outlet, om, none, want_mean ? P->partials : nullptr,
                                      R.s);
  } else if (R.use_mg) {
    // with the zero-mean projection the V-cycle's last sweep finishes the dots
    // (EFSI_SEPARATE_DOTS keeps them in their own kernel)
    static const bool separate = std::getenv("EFSI_SEPARATE_DOTS") != nullptr;
    const bool zero0 = R.zero0_ready;
    R.zero0_ready = false;
    EFSI_TRY(vcycle(R.P, R.P->r, R.P->z, R.prm->outlet, R.pre, R.coarse, R.post, want_mean, R.s,
                    want_mean && !separate ? R.P->delta : nullptr, &R.dots_fused, R.mixed, zero0));
  } else {
    EFSI_COUNTED launch_pdl(k_jacobi_precond, R.S.grid, R.S.block, 0, R.s, R.L, R.P->diag, R.P->r, R.P->z, want_mean ? 1 : 0,
                                                      R.P->partials, R.P->sc);
  }
  if (R.anchor) subtract_unreached_means(R.P, R.P->z, R.s);
  if (!want_mean) EFSI_COUNTED launch_pdl(k_set_zproj, 1, 32, 0, R.s, R.P->sc, 0);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

}  // namespace efsi

namespace efsi {

// Appends to the capture in progress on `cs`: the pressure reset of a zero
// right-hand side, k_dl_init, and a WHILE node whose body (captured on the
// plan's body stream) is one 16-iteration block plus k_dl_check.  Inside the
// body the launches keep their programmatic dependent launch attribute, and
// the V-cycle uses its per-level launches.
template <class Body>
static int build_device_loop(efsi_fv_plan* P, cudaStream_t cs, double* pressure, double tol, int max_iters, Body body) {
  cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
  unsigned long long id = 0;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  EFSI_CUDA_CHECK(cudaStreamGetCaptureInfo(cs, &status, &id, &g, &deps, &nd));
  EFSI_ARG_CHECK(status == cudaStreamCaptureStatusActive && g != nullptr, "the device-side loop needs a capturing stream");
  cudaGraphConditionalHandle h;
  EFSI_CUDA_CHECK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
  const LevelDev L0 = level_dev(P, 0);
  const Shape3& S0 = P->lv[0].shape;
  EFSI_COUNTED k_dl_zero_if_tiny<<<S0.grid, S0.block, 0, cs>>>(L0, pressure, (const CgScalars*)P->sc);
  EFSI_COUNTED k_dl_init<<<1, 32, 0, cs>>>(P->sc, tol, h);
  EFSI_CUDA_CHECK(cudaGetLastError());
  EFSI_CUDA_CHECK(cudaStreamGetCaptureInfo(cs, &status, &id, &g, &deps, &nd));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  EFSI_CUDA_CHECK(cudaGraphAddNode(&node, g, deps, nd, &cp));
  cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
  EFSI_CUDA_CHECK(cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies));
  if (P->body_stream == nullptr) EFSI_CUDA_CHECK(cudaStreamCreateWithFlags(&P->body_stream, cudaStreamNonBlocking));
  EFSI_CUDA_CHECK(cudaStreamBeginCaptureToGraph(P->body_stream, bodyg, nullptr, nullptr, 0,
                                                cudaStreamCaptureModeThreadLocal));
  const int keep_blocks = P->coarse_blocks;
  P->coarse_blocks = 0;
  int rc = body(P->body_stream);
  EFSI_COUNTED k_dl_check<<<1, 32, 0, P->body_stream>>>(P->sc, tol, max_iters, h);
  cudaGraph_t out = nullptr;
  const cudaError_t e = cudaStreamEndCapture(P->body_stream, &out);
  P->coarse_blocks = keep_blocks;
  if (rc != EFSI_OK) return rc;
  if (e != cudaSuccess) {
    set_error(std::string("capturing the device-side PCG loop body: ") + cudaGetErrorString(e));
    return EFSI_ERR_CUDA;
  }
  return EFSI_OK;
}

static void fill_device_stats(efsi_fv_plan* P, efsi_cg_stats* st) {
  const CgScalars* h = P->host_sc;
  st->iterations = h->dl_iter;
  st->converged = h->dl_converged;
  st->breakdown_code = h->code;
  st->breakdown_dAd = h->code_dAd;
  st->initial_relative_residual = h->dl_rel0;
  st->relative_residual = h->dl_rel;
  st->b_norm = h->dl_bnorm;
  st->used_mg = P->dl_used_mg;
  st->used_graphs = 1;
}

// The device-side loop after the preamble: inside the caller's stream
// capture, or as a graph of its own that is launched and waited for.
template <class Body>
static int pcg_device_loop(efsi_fv_plan* P, PcgRun& R, efsi_cg_stats* st, cudaStream_t s, double* pressure,
                           double tol, int max_iters, int64_t n0, Body body) {
  EFSI_CUDA_CHECK(cudaMemsetAsync(P->d0, 0, n0 * sizeof(double), s));
  EFSI_CUDA_CHECK(cudaMemsetAsync(P->d1, 0, n0 * sizeof(double), s));
  P->dl_used_mg = R.use_mg ? 1 : 0;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  EFSI_CUDA_CHECK(cudaStreamIsCapturing(s, &cs));
  if (cs == cudaStreamCaptureStatusActive) {
    EFSI_TRY(build_device_loop(P, s, pressure, tol, max_iters, body));
    st->converged = -1;  // read later with efsi_fv_pcg_device_stats
    st->used_mg = P->dl_used_mg;
    st->used_graphs = 1;
    return EFSI_OK;
  }
  // a graph of its own, ordered after the preamble by its launch on s
  EFSI_CUDA_CHECK(cudaStreamBeginCapture(P->cap_stream, cudaStreamCaptureModeThreadLocal));
  set_capturing(true);
  take_capture_count();
  int rc = build_device_loop(P, P->cap_stream, pressure, tol, max_iters, body);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(P->cap_stream, &g);
  set_capturing(false);
  const unsigned long long nodes = take_capture_count();
  cudaGraphExec_t ex = nullptr;
  if (rc == EFSI_OK && e == cudaSuccess) {
    const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
    if (ei != cudaSuccess) {
      set_error(std::string("instantiating the device-side PCG loop: ") + cudaGetErrorString(ei));
      rc = EFSI_ERR_CUDA;
    }
  } else if (rc == EFSI_OK) {
    set_error(std::string("capturing the device-side PCG loop: ") + cudaGetErrorString(e));
    rc = EFSI_ERR_CUDA;
  }
  if (g != nullptr) cudaGraphDestroy(g);
  if (rc != EFSI_OK) {
    cudaGetLastError();
    return rc;
  }
  EFSI_CUDA_CHECK(cudaGraphLaunch(ex, s));
  count_graph_launch(nodes);
  EFSI_CUDA_CHECK(cudaMemcpyAsync(P->host_sc, P->sc, sizeof(CgScalars), cudaMemcpyDeviceToHost, s));
  EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  cudaGraphExecDestroy(ex);
  if (P->host_sc->fault) {
    set_error("a plane-marching kernel's TMA stage did not complete in time");
    return EFSI_ERR_CUDA;
  }
  fill_device_stats(P, st);
  return EFSI_OK;
}

}  // namespace efsi

extern "C" {

int efsi_fv_pcg_solve(efsi_fv_plan* P, const double* rhs0, double* pressure, const efsi_pcg_params* prm,
                      efsi_cg_stats* st, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(rhs0 != nullptr && pressure != nullptr && prm != nullptr && st != nullptr, "null argument");
  cudaStream_t s = as_stream(stream);
  PcgRun R;
  R.mixed = false;
  R.learned = false;
  R.dots_fused = false;
  R.anchor = prm->outlet != 0 && P->ucomp_n > 0;
  R.P = P;
  R.prm = prm;
  R.s = s;
  R.L = level_dev(P, 0);
  R.S = P->lv[0].shape;
  const int max_iters = std::max(1, (int)prm->max_iters);
  const double tol = std::max(0.0, prm->tolerance);
  std::memset(st, 0, sizeof(*st));
  st->initial_relative_residual = INFINITY;
  st->relative_residual = INFINITY;
  const int outlet = prm->outlet;
  const bool remove_mean = prm->remove_mean != 0;
  // device_loop: no host reads; the loop runs on the device (WHILE node)
  const bool device = prm->device_loop != 0;
  EFSI_ARG_CHECK(!device || (prm->precond != 4 && prm->precond != 5),
                 "the device-side loop does not take the learned preconditioner (its fallback is a host decision)");
  EFSI_COUNTED k_reset_scalars<<<1, 32, 0, s>>>(P->sc);
  EFSI_TRY(ensure_rden(P, outlet, s));
  const bool coupled = P->cpl_nrows > 0;
  if (coupled) EFSI_COUNTED k_set_defer<<<1, 32, 0, s>>>(P->sc, 1);
  // fluid.py:6581 diagonal (Jacobi path and fallback).
  EFSI_COUNTED k_fv_diag<<<R.S.grid, R.S.block, 0, s>>>(R.L, P->diag, outlet);
  // b = -rhs - V-mean(-rhs)  (fluid.py:6589-6601); the free volume is reduced
  // in the same pass whether or not the mean is used.
  EFSI_COUNTED k_rhs_mean<<<R.S.grid, R.S.block, 0, s>>>(R.L, rhs0, -1.0, P->partials, P->sc);
  if (remove_mean) st->mean_projection_count += 1;
  if (R.anchor) st->unreached_set_mean_projection_count += 1;
  EFSI_COUNTED k_build_b<<<R.S.grid, R.S.block, 0, s>>>(R.L, rhs0, remove_mean ? 1 : 0, P->b, P->partials, P->sc);
  EFSI_LAUNCH_CHECK();
  if (!device) EFSI_TRY(read_scalars(R));
  const double b_norm = device ? 1.0 : std::sqrt(std::max(P->host_sc->bnorm2, 0.0));
  st->b_norm = b_norm;
  const int64_t n0 = P->lv[0].n;
  if (!device && b_norm <= 1.0e-30) {
    EFSI_CUDA_CHECK(cudaMemsetAsync(pressure, 0, n0 * sizeof(double), s));
    st->initial_relative_residual = 0.0;
    st->relative_residual = 0.0;
    st->converged = 1;
    return EFSI_OK;
  }
  // r = b - A p, mean projection, ||r||  (fluid.py:6613-6622).
  auto true_residual = [&]() -> int {
    EFSI_COUNTED k_true_residual<<<R.S.grid, R.S.block, 0, s>>>(R.L, pressure, P->b, P->r, outlet, remove_mean ? 1 : 0,
                                                   P->partials, P->sc);
    if (coupled) {
      // r -= C p, then the mean or <r, r>_V of the corrected residual
      EFSI_COUNTED k_couple<<<148, 256, 0, s>>>(P->cpl_rows, P->cpl_ptr, P->cpl_src, P->cpl_coef, P->cpl_n, pressure,
                                              P->r, 1);
      EFSI_COUNTED k_residual_reduce<<<R.S.grid, R.S.block, 0, s>>>(R.L, P->r, remove_mean ? 1 : 0, P->partials, P->sc);
    }
    if (R.anchor) {
      // r's unreached-component means, then <r, r>_V of the anchored residual
      subtract_unreached_means(P, P->r, s);
      st->unreached_set_mean_projection_count += 1;
      EFSI_COUNTED k_residual_reduce<<<R.S.grid, R.S.block, 0, s>>>(R.L, P->r, remove_mean ? 1 : 0, P->partials, P->sc);
    }
    if (remove_mean) {
      EFSI_COUNTED k_sub_mean_r<<<R.S.grid, R.S.block, 0, s>>>(R.L, P->r, P->partials, P->sc);
      st->mean_projection_count += 1;
    }
    EFSI_LAUNCH_CHECK();
    if (device) return EFSI_OK;
    EFSI_TRY(read_scalars(R));
    st->host_residual_checks += 1;
    return EFSI_OK;
  };
  EFSI_TRY(true_residual());
  double r_norm = device ? 1.0 : std::sqrt(std::max(P->host_sc->rr, 0.0));
  st->initial_relative_residual = r_norm / b_norm;
  st->relative_residual = st->initial_relative_residual;
  if (!device && r_norm <= tol * b_norm) {
    st->converged = 1;
    return EFSI_OK;
  }
  // 4: the learned network; the flexible beta of the V-cycle path applies to
  // it, and the 2/24/2 V-cycle (or Jacobi when no V-cycle applies) takes over
  // when it stalls.
  if (prm->precond == 4 || prm->precond == 5) {
    EFSI_ARG_CHECK(P->unet != nullptr && P->unet_in != nullptr,
                   "cg_preconditioner 'learned' needs a network (efsi_fv_set_learned_preconditioner)");
  }
  const bool mg_possible = P->n_levels > 1 && !prm->iface_active;
  R.learned = prm->precond == 4 || prm->precond == 5;
  const bool learned_fallback = prm->precond == 4;
  R.use_mg = R.learned || (mg_possible && (prm->precond == 1 || prm->precond == 2 || prm->precond == 3));
  // 3: the FP32 level-0 V-cycle.  It needs the plane-marching kernels on
  // level 0 with TMA maps of all three fields (mask rows of 16-byte multiples:
  // nz % 16 == 0) and no interface diagonal; otherwise the f64 V-cycle runs.
  R.mixed = R.use_mg && prm->precond == 3 && P->lv[0].march && P->lv[0].nz % 16 == 0 && !P->has_iface;
  R.pre = prm->precond == 2 ? 1 : 2;
  R.coarse = prm->precond == 2 ? 12 : 24;
  R.post = prm->precond == 2 ? 1 : 2;
  R.d_cur = P->d0;
  R.d_nxt = P->d1;
  // Initial preconditioning and rz (fluid.py:6644-6673).
  EFSI_TRY(precondition(R));
  if (remove_mean) st->mean_projection_count += 1;
  if (R.anchor) st->unreached_set_mean_projection_count += 1;
  EFSI_COUNTED launch_pdl(k_cg_dots<false, true>, R.S.grid, R.S.block, 0, s, R.L, P->r, P->z, nullptr, P->partials, P->sc);
  if (R.dots_fused) EFSI_COUNTED launch_pdl(k_clear_code, 1, 32, 0, s, P->sc);
  EFSI_LAUNCH_CHECK();
  if (!device) EFSI_TRY(read_scalars(R));
  double rz = device ? 1.0 : P->host_sc->rz;
  if (R.learned && learned_fallback && (!std::isfinite(rz) || rz <= 0.0)) {
    // the network's first z is not a descent direction: the V-cycle takes over
    R.learned = false;
    R.use_mg = mg_possible;
    EFSI_TRY(precondition(R));
    EFSI_COUNTED launch_pdl(k_cg_dots<false, true>, R.S.grid, R.S.block, 0, s, R.L, P->r, P->z, nullptr, P->partials, P->sc);
    EFSI_LAUNCH_CHECK();
    EFSI_TRY(read_scalars(R));
    rz = P->host_sc->rz;
  }
  if (!std::isfinite(rz) || std::fabs(rz) <= 1.0e-300) {
    // Downgrade to Jacobi; the reference does not re-project z here.
    R.use_mg = false;
    EFSI_COUNTED launch_pdl(k_jacobi_precond, R.S.grid, R.S.block, 0, s, R.L, P->diag, P->r, P->z, 0, P->partials, P->sc);
    EFSI_COUNTED launch_pdl(k_set_zproj, 1, 32, 0, s, P->sc, 0);
    EFSI_COUNTED launch_pdl(k_cg_dots<false, true>, R.S.grid, R.S.block, 0, s, R.L, P->r, P->z, nullptr, P->partials, P->sc);
    EFSI_LAUNCH_CHECK();
    EFSI_TRY(read_scalars(R));
    rz = P->host_sc->rz;
  }
  st->used_mg = R.use_mg ? 1 : 0;
  if (!std::isfinite(rz) || rz <= 0.0) {
    st->breakdown_reason = 1;
    return EFSI_OK;
  }
  R.copy_next = true;
  const int restart_interval = prm->iface_active ? 256 : 512;
  const double n0d = (double)n0;
  // --- launch pieces of one iteration -------------------------------------
  const bool tiled0 = P->lv[0].tiled;
  const unsigned tg0 = P->lv[0].tgrid;
  const dim3 tblk(kTK, kTJ);
  const bool march0 = P->lv[0].march;
  auto launch_spmv_operator = [&](bool copy, double* d_old, double* d_new) {
    if (march0) {
      bool done = false;
      EFSI_TIMED(KF_SPMV_DIR, (copy ? 25.0 : 33.0) * n0d, s,
                 done = launch_march_spmv(P, R.L, copy, P->z, d_old, d_new, P->Ad, outlet, P->partials, P->sc, s));
      if (done) return;
    }
    if (tiled0) {
      if (copy)
        EFSI_TIMED(KF_SPMV_DIR, 25.0 * n0d, s,
                   EFSI_COUNTED launch_pdl(kt_spmv_dir<true>, tg0, tblk, 0, s, R.L, P->z, d_old, d_new, P->Ad, outlet,
                                                                       P->partials, P->sc));
      else
        EFSI_TIMED(KF_SPMV_DIR, 33.0 * n0d, s,
                   EFSI_COUNTED launch_pdl(kt_spmv_dir<false>, tg0, tblk, 0, s, R.L, P->z, d_old, d_new, P->Ad, outlet,
                                                                        P->partials, P->sc));
      return;
    }
    if (copy)
      EFSI_TIMED(KF_SPMV_DIR, 25.0 * n0d, s,
                 EFSI_COUNTED launch_pdl(k_spmv_dir<true>, R.S.grid, R.S.block, 0, s, R.L, P->z, d_old, d_new, P->Ad, outlet,
                                                                              P->partials, P->sc));
    else
      EFSI_TIMED(KF_SPMV_DIR, 33.0 * n0d, s,
                 EFSI_COUNTED launch_pdl(k_spmv_dir<false>, R.S.grid, R.S.block, 0, s, R.L, P->z, d_old, d_new, P->Ad, outlet,
                                                                               P->partials, P->sc));
  };
  auto launch_spmv = [&](bool copy, double* d_old, double* d_new) {
    launch_spmv_operator(copy, d_old, d_new);
    if (coupled) {
      // Ad += C d, then <d, Ad>_V and alpha (the SpMV's finisher deferred them)
      EFSI_COUNTED launch_pdl(k_couple, 148, 256, 0, s, (const int32_t*)P->cpl_rows, (const int32_t*)P->cpl_ptr,
                              (const int32_t*)P->cpl_src, (const double*)P->cpl_coef, (const int32_t*)P->cpl_n,
                              (const double*)d_new, P->Ad, 0);
      EFSI_COUNTED launch_pdl(k_dot_alpha, R.S.grid, R.S.block, 0, s, R.L, (const double*)d_new, (const double*)P->Ad,
                              P->partials, P->sc);
    }
  };
  // The halves of an update on two streams: r and delta (which the
  // preconditioner reads) on `s`, x on the plan's side stream, joined back
  // by join_update() before the next SpMV.  Only the tiled multigrid path
  // splits, and only where the update forms no sums.
  static const bool no_split = std::getenv("EFSI_NO_SPLIT_UPDATE") != nullptr;
  const bool split_ok = !no_split && tiled0 && R.use_mg;
  static const bool no_zero0 = std::getenv("EFSI_NO_UPDATE_SWEEP0") != nullptr;
  const bool zero0_ok = !no_zero0 && P->lv[0].march && P->n_levels > 1;
  if (split_ok && P->side_stream == nullptr) {
    EFSI_CUDA_CHECK(cudaStreamCreateWithFlags(&P->side_stream, cudaStreamNonBlocking));
    EFSI_CUDA_CHECK(cudaEventCreateWithFlags(&P->ev_fork, cudaEventDisableTiming));
    EFSI_CUDA_CHECK(cudaEventCreateWithFlags(&P->ev_join, cudaEventDisableTiming));
  }
  bool joined = true;
  auto join_update = [&]() {
    if (!joined) cudaStreamWaitEvent(s, P->ev_join, 0);
    joined = true;
  };
  auto launch_update = [&](double* d, bool mean_now, bool want_rr, bool may_split = false) {
    if (may_split && split_ok && !mean_now && !want_rr) {
      cudaEventRecord(P->ev_fork, s);
      cudaStreamWaitEvent(P->side_stream, P->ev_fork, 0);
      EFSI_COUNTED kt_cg_update<true, 1><<<tg0, tblk, 0, P->side_stream>>>(R.L, pressure, d, P->r, P->Ad, P->delta, 0,
                                                                          0, P->partials, P->sc);
      cudaEventRecord(P->ev_join, P->side_stream);
      joined = false;
      // with the plane-marching f64 V-cycle next, the r half also forms its
      // first level-0 sweep (with the reciprocal denominators)
      const int o = outlet ? 1 : 0;
      if (zero0_ok && !R.learned && R.mixed) {
        EFSI_COUNTED launch_pdl(kt_cg_update_r_zero<float>, tg0, tblk, 0, s, R.L, P->r, (const double*)P->Ad, P->delta,
                                (const double*)nullptr, (float*)P->lv[0].pa32, (double)0.8f, outlet, P->sc);
        R.zero0_ready = true;
        return;
      }
      if (zero0_ok && P->rden_ok[o] && !R.learned && !R.mixed) {
        EFSI_COUNTED launch_pdl(kt_cg_update_r_zero<double>, tg0, tblk, 0, s, R.L, P->r, (const double*)P->Ad,
                                P->delta, (const double*)P->rden[o], (double*)P->lv[0].pa, (double)0.8f, outlet,
                                P->sc);
        R.zero0_ready = true;
        return;
      }
      EFSI_COUNTED launch_pdl(kt_cg_update<true, 2>, tg0, tblk, 0, s, R.L, pressure, d, P->r, P->Ad, P->delta, 0, 0,
                              P->partials, P->sc);
      return;
    }
    join_update();
    if (tiled0) {
      if (R.use_mg)
        EFSI_TIMED(KF_CG_UPDATE, 56.0 * n0d, s,
                   EFSI_COUNTED launch_pdl(kt_cg_update<true>, tg0, tblk, 0, s, R.L, pressure, d, P->r, P->Ad, P->delta,
                                                                        mean_now ? 1 : 0, want_rr ? 1 : 0,
                                                                        P->partials, P->sc));
      else
        EFSI_TIMED(KF_CG_UPDATE, 48.0 * n0d, s,
                   EFSI_COUNTED launch_pdl(kt_cg_update<false>, tg0, tblk, 0, s, R.L, pressure, d, P->r, P->Ad, nullptr,
                                                                         mean_now ? 1 : 0, want_rr ? 1 : 0,
                                                                         P->partials, P->sc));
      if (mean_now) EFSI_COUNTED launch_pdl(kt_sub_mean_xr, tg0, tblk, 0, s, R.L, pressure, P->r, P->partials, P->sc);
      return;
    }
    if (R.use_mg)
      EFSI_TIMED(KF_CG_UPDATE, 56.0 * n0d, s,
                 EFSI_COUNTED launch_pdl(k_cg_update<true>, R.S.grid, R.S.block, 0, s, R.L, pressure, d, P->r, P->Ad, P->delta,
                                                                               mean_now ? 1 : 0, want_rr ? 1 : 0,
                                                                               P->partials, P->sc));
    else
      EFSI_TIMED(KF_CG_UPDATE, 48.0 * n0d, s,
                 EFSI_COUNTED launch_pdl(k_cg_update<false>, R.S.grid, R.S.block, 0, s, R.L, pressure, d, P->r, P->Ad, nullptr,
                                                                                mean_now ? 1 : 0, want_rr ? 1 : 0,
                                                                                P->partials, P->sc));
    if (mean_now)
      EFSI_COUNTED launch_pdl(k_sub_mean_xr, R.S.grid, R.S.block, 0, s, R.L, pressure, P->r, P->partials, P->sc);
  };
  // every 16th iteration of an anchored solve (fluid.py:6682-6684): the
  // pressure's and the residual's unreached-component means, then <r, r>_V
  auto anchor_pressure_residual = [&](bool want_rr) {
    subtract_unreached_means(P, pressure, s);
    subtract_unreached_means(P, P->r, s);
    if (want_rr)
      EFSI_COUNTED launch_pdl(k_residual_reduce, R.S.grid, R.S.block, 0, s, R.L, (const double*)P->r, 0, P->partials,
                              P->sc);
  };
  auto launch_precond_dots = [&]() -> int {
    EFSI_TRY(precondition(R));
    if (R.dots_fused) return EFSI_OK;
    if (tiled0) {
      if (R.use_mg)
        EFSI_TIMED(KF_CG_DOTS, 25.0 * n0d, s,
                   EFSI_COUNTED launch_pdl(kt_cg_dots<true, false>, tg0, tblk, 0, s, R.L, P->r, P->z, P->delta, P->partials,
                                                                             P->sc));
      else
        EFSI_TIMED(KF_CG_DOTS, 17.0 * n0d, s,
                   EFSI_COUNTED launch_pdl(kt_cg_dots<false, false>, tg0, tblk, 0, s, R.L, P->r, P->z, nullptr, P->partials,
                                                                              P->sc));
      return EFSI_OK;
    }
    if (R.use_mg)
      EFSI_TIMED(KF_CG_DOTS, 25.0 * n0d, s,
                 EFSI_COUNTED launch_pdl(k_cg_dots<true, false>, R.S.grid, R.S.block, 0, s, R.L, P->r, P->z, P->delta,
                                                                                    P->partials, P->sc));
    else
      EFSI_TIMED(KF_CG_DOTS, 17.0 * n0d, s,
                 EFSI_COUNTED launch_pdl(k_cg_dots<false, false>, R.S.grid, R.S.block, 0, s, R.L, P->r, P->z, nullptr,
                                                                                     P->partials, P->sc));
    return EFSI_OK;
  };
  // --- one 16-iteration block (iterations 16k+1 .. 16k+16), optionally as a
  // CUDA graph.  `cont`: the block starts with the preconditioner and dots of
  // the previous block's last iteration; otherwise it starts a new direction.
  auto launch_block = [&](bool cont) -> int {
    if (cont) EFSI_TRY(launch_precond_dots());
    double* d[2] = {P->d0, P->d1};
    for (int j = 0; j < 16; ++j) {
      join_update();  // the previous x half reads the direction this SpMV rewrites two iterations on
      launch_spmv(!cont && j == 0, d[j & 1], d[(j + 1) & 1]);
      const bool last = (j == 15);
      // (the last update of the block is whole: the check reads x)
      launch_update(d[(j + 1) & 1], last && remove_mean, last && !remove_mean && !R.anchor, !last);
      if (last && R.anchor) anchor_pressure_residual(true);
      if (!last) EFSI_TRY(launch_precond_dots());
    }
    join_update();
    EFSI_LAUNCH_CHECK();
    return EFSI_OK;
  };
  auto run_block = [&](bool cont) -> int {
    if (!prm->use_graphs || P->graphs_disabled) return launch_block(cont);
    PcgGraphKey key{cont, R.use_mg, remove_mean, outlet, R.pre, R.coarse, R.post, pressure, R.mixed};
    key.learned = R.learned;
    key.coupled = coupled;
    key.anchor = R.anchor;
    cudaGraphExec_t exec = nullptr;
    for (auto& g : P->graphs)
      if (g.key == key) exec = g.exec;
    if (exec == nullptr) {
      // Capture on the plan's private stream (the caller's may be the legacy
      // default stream, which cannot be captured); the graph runs on `s`.
      cudaGraph_t graph = nullptr;
      const cudaStream_t launch_stream = s;
      s = P->cap_stream;
      R.s = P->cap_stream;
      set_capturing(true);
      take_capture_count();
      cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
      int rc = e == cudaSuccess ? launch_block(cont) : EFSI_ERR_CUDA;
      cudaError_t e2 = cudaStreamEndCapture(s, &graph);
      set_capturing(false);
      const unsigned long long nodes = take_capture_count();
      s = launch_stream;
      R.s = launch_stream;
      cudaError_t e3 = cudaSuccess;
      if (e == cudaSuccess && rc == EFSI_OK && e2 == cudaSuccess) e3 = cudaGraphInstantiate(&exec, graph, 0);
      if (graph != nullptr) cudaGraphDestroy(graph);
      if (e != cudaSuccess || rc != EFSI_OK || e2 != cudaSuccess || e3 != cudaSuccess) {
        // Record why and run this block with direct launches instead.
        P->graph_error = std::string("begin: ") + cudaGetErrorString(e) + "; block: " + std::to_string(rc) + " (" +
                         g_err + "); end: " + cudaGetErrorString(e2) + "; instantiate: " + cudaGetErrorString(e3);
        cudaGetLastError();
        P->graphs_disabled = true;
        return launch_block(cont);
      }
      P->graphs.push_back({key, exec, nodes});
    }
    unsigned long long nodes_now = 0;
    for (auto& g : P->graphs)
      if (g.exec == exec) nodes_now = g.nodes;
    EFSI_CUDA_CHECK(cudaGraphLaunch(exec, s));
    count_graph_launch(nodes_now);
    return EFSI_OK;
  };
  if (device) return pcg_device_loop(P, R, st, s, pressure, tol, max_iters, n0, [&](cudaStream_t bs) -> int {
    // one iteration block of the loop body: 16 x (direction + SpMV + alpha,
    // update, preconditioner + dots for the next one), as launch_block does
    // after its first iteration
    const cudaStream_t keep = s;
    s = bs;
    R.s = bs;
    double* d[2] = {P->d0, P->d1};
    int rc = EFSI_OK;
    for (int j = 0; j < 16 && rc == EFSI_OK; ++j) {
      join_update();
      launch_spmv(false, d[j & 1], d[(j + 1) & 1]);
      const bool last = (j == 15);
      launch_update(d[(j + 1) & 1], last && remove_mean, last && !remove_mean && !R.anchor, !last);
      if (last && R.anchor) anchor_pressure_residual(true);
      rc = launch_precond_dots();
    }
    join_update();
    s = keep;
    R.s = keep;
    return rc;
  });
  bool pending = false;  // preconditioner + dots of the previous iteration not launched yet
  int n_precond = 0;     // preconditioner applications inside the loop
  int it = 1;
  // the learned preconditioner must cut the residual by this factor over every
  // 16-iteration block, or the V-cycle takes over
  constexpr double kLearnedBlockReduction = 0.5;
  double learned_prev = st->initial_relative_residual;
  while (it <= max_iters) {
    const bool block = ((it - 1) % 16 == 0) && (it + 15 <= max_iters) && (pending || R.copy_next);
    if (block) {
      // d0 holds the current direction at every block start (16 swaps per block)
      EFSI_TRY(run_block(pending));
      n_precond += 15;
      it += 15;
      pending = false;
      R.copy_next = false;
    } else {
      if (pending) EFSI_TRY(launch_precond_dots());
      pending = false;
      double* d_old = ((it - 1) & 1) ? P->d1 : P->d0;
      double* d_new = ((it - 1) & 1) ? P->d0 : P->d1;
      launch_spmv(R.copy_next, d_old, d_new);
      R.copy_next = false;
      const bool mean_now = remove_mean && (it % 16 == 0);
      const bool anchor_now = R.anchor && (it % 16 == 0);
      const bool check_now = (it % 16 == 0) || it == max_iters;
      launch_update(d_new, mean_now, check_now && !mean_now && !anchor_now);
      if (anchor_now) anchor_pressure_residual(check_now && !mean_now);
      EFSI_LAUNCH_CHECK();
    }
    if (remove_mean && it % 16 == 0) st->mean_projection_count += 2;
    if (R.anchor && it % 16 == 0) st->unreached_set_mean_projection_count += 2;
    st->iterations = it;
    const bool check = (it % 16 == 0) || it == max_iters;
    if (!check) {
      pending = true;
      ++n_precond;
      ++it;
      continue;
    }
    EFSI_TRY(read_scalars(R));
    st->host_residual_checks += 1;
    r_norm = std::sqrt(std::max(P->host_sc->rr, 0.0));
    st->relative_residual = r_norm / b_norm;
    if (R.learned) {
      st->learned_iterations = it;
      st->learned_relative_residual = st->relative_residual;
    }
    if (st->relative_residual <= tol) {
      st->converged = 1;
      break;
    }
    const int code = P->host_sc->code;
    if (R.learned && learned_fallback && it < max_iters &&
        (code != 0 || !(st->relative_residual <= kLearnedBlockReduction * learned_prev))) {
      // fallback: restart from the exact residual with the V-cycle
      R.learned = false;
      R.use_mg = mg_possible;
      EFSI_TRY(true_residual());
      r_norm = std::sqrt(std::max(P->host_sc->rr, 0.0));
      st->relative_residual = r_norm / b_norm;
      if (st->relative_residual <= tol) {
        st->converged = 1;
        break;
      }
      EFSI_TRY(precondition(R));
      if (remove_mean) st->mean_projection_count += 1;
      if (R.anchor) st->unreached_set_mean_projection_count += 1;
      EFSI_COUNTED launch_pdl(k_cg_dots<false, true>, R.S.grid, R.S.block, 0, s, R.L, P->r, P->z, nullptr, P->partials, P->sc);
      EFSI_LAUNCH_CHECK();
      EFSI_TRY(read_scalars(R));
      rz = P->host_sc->rz;
      CgScalars* hs = P->host_sc;
      hs->code = 0;
      hs->code_dAd = 0.0;
      EFSI_CUDA_CHECK(cudaMemcpyAsync(&P->sc->code, &hs->code, sizeof(int), cudaMemcpyHostToDevice, s));
      EFSI_CUDA_CHECK(cudaMemcpyAsync(&P->sc->code_dAd, &hs->code_dAd, sizeof(double), cudaMemcpyHostToDevice, s));
      EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
      if (!std::isfinite(rz) || rz <= 0.0) {
        st->breakdown_reason = 3;
        break;
      }
      R.copy_next = true;
      pending = false;
      st->restart_count += 1;
      ++it;
      continue;
    }
    if (R.learned) learned_prev = st->relative_residual;
    if (code != 0) {
      st->breakdown_dAd = P->host_sc->code_dAd;
      if (it < max_iters) {
        EFSI_TRY(true_residual());
        r_norm = std::sqrt(std::max(P->host_sc->rr, 0.0));
        st->relative_residual = r_norm / b_norm;
        if (st->relative_residual <= tol) {
          st->converged = 1;
          break;
        }
        EFSI_TRY(precondition(R));
        if (remove_mean) st->mean_projection_count += 1;
        if (R.anchor) st->unreached_set_mean_projection_count += 1;
        EFSI_COUNTED launch_pdl(k_cg_dots<false, true>, R.S.grid, R.S.block, 0, s, R.L, P->r, P->z, nullptr, P->partials, P->sc);
        EFSI_LAUNCH_CHECK();
        EFSI_TRY(read_scalars(R));
        rz = P->host_sc->rz;
        if (std::isfinite(rz) && rz > 0.0) {
          // clear the device code (fluid.py:6728-6729)
          CgScalars* hs = P->host_sc;
          hs->code = 0;
          hs->code_dAd = 0.0;
          EFSI_CUDA_CHECK(cudaMemcpyAsync(&P->sc->code, &hs->code, sizeof(int), cudaMemcpyHostToDevice, s));
          EFSI_CUDA_CHECK(cudaMemcpyAsync(&P->sc->code_dAd, &hs->code_dAd, sizeof(double), cudaMemcpyHostToDevice, s));
          EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
          R.copy_next = true;
          pending = false;
          st->restart_count += 1;
          ++it;
          continue;
        }
      }
      st->breakdown_reason = 2;
      break;
    }
    if (it < max_iters && restart_interval > 0 && it % restart_interval == 0) {
      EFSI_TRY(true_residual());
      r_norm = std::sqrt(std::max(P->host_sc->rr, 0.0));
      st->relative_residual = r_norm / b_norm;
      if (st->relative_residual <= tol) {
        st->converged = 1;
        break;
      }
      EFSI_TRY(precondition(R));
      if (remove_mean) st->mean_projection_count += 1;
      if (R.anchor) st->unreached_set_mean_projection_count += 1;
      EFSI_COUNTED launch_pdl(k_cg_dots<false, true>, R.S.grid, R.S.block, 0, s, R.L, P->r, P->z, nullptr, P->partials, P->sc);
      EFSI_LAUNCH_CHECK();
      EFSI_TRY(read_scalars(R));
      rz = P->host_sc->rz;
      if (!std::isfinite(rz) || rz <= 0.0) {
        st->breakdown_reason = 3;
        break;
      }
      R.copy_next = true;
      pending = false;
      st->restart_count += 1;
      ++it;
      continue;
    }
    pending = true;
    ++n_precond;
    ++it;
  }
  // mean projections of z: one per preconditioner application
  if (remove_mean) st->mean_projection_count += n_precond;
  if (R.anchor) st->unreached_set_mean_projection_count += n_precond;
  EFSI_TRY(read_scalars(R));
  st->used_graphs = (prm->use_graphs && !P->graphs_disabled) ? 1 : 0;
  st->breakdown_code = P->host_sc->code;
  if (st->breakdown_dAd == 0.0) st->breakdown_dAd = P->host_sc->code_dAd;
  return EFSI_OK;
}

}  // extern "C"

namespace efsi {

// Sweeps with the reference's "sweep into tmp, copy back" structure
// (fluid.py:5862-5900); used by the non-PCG pressure solvers.
template <typename TP>
static int smooth_copy(efsi_fv_plan* P, int l, TP* p, const void* rhs, int outlet, int iterations, cudaStream_t s) {
  LevelBuf& B = P->lv[l];
  ProlongSrc none{nullptr, 0, 0, 0, 0.0f};
  const double om = (double)0.8f;
  for (int it = 0; it < std::max(0, iterations); ++it) {
    launch_sweep<TP, false, false>(P, l, p, rhs, (TP*)B.pb, outlet, om, none, nullptr, s);
    EFSI_CUDA_CHECK(cudaMemcpyAsync(p, B.pb, B.n * sizeof(TP), cudaMemcpyDeviceToDevice, s));
  }
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

}  // namespace efsi

extern "C" {

int efsi_fv_multigrid_solve(efsi_fv_plan* P, const double* rhs0, double* pressure, int32_t outlet,
                            int32_t iterations, int32_t cycles, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(cycles > 0, "multigrid_cycles must be positive");
  cudaStream_t s = as_stream(stream);
  const int nl = P->n_levels;
  if (nl <= 1) return smooth_copy<double>(P, 0, pressure, rhs0, outlet, std::max(1, (int)iterations), s);
  const float scale = P->uniform ? 1.0f : 0.7f;
  for (int cyc = 0; cyc < cycles; ++cyc) {
    for (int l = 0; l < nl - 1; ++l) {
      LevelDev L = level_dev(P, l);
      LevelBuf& B = P->lv[l];
      const LevelBuf& C = P->lv[l + 1];
      if (l == 0) {
        EFSI_TRY(smooth_copy<double>(P, 0, pressure, rhs0, outlet, 3, s));
        launch_restrict<double, false>(P, 0, pressure, rhs0, outlet, s);
      } else {
        EFSI_TRY(smooth_copy<float>(P, l, (float*)B.pa, B.rhs, outlet, 3, s));
        launch_restrict<float, false>(P, l, (const float*)B.pa, B.rhs, outlet, s);
      }
      // the restriction zeroes the coarse iterate (fluid.py:5383-5385)
      EFSI_CUDA_CHECK(cudaMemsetAsync(C.pa, 0, C.n * sizeof(float), s));
    }
    EFSI_TRY(smooth_copy<float>(P, nl - 1, (float*)P->lv[nl - 1].pa, P->lv[nl - 1].rhs, outlet, 36, s));
    for (int l = nl - 2; l >= 0; --l) {
      LevelDev L = level_dev(P, l);
      LevelBuf& B = P->lv[l];
      const LevelBuf& C = P->lv[l + 1];
      ProlongSrc pr{(const float*)C.pa, C.nx, C.ny, C.nz, scale};
      if (l == 0) {
        EFSI_COUNTED k_prolong<double><<<B.shape.grid, B.shape.block, 0, s>>>(L, pressure, pr);
        EFSI_TRY(smooth_copy<double>(P, 0, pressure, rhs0, outlet, 3, s));
      } else {
        EFSI_COUNTED k_prolong<float><<<B.shape.grid, B.shape.block, 0, s>>>(L, (float*)B.pa, pr);
        EFSI_TRY(smooth_copy<float>(P, l, (float*)B.pa, B.rhs, outlet, 3, s));
      }
    }
  }
  if (!P->uniform) EFSI_TRY(smooth_copy<double>(P, 0, pressure, rhs0, outlet, std::max(1, (int)iterations), s));
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_fv_jacobi_solve(efsi_fv_plan* P, const double* rhs0, double* pressure, int32_t outlet, int32_t iterations,
                         void* stream) {
  EFSI_TRY(level_zero_check(P));
  return smooth_copy<double>(P, 0, pressure, rhs0, outlet, (int)iterations, as_stream(stream));
}

}  // extern "C"

extern "C" {

// Benchmark helper (no counterpart in the reference): launch one level-0
// kernel family `reps` times back to back on the plan's own work buffers and
// report the mean CUDA-event duration per launch and its algorithmic bytes.
// Tile autotuner of the V-cycle's per-level launches.  For every level that
// launches its own kernels (those above the single-CTA tail), each candidate
// launch shape is timed with CUDA events over `reps` back-to-back units after
// two untimed ones -- on level 0 the PCG's direction SpMV and a whole V-cycle
// with the dots fused in, on a coarse level its plain sweep and restriction
// (the sweep alone on a coarsest level without a tail): the plane-marching kernels
// with 3 (the default), 1, 2, 4 or 6 blocks' worth of planes per SM and, on
// levels >= 1, the tiled / per-cell kernels.  A candidate replaces the best so
// far only when it is more than 3% faster.  Level 0 keeps the plane march
// whenever it can run (the PCG's dots are fused into its last sweep).  Every
// candidate computes the same rows; only the block partition of the z-mean /
// dot partial sums of level 0 follows the chosen shape.  Captured PCG graphs
// are dropped, so the next solve records the tuned launches.
int efsi_fv_autotune(efsi_fv_plan* P, int32_t reps, int32_t* choice, double* best_us, int32_t max_levels,
                     void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(reps > 0 && max_levels >= 0 && (max_levels == 0 || (choice != nullptr && best_us != nullptr)),
                 "invalid autotune arguments");
  cudaStream_t s = as_stream(stream);
  int dev = 0, nsm = 0;
  EFSI_CUDA_CHECK(cudaGetDevice(&dev));
  EFSI_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  for (int l = 0; l < max_levels; ++l) {
    choice[l] = -1;
    best_us[l] = 0.0;
  }
  const int nl = P->n_levels;
  const int last = P->tail_level < nl ? P->tail_level : nl;
  const ProlongSrc none{nullptr, 0, 0, 0, 0.0f};
  const double om = (double)0.8f;
  EFSI_TRY(ensure_rden(P, 0, s));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  EFSI_CUDA_CHECK(cudaEventCreate(&e0));
  EFSI_CUDA_CHECK(cudaEventCreate(&e1));
  int rc = EFSI_OK;
  for (int l = 0; l < last && rc == EFSI_OK; ++l) {
    LevelBuf& B = P->lv[l];
    std::vector<int> cands;
    if (B.march_ok) {
      cands = {3, 1, 2, 4, 6};
      if (l > 0) cands.push_back(0);
    } else {
      cands = {0};
    }
    auto apply = [&](int m) {
      if (m == 0) {
        B.march = false;
      } else {
        const MarchCfg mc = march_cfg(B.nx, B.ny, B.nz, nsm * m);
        B.march = true;
        B.mchunk = mc.chunk;
        B.mgrid = mc.grid;
      }
    };
    auto pair = [&]() {
      if (l == 0) {
        // level 0: the direction SpMV and a whole V-cycle with the PCG dots
        // fused in (every level-0 plane march of a PCG iteration)
        const LevelDev L0 = level_dev(P, 0);
        if (!launch_march_spmv(P, L0, false, P->z, P->d0, P->d1, P->Ad, 0, P->partials, P->sc, s))
          launch_sweep<double, true, false>(P, 0, (const double*)B.pa, P->r, (double*)B.pb, 0, om, none, nullptr, s);
        bool fused = false;
        if (vcycle(P, P->r, P->z, 0, 2, 24, 2, true, s, P->delta, &fused) != EFSI_OK) rc = EFSI_ERR_CUDA;
      } else {
        launch_sweep<float, false, false>(P, l, (const float*)B.pa, B.rhs, (float*)B.pb, 0, om, none, nullptr, s);
        if (l + 1 < nl) launch_restrict<float, false>(P, l, (const float*)B.pa, B.rhs, 0, s);
      }
    };
    int best = cands[0];
    float best_ms = 0.0f;
    for (size_t q = 0; q < cands.size(); ++q) {
      apply(cands[q]);
      for (int w = 0; w < 2; ++w) pair();
      cudaEventRecord(e0, s);
      for (int r = 0; r < reps; ++r) pair();
      cudaEventRecord(e1, s);
      cudaError_t e = cudaEventSynchronize(e1);
      if (e == cudaSuccess) e = cudaGetLastError();
      if (e != cudaSuccess) {
        set_error(std::string("autotune: ") + cudaGetErrorString(e));
        rc = EFSI_ERR_CUDA;
        break;
      }
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (q == 0 || ms < 0.97f * best_ms) {
        best = cands[q];
        best_ms = ms;
      }
    }
    apply(best);
    if (l < max_levels) {
      choice[l] = best;
      best_us[l] = 1000.0 * (double)best_ms / reps;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (PcgGraph& g : P->graphs) cudaGraphExecDestroy(g.exec);
  P->graphs.clear();
  return rc;
}

int efsi_fv_kernel_replay(efsi_fv_plan* P, int32_t family, int32_t reps, double* avg_ms, double* bytes_per_launch,
                          void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(reps > 0 && avg_ms && bytes_per_launch, "invalid replay arguments");
  cudaStream_t s = as_stream(stream);
  LevelDev L = level_dev(P, 0);
  const Shape3& S = P->lv[0].shape;
  const double n0 = (double)P->lv[0].n;
  ProlongSrc none{nullptr, 0, 0, 0, 0.0f};
  const double om = (double)0.8f;
  double bytes = 0.0;
  auto one = [&]() -> int {
    switch (family) {
      case KF_SPMV_DIR:
        bytes = 33.0 * n0;
        if (P->lv[0].march && launch_march_spmv(P, L, false, P->z, P->d0, P->d1, P->Ad, 0, P->partials, P->sc, s))
          break;
        if (P->lv[0].tiled)
          EFSI_COUNTED launch_pdl(kt_spmv_dir<false>, P->lv[0].tgrid, dim3(kTK, kTJ), 0, s, L, P->z, P->d0, P->d1, P->Ad, 0,
                                                                                    P->partials, P->sc);
        else
          EFSI_COUNTED launch_pdl(k_spmv_dir<false>, S.grid, S.block, 0, s, L, P->z, P->d0, P->d1, P->Ad, 0, P->partials,
                                                                    P->sc);
        break;
      case KF_SWEEP_L0:
        bytes = 25.0 * n0;
        launch_sweep<double, true, false>(P, 0, (const double*)P->lv[0].pa, P->r, (double*)P->lv[0].pb, 0, om, none,
                                          nullptr, s);
        break;
      case KF_CG_UPDATE:
        bytes = 56.0 * n0;
        if (P->lv[0].tiled)
          EFSI_COUNTED launch_pdl(kt_cg_update<true>, P->lv[0].tgrid, dim3(kTK, kTJ), 0, s, L, P->b, P->d0, P->diag, P->Ad,
                                                                                    P->delta, 0, 0, P->partials,
                                                                                    P->sc);
        else
          EFSI_COUNTED launch_pdl(k_cg_update<true>, S.grid, S.block, 0, s, L, P->b, P->d0, P->diag, P->Ad, P->delta, 0, 0,
                                                                    P->partials, P->sc);
        break;
      case KF_RESTRICT_L0: {
        if (P->n_levels < 2) {
          set_error("replay of the restriction needs two levels");
          return EFSI_ERR_ARG;
        }
        const LevelBuf& C = P->lv[1];
        // as in the V-cycle: with level 1's zero-guess sweep when it is fused
        float* cz = vcycle_fuses_zero(P, 1) ? (float*)C.pa : nullptr;
        bytes = 17.0 * n0 + (cz ? 9.0 : 4.0) * (double)C.n;
        launch_restrict<double, true>(P, 0, (const double*)P->lv[0].pa, P->r, 0, s, cz, (double)0.8f);
        break;
      }
      case KF_CG_DOTS:
        bytes = 25.0 * n0;
        if (P->lv[0].tiled)
          EFSI_COUNTED launch_pdl(kt_cg_dots<true, false>, P->lv[0].tgrid, dim3(kTK, kTJ), 0, s, L, P->r, P->z, P->delta,
                                                                                         P->partials, P->sc);
        else
          EFSI_COUNTED launch_pdl(k_cg_dots<true, false>, S.grid, S.block, 0, s, L, P->r, P->z, P->delta, P->partials, P->sc);
        break;
      case 16:  // zero-guess level-0 sweep
        bytes = 17.0 * n0;
        launch_sweep<double, true, true>(P, 0, nullptr, P->r, (double*)P->lv[0].pb, 0, om, none, nullptr, s);
        break;
      case 17: {  // level-0 sweep with the prolongation from level 1 fused in
        if (P->n_levels < 2) {
          set_error("replay of the prolongation sweep needs two levels");
          return EFSI_ERR_ARG;
        }
        const LevelBuf& C = P->lv[1];
        ProlongSrc pr{(const float*)C.pa, C.nx, C.ny, C.nz, P->uniform ? 1.0f : 0.7f};
        bytes = 25.0 * n0 + 4.0 * (double)C.n;
        launch_sweep<double, true, false>(P, 0, (const double*)P->lv[0].pa, P->r, (double*)P->lv[0].pb, 0, om, pr,
                                          nullptr, s);
        break;
      }
      case 18: {  // the V-cycle's last level-0 sweep with the PCG dots finished in it
        bool fused = false;
        bytes = 33.0 * n0;
        launch_sweep<double, true, false>(P, 0, (const double*)P->lv[0].pa, P->r, (double*)P->lv[0].pb, 0, om, none,
                                          P->partials, s, P->delta, &fused);
        break;
      }
      case 19: {  // one whole MG preconditioner application (2 / 24 / 2), dots included
        bool fused = false;
        bytes = 0.0;  // time only
        EFSI_TRY(vcycle(P, P->r, P->z, 0, 2, 24, 2, true, s, P->delta, &fused));
        break;
      }
      default:
        set_error("family not supported by the replay");
        return EFSI_ERR_ARG;
    }
    return EFSI_OK;
  };
  EFSI_TRY(one());  // warm-up
  cudaEvent_t a, b;
  EFSI_CUDA_CHECK(cudaEventCreate(&a));
  EFSI_CUDA_CHECK(cudaEventCreate(&b));
  EFSI_CUDA_CHECK(cudaEventRecord(a, s));
  for (int q = 0; q < reps; ++q) EFSI_TRY(one());
  EFSI_CUDA_CHECK(cudaEventRecord(b, s));
  EFSI_CUDA_CHECK(cudaEventSynchronize(b));
  float ms = 0.0f;
  EFSI_CUDA_CHECK(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  EFSI_LAUNCH_CHECK();
  *avg_ms = (double)ms / reps;
  *bytes_per_launch = bytes;
  return EFSI_OK;
}

}  // extern "C"

namespace efsi {
namespace {
__global__ void k_cg_alpha(CgScalars* sc) { cg_alpha_step(sc, sc->dAd); }
__global__ void k_cg_beta(CgScalars* sc, int mg) { cg_beta_step(sc, sc->rz_new, sc->beta_num, mg != 0); }
}  // namespace
}  // namespace efsi

extern "C" {

int efsi_cg_scalars_write(efsi_fv_plan* P, const efsi_cg_scalar_values* v, void* stream) {
  EFSI_ARG_CHECK(P != nullptr && v != nullptr, "null argument");
  cudaStream_t s = as_stream(stream);
  CgScalars* h = P->host_sc;
  EFSI_CUDA_CHECK(cudaMemcpyAsync(h, P->sc, sizeof(CgScalars), cudaMemcpyDeviceToHost, s));
  EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  h->rz = v->rz;
  h->rz_new = v->rz_new;
  h->dAd = v->dAd;
  h->beta_num = v->beta_numerator;
  h->alpha = v->alpha;
  h->beta = v->beta;
  h->code_dAd = v->breakdown_dAd;
  h->code = v->breakdown_code;
  EFSI_CUDA_CHECK(cudaMemcpyAsync(P->sc, h, sizeof(CgScalars), cudaMemcpyHostToDevice, s));
  EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  return EFSI_OK;
}

int efsi_cg_scalars_read(efsi_fv_plan* P, efsi_cg_scalar_values* v, void* stream) {
  EFSI_ARG_CHECK(P != nullptr && v != nullptr, "null argument");
  cudaStream_t s = as_stream(stream);
  const CgScalars* h = P->host_sc;
  EFSI_CUDA_CHECK(cudaMemcpyAsync(P->host_sc, P->sc, sizeof(CgScalars), cudaMemcpyDeviceToHost, s));
  EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  v->rz = h->rz;
  v->rz_new = h->rz_new;
  v->dAd = h->dAd;
  v->beta_numerator = h->beta_num;
  v->alpha = h->alpha;
  v->beta = h->beta;
  v->breakdown_dAd = h->code_dAd;
  v->breakdown_code = h->code;
  return EFSI_OK;
}

int efsi_cg_compute_alpha(efsi_fv_plan* P, void* stream) {
  EFSI_ARG_CHECK(P != nullptr, "null plan");
  EFSI_COUNTED k_cg_alpha<<<1, 1, 0, as_stream(stream)>>>(P->sc);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_cg_compute_beta(efsi_fv_plan* P, int32_t use_mg, void* stream) {
  EFSI_ARG_CHECK(P != nullptr, "null plan");
  EFSI_COUNTED k_cg_beta<<<1, 1, 0, as_stream(stream)>>>(P->sc, use_mg);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

}  // extern "C"

extern "C" {

int efsi_fv_set_learned_preconditioner(efsi_fv_plan* P, efsi_unet* net, void* stream) {
  EFSI_TRY(level_zero_check(P));
  cudaStream_t s = as_stream(stream);
  EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  if (net == nullptr) {
    P->unet = nullptr;
    return EFSI_OK;
  }
  const LevelBuf& B = P->lv[0];
  EFSI_TRY(unet_prepare(net, B.nx, B.ny, B.nz));
  if (P->unet_in == nullptr) EFSI_CUDA_CHECK(cudaMalloc(&P->unet_in, (size_t)B.n * 16 * sizeof(__nv_bfloat16)));
  // finest width per axis, for the input's width channels
  const float* w[3] = {B.wx, B.wy, B.wz};
  const int n[3] = {B.nx, B.ny, B.nz};
  for (int a = 0; a < 3; ++a) {
    std::vector<float> h((size_t)n[a]);
    EFSI_CUDA_CHECK(cudaMemcpy(h.data(), w[a], n[a] * sizeof(float), cudaMemcpyDeviceToHost));
    P->unet_wmin[a] = *std::min_element(h.begin(), h.end());
  }
  P->unet = net;
  // graphs captured with another network's buffers are not reused
  for (PcgGraph& g : P->graphs) cudaGraphExecDestroy(g.exec);
  P->graphs.clear();
  return EFSI_OK;
}

int efsi_fv_set_unreached_components(efsi_fv_plan* P, const int32_t* comp, int32_t ncomp, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(ncomp >= 0 && ncomp <= kMaxUnreachedComponents, "ncomp must lie in [0, 256]");
  EFSI_ARG_CHECK(ncomp == 0 || comp != nullptr, "null component array");
  cudaStream_t s = as_stream(stream);
  if (ncomp > 0) {
    const size_t n = (size_t)P->lv[0].n;
    if (P->ucomp == nullptr) EFSI_CUDA_CHECK(cudaMalloc(&P->ucomp, n * sizeof(int32_t)));
    if (P->ucomp_acc == nullptr)
      EFSI_CUDA_CHECK(cudaMalloc(&P->ucomp_acc, 2 * kMaxUnreachedComponents * sizeof(double)));
    EFSI_CUDA_CHECK(cudaMemcpyAsync(P->ucomp, comp, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  }
  P->ucomp_n = ncomp;
  return EFSI_OK;
}

int efsi_fv_subtract_unreached_means(efsi_fv_plan* P, double* field, double* sums_host, double* volumes_host,
                                     void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(field != nullptr, "null field");
  if (P->ucomp_n <= 0) return EFSI_OK;
  cudaStream_t s = as_stream(stream);
  subtract_unreached_means(P, field, s);
  EFSI_LAUNCH_CHECK();
  if (sums_host != nullptr || volumes_host != nullptr) {
    const int nc = P->ucomp_n;
    if (sums_host != nullptr)
      EFSI_CUDA_CHECK(cudaMemcpyAsync(sums_host, P->ucomp_acc, nc * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (volumes_host != nullptr)
      EFSI_CUDA_CHECK(cudaMemcpyAsync(volumes_host, P->ucomp_acc + kMaxUnreachedComponents, nc * sizeof(double),
                                      cudaMemcpyDeviceToHost, s));
    EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  }
  return EFSI_OK;
}

int efsi_fv_set_interface_coupling(efsi_fv_plan* P, int32_t nrows, const int32_t* rows, const int32_t* row_ptr,
                                   const int32_t* src, const double* coef, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(nrows >= 0, "nrows must be non-negative");
  cudaStream_t s = as_stream(stream);
  EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  if (P->cpl_n == nullptr) EFSI_CUDA_CHECK(cudaMalloc(&P->cpl_n, sizeof(int32_t)));
  if (nrows == 0) {
    const int32_t zero = 0;
    EFSI_CUDA_CHECK(cudaMemcpy(P->cpl_n, &zero, sizeof(int32_t), cudaMemcpyHostToDevice));
    P->cpl_nrows = 0;
    return EFSI_OK;
  }
  EFSI_ARG_CHECK(rows != nullptr && row_ptr != nullptr && src != nullptr && coef != nullptr, "null coupling array");
  // the rows are validated on the host before they reach a kernel
  std::vector<int32_t> h_rows((size_t)nrows), h_ptr((size_t)nrows + 1);
  EFSI_CUDA_CHECK(cudaMemcpy(h_rows.data(), rows, nrows * sizeof(int32_t), cudaMemcpyDeviceToHost));
  EFSI_CUDA_CHECK(cudaMemcpy(h_ptr.data(), row_ptr, (nrows + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost));
  const int64_t n0 = P->lv[0].n;
  EFSI_ARG_CHECK(h_ptr[0] == 0, "row_ptr must start at 0");
  for (int32_t r = 0; r < nrows; ++r) {
    EFSI_ARG_CHECK(h_rows[r] >= 0 && h_rows[r] < n0, "coupling row cell out of range");
    EFSI_ARG_CHECK(h_ptr[r + 1] >= h_ptr[r], "row_ptr must not decrease");
    if (r > 0) EFSI_ARG_CHECK(h_rows[r] > h_rows[r - 1], "coupling rows must be distinct, in increasing order");
  }
  const int32_t nent = h_ptr[nrows];
  std::vector<int32_t> h_src((size_t)std::max(nent, 1));
  std::vector<double> h_coef((size_t)std::max(nent, 1));
  if (nent > 0) {
    EFSI_CUDA_CHECK(cudaMemcpy(h_src.data(), src, nent * sizeof(int32_t), cudaMemcpyDeviceToHost));
    EFSI_CUDA_CHECK(cudaMemcpy(h_coef.data(), coef, nent * sizeof(double), cudaMemcpyDeviceToHost));
  }
  for (int32_t e = 0; e < nent; ++e) EFSI_ARG_CHECK(h_src[e] >= 0 && h_src[e] < n0, "coupling source cell out of range");
  if (P->cpl_cap_rows < nrows || P->cpl_cap_ent < nent) {
    // new buffers: graphs that captured the old pointers are dropped
    for (PcgGraph& g : P->graphs) cudaGraphExecDestroy(g.exec);
    P->graphs.clear();
    cudaFree(P->cpl_rows);
    cudaFree(P->cpl_ptr);
    cudaFree(P->cpl_src);
    cudaFree(P->cpl_coef);
    P->cpl_rows = P->cpl_ptr = P->cpl_src = nullptr;
    P->cpl_coef = nullptr;
    P->cpl_cap_rows = P->cpl_cap_ent = 0;
    const int64_t cr = std::max<int64_t>(nrows, 2 * P->cpl_cap_rows), ce = std::max<int64_t>(std::max(nent, 1), 1);
    EFSI_CUDA_CHECK(cudaMalloc(&P->cpl_rows, cr * sizeof(int32_t)));
    EFSI_CUDA_CHECK(cudaMalloc(&P->cpl_ptr, (cr + 1) * sizeof(int32_t)));
    EFSI_CUDA_CHECK(cudaMalloc(&P->cpl_src, ce * sizeof(int32_t)));
    EFSI_CUDA_CHECK(cudaMalloc(&P->cpl_coef, ce * sizeof(double)));
    P->cpl_cap_rows = cr;
    P->cpl_cap_ent = ce;
  }
  EFSI_CUDA_CHECK(cudaMemcpy(P->cpl_rows, h_rows.data(), nrows * sizeof(int32_t), cudaMemcpyHostToDevice));
  EFSI_CUDA_CHECK(cudaMemcpy(P->cpl_ptr, h_ptr.data(), (nrows + 1) * sizeof(int32_t), cudaMemcpyHostToDevice));
  if (nent > 0) {
    EFSI_CUDA_CHECK(cudaMemcpy(P->cpl_src, h_src.data(), nent * sizeof(int32_t), cudaMemcpyHostToDevice));
    EFSI_CUDA_CHECK(cudaMemcpy(P->cpl_coef, h_coef.data(), nent * sizeof(double), cudaMemcpyHostToDevice));
  }
  EFSI_CUDA_CHECK(cudaMemcpy(P->cpl_n, &nrows, sizeof(int32_t), cudaMemcpyHostToDevice));
  P->cpl_nrows = nrows;
  return EFSI_OK;
}

int efsi_fv_copy_rhs(efsi_fv_plan* P, double* out, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(out != nullptr, "null output");
  EFSI_CUDA_CHECK(cudaMemcpyAsync(out, P->b, P->lv[0].n * sizeof(double), cudaMemcpyDeviceToDevice, as_stream(stream)));
  return EFSI_OK;
}

int efsi_fv_learned_input(efsi_fv_plan* P, const double* r, void* input, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(r != nullptr && input != nullptr, "null argument");
  EFSI_ARG_CHECK(P->unet != nullptr, "no learned preconditioner attached (its finest widths define the input)");
  cudaStream_t s = as_stream(stream);
  const LevelDev L = level_dev(P, 0);
  const Shape3 S = P->lv[0].shape;
  // the free volume and r's RMS as the solve computes them
  EFSI_COUNTED k_rhs_mean<<<S.grid, S.block, 0, s>>>(L, r, 0.0, P->partials, P->sc);
  EFSI_COUNTED k_learned_sumsq<<<S.grid, S.block, 0, s>>>(L, r, nullptr, P->partials, P->sc);
  EFSI_COUNTED k_learned_pack<<<S.grid, S.block, 0, s>>>(L, r, nullptr, static_cast<__nv_bfloat16*>(input),
                                                         P->unet_wmin[0], P->unet_wmin[1], P->unet_wmin[2],
                                                         (const CgScalars*)P->sc);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_fv_learned_presmooth(efsi_fv_plan* P, const double* r, double* z, int32_t outlet, void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(r != nullptr && z != nullptr, "null argument");
  cudaStream_t s = as_stream(stream);
  const ProlongSrc none{nullptr, 0, 0, 0, 0.0f};
  const double om = (double)0.8f;
  double* za = static_cast<double*>(P->lv[0].pa);
  launch_sweep<double, true, true>(P, 0, nullptr, r, za, outlet, om, none, nullptr, s);
  launch_sweep<double, true, false>(P, 0, za, r, z, outlet, om, none, nullptr, s);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

}  // extern "C"

extern "C" const char* efsi_fv_graph_error(efsi_fv_plan* P) { return P ? P->graph_error.c_str() : ""; }

extern "C" int efsi_fv_pcg_device_stats(efsi_fv_plan* P, efsi_cg_stats* st, void* stream) {
  EFSI_ARG_CHECK(P != nullptr && st != nullptr, "null argument");
  cudaStream_t s = as_stream(stream);
  EFSI_CUDA_CHECK(cudaMemcpyAsync(P->host_sc, P->sc, sizeof(CgScalars), cudaMemcpyDeviceToHost, s));
  EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  std::memset(st, 0, sizeof(*st));
  if (P->host_sc->fault) {
    set_error("a plane-marching kernel's TMA stage did not complete in time");
    return EFSI_ERR_CUDA;
  }
  fill_device_stats(P, st);
  return EFSI_OK;
}

// Whole-step graphs: everything the library launches on `stream` between
// begin and end is captured (the caller's stream must not be the legacy
// default stream); launch replays it.
struct efsi_step_graph {
  cudaGraphExec_t exec = nullptr;
  unsigned long long nodes = 0;
};

extern "C" int efsi_step_graph_begin(void* stream) {
  cudaStream_t s = as_stream(stream);
  EFSI_ARG_CHECK(s != nullptr && s != cudaStreamLegacy && s != cudaStreamPerThread,
                 "a step graph is captured on a created stream, not the default stream");
  EFSI_CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  set_capturing(true);
  take_capture_count();
  return EFSI_OK;
}

extern "C" int efsi_step_graph_end(void* stream, efsi_step_graph** out) {
  EFSI_ARG_CHECK(out != nullptr, "null output");
  *out = nullptr;
  cudaStream_t s = as_stream(stream);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &g);
  set_capturing(false);
  const unsigned long long nodes = take_capture_count();
  if (e != cudaSuccess) {
    if (g != nullptr) cudaGraphDestroy(g);
    cudaGetLastError();
    set_error(std::string("step graph capture: ") + cudaGetErrorString(e));
    return EFSI_ERR_CUDA;
  }
  cudaGraphExec_t ex = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    cudaGetLastError();
    set_error(std::string("step graph instantiation: ") + cudaGetErrorString(ei));
    return EFSI_ERR_CUDA;
  }
  efsi_step_graph* G = new efsi_step_graph();
  G->exec = ex;
  G->nodes = nodes;
  *out = G;
  return EFSI_OK;
}

extern "C" int efsi_step_graph_launch(efsi_step_graph* G, void* stream) {
  EFSI_ARG_CHECK(G != nullptr && G->exec != nullptr, "null step graph");
  EFSI_CUDA_CHECK(cudaGraphLaunch(G->exec, as_stream(stream)));
  count_graph_launch(G->nodes);
  return EFSI_OK;
}

extern "C" int efsi_step_graph_destroy(efsi_step_graph* G) {
  if (G == nullptr) return EFSI_OK;
  if (G->exec != nullptr) cudaGraphExecDestroy(G->exec);
  delete G;
  return EFSI_OK;
}

extern "C" int efsi_fv_coarse_kernel_blocks(efsi_fv_plan* P, int32_t* blocks) {
  EFSI_ARG_CHECK(P != nullptr && blocks != nullptr, "null argument");
  *blocks = P->coarse_blocks;
  if (P->coarse_blocks == 0) set_error(P->coarse_note);
  return EFSI_OK;
}
