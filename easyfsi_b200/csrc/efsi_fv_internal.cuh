// Internal definitions shared by the fluid translation units of the
// easyfsi_b200 library (plan layout, per-level device view, mask bits).
#pragma once

#include <vector>

#include "efsi_common.cuh"

namespace efsi {

// ---------------------------------------------------------------------------
// Mask bits
// ---------------------------------------------------------------------------
enum : unsigned {
  M_XM = 1u,
  M_XP = 2u,
  M_YM = 4u,
  M_YP = 8u,
  M_ZM = 16u,
  M_ZP = 32u,
  M_FLUID = 64u,  // obstacle == 0
  M_SOLID = 128u  // obstacle == 1
};

struct LevelDev {
  int nx, ny, nz;
  const double* cxm;
  const double* cxp;
  const double* cym;
  const double* cyp;
  const double* czm;
  const double* czp;
  double oz;  // outlet diagonal term 2 / wz[0]^2
  const float* wx;
  const float* wy;
  const float* wz;
  const float* cdx_f;  // f32 centre distances as loaded by the reference
  const float* cdy_f;
  const float* cdz_f;
  const uint8_t* mask;
  const float* fw;     // clamped Dirichlet face weight per cell, or null
  const void* iface;   // interface diagonal: double (level 0) / float (coarse), or null
};

struct CgScalars {
  double rz, rz_new, dAd, rr, beta_num, alpha, beta;
  double mean_z, mean_x, mean_r, mean_b, free_vol, bnorm2, code_dAd, dot;
  int code;
  int zproj;  // 1: consumers of z apply the zero-mean projection on the fly
  unsigned ticket;
};

__device__ __forceinline__ int64_t cidx(int i, int j, int k, int ny, int nz) {
  return ((int64_t)i * ny + j) * nz + k;
}

__device__ __forceinline__ double vol64(const LevelDev& L, int i, int j, int k) {
  return (double)__ldg(L.wx + i) * (double)__ldg(L.wy + j) * (double)__ldg(L.wz + k);
}

template <typename TP>
__device__ __forceinline__ double iface_at(const LevelDev& L, int64_t c) {
  if (L.iface == nullptr) return 0.0;
  return (double)__ldg(reinterpret_cast<const TP*>(L.iface) + c);
}

// fluid.py:4080-4221: neighbour sum and denominator of one row.  `val(cell)`
// returns the (possibly on-the-fly) iterate at a neighbour.
template <class V>
__device__ __forceinline__ void stencil(const LevelDev& L, const V& val, int i, int j, int k, int64_t c, unsigned m,
                                        int outlet, double& ns, double& den) {
  const int64_t sx = (int64_t)L.ny * L.nz, sy = L.nz;
  ns = 0.0;
  den = 0.0;
  const float* fw = L.fw;
  if (m & M_XM) {
    double co = __ldg(L.cxm + i);
    if (fw) co *= (double)__ldg(fw + c);
    ns += co * val(c - sx, i - 1, j, k);
    den += co;
  }
  if (m & M_XP) {
    double co = __ldg(L.cxp + i);
    if (fw) co *= (double)__ldg(fw + c + sx);
    ns += co * val(c + sx, i + 1, j, k);
    den += co;
  }
  if (m & M_YM) {
    double co = __ldg(L.cym + j);
    if (fw) co *= (double)__ldg(fw + c);
    ns += co * val(c - sy, i, j - 1, k);
    den += co;
  }
  if (m & M_YP) {
    double co = __ldg(L.cyp + j);
    if (fw) co *= (double)__ldg(fw + c + sy);
    ns += co * val(c + sy, i, j + 1, k);
    den += co;
  }
  if (m & M_ZM) {
    double co = __ldg(L.czm + k);
    if (fw) co *= (double)__ldg(fw + c);
    ns += co * val(c - 1, i, j, k - 1);
    den += co;
  }
  if (m & M_ZP) {
    double co = __ldg(L.czp + k);
    if (fw) co *= (double)__ldg(fw + c + 1);
    ns += co * val(c + 1, i, j, k + 1);
    den += co;
  }
  if (outlet && k == 0) den += L.oz;
}

}  // namespace efsi

namespace efsi {
// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------

struct LevelBuf {
  int nx, ny, nz;
  int64_t n;
  double* coef = nullptr;   // cxm cxp cym cyp czm czp
  uint8_t* mask = nullptr;
  float* fw = nullptr;      // allocated lazily when Dirichlet rows are active
  int32_t* obs = nullptr;   // coarse obstacle (levels >= 1)
  int32_t* va = nullptr;    // coarse Dirichlet flags
  float* vw = nullptr;
  void* iface = nullptr;    // coarse interface diagonal (float) when active
  // V-cycle work: three iterate buffers and the rhs (coarse) of the level.
  void* pa = nullptr;
  void* pb = nullptr;
  float* rhs = nullptr;     // coarse rhs (levels >= 1)
  const float *wx, *wy, *wz;
  const float *cdx, *cdy, *cdz;
  double oz = 0.0;
  Shape3 shape;
};

}  // namespace efsi

struct efsi_fv_plan {
  int n_levels = 0;
  int uniform = 0;
  std::vector<efsi::LevelBuf> lv;
  // level-0 CG vectors
  double *r = nullptr, *z = nullptr, *d0 = nullptr, *d1 = nullptr, *Ad = nullptr, *delta = nullptr, *b = nullptr,
         *diag = nullptr;
  double* partials = nullptr;
  size_t partials_len = 0;
  double* aux = nullptr;  // 16 doubles of statistics scratch
  efsi::CgScalars* sc = nullptr;
  efsi::CgScalars* host_sc = nullptr;  // pinned readback
  bool has_vdir = false;
  bool has_iface = false;
  const double* iface0 = nullptr;  // caller's level-0 interface diagonal
  const int32_t* obstacle0 = nullptr;  // caller's level-0 obstacle (legacy Jacobi)
};


namespace efsi {
LevelDev level_dev(const efsi_fv_plan* P, int l);
int level_zero_check(const efsi_fv_plan* P);
}  // namespace efsi
