// Internal definitions shared by the fluid translation units of the
// easyfsi_b200 library (plan layout, per-level device view, mask bits).
#pragma once

#include <deque>
#include <string>
#include <vector>

#include <cuda.h>

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
  double learned_num;  // <r', n>_V of the learned coarse correction (its 1-D Galerkin scale)
  // device-side loop (efsi_pcg_params::device_loop): iterations done, the
  // relative residuals, b_norm, converged flag
  double dl_bnorm, dl_rel0, dl_rel;
  int dl_iter, dl_converged;
  int code;
  int zproj;  // 1: consumers of z apply the zero-mean projection on the fly
  unsigned ticket;
  int fault;  // a plane-marching kernel's stage copy did not complete in time
  int defer_alpha;  // interface couplings follow the SpMV: its finisher stores dAd only
};

// fluid.py:4567-4574 _cg_compute_alpha_kernel on the device scalars: alpha =
// rz / dAd, or breakdown code 1 (and the first offending dAd) when dAd <= 0.
// Shared by every SpMV finisher and by efsi_cg_compute_alpha.
__device__ __forceinline__ void cg_alpha_step(CgScalars* sc, double dAd);

// The SpMV finishers: alpha now, or (interface couplings still to come) only
// the operator's part of dAd.
__device__ __forceinline__ void spmv_alpha(CgScalars* sc, double dAd) {
  if (sc->defer_alpha)
    sc->dAd = dAd;
  else
    cg_alpha_step(sc, dAd);
}

__device__ __forceinline__ void cg_alpha_step(CgScalars* sc, double dAd) {
  sc->dAd = dAd;
  sc->alpha = 0.0;
  if (dAd <= 0.0) {
    if (sc->code == 0) sc->code_dAd = dAd;
    sc->code = 1;
  } else {
    sc->alpha = sc->rz / dAd;
  }
}

// fluid.py:4590-4601 _cg_compute_beta_kernel on the device scalars: the
// flexible (Polak-Ribiere, clamped at 0) beta with the multigrid
// preconditioner, Fletcher-Reeves otherwise; breakdown code 2 when rz <=
// 1e-300 or rz_new <= 0.  Shared by every dots finisher and by
// efsi_cg_compute_beta.
__device__ __forceinline__ void cg_beta_step(CgScalars* sc, double rz_new, double beta_num, bool mg) {
  const double rz = sc->rz;
  sc->rz_new = rz_new;
  sc->beta_num = beta_num;
  double beta = 0.0;
  if (rz <= 1.0e-300 || rz_new <= 0.0) {
    sc->code = 2;
  } else if (mg) {
    beta = beta_num / rz;
    if (beta < 0.0) beta = 0.0;
  } else {
    beta = rz_new / rz;
  }
  sc->beta = beta;
}

// Coarse iterate whose prolongation p += scale * p_coarse is fused into a sweep.
struct ProlongSrc {
  const float* pc;  // coarse iterate, null when no prolongation is fused
  int cnx, cny, cnz;
  float scale;
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

// fluid.py:4080-4221: neighbour sum and denominator of one row.  `val(cell,
// i, j, k)` returns the (possibly on-the-fly) iterate at a neighbour.  All six
// neighbour values, coefficients and face weights are loaded unconditionally
// (a wall face reads the cell itself) so the loads do not wait for the mask;
// the mask then selects the open faces in the reference's order x-, x+, y-,
// y+, z-, z+.
template <class V>
__device__ __forceinline__ void stencil(const LevelDev& L, const V& val, int i, int j, int k, int64_t c, unsigned m,
                                        int outlet, double& ns, double& den) {
  const int64_t sx = (int64_t)L.ny * L.nz, sy = L.nz;
  const bool hxm = i > 0, hxp = i < L.nx - 1, hym = j > 0, hyp = j < L.ny - 1, hzm = k > 0, hzp = k < L.nz - 1;
  const int64_t cxm = hxm ? c - sx : c, cxp = hxp ? c + sx : c;
  const int64_t cym = hym ? c - sy : c, cyp = hyp ? c + sy : c;
  const int64_t czm = hzm ? c - 1 : c, czp = hzp ? c + 1 : c;
  const double vxm = val(cxm, hxm ? i - 1 : i, j, k);
  const double vxp = val(cxp, hxp ? i + 1 : i, j, k);
  const double vym = val(cym, i, hym ? j - 1 : j, k);
  const double vyp = val(cyp, i, hyp ? j + 1 : j, k);
  const double vzm = val(czm, i, j, hzm ? k - 1 : k);
  const double vzp = val(czp, i, j, hzp ? k + 1 : k);
  double kxm = __ldg(L.cxm + i), kxp = __ldg(L.cxp + i);
  double kym = __ldg(L.cym + j), kyp = __ldg(L.cyp + j);
  double kzm = __ldg(L.czm + k), kzp = __ldg(L.czp + k);
  if (L.fw != nullptr) {
    const double fc = (double)__ldg(L.fw + c);
    kxm *= fc;
    kxp *= (double)__ldg(L.fw + cxp);
    kym *= fc;
    kyp *= (double)__ldg(L.fw + cyp);
    kzm *= fc;
    kzp *= (double)__ldg(L.fw + czp);
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
  float* pa32 = nullptr;    // level 0: FP32 iterates of the mixed-precision V-cycle
  float* pb32 = nullptr;
  float* rhs = nullptr;     // coarse rhs (levels >= 1)
  const float *wx, *wy, *wz;
  const float *cdx, *cdy, *cdz;
  double oz = 0.0;
  Shape3 shape;
  bool tiled = false;  // the tiled 32 x 8 x 4 kernels run on this level
  unsigned tgrid = 1;  // their grid-stride grid size
  bool march = false;  // the plane-marching stencil kernels run on this level
  bool march_ok = false;  // they can (set at plan creation; the autotuner may switch them off)
  int mchunk = 2;      // their planes per block
  unsigned mgrid = 1;  // and grid size
  int spchunk = 2;      // the direction SpMV's (two blocks per SM)
  unsigned spgrid = 1;
};

}  // namespace efsi

struct efsi_unet;

struct PcgGraphKey {
  bool cont, use_mg, remove_mean;
  int outlet, pre, coarse, post;
  const double* pressure;
  bool mixed;  // FP32 level-0 V-cycle
  bool learned = false;  // the learned preconditioner
  bool coupled = false;  // interface-coupling kernels follow the SpMV
  bool anchor = false;   // unreached-component means are subtracted
  bool operator==(const PcgGraphKey& o) const {
    return learned == o.learned && coupled == o.coupled && anchor == o.anchor && cont == o.cont && use_mg == o.use_mg && remove_mean == o.remove_mean && outlet == o.outlet &&
           pre == o.pre && coarse == o.coarse && post == o.post && pressure == o.pressure && mixed == o.mixed;
  }
};

struct PcgGraph {
  PcgGraphKey key;
  cudaGraphExec_t exec;
  unsigned long long nodes;  // kernel launches per replay
};

// A TMA descriptor of one level field, cached per plan (encoded on the host
// at first use; the plane-marching kernels take it by value).
struct PlaneMap {
  const void* ptr;
  int level;
  int kind;  // 0: value tile with halo, 1: right-hand side tile, 2: mask tile
  alignas(64) CUtensorMap map;
};

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
  double* bicg_work = nullptr;  // BiCGSTAB fallback's nine level-0 work vectors, allocated at its first use
  double* report_buf = nullptr;  // 54 doubles of the final divergence report
  double* rden[2] = {nullptr, nullptr};  // level-0 reciprocal row denominators (outlet off / on)
  bool rden_ok[2] = {false, false};      // current for the masks and weights set last
  int32_t* ucomp = nullptr;      // unreached component of every level-0 cell (-1: none)
  int ucomp_n = 0;               // components anchored by an outlet solve (0: none)
  double* ucomp_acc = nullptr;   // per component: volume-weighted sums [256], volumes [256]
  efsi_unet* unet = nullptr;    // learned preconditioner (code 4), not owned
  void* unet_in = nullptr;      // its BF16 input [n0][16]
  float unet_wmin[3] = {1.0f, 1.0f, 1.0f};  // finest level-0 width per axis
  // interface-coupling terms of the level-0 operator as rows of (source cell,
  // coefficient) entries per receiving cell; the row count lives on the
  // device (cpl_n) so captured graphs stay valid when the couplings change
  int32_t* cpl_rows = nullptr;
  int32_t* cpl_ptr = nullptr;
  int32_t* cpl_src = nullptr;
  double* cpl_coef = nullptr;
  int32_t* cpl_n = nullptr;
  int64_t cpl_cap_rows = 0, cpl_cap_ent = 0;
  int cpl_nrows = 0;  // host copy
  efsi::CgScalars* sc = nullptr;
  efsi::CgScalars* host_sc = nullptr;  // pinned readback
  bool has_vdir = false;
  bool has_iface = false;
  const double* iface0 = nullptr;  // caller's level-0 interface diagonal
  const int32_t* obstacle0 = nullptr;  // caller's level-0 obstacle (legacy Jacobi)
  std::vector<PcgGraph> graphs;        // instantiated 16-iteration PCG blocks
  cudaStream_t cap_stream = nullptr;   // private stream used for graph capture
  cudaStream_t body_stream = nullptr;  // captures the body of the device-side PCG loop
  cudaStream_t side_stream = nullptr;  // the x half of a split CG update
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int dl_used_mg = 0;                  // preconditioner kind of the last device-side loop
  bool graphs_disabled = false;        // a capture failed; blocks run as direct launches
  int tail_level = 1 << 30;            // first level run by the single-CTA V-cycle tail
  size_t tail_smem_bytes = 0;
  int tail_foff[12] = {0};
  int tail_moff[12] = {0};
  int tail_coff[12] = {0};
  int tail_noff[12] = {0};
  int coarse_blocks = 0;               // grid of the cooperative coarse-level kernel (0: per-level launches)
  int coarse_first = 1;                // first level the coarse-level kernel runs
  int coarse_cluster = 0;              // 1: one thread-block cluster of coarse_blocks CTAs, hardware barriers
  unsigned* coarse_bar = nullptr;      // its grid barrier: arrivals, generation
  std::string coarse_note;             // why the per-level launches run instead
  std::string graph_error;
  std::deque<PlaneMap> maps;  // deque: descriptors stay in place as the cache grows
};


namespace efsi {
LevelDev level_dev(const efsi_fv_plan* P, int l);
int level_zero_check(const efsi_fv_plan* P);
}  // namespace efsi
