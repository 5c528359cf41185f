// CPU oracle, fluid part -- TEST INFRASTRUCTURE ONLY (see oracle_common.h).
//
// Restates simulation_core/fluid.py of the reference: divergence, the FV
// pressure operator and its Jacobi smoother, the multigrid transfer operators,
// the flexible MG/Jacobi preconditioned CG driver, the gradient correction,
// the predictor and the body-force spreading.  Citations are file:line in the
// reference tree.
#include "oracle_common.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Literal f32 kernel arguments of the reference: omega=0.8 and the graded
// coarse correction 0.7 are passed as ti.f32 (fluid.py:4243, 5399).
inline double f32arg(double v) { return (double)(float)v; }

inline double clamp01(double v) { return std::min(std::max(v, 0.0), 1.0); }

// fluid.py:4080-4221 _fv_pressure_neighbor_sum_denominator.
template <typename TP>
inline void nb_sum_den(const efo_level& L, const TP* p, const int32_t* obs, const int32_t* va,
                       const r32* vw, int i, int j, int k, int outlet, double& ns, double& den) {
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const int64_t c = efo_idx(i, j, k, ny, nz);
  const int64_t sx = (int64_t)ny * nz, sy = nz;
  ns = 0.0;
  den = 0.0;
  auto fw = [&](int64_t cell) -> double {
    if (va != nullptr && va[cell] != 0) return clamp01((double)vw[cell]);
    return 1.0;
  };
  if (i > 0 && obs[c - sx] == 0) {
    double w = fw(c);
    double coeff = 1.0 / ((double)L.wx[i] * (double)L.cdx[i]);
    ns += coeff * w * (double)p[c - sx];
    den += coeff * w;
  }
  if (i < nx - 1 && obs[c + sx] == 0) {
    double w = fw(c + sx);
    double coeff = 1.0 / ((double)L.wx[i] * (double)L.cdx[i + 1]);
    ns += coeff * w * (double)p[c + sx];
    den += coeff * w;
  }
  if (j > 0 && obs[c - sy] == 0) {
    double w = fw(c);
    double coeff = 1.0 / ((double)L.wy[j] * (double)L.cdy[j]);
    ns += coeff * w * (double)p[c - sy];
    den += coeff * w;
  }
  if (j < ny - 1 && obs[c + sy] == 0) {
    double w = fw(c + sy);
    double coeff = 1.0 / ((double)L.wy[j] * (double)L.cdy[j + 1]);
    ns += coeff * w * (double)p[c + sy];
    den += coeff * w;
  }
  if (k > 0 && obs[c - 1] == 0) {
    double w = fw(c);
    double coeff = 1.0 / ((double)L.wz[k] * (double)L.cdz[k]);
    ns += coeff * w * (double)p[c - 1];
    den += coeff * w;
  }
  if (k < nz - 1 && obs[c + 1] == 0) {
    double w = fw(c + 1);
    double coeff = 1.0 / ((double)L.wz[k] * (double)L.cdz[k + 1]);
    ns += coeff * w * (double)p[c + 1];
    den += coeff * w;
  }
  if (outlet == 1 && k == 0) {
    den += 2.0 / ((double)L.wz[k] * (double)L.wz[k]);
  }
}

inline int64_t ncells(const efo_level& L) { return (int64_t)L.nx * L.ny * L.nz; }

// Cell volume promoted to f64 as in the weighted dot (fluid.py:4538-4545).
inline double vol64(const efo_level& L, int i, int j, int k) {
  return (double)L.wx[i] * (double)L.wy[j] * (double)L.wz[k];
}

template <typename TI>
inline double iface_at(const TI* d, int64_t c) {
  return d == nullptr ? 0.0 : (double)d[c];
}

// fluid.py:4224-4273 _pressure_fv_jacobi_kernel (one sweep, out of place).
template <typename TP, typename TI>
void jacobi_sweep(const efo_level& L, const TP* p, const TP* rhs, const TI* iface, const int32_t* obs,
                  const int32_t* va, const r32* vw, TP* tmp, int outlet, double omega) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k) {
        const int64_t c = efo_idx(i, j, k, L.ny, L.nz);
        if (obs[c] == 1) {
          tmp[c] = (TP)0;
          continue;
        }
        double ns, den;
        nb_sum_den(L, p, obs, va, vw, i, j, k, outlet, ns, den);
        den += iface_at(iface, c);
        if (den <= 0.0) {
          tmp[c] = (TP)0;
        } else {
          double jv = (ns - (double)rhs[c]) / den;
          double pc = (double)p[c];
          tmp[c] = (TP)(pc + omega * (jv - pc));
        }
      }
}

template <typename TP, typename TI>
void smooth(const efo_level& L, TP* p, const TP* rhs, const TI* iface, const int32_t* obs, const int32_t* va,
            const r32* vw, TP* tmp, int outlet, int iterations, double omega) {
  // fluid.py:5862-5900: sweep then copy tmp -> pressure.
  const int64_t n = ncells(L);
  for (int it = 0; it < std::max(0, iterations); ++it) {
    jacobi_sweep(L, p, rhs, iface, obs, va, vw, tmp, outlet, omega);
    std::memcpy(p, tmp, sizeof(TP) * n);
  }
}

// fluid.py:5262-5307 _mg_compute_residual_kernel.
template <typename TP, typename TI>
void mg_residual(const efo_level& L, const TP* p, const TP* rhs, const TI* iface, const int32_t* obs,
                 const int32_t* va, const r32* vw, TP* res, int outlet) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k) {
        const int64_t c = efo_idx(i, j, k, L.ny, L.nz);
        if (obs[c] == 1) {
          res[c] = (TP)0;
          continue;
        }
        double ns, den;
        nb_sum_den(L, p, obs, va, vw, i, j, k, outlet, ns, den);
        den += iface_at(iface, c);
        double applied = ns - den * (double)p[c];
        res[c] = (TP)((double)rhs[c] - applied);
      }
}

// f32 accumulator of the restriction (fluid.py:5331-5366): the locals are
// declared with the default f32 type, so every += rounds to f32.  A product of
// an f64 fine value with the f32 volume is formed in f64 first.
inline void acc32(r32& s, double v, r32 vol) { s = (r32)((double)s + v * (double)vol); }
inline void acc32(r32& s, float v, r32 vol) { s = (r32)(s + (r32)v * vol); }

// fluid.py:5310-5388 _mg_restrict_residual_kernel.
template <typename TF, typename TFI>
void mg_restrict(const efo_level& F, const TF* fine_res, const TFI* fine_iface, const int32_t* fobs,
                 const int32_t* fva, const r32* fvw, const efo_level& C, r32* crhs, r32* ciface, r32* cp,
                 r32* ctmp, r32* cres, int32_t* cobs, int32_t* cva, r32* cvw) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < C.nx; ++i)
    for (int j = 0; j < C.ny; ++j)
      for (int k = 0; k < C.nz; ++k) {
        r32 wres = 0, wdiag = 0, free_vol = 0, vdw = 0;
        int obstacle_count = 0, vdc = 0;
        for (int oi = 0; oi < 2; ++oi)
          for (int oj = 0; oj < 2; ++oj)
            for (int ok = 0; ok < 2; ++ok) {
              int fi = 2 * i + oi, fj = 2 * j + oj, fk = 2 * k + ok;
              if (fi < F.nx && fj < F.ny && fk < F.nz) {
                int64_t f = efo_idx(fi, fj, fk, F.ny, F.nz);
                if (fva != nullptr && fva[f] != 0) {
                  vdc += 1;
                  vdw = std::max(vdw, fvw[f]);
                }
                if (fobs[f] == 1) {
                  obstacle_count += 1;
                } else {
                  r32 vol = F.wx[fi] * F.wy[fj] * F.wz[fk];
                  acc32(wres, fine_res[f], vol);
                  if (fine_iface != nullptr) acc32(wdiag, fine_iface[f], vol);
                  free_vol += vol;
                }
              }
            }
        int64_t c = efo_idx(i, j, k, C.ny, C.nz);
        if (obstacle_count > 0) {
          cobs[c] = 1;
          crhs[c] = 0;
          ciface[c] = 0;
        } else {
          cobs[c] = 0;
          r32 denom = std::max(free_vol, (r32)1.0e-30);
          crhs[c] = wres / denom;
          ciface[c] = wdiag / denom;
        }
        if (vdc > 0) {
          cva[c] = 1;
          cvw[c] = vdw;
        } else {
          cva[c] = 0;
          cvw[c] = 0;
        }
        cp[c] = 0;
        ctmp[c] = 0;
        cres[c] = 0;
      }
}

// fluid.py:5391-5406 _mg_prolongate_add_kernel.
template <typename TF>
void mg_prolong(const efo_level& F, TF* fp, const int32_t* fobs, const efo_level& C, const r32* cp, double scale) {
  const r32 s = (r32)scale;
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < F.nx; ++i)
    for (int j = 0; j < F.ny; ++j)
      for (int k = 0; k < F.nz; ++k) {
        int64_t f = efo_idx(i, j, k, F.ny, F.nz);
        if (fobs[f] == 0) {
          int ci = std::min(i / 2, C.nx - 1), cj = std::min(j / 2, C.ny - 1), ck = std::min(k / 2, C.nz - 1);
          r32 corr = s * cp[efo_idx(ci, cj, ck, C.ny, C.nz)];
          fp[f] = (TF)(fp[f] + (TF)corr);
        }
      }
}

// fluid.py:4534-4546 _weighted_dot_kernel.
template <typename TA, typename TB>
double weighted_dot(const efo_level& L, const int32_t* obs, const TA* a, const TB* b) {
  double total = 0.0;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : total)
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k) {
        int64_t c = efo_idx(i, j, k, L.ny, L.nz);
        if (obs[c] == 0) total += (double)a[c] * (double)b[c] * vol64(L, i, j, k);
      }
  return total;
}

// fluid.py:4677-4693 _weighted_mean_to_cg_field_kernel.
double weighted_mean(const efo_level& L, const int32_t* obs, const double* f, double multiplier) {
  double total = 0.0, vol = 0.0;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : total, vol)
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k) {
        int64_t c = efo_idx(i, j, k, L.ny, L.nz);
        if (obs[c] == 0) {
          double v = vol64(L, i, j, k);
          total += f[c] * v;
          vol += v;
        }
      }
  return vol > 0.0 ? multiplier * total / vol : 0.0;
}

// fluid.py:4716-4726 _subtract_weighted_mean_device.
void subtract_mean(const efo_level& L, const int32_t* obs, double* f) {
  double m = weighted_mean(L, obs, f, 1.0);
  const int64_t n = ncells(L);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c) f[c] = (obs[c] == 0) ? f[c] - m : 0.0;
}

// fluid.py:4312-4345 _fv_laplacian_apply_kernel (the row-list / slot terms are
// inactive when no interface rows exist, which the callers guarantee).
void fv_apply(const efo_level& L, const int32_t* obs, const int32_t* va, const r32* vw, const double* iface,
              const double* p, double* out, int outlet) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k) {
        int64_t c = efo_idx(i, j, k, L.ny, L.nz);
        if (obs[c] == 1) {
          out[c] = 0.0;
          continue;
        }
        double ns, den;
        nb_sum_den(L, p, obs, va, vw, i, j, k, outlet, ns, den);
        out[c] = (den + iface_at(iface, c)) * p[c] - ns;
      }
}

// fluid.py:4280-4309 _fv_diagonal_kernel.
void fv_diagonal(const efo_level& L, const int32_t* obs, const int32_t* va, const r32* vw, const double* iface,
                 double* diag, int outlet) {
  std::vector<double> zero(1, 0.0);
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k) {
        int64_t c = efo_idx(i, j, k, L.ny, L.nz);
        if (obs[c] == 1) {
          diag[c] = 0.0;
          continue;
        }
        double ns, den;
        nb_sum_den(L, diag, obs, va, vw, i, j, k, outlet, ns, den);
        diag[c] = den + iface_at(iface, c);
      }
}

struct Levels {
  int n;
  const efo_level* L;
  // Per-level state.  Level 0 uses the caller's f64 arrays; coarse levels are
  // f32 in the reference (fluid.py:1055-1075).
  std::vector<std::vector<r32>> p, tmp, rhs, res, iface, vw;
  std::vector<std::vector<int32_t>> obs, va;
  explicit Levels(int n_, const efo_level* L_) : n(n_), L(L_) {
    p.resize(n);
    tmp.resize(n);
    rhs.resize(n);
    res.resize(n);
    iface.resize(n);
    vw.resize(n);
    obs.resize(n);
    va.resize(n);
    for (int l = 1; l < n; ++l) {
      int64_t m = ncells(L[l]);
      p[l].assign(m, 0);
      tmp[l].assign(m, 0);
      rhs[l].assign(m, 0);
      res[l].assign(m, 0);
      iface[l].assign(m, 0);
      vw[l].assign(m, 0);
      obs[l].assign(m, 0);
      va[l].assign(m, 0);
    }
  }
};

struct Fine {
  const int32_t* obs;
  const int32_t* va;
  const r32* vw;
  const double* iface;  // may be null (zero)
};

// One V-cycle with zero initial guess: fluid.py:6085-6262
// _apply_fv_multigrid_preconditioner.  The level-0 arrays (pressure, tmp,
// rhs, residual) are f64 (cg_z, cg_Ad, cg_mg_rhs, cg_mg_residual).
void vcycle(Levels& lv, const Fine& fine, const double* r, double* z, double* tmp0, double* rhs0, double* res0,
            int outlet, int pre, int coarse, int post, double scale) {
  const efo_level& L0 = lv.L[0];
  const int64_t n0 = ncells(L0);
  // fluid.py:4485-4500 _pcg_prepare_mg_level0_kernel.
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n0; ++c) {
    z[c] = 0.0;
    tmp0[c] = 0.0;
    res0[c] = 0.0;
    rhs0[c] = (fine.obs[c] == 1) ? 0.0 : -r[c];
  }
  const double omega = f32arg(0.8);
  pre = std::max(1, pre);
  coarse = std::max(1, coarse);
  post = std::max(1, post);
  if (lv.n <= 1) {
    smooth(L0, z, rhs0, fine.iface, fine.obs, fine.va, fine.vw, tmp0, outlet, std::max(pre + post, coarse), omega);
    return;
  }
  auto obs_at = [&](int l) -> const int32_t* { return l == 0 ? fine.obs : lv.obs[l].data(); };
  auto va_at = [&](int l) -> const int32_t* { return l == 0 ? fine.va : lv.va[l].data(); };
  auto vw_at = [&](int l) -> const r32* { return l == 0 ? fine.vw : lv.vw[l].data(); };
  for (int l = 0; l < lv.n - 1; ++l) {
    if (l == 0) {
      smooth(L0, z, (const double*)rhs0, fine.iface, fine.obs, fine.va, fine.vw, tmp0, outlet, pre, omega);
      mg_residual(L0, (const double*)z, (const double*)rhs0, fine.iface, fine.obs, fine.va, fine.vw, res0, outlet);
      mg_restrict(L0, (const double*)res0, fine.iface, fine.obs, fine.va, fine.vw, lv.L[1], lv.rhs[1].data(),
                  lv.iface[1].data(), lv.p[1].data(), lv.tmp[1].data(), lv.res[1].data(), lv.obs[1].data(),
                  lv.va[1].data(), lv.vw[1].data());
    } else {
      smooth(lv.L[l], lv.p[l].data(), (const r32*)lv.rhs[l].data(), (const r32*)lv.iface[l].data(), obs_at(l),
             va_at(l), vw_at(l), lv.tmp[l].data(), outlet, pre, omega);
      mg_residual(lv.L[l], (const r32*)lv.p[l].data(), (const r32*)lv.rhs[l].data(), (const r32*)lv.iface[l].data(),
                  obs_at(l), va_at(l), vw_at(l), lv.res[l].data(), outlet);
      mg_restrict(lv.L[l], (const r32*)lv.res[l].data(), (const r32*)lv.iface[l].data(), obs_at(l), va_at(l),
                  vw_at(l), lv.L[l + 1], lv.rhs[l + 1].data(), lv.iface[l + 1].data(), lv.p[l + 1].data(),
                  lv.tmp[l + 1].data(), lv.res[l + 1].data(), lv.obs[l + 1].data(), lv.va[l + 1].data(),
                  lv.vw[l + 1].data());
    }
  }
  const int lc = lv.n - 1;
  smooth(lv.L[lc], lv.p[lc].data(), (const r32*)lv.rhs[lc].data(), (const r32*)lv.iface[lc].data(), obs_at(lc),
         va_at(lc), vw_at(lc), lv.tmp[lc].data(), outlet, coarse, omega);
  for (int l = lv.n - 2; l >= 0; --l) {
    if (l == 0) {
      mg_prolong(L0, z, fine.obs, lv.L[1], lv.p[1].data(), scale);
      smooth(L0, z, (const double*)rhs0, fine.iface, fine.obs, fine.va, fine.vw, tmp0, outlet, post, omega);
    } else {
      mg_prolong(lv.L[l], lv.p[l].data(), obs_at(l), lv.L[l + 1], lv.p[l + 1].data(), scale);
      smooth(lv.L[l], lv.p[l].data(), (const r32*)lv.rhs[l].data(), (const r32*)lv.iface[l].data(), obs_at(l),
             va_at(l), vw_at(l), lv.tmp[l].data(), outlet, post, omega);
    }
  }
}

// fluid.py:4503-4516 _apply_jacobi_preconditioner_kernel.
void jacobi_precond(int64_t n, const int32_t* obs, const double* diag, const double* r, double* z) {
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c) {
    if (obs[c] == 1)
      z[c] = 0.0;
    else
      z[c] = diag[c] > 0.0 ? r[c] / diag[c] : 0.0;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// C entry points (host arrays, C order (nx, ny, nz), k fastest).
// ---------------------------------------------------------------------------

// fluid.py:3451-3486 _compute_divergence_kernel.
EFO_API void efo_compute_divergence(const efo_level* Lp, const int32_t* obs, const r32* vel, int outlet, r32* div) {
  const efo_level& L = *Lp;
  const int64_t sx = (int64_t)L.ny * L.nz, sy = L.nz;
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k) {
        int64_t c = efo_idx(i, j, k, L.ny, L.nz);
        if (obs[c] == 1) {
          div[c] = 0;
          continue;
        }
        r32 lx = 0, rx = 0, by = 0, fy = 0, bz = 0, tz = 0;
        if (i > 0 && obs[c - sx] == 0) lx = vel[3 * c + 0];
        if (i < L.nx - 1 && obs[c + sx] == 0) rx = vel[3 * (c + sx) + 0];
        if (j > 0 && obs[c - sy] == 0) by = vel[3 * c + 1];
        if (j < L.ny - 1 && obs[c + sy] == 0) fy = vel[3 * (c + sy) + 1];
        if (outlet == 1 && k == 0)
          bz = vel[3 * c + 2];
        else if (k > 0 && obs[c - 1] == 0)
          bz = vel[3 * c + 2];
        if (k < L.nz - 1 && obs[c + 1] == 0) tz = vel[3 * (c + 1) + 2];
        div[c] = (rx - lx) / L.wx[i] + (fy - by) / L.wy[j] + (tz - bz) / L.wz[k];
      }
}

// fluid.py:5228-5243 _mg_prepare_level0_kernel.
EFO_API void efo_mg_prepare_level0(const efo_level* Lp, const int32_t* obs, const r32* div, const r32* src,
                                   const double* iface_rhs, float rhs_scale, double* rhs) {
  const int64_t n = ncells(*Lp);
  const r32 s = (r32)rhs_scale;
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < n; ++c) {
    if (obs[c] == 1)
      rhs[c] = 0.0;
    else
      rhs[c] = (double)(r32)(s * (r32)(div[c] - src[c])) - (iface_rhs ? iface_rhs[c] : 0.0);
  }
}

EFO_API void efo_fv_apply(const efo_level* Lp, const int32_t* obs, const int32_t* va, const r32* vw,
                          const double* iface, const double* p, double* out, int outlet) {
  fv_apply(*Lp, obs, va, vw, iface, p, out, outlet);
}

EFO_API void efo_fv_diagonal(const efo_level* Lp, const int32_t* obs, const int32_t* va, const r32* vw,
                             const double* iface, double* diag, int outlet) {
  fv_diagonal(*Lp, obs, va, vw, iface, diag, outlet);
}

EFO_API double efo_weighted_dot(const efo_level* Lp, const int32_t* obs, const double* a, const double* b) {
  return weighted_dot(*Lp, obs, a, b);
}

EFO_API void efo_jacobi_sweep_f64(const efo_level* Lp, const double* p, const double* rhs, const double* iface,
                                  const int32_t* obs, const int32_t* va, const r32* vw, double* tmp, int outlet,
                                  double omega) {
  jacobi_sweep(*Lp, p, rhs, iface, obs, va, vw, tmp, outlet, f32arg(omega));
}

EFO_API void efo_jacobi_sweep_r32(const efo_level* Lp, const r32* p, const r32* rhs, const r32* iface,
                                  const int32_t* obs, const int32_t* va, const r32* vw, r32* tmp, int outlet,
                                  double omega) {
  jacobi_sweep(*Lp, p, rhs, iface, obs, va, vw, tmp, outlet, f32arg(omega));
}

EFO_API void efo_mg_residual_f64(const efo_level* Lp, const double* p, const double* rhs, const double* iface,
                                 const int32_t* obs, const int32_t* va, const r32* vw, double* res, int outlet) {
  mg_residual(*Lp, p, rhs, iface, obs, va, vw, res, outlet);
}

EFO_API void efo_mg_restrict_f64(const efo_level* F, const double* fres, const double* fiface, const int32_t* fobs,
                                 const int32_t* fva, const r32* fvw, const efo_level* C, r32* crhs, r32* ciface,
                                 int32_t* cobs, int32_t* cva, r32* cvw) {
  std::vector<r32> cp(ncells(*C)), ctmp(ncells(*C)), cres(ncells(*C));
  mg_restrict(*F, fres, fiface, fobs, fva, fvw, *C, crhs, ciface, cp.data(), ctmp.data(), cres.data(), cobs, cva,
              cvw);
}

EFO_API void efo_mg_prolong_f64(const efo_level* F, double* fp, const int32_t* fobs, const efo_level* C,
                                const r32* cp, double scale) {
  mg_prolong(*F, fp, fobs, *C, cp, f32arg(scale));
}

// V-cycle preconditioner on its own (zero initial guess); z receives M^-1 r.
EFO_API void efo_mg_vcycle(int n_levels, const efo_level* levels, const int32_t* obs, const int32_t* va,
                           const r32* vw, const double* iface, const double* r, double* z, int outlet, int pre,
                           int coarse, int post, int uniform_grid) {
  Levels lv(n_levels, levels);
  const int64_t n0 = ncells(levels[0]);
  std::vector<double> tmp0(n0), rhs0(n0), res0(n0);
  Fine fine{obs, va, vw, iface};
  vcycle(lv, fine, r, z, tmp0.data(), rhs0.data(), res0.data(), outlet, pre, coarse, post,
         f32arg(uniform_grid ? 1.0 : 0.7));
}

typedef struct efo_cg_stats {
  int32_t iterations;
  int32_t converged;
  int32_t breakdown_code;    // device code (1: dAd<=0, 2: rz<=0)
  int32_t breakdown_reason;  // 0 none, 1 initial dot, 2 device scalar, 3 restart dot
  int32_t host_residual_checks;
  int32_t restart_count;
  int32_t mean_projection_count;
  int32_t used_mg;
  double initial_relative_residual;
  double relative_residual;
  double breakdown_dAd;
  double b_norm;
  int32_t unreached_set_mean_projection_count;
} efo_cg_stats;

// fluid.py:4905-4981 _accumulate_unreached_component_means_kernel and
// _subtract_unreached_component_means_kernel: comp[c] is the component of an
// anchored (outlet-unreached) cell, -1 elsewhere; each component's
// volume-weighted mean (f64 volumes of the f32 widths) is subtracted from the
// field on its cells.
static void subtract_components(const efo_level& L, const int32_t* comp, int ncomp, double* f) {
  if (comp == nullptr || ncomp <= 0) return;
  std::vector<double> sum(ncomp, 0.0), vol(ncomp, 0.0);
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k) {
        const int64_t c = ((int64_t)i * L.ny + j) * L.nz + k;
        const int q = comp[c];
        if (q < 0 || q >= ncomp) continue;
        const double v = (double)L.wx[i] * (double)L.wy[j] * (double)L.wz[k];
        sum[q] += f[c] * v;
        vol[q] += v;
      }
  for (int64_t c = 0; c < ncells(L); ++c) {
    const int q = comp[c];
    if (q < 0 || q >= ncomp || !(vol[q] > 0.0)) continue;
    f[c] -= sum[q] / vol[q];
  }
}

// fluid.py:6535-6811 _solve_pressure_poisson_fv_cg (no interface row list).
//   rhs_in     : the f64 level-0 rhs _mg_rhs[0] built by efo_mg_prepare_level0
//   pressure   : warm start in, solution out (f64)
//   precond    : 0 jacobi, 1 fv_multigrid (2/24/2), 2 fv_multigrid_light (1/12/1)
//   comp/ncomp : with an outlet, the unreached components anchored where the
//                reference calls _subtract_unreached_set_mean_device
//                (fluid.py:6582-6789); null / 0 for none
EFO_API void efo_fv_pcg_solve_anchored(int n_levels, const efo_level* levels, const int32_t* obs, const int32_t* va,
                                       const r32* vw, const double* iface, const double* rhs_in, double* pressure,
                                       int outlet, int max_iters_in, double tolerance, int precond, int remove_mean,
                                       int uniform_grid, int iface_active, const int32_t* comp, int ncomp,
                                       efo_cg_stats* st) {
  const efo_level& L = levels[0];
  const int64_t n = ncells(L);
  const bool anchor = outlet != 0 && comp != nullptr && ncomp > 0;
  const int max_iters = std::max(1, max_iters_in);
  const double tol = std::max(0.0, tolerance);
  std::memset(st, 0, sizeof(*st));
  st->initial_relative_residual = INFINITY;
  st->relative_residual = INFINITY;
  int code = 0;
  double code_dAd = 0.0;
  std::vector<double> diag(n), r(n), z(n), d(n), Ad(n), r_old(n), rhs_cg(n), mg_rhs(n), mg_res(n);
  std::vector<double> rhs0(rhs_in, rhs_in + n);
  Levels lv(n_levels, levels);
  Fine fine{obs, va, vw, iface};
  fv_diagonal(L, obs, va, vw, iface, diag.data(), outlet);
  auto anchor_field = [&](double* f) {
    if (!anchor) return;
    subtract_components(L, comp, ncomp, f);
    st->unreached_set_mean_projection_count += 1;
  };
  anchor_field(rhs0.data());
  if (remove_mean) {
    double mean = weighted_mean(L, obs, rhs0.data(), -1.0);
    st->mean_projection_count += 1;
    for (int64_t c = 0; c < n; ++c) z[c] = (obs[c] == 1) ? 0.0 : -rhs0[c] - mean;
  } else {
    for (int64_t c = 0; c < n; ++c) z[c] = (obs[c] == 1) ? 0.0 : -rhs0[c] - 0.0;
  }
  rhs_cg = z;
  double b_norm = std::sqrt(std::max(weighted_dot(L, obs, z.data(), z.data()), 0.0));
  st->b_norm = b_norm;
  if (b_norm <= 1.0e-30) {
    std::memset(pressure, 0, sizeof(double) * n);
    st->initial_relative_residual = 0.0;
    st->relative_residual = 0.0;
    st->converged = 1;
    return;
  }
  auto exact_residual = [&]() {
    fv_apply(L, obs, va, vw, iface, pressure, Ad.data(), outlet);
    for (int64_t c = 0; c < n; ++c) r[c] = (obs[c] == 1) ? 0.0 : 1.0 * rhs_cg[c] + -1.0 * Ad[c];
    anchor_field(r.data());
    if (remove_mean) {
      subtract_mean(L, obs, r.data());
      st->mean_projection_count += 1;
    }
    double rr = weighted_dot(L, obs, r.data(), r.data());
    st->host_residual_checks += 1;
    return std::sqrt(std::max(rr, 0.0));
  };
  // Initial residual r = b - A p  (fluid.py:6613-6622).
  fv_apply(L, obs, va, vw, iface, pressure, Ad.data(), outlet);
  for (int64_t c = 0; c < n; ++c) r[c] = (obs[c] == 1) ? 0.0 : 1.0 * z[c] + -1.0 * Ad[c];
  anchor_field(r.data());
  if (remove_mean) {
    subtract_mean(L, obs, r.data());
    st->mean_projection_count += 1;
  }
  double rr = weighted_dot(L, obs, r.data(), r.data());
  st->host_residual_checks += 1;
  double r_norm = std::sqrt(std::max(rr, 0.0));
  st->initial_relative_residual = r_norm / b_norm;
  st->relative_residual = st->initial_relative_residual;
  if (r_norm <= tol * b_norm) {
    st->converged = 1;
    return;
  }
  bool use_mg = n_levels > 1 && !iface_active && (precond == 1 || precond == 2);
  const int pre = precond == 2 ? 1 : 2, coarse = precond == 2 ? 12 : 24, post = precond == 2 ? 1 : 2;
  const double scale = f32arg(uniform_grid ? 1.0 : 0.7);
  std::vector<double> tmp0(n);
  auto apply_precond = [&]() {
    if (use_mg)
      vcycle(lv, fine, r.data(), z.data(), tmp0.data(), mg_rhs.data(), mg_res.data(), outlet, pre, coarse, post,
             scale);
    else
      jacobi_precond(n, obs, diag.data(), r.data(), z.data());
  };
  auto project_z = [&]() {
    anchor_field(z.data());
    if (remove_mean) {
      subtract_mean(L, obs, z.data());
      st->mean_projection_count += 1;
    }
  };
  apply_precond();
  project_z();
  double rz = weighted_dot(L, obs, r.data(), z.data());
  if (!std::isfinite(rz) || std::fabs(rz) <= 1.0e-300) {
    use_mg = false;
    jacobi_precond(n, obs, diag.data(), r.data(), z.data());
    rz = weighted_dot(L, obs, r.data(), z.data());
  }
  st->used_mg = use_mg ? 1 : 0;
  if (!std::isfinite(rz) || rz <= 0.0) {
    st->breakdown_reason = 1;
    return;
  }
  d = z;
  const int check_interval = 16;
  const int restart_interval = iface_active ? 256 : 512;
  for (int it = 1; it <= max_iters; ++it) {
    fv_apply(L, obs, va, vw, iface, d.data(), Ad.data(), outlet);
    double dAd = weighted_dot(L, obs, d.data(), Ad.data());
    // fluid.py:4567-4574 _cg_compute_alpha_kernel.
    double alpha = 0.0;
    if (dAd <= 0.0) {
      if (code == 0) code_dAd = dAd;
      code = 1;
    } else {
      alpha = rz / dAd;
    }
    // fluid.py:4577-4587 _cg_apply_alpha_kernel.
    for (int64_t c = 0; c < n; ++c) {
      if (obs[c] == 1) {
        r_old[c] = 0.0;
        pressure[c] = 0.0;
        r[c] = 0.0;
      } else {
        r_old[c] = r[c];
        pressure[c] += alpha * d[c];
        r[c] -= alpha * Ad[c];
      }
    }
    if (anchor && it % 16 == 0) {
      anchor_field(pressure);
      anchor_field(r.data());
    }
    if (remove_mean && it % 16 == 0) {
      subtract_mean(L, obs, pressure);
      subtract_mean(L, obs, r.data());
      st->mean_projection_count += 2;
    }
    st->iterations = it;
    bool check = (it % check_interval == 0) || it == max_iters;
    if (check) {
      rr = weighted_dot(L, obs, r.data(), r.data());
      st->host_residual_checks += 1;
      r_norm = std::sqrt(std::max(rr, 0.0));
      st->relative_residual = r_norm / b_norm;
      if (st->relative_residual <= tol) {
        st->converged = 1;
        break;
      }
      if (code != 0) {
        st->breakdown_dAd = code_dAd;
        if (it < max_iters) {
          r_norm = exact_residual();
          st->relative_residual = r_norm / b_norm;
          if (st->relative_residual <= tol) {
            st->converged = 1;
            break;
          }
          apply_precond();
          project_z();
          rz = weighted_dot(L, obs, r.data(), z.data());
          if (std::isfinite(rz) && rz > 0.0) {
            d = z;
            code = 0;
            code_dAd = 0.0;
            st->restart_count += 1;
            continue;
          }
        }
        st->breakdown_reason = 2;
        break;
      }
      if (it < max_iters && restart_interval > 0 && it % restart_interval == 0) {
        r_norm = exact_residual();
        st->relative_residual = r_norm / b_norm;
        if (st->relative_residual <= tol) {
          st->converged = 1;
          break;
        }
        apply_precond();
        project_z();
        rz = weighted_dot(L, obs, r.data(), z.data());
        if (!std::isfinite(rz) || rz <= 0.0) {
          st->breakdown_reason = 3;
          break;
        }
        d = z;
        st->restart_count += 1;
        continue;
      }
    }
    apply_precond();
    project_z();
    double rz_new = weighted_dot(L, obs, r.data(), z.data());
    double beta_num = 0.0;
    if (use_mg) {
      for (int64_t c = 0; c < n; ++c) Ad[c] = (obs[c] == 1) ? 0.0 : 1.0 * r[c] + -1.0 * r_old[c];
      beta_num = weighted_dot(L, obs, z.data(), Ad.data());
    }
    // fluid.py:4590-4601 _cg_compute_beta_kernel.
    double beta = 0.0;
    if (rz <= 1.0e-300 || rz_new <= 0.0) {
      code = 2;
    } else if (use_mg) {
      beta = beta_num / rz;
      if (beta < 0.0) beta = 0.0;
    } else {
      beta = rz_new / rz;
    }
    // fluid.py:4604-4611 _cg_update_direction_and_rz_kernel.
    for (int64_t c = 0; c < n; ++c) d[c] = (obs[c] == 1) ? 0.0 : z[c] + beta * d[c];
    rz = rz_new;
  }
  st->breakdown_code = code;
  if (st->breakdown_dAd == 0.0) st->breakdown_dAd = code_dAd;
}

EFO_API void efo_fv_pcg_solve(int n_levels, const efo_level* levels, const int32_t* obs, const int32_t* va,
                              const r32* vw, const double* iface, const double* rhs_in, double* pressure,
                              int outlet, int max_iters_in, double tolerance, int precond, int remove_mean,
                              int uniform_grid, int iface_active, efo_cg_stats* st) {
  efo_fv_pcg_solve_anchored(n_levels, levels, obs, va, vw, iface, rhs_in, pressure, outlet, max_iters_in, tolerance,
                            precond, remove_mean, uniform_grid, iface_active, nullptr, 0, st);
}

// fluid.py:5992-6083 _solve_pressure_poisson_fv_multigrid (standalone cycles);
// pressure is the level-0 iterate (warm start), rhs0 the f64 level-0 rhs.
EFO_API void efo_fv_multigrid_solve(int n_levels, const efo_level* levels, const int32_t* obs, const int32_t* va,
                                    const r32* vw, const double* iface, const double* rhs0, double* pressure,
                                    int outlet, int iterations, int cycles, int uniform_grid) {
  const efo_level& L0 = levels[0];
  const int64_t n0 = ncells(L0);
  const double omega = f32arg(0.8);
  std::vector<double> tmp0(n0, 0.0), res0(n0, 0.0);
  if (n_levels <= 1) {
    smooth(L0, pressure, rhs0, iface, obs, va, vw, tmp0.data(), outlet, std::max(1, iterations), omega);
    return;
  }
  Levels lv(n_levels, levels);
  const double scale = f32arg(uniform_grid ? 1.0 : 0.7);
  auto obs_at = [&](int l) -> const int32_t* { return l == 0 ? obs : lv.obs[l].data(); };
  auto va_at = [&](int l) -> const int32_t* { return l == 0 ? va : lv.va[l].data(); };
  auto vw_at = [&](int l) -> const r32* { return l == 0 ? vw : lv.vw[l].data(); };
  for (int cyc = 0; cyc < cycles; ++cyc) {
    for (int l = 0; l < n_levels - 1; ++l) {
      if (l == 0) {
        smooth(L0, pressure, rhs0, iface, obs, va, vw, tmp0.data(), outlet, 3, omega);
        mg_residual(L0, (const double*)pressure, rhs0, iface, obs, va, vw, res0.data(), outlet);
        mg_restrict(L0, (const double*)res0.data(), iface, obs, va, vw, lv.L[1], lv.rhs[1].data(),
                    lv.iface[1].data(), lv.p[1].data(), lv.tmp[1].data(), lv.res[1].data(), lv.obs[1].data(),
                    lv.va[1].data(), lv.vw[1].data());
      } else {
        smooth(lv.L[l], lv.p[l].data(), (const r32*)lv.rhs[l].data(), (const r32*)lv.iface[l].data(), obs_at(l),
               va_at(l), vw_at(l), lv.tmp[l].data(), outlet, 3, omega);
        mg_residual(lv.L[l], (const r32*)lv.p[l].data(), (const r32*)lv.rhs[l].data(),
                    (const r32*)lv.iface[l].data(), obs_at(l), va_at(l), vw_at(l), lv.res[l].data(), outlet);
        mg_restrict(lv.L[l], (const r32*)lv.res[l].data(), (const r32*)lv.iface[l].data(), obs_at(l), va_at(l),
                    vw_at(l), lv.L[l + 1], lv.rhs[l + 1].data(), lv.iface[l + 1].data(), lv.p[l + 1].data(),
                    lv.tmp[l + 1].data(), lv.res[l + 1].data(), lv.obs[l + 1].data(), lv.va[l + 1].data(),
                    lv.vw[l + 1].data());
      }
    }
    const int lc = n_levels - 1;
    smooth(lv.L[lc], lv.p[lc].data(), (const r32*)lv.rhs[lc].data(), (const r32*)lv.iface[lc].data(), obs_at(lc),
           va_at(lc), vw_at(lc), lv.tmp[lc].data(), outlet, 36, omega);
    for (int l = n_levels - 2; l >= 0; --l) {
      if (l == 0) {
        mg_prolong(L0, pressure, obs, lv.L[1], lv.p[1].data(), scale);
        smooth(L0, pressure, rhs0, iface, obs, va, vw, tmp0.data(), outlet, 3, omega);
      } else {
        mg_prolong(lv.L[l], lv.p[l].data(), obs_at(l), lv.L[l + 1], lv.p[l + 1].data(), scale);
        smooth(lv.L[l], lv.p[l].data(), (const r32*)lv.rhs[l].data(), (const r32*)lv.iface[l].data(), obs_at(l),
               va_at(l), vw_at(l), lv.tmp[l].data(), outlet, 3, omega);
      }
    }
  }
  if (!uniform_grid) smooth(L0, pressure, rhs0, iface, obs, va, vw, tmp0.data(), outlet, std::max(1, iterations), omega);
}

// fluid.py:5538-5582 _subtract_pressure_gradient_kernel.
EFO_API void efo_subtract_pressure_gradient(const efo_level* Lp, const int32_t* obs, const int32_t* va,
                                            const r32* vw, const r32* vvalue, const double* p, float dt_over_rho,
                                            int outlet, r32* vel) {
  const efo_level& L = *Lp;
  const int64_t sx = (int64_t)L.ny * L.nz, sy = L.nz;
  const double dtr = (double)(r32)dt_over_rho;
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k) {
        int64_t c = efo_idx(i, j, k, L.ny, L.nz);
        if (obs[c] == 1) {
          vel[3 * c] = vel[3 * c + 1] = vel[3 * c + 2] = 0;
          continue;
        }
        double center = p[c];
        double g[3] = {0.0, 0.0, 0.0};
        if (i > 0 && obs[c - sx] == 0) g[0] = (center - p[c - sx]) / (double)L.cdx[i];
        if (j > 0 && obs[c - sy] == 0) g[1] = (center - p[c - sy]) / (double)L.cdy[j];
        if (k > 0 && obs[c - 1] == 0)
          g[2] = (center - p[c - 1]) / (double)L.cdz[k];
        else if (outlet == 1 && k == 0)
          g[2] = 2.0 * center / (double)L.wz[k];
        double cw = 1.0;
        if (va != nullptr && va[c] != 0) {
          cw = (double)std::min(std::max(vw[c], (r32)0), (r32)1);
          if (cw <= 0.0) {
            vel[3 * c] = vvalue[3 * c];
            vel[3 * c + 1] = vvalue[3 * c + 1];
            vel[3 * c + 2] = vvalue[3 * c + 2];
          }
        }
        if (cw > 0.0) {
          for (int a = 0; a < 3; ++a) vel[3 * c + a] -= (r32)(cw * dtr * g[a]);
        }
      }
}

// fluid.py:5529-5536 _apply_closed_boundary_no_normal_flow_kernel.
EFO_API void efo_apply_closed_boundary(const efo_level* Lp, int outlet, r32* vel) {
  const efo_level& L = *Lp;
  for (int j = 0; j < L.ny; ++j)
    for (int k = 0; k < L.nz; ++k) vel[3 * efo_idx(0, j, k, L.ny, L.nz) + 0] = 0;
  for (int i = 0; i < L.nx; ++i)
    for (int k = 0; k < L.nz; ++k) vel[3 * efo_idx(i, 0, k, L.ny, L.nz) + 1] = 0;
  if (outlet == 0)
    for (int i = 0; i < L.nx; ++i)
      for (int j = 0; j < L.ny; ++j) vel[3 * efo_idx(i, j, 0, L.ny, L.nz) + 2] = 0;
}

// fluid.py:2549-2593 _apply_velocity_dirichlet_boundary_rows_kernel (state part).
EFO_API void efo_apply_velocity_dirichlet_rows(int64_t n, const int32_t* obs, const int32_t* va, const r32* vvalue,
                                               r32* vel) {
  for (int64_t c = 0; c < n; ++c)
    if (va[c] != 0 && obs[c] == 0)
      for (int a = 0; a < 3; ++a) vel[3 * c + a] = vvalue[3 * c + a];
}

// fluid.py:5762-5766 _apply_zmin_no_backflow_kernel.
EFO_API void efo_apply_zmin_no_backflow(const efo_level* Lp, const int32_t* obs, r32* vel) {
  const efo_level& L = *Lp;
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j) {
      int64_t c = efo_idx(i, j, 0, L.ny, L.nz);
      if (obs[c] == 0 && vel[3 * c + 2] > 0) vel[3 * c + 2] = 0;
    }
}

namespace {

// fluid.py:2407-2433 _axis_grid_coordinate_device.
inline r32 axis_coord(r32 v, const r32* faces, const r32* centers, int count) {
  r32 coord = 0;
  if (v <= centers[0]) {
    r32 hw = std::max(centers[0] - faces[0], (r32)1.0e-18);
    coord = (r32)(-0.5) * (centers[0] - v) / hw;
  } else if (v >= centers[count - 1]) {
    r32 hw = std::max(faces[count] - centers[count - 1], (r32)1.0e-18);
    coord = (r32)(count - 1) + (r32)0.5 * (v - centers[count - 1]) / hw;
  } else {
    int lo = 0, hi = count - 1;
    while (hi - lo > 1) {
      int mid = (lo + hi) / 2;
      if (v >= centers[mid])
        lo = mid;
      else
        hi = mid;
    }
    hi = std::min(lo + 1, count - 1);
    r32 dist = std::max(centers[hi] - centers[lo], (r32)1.0e-18);
    coord = (r32)lo + (v - centers[lo]) / dist;
  }
  return coord;
}

inline int ifloor(r32 v) { return (int)std::floor(v); }

// fluid.py:2383-2404 _sample_velocity_prev_trilinear.
inline void sample_prev(const efo_level& L, const int32_t* obs, const r32* vp, r32 gx, r32 gy, r32 gz,
                        const r32* fallback, r32* out) {
  int i0 = std::min(std::max(ifloor(gx), 0), L.nx - 2);
  int j0 = std::min(std::max(ifloor(gy), 0), L.ny - 2);
  int k0 = std::min(std::max(ifloor(gz), 0), L.nz - 2);
  r32 tx = std::min(std::max(gx - (r32)i0, (r32)0), (r32)1);
  r32 ty = std::min(std::max(gy - (r32)j0, (r32)0), (r32)1);
  r32 tz = std::min(std::max(gz - (r32)k0, (r32)0), (r32)1);
  r32 val[3] = {0, 0, 0};
  r32 fw = 0;
  for (int oi = 0; oi < 2; ++oi)
    for (int oj = 0; oj < 2; ++oj)
      for (int ok = 0; ok < 2; ++ok) {
        r32 wx = oi == 0 ? (r32)1 - tx : tx;
        r32 wy = oj == 0 ? (r32)1 - ty : ty;
        r32 wz = ok == 0 ? (r32)1 - tz : tz;
        r32 w = wx * wy * wz;
        int64_t c = efo_idx(i0 + oi, j0 + oj, k0 + ok, L.ny, L.nz);
        if (obs[c] == 0) {
          for (int a = 0; a < 3; ++a) val[a] += w * vp[3 * c + a];
          fw += w;
        }
      }
  if (fw > (r32)1.0e-12) {
    for (int a = 0; a < 3; ++a) out[a] = val[a] / fw;
  } else {
    for (int a = 0; a < 3; ++a) out[a] = fallback[a];
  }
}

}  // namespace

// fluid.py:2447-2527 _predict_kernel (velocity_prev is the copied state).
EFO_API void efo_predict(const efo_grid* G, const int32_t* obs, const r32* vp, float dt_in, float nu_in, int rk2,
                         r32* vel) {
  const efo_level& L = G->l0;
  const r32 dt = (r32)dt_in, nu = (r32)nu_in;
  const int64_t sx = (int64_t)L.ny * L.nz, sy = L.nz;
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k) {
        int64_t c = efo_idx(i, j, k, L.ny, L.nz);
        if (obs[c] == 1) {
          vel[3 * c] = vel[3 * c + 1] = vel[3 * c + 2] = 0;
          continue;
        }
        const r32* center = vp + 3 * c;
        r32 x = G->cx[i], y = G->cy[j], z = G->cz[k];
        r32 trace[3] = {center[0], center[1], center[2]};
        if (rk2) {
          r32 mx = x - (r32)0.5 * dt * center[0];
          r32 my = y - (r32)0.5 * dt * center[1];
          r32 mz = z - (r32)0.5 * dt * center[2];
          sample_prev(L, obs, vp, axis_coord(mx, G->fx, G->cx, L.nx), axis_coord(my, G->fy, G->cy, L.ny),
                      axis_coord(mz, G->fz, G->cz, L.nz), center, trace);
        }
        r32 bx = x - dt * trace[0], by = y - dt * trace[1], bz = z - dt * trace[2];
        r32 adv[3];
        sample_prev(L, obs, vp, axis_coord(bx, G->fx, G->cx, L.nx), axis_coord(by, G->fy, G->cy, L.ny),
                    axis_coord(bz, G->fz, G->cz, L.nz), center, adv);
        r32 fxb[3] = {0, 0, 0}, fxf[3] = {0, 0, 0}, fyb[3] = {0, 0, 0}, fyf[3] = {0, 0, 0}, fzb[3] = {0, 0, 0},
            fzf[3] = {0, 0, 0};
        if (i > 0 && obs[c - sx] == 0)
          for (int a = 0; a < 3; ++a) fxb[a] = (center[a] - vp[3 * (c - sx) + a]) / L.cdx[i];
        if (i < L.nx - 1 && obs[c + sx] == 0)
          for (int a = 0; a < 3; ++a) fxf[a] = (vp[3 * (c + sx) + a] - center[a]) / L.cdx[i + 1];
        if (j > 0 && obs[c - sy] == 0)
          for (int a = 0; a < 3; ++a) fyb[a] = (center[a] - vp[3 * (c - sy) + a]) / L.cdy[j];
        if (j < L.ny - 1 && obs[c + sy] == 0)
          for (int a = 0; a < 3; ++a) fyf[a] = (vp[3 * (c + sy) + a] - center[a]) / L.cdy[j + 1];
        if (k > 0 && obs[c - 1] == 0)
          for (int a = 0; a < 3; ++a) fzb[a] = (center[a] - vp[3 * (c - 1) + a]) / L.cdz[k];
        if (k < L.nz - 1 && obs[c + 1] == 0)
          for (int a = 0; a < 3; ++a) fzf[a] = (vp[3 * (c + 1) + a] - center[a]) / L.cdz[k + 1];
        r32 dtnu = dt * nu;
        for (int a = 0; a < 3; ++a) {
          r32 lap = (fxf[a] - fxb[a]) / L.wx[i] + (fyf[a] - fyb[a]) / L.wy[j] + (fzf[a] - fzb[a]) / L.wz[k];
          vel[3 * c + a] = adv[a] + dtnu * lap;
        }
      }
}

// fluid.py:3196-3273 _spread_surface_forces_kernel (force density into `force`).
EFO_API void efo_spread_surface_forces(const efo_grid* G, const int32_t* obs, const r32* pos, const r32* fsurf,
                                       int vertex_count, float cx_, float cy_, float cz_, float sign_,
                                       r32* force, double* report /* 3 surface, 3 grid */) {
  const efo_level& L = G->l0;
  const int64_t n = ncells(L);
  for (int64_t c = 0; c < 3 * n; ++c) force[c] = 0;
  for (int a = 0; a < 6; ++a) report[a] = 0.0;
  const r32 cen[3] = {(r32)cx_, (r32)cy_, (r32)cz_};
  const r32 sign = (r32)sign_;
  for (int v = 0; v < vertex_count; ++v) {
    r32 p[3], f[3], ff[3];
    for (int a = 0; a < 3; ++a) {
      p[a] = pos[3 * v + a] + cen[a];
      f[a] = fsurf[3 * v + a];
      ff[a] = sign * f[a];
      report[a] += f[a];
    }
    r32 gx = axis_coord(p[0], G->fx, G->cx, L.nx), gy = axis_coord(p[1], G->fy, G->cy, L.ny),
        gz = axis_coord(p[2], G->fz, G->cz, L.nz);
    int bi = ifloor(gx), bj = ifloor(gy), bk = ifloor(gz);
    r32 tx = gx - (r32)bi, ty = gy - (r32)bj, tz = gz - (r32)bk;
    r32 wsum = 0;
    for (int pass = 0; pass < 2; ++pass)
      for (int oi = 0; oi < 2; ++oi)
        for (int oj = 0; oj < 2; ++oj)
          for (int ok = 0; ok < 2; ++ok) {
            int ii = bi + oi, jj = bj + oj, kk = bk + ok;
            if (ii < 0 || ii >= L.nx || jj < 0 || jj >= L.ny || kk < 0 || kk >= L.nz) continue;
            r32 w = (oi == 0 ? (r32)1 - tx : tx) * (oj == 0 ? (r32)1 - ty : ty) * (ok == 0 ? (r32)1 - tz : tz);
            int64_t c = efo_idx(ii, jj, kk, L.ny, L.nz);
            if (obs[c] != 0) continue;
            if (pass == 0) {
              wsum += w;
            } else if (wsum > (r32)0) {
              r32 wn = w / wsum;
              r32 vol = L.wx[ii] * L.wy[jj] * L.wz[kk];
              for (int a = 0; a < 3; ++a) {
                r32 cf = ff[a] * wn;
                force[3 * c + a] += cf / vol;
                report[3 + a] += cf;
              }
            }
          }
  }
}

// fluid.py:3301-3328 _apply_body_force_kernel (state part).
EFO_API void efo_apply_body_force(const efo_level* Lp, const int32_t* obs, const r32* force, float dt_in,
                                  float rho_in, r32* vel) {
  const efo_level& L = *Lp;
  const r32 dt = (r32)dt_in, rho = (r32)rho_in;
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k) {
        int64_t c = efo_idx(i, j, k, L.ny, L.nz);
        if (obs[c] == 0)
          for (int a = 0; a < 3; ++a) vel[3 * c + a] += force[3 * c + a] * (dt / rho);
      }
}

// fluid.py:4345-4456, the interface-coupling terms of
// _fv_laplacian_apply_kernel, added to `out` after the FV operator: each
// coupling (owner, neighbour, transmissibility T > 0) between two fluid cells
// subtracts T / V_owner * p[neighbour] from the owner's row and
// T / V_neighbour * p[owner] from the neighbour's.  The explicit row list is
// used when row_count > 0, else the per-cell slots (active count, first
// neighbour / coefficient, then n_extra extra slots; at most 16 slots in
// all).  Cell volumes are the f32 products of the widths
// (fluid.py:2861-2862).  Sequential order here; the reference adds atomically.
EFO_API void efo_fv_interface_coupling(const efo_level* Lp, const int32_t* obs, const double* p, double* out,
                                       const int32_t* active, const int32_t* nb, const double* coef,
                                       const int32_t* extra_nb, const double* extra_coef, int n_extra,
                                       int row_count, const int32_t* row_owner, const int32_t* row_neighbor,
                                       const double* row_t) {
  const efo_level& L = *Lp;
  auto inside = [&](int i, int j, int k) { return 0 <= i && i < L.nx && 0 <= j && j < L.ny && 0 <= k && k < L.nz; };
  auto vol = [&](int i, int j, int k) {
    const r32 v = L.wx[i] * L.wy[j] * L.wz[k];
    return (double)std::max(v, (r32)1.0e-30);
  };
  auto couple = [&](int i, int j, int k, int ni, int nj, int nk, double t) {
    const int64_t c = efo_idx(i, j, k, L.ny, L.nz), cn = efo_idx(ni, nj, nk, L.ny, L.nz);
    out[c] += -(t / vol(i, j, k)) * p[cn];
    out[cn] += -(t / vol(ni, nj, nk)) * p[c];
  };
  if (row_count > 0) {
    const int limit = std::min(row_count, L.nx * L.ny * L.nz);
    for (int r = 0; r < limit; ++r) {
      const int i = row_owner[3 * r], j = row_owner[3 * r + 1], k = row_owner[3 * r + 2];
      const int ni = row_neighbor[3 * r], nj = row_neighbor[3 * r + 1], nk = row_neighbor[3 * r + 2];
      const double t = row_t[r];
      if (inside(i, j, k) && inside(ni, nj, nk) && obs[efo_idx(i, j, k, L.ny, L.nz)] == 0 &&
          obs[efo_idx(ni, nj, nk, L.ny, L.nz)] == 0 && t > 0.0)
        couple(i, j, k, ni, nj, nk, t);
    }
    return;
  }
  for (int i = 0; i < L.nx; ++i)
    for (int j = 0; j < L.ny; ++j)
      for (int k = 0; k < L.nz; ++k) {
        const int64_t c = efo_idx(i, j, k, L.ny, L.nz);
        if (!(active[c] > 0 && obs[c] == 0)) continue;
        const int slots = std::min(active[c], 1 + n_extra);
        for (int s = 0; s < slots; ++s) {
          const int32_t* q = s == 0 ? nb + 3 * c : extra_nb + 3 * (c * n_extra + (s - 1));
          const double t = s == 0 ? coef[c] : extra_coef[c * n_extra + (s - 1)];
          const int ni = q[0], nj = q[1], nk = q[2];
          if (inside(ni, nj, nk) && obs[efo_idx(ni, nj, nk, L.ny, L.nz)] == 0 && t > 0.0) couple(i, j, k, ni, nj, nk, t);
        }
      }
}

// ---------------------------------------------------------------------------
// z-min outlet pressure reachability and the unreached components
// (CartesianFluidSolver.mark_hibm_pressure_outlet_disconnected_nonprojectable_cells,
// fluid.py:1649-1876, 4764-4910).  Restated as the reference's Jacobi sweeps:
// seed the fluid z = 0 cells, expand until nothing changes (a cell joins from a
// reached neighbour through a face whose upper cell has no Dirichlet row and
// no barrier), then label the unreached fluid cells with the smallest linear
// index of their component (same face rule, min-label sweeps in place) and
// number the components by increasing raw label, stored as -(rank + 1).
// Outputs: reachable (0/1) and label per cell; returns the unreached count,
// and component count / sweeps / convergence through `info`
// (info[0] components, [1] reachability sweeps, [2] converged, [3] labels
// converged, [4] component overflow).
// ---------------------------------------------------------------------------
EFO_API int64_t efo_outlet_reachability(int nx, int ny, int nz, const int32_t* obs, const int32_t* vdir,
                                        const int32_t* barrier, int32_t* reach, int32_t* label, int64_t* info) {
  const int64_t n = (int64_t)nx * ny * nz;
  auto at = [&](const int32_t* a, int i, int j, int k) { return a == nullptr ? 0 : a[efo_idx(i, j, k, ny, nz)]; };
  // face (lower, upper) between cell c and its neighbour, passable iff the
  // upper cell has no Dirichlet row and no barrier (fluid.py:1649-1698)
  auto face_open = [&](int ui, int uj, int uk) { return at(vdir, ui, uj, uk) == 0 && at(barrier, ui, uj, uk) == 0; };
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k)
        reach[efo_idx(i, j, k, ny, nz)] =
            (at(obs, i, j, k) == 0 && at(barrier, i, j, k) == 0 && k == 0 && at(vdir, i, j, k) == 0) ? 1 : 0;
  const int64_t max_sweeps = std::max<int64_t>(1, 32 * (int64_t)(nx + ny + nz));
  std::vector<int32_t> next(reach, reach + n);
  int64_t sweeps = 0;
  bool converged = false;
  for (int64_t s = 0; s < max_sweeps; ++s) {
    int64_t changed = 0;
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) {
          const int64_t c = efo_idx(i, j, k, ny, nz);
          int32_t r = reach[c];
          if (at(obs, i, j, k) == 0 && at(barrier, i, j, k) == 0 && r == 0) {
            const bool hit = (i > 0 && at(reach, i - 1, j, k) != 0 && face_open(i, j, k)) ||
                             (i < nx - 1 && at(reach, i + 1, j, k) != 0 && face_open(i + 1, j, k)) ||
                             (j > 0 && at(reach, i, j - 1, k) != 0 && face_open(i, j, k)) ||
                             (j < ny - 1 && at(reach, i, j + 1, k) != 0 && face_open(i, j + 1, k)) ||
                             (k > 0 && at(reach, i, j, k - 1) != 0 && face_open(i, j, k)) ||
                             (k < nz - 1 && at(reach, i, j, k + 1) != 0 && face_open(i, j, k + 1));
            if (hit) {
              r = 1;
              changed += 1;
            }
          }
          next[c] = r;
        }
    std::copy(next.begin(), next.end(), reach);
    sweeps += 1;
    if (changed == 0) {
      converged = true;
      break;
    }
  }
  int64_t unreached = 0;
  auto open_cell = [&](int i, int j, int k) {
    return at(obs, i, j, k) == 0 && at(barrier, i, j, k) == 0 && at(reach, i, j, k) == 0;
  };
  const int32_t none = 1 << 30;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const int64_t c = efo_idx(i, j, k, ny, nz);
        label[c] = open_cell(i, j, k) ? (int32_t)c : none;
        if (open_cell(i, j, k)) unreached += 1;
      }
  int64_t components = 0;
  bool labels_converged = true, overflow = false;
  if (unreached > 0) {
    labels_converged = false;
    // fluid.py:4776-4845: a neighbour contributes through a face whose upper
    // cell has no barrier and no Dirichlet row, if it is fluid and unreached
    auto nb_ok = [&](int ni, int nj, int nk, int ui, int uj, int uk) {
      return at(obs, ni, nj, nk) == 0 && at(barrier, ui, uj, uk) == 0 && at(reach, ni, nj, nk) == 0 &&
             at(vdir, ui, uj, uk) == 0;
    };
    for (int64_t s = 0; s < max_sweeps; ++s) {
      int64_t changed = 0;
      for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
          for (int k = 0; k < nz; ++k) {
            if (!open_cell(i, j, k)) continue;
            const int64_t c = efo_idx(i, j, k, ny, nz);
            int32_t best = label[c];
            if (i > 0 && nb_ok(i - 1, j, k, i, j, k)) best = std::min(best, label[efo_idx(i - 1, j, k, ny, nz)]);
            if (i < nx - 1 && nb_ok(i + 1, j, k, i + 1, j, k))
              best = std::min(best, label[efo_idx(i + 1, j, k, ny, nz)]);
            if (j > 0 && nb_ok(i, j - 1, k, i, j, k)) best = std::min(best, label[efo_idx(i, j - 1, k, ny, nz)]);
            if (j < ny - 1 && nb_ok(i, j + 1, k, i, j + 1, k))
              best = std::min(best, label[efo_idx(i, j + 1, k, ny, nz)]);
            if (k > 0 && nb_ok(i, j, k - 1, i, j, k)) best = std::min(best, label[efo_idx(i, j, k - 1, ny, nz)]);
            if (k < nz - 1 && nb_ok(i, j, k + 1, i, j, k + 1))
              best = std::min(best, label[efo_idx(i, j, k + 1, ny, nz)]);
            if (best < label[c]) {
              label[c] = best;
              changed += 1;
            }
          }
      if (changed == 0) {
        labels_converged = true;
        break;
      }
    }
    // fluid.py:4885-4910: rank the raw labels; up to 256 components
    std::vector<int32_t> raw;
    for (int64_t c = 0; c < n; ++c)
      if (label[c] >= 0 && label[c] < none) raw.push_back(label[c]);
    std::sort(raw.begin(), raw.end());
    raw.erase(std::unique(raw.begin(), raw.end()), raw.end());
    const int64_t capacity = 256;  // HIBM_PRESSURE_COMPONENT_CAPACITY (fluid.py:17)
    components = std::min<int64_t>((int64_t)raw.size(), capacity);
    overflow = (int64_t)raw.size() > capacity;
    for (int64_t c = 0; c < n; ++c) {
      if (!(label[c] >= 0 && label[c] < none)) continue;
      const auto it = std::lower_bound(raw.begin(), raw.begin() + components, label[c]);
      if (it != raw.begin() + components && *it == label[c]) label[c] = -(int32_t)(it - raw.begin()) - 1;
    }
  }
  info[0] = components;
  info[1] = sweeps;
  info[2] = converged ? 1 : 0;
  info[3] = labels_converged ? 1 : 0;
  info[4] = overflow ? 1 : 0;
  return unreached;
}

// ---------------------------------------------------------------------------
// fluid.py:6264-6533 _continue_pressure_poisson_fv_bicgstab: the BiCGSTAB
// fallback (right Jacobi preconditioning, fluid.py:4614-4661 vector kernels),
// on the level-0 system with rhs `rhs`, from the pressure in `p`.  Every
// breakdown restarts from the true residual until the last iteration, as the
// reference does; remove_mean applies the zero-mean projection where the
// reference's project_field does (no unreached-set anchoring here).
// stats: [0] iterations, [1] converged, [2] restarts, [3] breakdown code
// (0 none, 1 shadow dot, 2 recurrence scalar, 3 beta, 4 alpha denominator,
// 5 alpha, 6 omega denominator, 7 omega, 8 not converged);
// rel_res: the final relative residual.
// ---------------------------------------------------------------------------
EFO_API void efo_bicgstab(const efo_level* Lp, const int32_t* obs, const double* rhs, double* p, int outlet,
                          int max_iters, double tol, double b_norm, int remove_mean, int64_t* stats,
                          double* rel_res) {
  const efo_level& L = *Lp;
  const int64_t n = ncells(L);
  std::vector<double> r(n), r_old(n), d(n, 0.0), Ad(n, 0.0), z(n, 0.0), s(n, 0.0), t(n, 0.0), diag(n);
  fv_diagonal(L, obs, nullptr, nullptr, nullptr, diag.data(), outlet);
  auto project = [&](double* f) {
    if (remove_mean) subtract_mean(L, obs, f);
  };
  auto dot = [&](const std::vector<double>& a, const std::vector<double>& b) {
    return weighted_dot(L, obs, a.data(), b.data());
  };
  auto true_residual = [&]() {
    fv_apply(L, obs, nullptr, nullptr, nullptr, p, Ad.data(), outlet);
    for (int64_t c = 0; c < n; ++c) r[c] = 1.0 * rhs[c] + -1.0 * Ad[c];
    project(r.data());
  };
  auto reset = [&]() {  // fluid.py:4614-4627
    for (int64_t c = 0; c < n; ++c) {
      r_old[c] = obs[c] == 1 ? 0.0 : r[c];
      d[c] = Ad[c] = s[c] = t[c] = 0.0;
    }
  };
  const int iters = std::max(1, max_iters);
  const double tolerance = std::max(0.0, tol), floor = 1.0e-300;
  int64_t it_done = 0, restarts = 0, code = 0;
  bool converged = false;
  double rr;
  true_residual();
  rr = std::sqrt(std::max(dot(r, r), 0.0)) / b_norm;
  if (rr <= tolerance) converged = true;
  double rho_prev = 1.0, alpha = 1.0, omega = 1.0;
  if (!converged) reset();
  for (int it = 1; it <= iters && !converged; ++it) {
    const double rho = dot(r_old, r);
    auto restart = [&](int why) -> bool {  // true: give up
      if (it >= iters) {
        code = why;
        return true;
      }
      return false;
    };
    if (!std::isfinite(rho) || std::fabs(rho) <= floor) {
      if (restart(1)) break;
      true_residual();
      rr = std::sqrt(std::max(dot(r, r), 0.0)) / b_norm;
      it_done = it;
      if (rr <= tolerance) {
        converged = true;
        break;
      }
      reset();
      rho_prev = alpha = omega = 1.0;
      restarts += 1;
      continue;
    }
    double beta = 0.0;
    if (it > 1) {
      if (!std::isfinite(rho_prev) || std::fabs(rho_prev) <= floor || !std::isfinite(omega) ||
          std::fabs(omega) <= floor) {
        if (restart(2)) break;
        true_residual();
        reset();
        rho_prev = alpha = omega = 1.0;
        restarts += 1;
        continue;
      }
      beta = (rho / rho_prev) * (alpha / omega);
      if (!std::isfinite(beta)) {
        if (restart(3)) break;
        true_residual();
        reset();
        rho_prev = alpha = omega = 1.0;
        restarts += 1;
        continue;
      }
    }
    for (int64_t c = 0; c < n; ++c) d[c] = obs[c] == 1 ? 0.0 : r[c] + beta * (d[c] - omega * Ad[c]);
    jacobi_precond(n, obs, diag.data(), d.data(), z.data());
    project(z.data());
    fv_apply(L, obs, nullptr, nullptr, nullptr, z.data(), Ad.data(), outlet);
    const double alpha_den = dot(r_old, Ad);
    if (!std::isfinite(alpha_den) || std::fabs(alpha_den) <= floor) {
      if (restart(4)) break;
      true_residual();
      reset();
      rho_prev = alpha = omega = 1.0;
      restarts += 1;
      continue;
    }
    alpha = rho / alpha_den;
    if (!std::isfinite(alpha)) {
      if (restart(5)) break;
      true_residual();
      reset();
      rho_prev = alpha = omega = 1.0;
      restarts += 1;
      continue;
    }
    for (int64_t c = 0; c < n; ++c) {
      if (obs[c] == 1) {
        p[c] = 0.0;
        s[c] = 0.0;
      } else {
        p[c] += alpha * z[c];
        s[c] = r[c] - alpha * Ad[c];
      }
    }
    project(s.data());
    rr = std::sqrt(std::max(dot(s, s), 0.0)) / b_norm;
    it_done = it;
    if (rr <= tolerance) {
      r = s;
      converged = true;
      break;
    }
    jacobi_precond(n, obs, diag.data(), s.data(), z.data());
    project(z.data());
    fv_apply(L, obs, nullptr, nullptr, nullptr, z.data(), t.data(), outlet);
    const double ts = dot(t, s), tt = dot(t, t);
    if (!std::isfinite(tt) || std::fabs(tt) <= floor) {
      if (restart(6)) break;
      r = s;
      project(r.data());
      reset();
      rho_prev = alpha = omega = 1.0;
      restarts += 1;
      continue;
    }
    omega = ts / tt;
    if (!std::isfinite(omega) || std::fabs(omega) <= floor) {
      if (restart(7)) break;
      r = s;
      project(r.data());
      reset();
      rho_prev = alpha = omega = 1.0;
      restarts += 1;
      continue;
    }
    for (int64_t c = 0; c < n; ++c) {
      if (obs[c] == 1) {
        p[c] = 0.0;
        r[c] = 0.0;
      } else {
        p[c] += omega * z[c];
        r[c] = s[c] - omega * t[c];
      }
    }
    if (it % 16 == 0) {
      project(p);
      project(r.data());
    }
    rr = std::sqrt(std::max(dot(r, r), 0.0)) / b_norm;
    it_done = it;
    if (rr <= tolerance) {
      converged = true;
      break;
    }
    rho_prev = rho;
  }
  if (!converged && code == 0) code = 8;
  stats[0] = it_done;
  stats[1] = converged ? 1 : 0;
  stats[2] = restarts;
  stats[3] = code;
  *rel_res = rr;
}
