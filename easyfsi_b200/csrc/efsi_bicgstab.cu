// The BiCGSTAB fallback of the FV pressure solve
// (CartesianFluidSolver._continue_pressure_poisson_fv_bicgstab, fluid.py:6264-6533).
//
// The reference runs it as a host loop over device kernels with a host read
// of every inner product; so does this one.  It is built on the plan's own
// level-0 operator, diagonal, Jacobi preconditioner and weighted dot (the
// same entry points the PCG path uses), plus the five vector updates of
// fluid.py:4519-4531 and 4614-4661 below.
#include <cmath>
#include <vector>

#include "efsi_fv_internal.cuh"

namespace efsi {
namespace {

__device__ __forceinline__ bool solid(const uint8_t* mask, int64_t c) { return (mask[c] & M_SOLID) != 0; }
__device__ __forceinline__ bool fluid(const uint8_t* mask, int64_t c) { return (mask[c] & M_FLUID) != 0; }

#define EFSI_GRID_STRIDE(c, n) \
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < (n); c += (int64_t)gridDim.x * blockDim.x)

// fluid.py:4519-4531 with a = 1, b = -1: r = rhs - A p
__global__ void k_bicg_residual(int64_t n, const uint8_t* __restrict__ mask, const double* __restrict__ rhs,
                                const double* __restrict__ Ap, double* __restrict__ r) {
  EFSI_GRID_STRIDE(c, n) r[c] = solid(mask, c) ? 0.0 : 1.0 * rhs[c] + -1.0 * Ap[c];
}

// fluid.py:4614-4627
__global__ void k_bicg_reset(int64_t n, const uint8_t* __restrict__ mask, const double* __restrict__ r,
                             double* __restrict__ r_old, double* __restrict__ d, double* __restrict__ Ad,
                             double* __restrict__ s, double* __restrict__ t) {
  EFSI_GRID_STRIDE(c, n) {
    r_old[c] = solid(mask, c) ? 0.0 : r[c];
    d[c] = 0.0;
    Ad[c] = 0.0;
    s[c] = 0.0;
    t[c] = 0.0;
  }
}

// fluid.py:4630-4637
__global__ void k_bicg_direction(int64_t n, const uint8_t* __restrict__ mask, const double* __restrict__ r,
                                 double* __restrict__ d, const double* __restrict__ Ad, double beta, double omega) {
  EFSI_GRID_STRIDE(c, n) d[c] = solid(mask, c) ? 0.0 : r[c] + beta * (d[c] - omega * Ad[c]);
}

// fluid.py:4640-4649
__global__ void k_bicg_alpha(int64_t n, const uint8_t* __restrict__ mask, double* __restrict__ p,
                             const double* __restrict__ z, const double* __restrict__ r,
                             const double* __restrict__ Ad, double* __restrict__ s, double alpha) {
  EFSI_GRID_STRIDE(c, n) {
    if (solid(mask, c)) {
      p[c] = 0.0;
      s[c] = 0.0;
    } else {
      p[c] += alpha * z[c];
      s[c] = r[c] - alpha * Ad[c];
    }
  }
}

// fluid.py:4652-4661
__global__ void k_bicg_omega(int64_t n, const uint8_t* __restrict__ mask, double* __restrict__ p,
                             const double* __restrict__ z, const double* __restrict__ s,
                             const double* __restrict__ t, double* __restrict__ r, double omega) {
  EFSI_GRID_STRIDE(c, n) {
    if (solid(mask, c)) {
      p[c] = 0.0;
      r[c] = 0.0;
    } else {
      p[c] += omega * z[c];
      r[c] = s[c] - omega * t[c];
    }
  }
}

// fluid.py:4716-4726: f -= its volume-weighted fluid mean; 0 off the fluid
__global__ void k_bicg_sub_mean(int64_t n, const uint8_t* __restrict__ mask, double* __restrict__ f, double m) {
  EFSI_GRID_STRIDE(c, n) f[c] = fluid(mask, c) ? f[c] - m : 0.0;
}

__global__ void k_bicg_fill(int64_t n, double* __restrict__ f, double v) { EFSI_GRID_STRIDE(c, n) f[c] = v; }

#undef EFSI_GRID_STRIDE

}  // namespace
}  // namespace efsi

using namespace efsi;

extern "C" {

int efsi_fv_bicgstab(efsi_fv_plan* P, const double* rhs, double* pressure, int32_t outlet, int32_t max_iters,
                     double tolerance, double b_norm, int32_t remove_mean, int64_t* stats, double* relative_residual,
                     void* stream) {
  EFSI_TRY(level_zero_check(P));
  EFSI_ARG_CHECK(rhs != nullptr && pressure != nullptr && stats != nullptr && relative_residual != nullptr,
                 "null argument");
  EFSI_ARG_CHECK(std::isfinite(b_norm) && b_norm > 0.0, "b_norm must be a finite positive number");
  cudaStream_t s = as_stream(stream);
  const LevelDev L = level_dev(P, 0);
  const int64_t n = P->lv[0].n;
  const uint8_t* mask = L.mask;
  const unsigned grid = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16);
  // work vectors: r, r_old, d, Ad, z, s, t, diag, ones; the plan keeps them
  // from the first fallback on (level 0 never changes size within a plan)
  if (P->bicg_work == nullptr) EFSI_CUDA_CHECK(cudaMalloc(&P->bicg_work, 9 * (size_t)n * sizeof(double)));
  double* w = P->bicg_work;
  double *r = w, *r_old = w + n, *d = w + 2 * n, *Ad = w + 3 * n, *z = w + 4 * n, *sv = w + 5 * n, *t = w + 6 * n,
         *diag = w + 7 * n, *ones = w + 8 * n;
  int status = EFSI_OK;
  auto run = [&]() -> int {
    EFSI_TRY(efsi_fv_diagonal(P, diag, outlet, stream));
    double free_vol = 0.0;
    if (remove_mean) {
      EFSI_COUNTED k_bicg_fill<<<grid, 256, 0, s>>>(n, ones, 1.0);
      EFSI_TRY(efsi_weighted_dot(P, ones, ones, &free_vol, stream));
    }
    auto dot = [&](const double* a, const double* b, double& out) { return efsi_weighted_dot(P, a, b, &out, stream); };
    // with an outlet and unreached components: their means first
    // (fluid.py:6282-6296 project_field / project_pressure_and_residual)
    const bool anchor = outlet != 0 && P->ucomp_n > 0;
    auto project = [&](double* f) -> int {
      if (anchor) EFSI_TRY(efsi_fv_subtract_unreached_means(P, f, nullptr, nullptr, stream));
      if (!remove_mean) return EFSI_OK;
      double sum = 0.0;
      EFSI_TRY(dot(f, ones, sum));
      const double m = free_vol > 0.0 ? sum / free_vol : 0.0;
      EFSI_COUNTED k_bicg_sub_mean<<<grid, 256, 0, s>>>(n, mask, f, m);
      return EFSI_OK;
    };
    auto true_residual = [&]() -> int {
      EFSI_TRY(efsi_fv_apply(P, pressure, Ad, outlet, stream));
      EFSI_COUNTED k_bicg_residual<<<grid, 256, 0, s>>>(n, mask, rhs, Ad, r);
      return project(r);
    };
    auto reset = [&]() { EFSI_COUNTED k_bicg_reset<<<grid, 256, 0, s>>>(n, mask, r, r_old, d, Ad, sv, t); };
    auto norm_of = [&](const double* f, double& out) -> int {
      double q = 0.0;
      EFSI_TRY(dot(f, f, q));
      out = std::sqrt(std::max(q, 0.0)) / b_norm;
      return EFSI_OK;
    };
    const int iters = std::max(1, (int)max_iters);
    const double tol = std::max(0.0, tolerance), floor_v = 1.0e-300;
    int64_t it_done = 0, restarts = 0, code = 0;
    bool converged = false;
    double rr = 0.0;
    EFSI_TRY(true_residual());
    EFSI_TRY(norm_of(r, rr));
    if (rr <= tol) converged = true;
    double rho_prev = 1.0, alpha = 1.0, omega = 1.0;
    if (!converged) reset();
    for (int it = 1; it <= iters && !converged; ++it) {
      double rho = 0.0;
      EFSI_TRY(dot(r_old, r, rho));
      const bool last = it >= iters;
      if (!std::isfinite(rho) || std::fabs(rho) <= floor_v) {
        if (last) {
          code = 1;
          break;
        }
        EFSI_TRY(true_residual());
        EFSI_TRY(norm_of(r, rr));
        it_done = it;
        if (rr <= tol) {
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
        const bool bad_prev = !std::isfinite(rho_prev) || std::fabs(rho_prev) <= floor_v || !std::isfinite(omega) ||
                              std::fabs(omega) <= floor_v;
        if (!bad_prev) beta = (rho / rho_prev) * (alpha / omega);
        if (bad_prev || !std::isfinite(beta)) {
          if (last) {
            code = bad_prev ? 2 : 3;
            break;
          }
          EFSI_TRY(true_residual());
          reset();
          rho_prev = alpha = omega = 1.0;
          restarts += 1;
          continue;
        }
      }
      EFSI_COUNTED k_bicg_direction<<<grid, 256, 0, s>>>(n, mask, r, d, Ad, beta, omega);
      EFSI_TRY(efsi_apply_jacobi_preconditioner(P, diag, d, z, stream));
      EFSI_TRY(project(z));
      EFSI_TRY(efsi_fv_apply(P, z, Ad, outlet, stream));
      double alpha_den = 0.0;
      EFSI_TRY(dot(r_old, Ad, alpha_den));
      const bool bad_den = !std::isfinite(alpha_den) || std::fabs(alpha_den) <= floor_v;
      if (!bad_den) alpha = rho / alpha_den;
      if (bad_den || !std::isfinite(alpha)) {
        if (last) {
          code = bad_den ? 4 : 5;
          break;
        }
        EFSI_TRY(true_residual());
        reset();
        rho_prev = alpha = omega = 1.0;
        restarts += 1;
        continue;
      }
      EFSI_COUNTED k_bicg_alpha<<<grid, 256, 0, s>>>(n, mask, pressure, z, r, Ad, sv, alpha);
      EFSI_TRY(project(sv));
      EFSI_TRY(norm_of(sv, rr));
      it_done = it;
      if (rr <= tol) {
        EFSI_CUDA_CHECK(cudaMemcpyAsync(r, sv, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        converged = true;
        break;
      }
      EFSI_TRY(efsi_apply_jacobi_preconditioner(P, diag, sv, z, stream));
      EFSI_TRY(project(z));
      EFSI_TRY(efsi_fv_apply(P, z, t, outlet, stream));
      double ts = 0.0, tt = 0.0;
      EFSI_TRY(dot(t, sv, ts));
      EFSI_TRY(dot(t, t, tt));
      const bool bad_tt = !std::isfinite(tt) || std::fabs(tt) <= floor_v;
      if (!bad_tt) omega = ts / tt;
      if (bad_tt || !std::isfinite(omega) || std::fabs(omega) <= floor_v) {
        if (last) {
          code = bad_tt ? 6 : 7;
          break;
        }
        EFSI_CUDA_CHECK(cudaMemcpyAsync(r, sv, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        EFSI_TRY(project(r));
        reset();
        rho_prev = alpha = omega = 1.0;
        restarts += 1;
        continue;
      }
      EFSI_COUNTED k_bicg_omega<<<grid, 256, 0, s>>>(n, mask, pressure, z, sv, t, r, omega);
      if (it % 16 == 0) {
        EFSI_TRY(project(pressure));
        EFSI_TRY(project(r));
      }
      EFSI_TRY(norm_of(r, rr));
      it_done = it;
      if (rr <= tol) {
        converged = true;
        break;
      }
      rho_prev = rho;
    }
    if (!converged && code == 0) code = 8;
    EFSI_LAUNCH_CHECK();
    EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
    stats[0] = it_done;
    stats[1] = converged ? 1 : 0;
    stats[2] = restarts;
    stats[3] = code;
    *relative_residual = rr;
    return EFSI_OK;
  };
  status = run();
  const cudaError_t sync = cudaStreamSynchronize(s);
  if (status == EFSI_OK && sync != cudaSuccess) {
    set_error(std::string("efsi_fv_bicgstab: ") + cudaGetErrorString(sync));
    return EFSI_ERR_CUDA;
  }
  return status;
}

}  // extern "C"
