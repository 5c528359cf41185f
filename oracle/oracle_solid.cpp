// CPU oracle, solid and coupling part -- TEST INFRASTRUCTURE ONLY (see
// oracle_common.h).
//
// Restates simulation_core/neo_hookean_mpm.py (the MLS/APIC-MPM substep) and
// the marker part of simulation_core/hibm_mpm.py (pressure traction sampling,
// marker forces, marker -> particle force spreading, particle -> marker surface
// feedback).  The spreading and feedback loops are the reference's brute-force
// O(markers x particles) loops, kept as such: that is the algorithm the CUDA
// path's binned version must agree with.
#include "oracle_common.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef double m3d[3][3];

inline double det3(const m3d a) {
  return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
         a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
}

// One-sided Jacobi SVD (Hestenes 1958; see Demmel & Veselic, "Jacobi's method
// is more accurate than QR", SIAM J. Matrix Anal. Appl. 13(4), 1992): rotate
// column pairs of A until they are mutually orthogonal; A V = U S.  Returns
// U, s (descending, >= 0) and V with det(V) = +1 (det(U) = sign(det A)).
void svd3(const m3d A_in, m3d U, double s[3], m3d V) {
  m3d A;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      A[i][j] = A_in[i][j];
      V[i][j] = (i == j) ? 1.0 : 0.0;
    }
  for (int sweep = 0; sweep < 30; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        double alpha = 0, beta = 0, gamma = 0;
        for (int i = 0; i < 3; ++i) {
          alpha += A[i][p] * A[i][p];
          beta += A[i][q] * A[i][q];
          gamma += A[i][p] * A[i][q];
        }
        if (gamma == 0.0) continue;
        double scale = std::sqrt(alpha * beta);
        if (scale > 0.0) off = std::max(off, std::fabs(gamma) / scale);
        if (std::fabs(gamma) <= 1.0e-15 * scale) continue;
        double zeta = (beta - alpha) / (2.0 * gamma);
        double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        double c = 1.0 / std::sqrt(1.0 + t * t);
        double sn = c * t;
        for (int i = 0; i < 3; ++i) {
          double ap = A[i][p], aq = A[i][q];
          A[i][p] = c * ap - sn * aq;
          A[i][q] = sn * ap + c * aq;
          double vp = V[i][p], vq = V[i][q];
          V[i][p] = c * vp - sn * vq;
          V[i][q] = sn * vp + c * vq;
        }
      }
    if (off <= 1.0e-15) break;
  }
  for (int j = 0; j < 3; ++j) s[j] = std::sqrt(A[0][j] * A[0][j] + A[1][j] * A[1][j] + A[2][j] * A[2][j]);
  // Sort descending (columns of A and V move together).
  int order[3] = {0, 1, 2};
  std::sort(order, order + 3, [&](int a, int b) { return s[a] > s[b]; });
  m3d A2, V2;
  double s2[3];
  for (int j = 0; j < 3; ++j) {
    s2[j] = s[order[j]];
    for (int i = 0; i < 3; ++i) {
      A2[i][j] = A[i][order[j]];
      V2[i][j] = V[i][order[j]];
    }
  }
  if (det3(V2) < 0.0)
    for (int i = 0; i < 3; ++i) {
      V2[i][2] = -V2[i][2];
      A2[i][2] = -A2[i][2];
    }
  for (int j = 0; j < 3; ++j) {
    s[j] = s2[j];
    for (int i = 0; i < 3; ++i) V[i][j] = V2[i][j];
  }
  for (int j = 0; j < 2; ++j)
    for (int i = 0; i < 3; ++i) U[i][j] = s[j] > 1.0e-300 ? A2[i][j] / s[j] : (i == j ? 1.0 : 0.0);
  if (s[2] > 1.0e-12 * std::max(s[0], 1.0e-300)) {
    for (int i = 0; i < 3; ++i) U[i][2] = A2[i][2] / s[2];
  } else {
    // Rank-deficient: complete U with the cross product; sign from det(A).
    double cx = U[1][0] * U[2][1] - U[2][0] * U[1][1];
    double cy = U[2][0] * U[0][1] - U[0][0] * U[2][1];
    double cz = U[0][0] * U[1][1] - U[1][0] * U[0][1];
    double sg = det3(A_in) < 0.0 ? -1.0 : 1.0;
    U[0][2] = sg * cx;
    U[1][2] = sg * cy;
    U[2][2] = sg * cz;
  }
}

// Deformation clamp of neo_hookean_mpm.py:720-748.  Writes the clamped F to Fp
// and returns 1 when the reference would count a clamp (and write F back).
// When no clamp is required the stress is evaluated on F itself (the reference
// evaluates it on its f32 SVD reconstruction, equal to F to f32 round-off).
int clamp_deformation(const r32 F[9], r32 Fp[9]) {
  m3d A;
  double frob2 = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      A[i][j] = (double)F[3 * i + j];
      frob2 += A[i][j] * A[i][j];
    }
  double det = det3(A);
  // Cheap sufficient test: sigma_max <= ||F||_F and
  // sigma_min >= |det| / (sigma_1 sigma_2) >= 2 |det| / ||F||_F^2.
  if (det > 0.0 && frob2 <= 99.99 * 99.99 && 2.0 * det >= 0.0101 * frob2) {
    for (int a = 0; a < 9; ++a) Fp[a] = F[a];
    return 0;
  }
  m3d U, V;
  double s[3];
  svd3(A, U, s, V);
  double sign3 = 1.0;
  if (det < 0.0) {  // reference SVD keeps U, V proper rotations, sigma_3 < 0
    sign3 = -1.0;
    for (int i = 0; i < 3; ++i) U[i][2] = -U[i][2];
  }
  r32 raw[3] = {(r32)s[0], (r32)s[1], (r32)(sign3 * s[2])};
  int clamped = 0;
  double c[3];
  for (int a = 0; a < 3; ++a) {
    r32 cs = std::min(std::max((r32)std::fabs(raw[a]), (r32)1.0e-2), (r32)1.0e2);
    if (std::fabs(cs - raw[a]) > (r32)1.0e-6) clamped = 1;
    c[a] = (double)cs;
  }
  r32 rawF[9];
  for (int a = 0; a < 9; ++a) rawF[a] = F[a];
  r32 rawJ = rawF[0] * (rawF[4] * rawF[8] - rawF[5] * rawF[7]) - rawF[1] * (rawF[3] * rawF[8] - rawF[5] * rawF[6]) +
             rawF[2] * (rawF[3] * rawF[7] - rawF[4] * rawF[6]);
  if (rawJ <= (r32)0) clamped = 1;
  if (!clamped) {
    for (int a = 0; a < 9; ++a) Fp[a] = F[a];
    return 0;
  }
  m3d P;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) P[i][j] = U[i][0] * c[0] * V[j][0] + U[i][1] * c[1] * V[j][1] + U[i][2] * c[2] * V[j][2];
  if (det3(P) <= 0.0)
    for (int i = 0; i < 3; ++i) P[i][2] = -P[i][2];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Fp[3 * i + j] = (r32)P[i][j];
  return 1;
}

inline void quad_weights(r32 fx, r32 w[3]) {
  // neo_hookean_mpm.py:688-693 _weights.
  w[0] = (r32)0.5 * ((r32)1.5 - fx) * ((r32)1.5 - fx);
  w[1] = (r32)0.75 - (fx - (r32)1.0) * (fx - (r32)1.0);
  w[2] = (r32)0.5 * (fx - (r32)0.5) * (fx - (r32)0.5);
}

}  // namespace

// MPM state (host arrays, particle-major AoS like the reference's Taichi fields).
typedef struct efo_mpm {
  int32_t particle_count;
  int32_t nx, ny, nz;
  double bmin[3];
  double dx[3];
  r32* x;      // (P,3)
  r32* v;      // (P,3)
  r32* C;      // (P,3,3)
  r32* F;      // (P,3,3)
  const r32* mass;
  const r32* volume;
  const r32* fext;  // (P,3)
  const int32_t* fixed;
  const int32_t* region;
  const r32* rest_x;
  r32* normal;            // surface_normal (P,3)
  r32* area;              // area_weight_m2
  const r32* rest_normal;
  const r32* rest_area;
  r32* grid_mass;  // (G)
  r32* grid_vel;   // (G,3)
  r32* grid_force;
} efo_mpm;

namespace {

inline int stencil_oob(const efo_mpm& S, const r32 X[3]) {
  int oob = 0;
  const int n[3] = {S.nx, S.ny, S.nz};
  for (int a = 0; a < 3; ++a)
    if (X[a] < (r32)0.5 || X[a] >= (r32)n[a] - (r32)1.5) oob = 1;
  return oob;
}

inline void grid_coord(const efo_mpm& S, const r32* x, r32 X[3]) {
  for (int a = 0; a < 3; ++a) X[a] = (x[a] - (r32)S.bmin[a]) / (r32)S.dx[a];
}

// neo_hookean_mpm.py:674-685 _update_surface_geometry_from_deformation.
void surface_geometry(const efo_mpm& S, int p) {
  r32 ra = S.rest_area[p];
  const r32* rn = S.rest_normal + 3 * p;
  r32 rnn = std::sqrt(rn[0] * rn[0] + rn[1] * rn[1] + rn[2] * rn[2]);
  if (!(ra > (r32)0 && rnn > (r32)1.0e-12)) return;
  const r32* F = S.F + 9 * p;
  r32 J = F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) + F[2] * (F[3] * F[7] - F[4] * F[6]);
  if (!(J > (r32)1.0e-12)) return;
  // cofactor matrix = J * F^-T
  r32 cof[9] = {F[4] * F[8] - F[5] * F[7], F[5] * F[6] - F[3] * F[8], F[3] * F[7] - F[4] * F[6],
                F[2] * F[7] - F[1] * F[8], F[0] * F[8] - F[2] * F[6], F[1] * F[6] - F[0] * F[7],
                F[1] * F[5] - F[2] * F[4], F[2] * F[3] - F[0] * F[5], F[0] * F[4] - F[1] * F[3]};
  r32 av[3];
  for (int i = 0; i < 3; ++i) av[i] = cof[3 * i] * rn[0] + cof[3 * i + 1] * rn[1] + cof[3 * i + 2] * rn[2];
  r32 sc = std::sqrt(av[0] * av[0] + av[1] * av[1] + av[2] * av[2]);
  if (sc > (r32)1.0e-12) {
    for (int a = 0; a < 3; ++a) S.normal[3 * p + a] = av[a] / sc;
    S.area[p] = ra * sc;
  }
}

}  // namespace

// Report snapshot layout of neo_hookean_mpm.py:909-958 (28 floats + 6 counts).
typedef struct efo_mpm_report {
  double values[28];
  int64_t counts[6];
} efo_mpm_report;

// neo_hookean_mpm.py:696-959 _step_kernel.
EFO_API void efo_mpm_step(efo_mpm* Sp, float dt_in, float mu_in, float lambda_in, float damping_in, int primary_id,
                          int secondary_id, efo_mpm_report* rep) {
  efo_mpm& S = *Sp;
  const r32 dt = (r32)dt_in, mu = (r32)mu_in, lam = (r32)lambda_in, damping = (r32)damping_in;
  const int64_t G = (int64_t)S.nx * S.ny * S.nz;
  const int P = S.particle_count;
  const r32 dxr[3] = {(r32)S.dx[0], (r32)S.dx[1], (r32)S.dx[2]};
  const r32 inv4[3] = {(r32)(4.0 / (S.dx[0] * S.dx[0])), (r32)(4.0 / (S.dx[1] * S.dx[1])),
                       (r32)(4.0 / (S.dx[2] * S.dx[2]))};
  std::memset(S.grid_mass, 0, sizeof(r32) * G);
  std::memset(S.grid_vel, 0, sizeof(r32) * 3 * G);
  std::memset(S.grid_force, 0, sizeof(r32) * 3 * G);
  double pmom[3] = {0, 0, 0}, fsum[3] = {0, 0, 0}, msum = 0, vsum = 0, mom2 = 0, maxJ = 0;
  int64_t oob = 0, clamps = 0;
#pragma omp parallel for schedule(static) reduction(+ : pmom[:3], fsum[:3], msum, vsum, mom2, oob, clamps) \
    reduction(max : maxJ)
  for (int p = 0; p < P; ++p) {
    r32 X[3];
    grid_coord(S, S.x + 3 * p, X);
    int base[3];
    r32 fx[3], w[3][3];
    for (int a = 0; a < 3; ++a) {
      base[a] = (int)std::floor(X[a] - (r32)0.5);
      fx[a] = X[a] - (r32)base[a];
      quad_weights(fx[a], w[a]);
    }
    r32 Fp[9];
    if (clamp_deformation(S.F + 9 * p, Fp)) {
      clamps += 1;
      for (int a = 0; a < 9; ++a) S.F[9 * p + a] = Fp[a];
    }
    // J and log J in f64 (det F / log J evaluation), the inverse in r32.
    double J = (double)Fp[0] * ((double)Fp[4] * Fp[8] - (double)Fp[5] * Fp[7]) -
               (double)Fp[1] * ((double)Fp[3] * Fp[8] - (double)Fp[5] * Fp[6]) +
               (double)Fp[2] * ((double)Fp[3] * Fp[7] - (double)Fp[4] * Fp[6]);
    r32 Jr = (r32)J;
    r32 cof[9] = {Fp[4] * Fp[8] - Fp[5] * Fp[7], Fp[5] * Fp[6] - Fp[3] * Fp[8], Fp[3] * Fp[7] - Fp[4] * Fp[6],
                  Fp[2] * Fp[7] - Fp[1] * Fp[8], Fp[0] * Fp[8] - Fp[2] * Fp[6], Fp[1] * Fp[6] - Fp[0] * Fp[7],
                  Fp[1] * Fp[5] - Fp[2] * Fp[4], Fp[2] * Fp[3] - Fp[0] * Fp[5], Fp[0] * Fp[4] - Fp[1] * Fp[3]};
    // F^-T = cof / J  (cof is the cofactor matrix, i.e. (adj F)^T)
    r32 FinvT[9];
    for (int a = 0; a < 9; ++a) FinvT[a] = cof[a] / Jr;
    r32 lnJ = (r32)std::log(J);
    r32 Pm[9];
    for (int a = 0; a < 9; ++a) Pm[a] = mu * (Fp[a] - FinvT[a]) + lam * lnJ * FinvT[a];
    // stress = -dt V (P F^T) diag(4/dx^2)
    r32 sv = -dt * S.volume[p];
    r32 affine[9];
    const r32* Cp = S.C + 9 * p;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        r32 pf = Pm[3 * i + 0] * Fp[3 * j + 0] + Pm[3 * i + 1] * Fp[3 * j + 1] + Pm[3 * i + 2] * Fp[3 * j + 2];
        affine[3 * i + j] = sv * (pf * inv4[j]) + S.mass[p] * Cp[3 * i + j];
      }
    r32 mom[3], fe[3];
    for (int a = 0; a < 3; ++a) {
      mom[a] = S.mass[p] * S.v[3 * p + a];
      fe[a] = S.fext[3 * p + a];
    }
    if (S.fixed[p] != 0) {
      for (int a = 0; a < 3; ++a) mom[a] = fe[a] = 0;
      for (int a = 0; a < 9; ++a) affine[a] = 0;
    }
    for (int a = 0; a < 3; ++a) {
      pmom[a] += mom[a];
      fsum[a] += fe[a];
    }
    msum += S.mass[p];
    vsum += S.volume[p];
    mom2 += (double)(mom[0] * mom[0] + mom[1] * mom[1] + mom[2] * mom[2]);
    maxJ = std::max(maxJ, std::fabs((double)Jr));
    if (stencil_oob(S, X)) {
      oob += 1;
      continue;
    }
    for (int ox = 0; ox < 3; ++ox)
      for (int oy = 0; oy < 3; ++oy)
        for (int oz = 0; oz < 3; ++oz) {
          r32 wt = w[0][ox] * w[1][oy] * w[2][oz];
          r32 dpos[3] = {((r32)ox - fx[0]) * dxr[0], ((r32)oy - fx[1]) * dxr[1], ((r32)oz - fx[2]) * dxr[2]};
          int64_t node = efo_idx(base[0] + ox, base[1] + oy, base[2] + oz, S.ny, S.nz);
          r32 add_m = wt * S.mass[p];
#pragma omp atomic
          S.grid_mass[node] += add_m;
          for (int a = 0; a < 3; ++a) {
            r32 ad = affine[3 * a + 0] * dpos[0] + affine[3 * a + 1] * dpos[1] + affine[3 * a + 2] * dpos[2];
            r32 m = wt * (mom[a] + ad);
            r32 f = wt * fe[a];
#pragma omp atomic
            S.grid_vel[3 * node + a] += m;
#pragma omp atomic
            S.grid_force[3 * node + a] += f;
          }
        }
  }
  double tmom[3] = {0, 0, 0}, gmom[3] = {0, 0, 0}, maxspeed = 0;
  int64_t active = 0;
#pragma omp parallel for schedule(static) reduction(+ : tmom[:3], gmom[:3], active) reduction(max : maxspeed)
  for (int64_t g = 0; g < G; ++g) {
    r32 m = S.grid_mass[g];
    if (m > (r32)1.0e-20) {
      r32 vv[3], tv[3];
      for (int a = 0; a < 3; ++a) {
        vv[a] = S.grid_vel[3 * g + a] / m;
        vv[a] += dt * S.grid_force[3 * g + a] / m;
        tv[a] = vv[a];
        vv[a] *= damping;
        S.grid_vel[3 * g + a] = vv[a];
        tmom[a] += (double)(m * tv[a]);
        gmom[a] += (double)(m * vv[a]);
      }
      active += 1;
      maxspeed = std::max(maxspeed, (double)std::sqrt(vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2]));
    }
  }
  double psum_d[3] = {0, 0, 0}, psum_v[3] = {0, 0, 0}, ssum_d[3] = {0, 0, 0}, ssum_v[3] = {0, 0, 0};
  int64_t pc = 0, sc = 0;
#pragma omp parallel for schedule(static) reduction(+ : psum_d[:3], psum_v[:3], ssum_d[:3], ssum_v[:3], pc, sc)
  for (int p = 0; p < P; ++p) {
    r32 X[3];
    grid_coord(S, S.x + 3 * p, X);
    if (!stencil_oob(S, X)) {
      int base[3];
      r32 fx[3], w[3][3];
      for (int a = 0; a < 3; ++a) {
        base[a] = (int)std::floor(X[a] - (r32)0.5);
        fx[a] = X[a] - (r32)base[a];
        quad_weights(fx[a], w[a]);
      }
      r32 nv[3] = {0, 0, 0}, nC[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int ox = 0; ox < 3; ++ox)
        for (int oy = 0; oy < 3; ++oy)
          for (int oz = 0; oz < 3; ++oz) {
            r32 wt = w[0][ox] * w[1][oy] * w[2][oz];
            r32 dpos[3] = {((r32)ox - fx[0]) * dxr[0], ((r32)oy - fx[1]) * dxr[1], ((r32)oz - fx[2]) * dxr[2]};
            int64_t node = efo_idx(base[0] + ox, base[1] + oy, base[2] + oz, S.ny, S.nz);
            const r32* gv = S.grid_vel + 3 * node;
            r32 q[3] = {(r32)4.0 * dpos[0] / (dxr[0] * dxr[0]), (r32)4.0 * dpos[1] / (dxr[1] * dxr[1]),
                        (r32)4.0 * dpos[2] / (dxr[2] * dxr[2])};
            for (int a = 0; a < 3; ++a) {
              nv[a] += wt * gv[a];
              for (int b = 0; b < 3; ++b) nC[3 * a + b] += wt * (gv[a] * q[b]);
            }
          }
      if (S.fixed[p] == 0) {
        for (int a = 0; a < 3; ++a) {
          S.v[3 * p + a] = nv[a];
          S.x[3 * p + a] += dt * nv[a];
        }
        for (int a = 0; a < 9; ++a) S.C[9 * p + a] = nC[a];
        r32 Fo[9];
        for (int a = 0; a < 9; ++a) Fo[a] = S.F[9 * p + a];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            r32 acc = 0;
            for (int k = 0; k < 3; ++k) acc += (((i == k) ? (r32)1 : (r32)0) + dt * nC[3 * i + k]) * Fo[3 * k + j];
            S.F[9 * p + 3 * i + j] = acc;
          }
      }
    }
    if (S.fixed[p] != 0) {
      for (int a = 0; a < 3; ++a) S.v[3 * p + a] = 0;
      for (int a = 0; a < 9; ++a) {
        S.C[9 * p + a] = 0;
        S.F[9 * p + a] = (a % 4 == 0) ? (r32)1 : (r32)0;
      }
    }
    surface_geometry(S, p);
    r32 Xr[3];
    grid_coord(S, S.x + 3 * p, Xr);
    if (!stencil_oob(S, Xr)) {
      if (S.region[p] == primary_id) {
        for (int a = 0; a < 3; ++a) {
          psum_d[a] += S.x[3 * p + a] - S.rest_x[3 * p + a];
          psum_v[a] += S.v[3 * p + a];
        }
        pc += 1;
      } else if (S.region[p] == secondary_id) {
        for (int a = 0; a < 3; ++a) {
          ssum_d[a] += S.x[3 * p + a] - S.rest_x[3 * p + a];
          ssum_v[a] += S.v[3 * p + a];
        }
        sc += 1;
      }
    }
  }
  if (rep == nullptr) return;
  // Radial diagnostics (neo_hookean_mpm.py:876-898).
  double csum[3] = {0, 0, 0}, rsum[3] = {0, 0, 0};
  int64_t ccount = 0;
  for (int p = 0; p < P; ++p) {
    r32 X[3];
    grid_coord(S, S.x + 3 * p, X);
    if (!stencil_oob(S, X)) {
      for (int a = 0; a < 3; ++a) {
        csum[a] += S.x[3 * p + a];
        rsum[a] += S.rest_x[3 * p + a];
      }
      ccount += 1;
    }
  }
  double cnt = (double)std::max<int64_t>(ccount, 1);
  double cc[3], rc[3];
  for (int a = 0; a < 3; ++a) {
    cc[a] = csum[a] / cnt;
    rc[a] = rsum[a] / cnt;
  }
  double stretch_sum = 0, stretch_err = 0;
  int64_t stretch_count = 0;
  for (int p = 0; p < P; ++p) {
    r32 X[3];
    grid_coord(S, S.x + 3 * p, X);
    if (stencil_oob(S, X)) continue;
    double rr = 0, cr = 0;
    for (int a = 0; a < 3; ++a) {
      double d1 = S.rest_x[3 * p + a] - rc[a], d2 = S.x[3 * p + a] - cc[a];
      rr += d1 * d1;
      cr += d2 * d2;
    }
    rr = std::sqrt(rr);
    if (rr > 1.0e-12) {
      double st = std::sqrt(cr) / rr;
      stretch_sum += st;
      stretch_count += 1;
      stretch_err = std::max(stretch_err, std::fabs(st - 1.0));
    }
  }
  double expected[3], en = 0, tr = 0;
  for (int a = 0; a < 3; ++a) {
    expected[a] = pmom[a] + (double)dt * fsum[a];
    en += expected[a] * expected[a];
    tr += (tmom[a] - expected[a]) * (tmom[a] - expected[a]);
  }
  double denom = std::max(std::max(std::sqrt(en), std::sqrt(mom2)), 1.0e-20);
  double* v = rep->values;
  v[0] = msum;
  v[1] = vsum;
  for (int a = 0; a < 3; ++a) {
    v[2 + a] = pmom[a];
    v[5 + a] = gmom[a];
    v[8 + a] = fsum[a];
    v[16 + a] = psum_d[a];
    v[19 + a] = psum_v[a];
    v[22 + a] = ssum_d[a];
    v[25 + a] = ssum_v[a];
  }
  v[11] = std::sqrt(tr) / denom;
  v[12] = maxspeed;
  v[13] = maxJ;
  v[14] = stretch_sum;
  v[15] = stretch_err;
  rep->counts[0] = active;
  rep->counts[1] = oob;
  rep->counts[2] = clamps;
  rep->counts[3] = stretch_count;
  rep->counts[4] = pc;
  rep->counts[5] = sc;
}

EFO_API int efo_clamp_deformation(const r32* F, r32* Fp) { return clamp_deformation(F, Fp); }

// --------------------------------------------------------------------------
// HIBM markers (hibm_mpm.py).
// --------------------------------------------------------------------------

namespace {

inline r32 axis_coord_m(r32 v, const r32* faces, const r32* centers, int count) {
  // hibm_mpm.py:911-939 (same law as fluid.py:2407-2433).
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

// hibm_mpm.py:981-1009 _sample_pressure_trilinear (obstacle-masked).
inline double sample_p(const efo_grid* G, const int32_t* obs, const double* p, r32 gx, r32 gy, r32 gz, double& fw) {
  const efo_level& L = G->l0;
  int i0 = std::min(std::max((int)std::floor(gx), 0), L.nx - 2);
  int j0 = std::min(std::max((int)std::floor(gy), 0), L.ny - 2);
  int k0 = std::min(std::max((int)std::floor(gz), 0), L.nz - 2);
  r32 tx = std::min(std::max(gx - (r32)i0, (r32)0), (r32)1);
  r32 ty = std::min(std::max(gy - (r32)j0, (r32)0), (r32)1);
  r32 tz = std::min(std::max(gz - (r32)k0, (r32)0), (r32)1);
  double val = 0.0;
  fw = 0.0;
  for (int oi = 0; oi < 2; ++oi)
    for (int oj = 0; oj < 2; ++oj)
      for (int ok = 0; ok < 2; ++ok) {
        r32 w = (oi == 0 ? (r32)1 - tx : tx) * (oj == 0 ? (r32)1 - ty : ty) * (ok == 0 ? (r32)1 - tz : tz);
        int64_t c = efo_idx(i0 + oi, j0 + oj, k0 + ok, L.ny, L.nz);
        if (obs[c] == 0) {
          val += (double)w * p[c];
          fw += (double)w;
        }
      }
  if (fw > 1.0e-12) val /= fw;
  return val;
}

}  // namespace

typedef struct efo_traction_report {
  int64_t valid;
  int64_t invalid;
  int64_t two_sided;
  int64_t one_sided;
  double max_abs_traction;
} efo_traction_report;

// hibm_mpm.py:2253-2432 _sample_pressure_only_marker_tractions_kernel.
EFO_API void efo_sample_pressure_tractions(const efo_grid* G, const int32_t* obs, const double* p, int marker_count,
                                           const r32* xg, const r32* ng, const int32_t* region, int two_sided,
                                           int one_sided_region, float one_sided_ref, double* t, int32_t* valid,
                                           efo_traction_report* rep) {
  const efo_level& L = G->l0;
  std::memset(rep, 0, sizeof(*rep));
  for (int m = 0; m < marker_count; ++m) {
    const r32* x = xg + 3 * m;
    const r32* n = ng + 3 * m;
    r32 g[3] = {axis_coord_m(x[0], G->fx, G->cx, L.nx), axis_coord_m(x[1], G->fy, G->cy, L.ny),
                axis_coord_m(x[2], G->fz, G->cz, L.nz)};
    double pw;
    double pr = sample_p(G, obs, p, g[0], g[1], g[2], pw);
    double tr[3] = {-pr * (double)n[0], -pr * (double)n[1], -pr * (double)n[2]};
    bool ok = pw > 1.0e-12;
    if (two_sided) {
      int in = std::min(std::max((int)std::floor(g[0]), 0), L.nx - 1);
      int jn = std::min(std::max((int)std::floor(g[1]), 0), L.ny - 1);
      int kn = std::min(std::max((int)std::floor(g[2]), 0), L.nz - 1);
      r32 nsi = std::fabs(n[0]) / L.wx[in] + std::fabs(n[1]) / L.wy[jn] + std::fabs(n[2]) / L.wz[kn];
      r32 h = (r32)1.0 / std::max(nsi, (r32)1.0e-12);
      double outside = 0.0, inside = 0.0;
      int of = 0, inf = 0;
      for (int pi = 0; pi < 3; ++pi) {
        r32 mul = (r32)(pi + 1);
        r32 op[3], ip[3];
        for (int a = 0; a < 3; ++a) {
          op[a] = x[a] + mul * h * n[a];
          ip[a] = x[a] - mul * h * n[a];
        }
        double w;
        double so = sample_p(G, obs, p, axis_coord_m(op[0], G->fx, G->cx, L.nx),
                             axis_coord_m(op[1], G->fy, G->cy, L.ny), axis_coord_m(op[2], G->fz, G->cz, L.nz), w);
        if (of == 0 && w > 1.0e-12) {
          outside = so;
          of = 1;
        }
        double si = sample_p(G, obs, p, axis_coord_m(ip[0], G->fx, G->cx, L.nx),
                             axis_coord_m(ip[1], G->fy, G->cy, L.ny), axis_coord_m(ip[2], G->fz, G->cz, L.nz), w);
        if (inf == 0 && w > 1.0e-12) {
          inside = si;
          inf = 1;
        }
      }
      const double ref = (double)(r32)one_sided_ref;
      if (one_sided_region != -1 && region[m] == one_sided_region && inf) {
        for (int a = 0; a < 3; ++a) tr[a] = (inside - ref) * (double)n[a];
        ok = true;
        rep->one_sided += 1;
      } else if (one_sided_region != -1 && region[m] == one_sided_region && of) {
        for (int a = 0; a < 3; ++a) tr[a] = (ref - outside) * (double)n[a];
        ok = true;
        rep->one_sided += 1;
      } else if (of && inf) {
        for (int a = 0; a < 3; ++a) tr[a] = (inside - outside) * (double)n[a];
        ok = true;
        rep->two_sided += 1;
      } else {
        ok = false;
      }
    }
    if (ok) {
      for (int a = 0; a < 3; ++a) t[3 * m + a] = tr[a];
      valid[m] = 1;
      rep->valid += 1;
      rep->max_abs_traction =
          std::max(rep->max_abs_traction, std::sqrt(tr[0] * tr[0] + tr[1] * tr[1] + tr[2] * tr[2]));
    } else {
      t[3 * m] = t[3 * m + 1] = t[3 * m + 2] = 0.0;
      valid[m] = 0;
      rep->invalid += 1;
    }
  }
}

// hibm_mpm.py:903-909 _compute_marker_forces_kernel.
EFO_API void efo_compute_marker_forces(int marker_count, const double* t, const r32* A, double* F) {
  for (int m = 0; m < marker_count; ++m)
    for (int a = 0; a < 3; ++a) F[3 * m + a] = t[3 * m + a] * (double)A[m];
}

namespace {
inline bool finite3(const r32* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }
inline bool finite3d(const double* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }
// hibm_mpm.py:4838-4848 _marker_particle_shape_weight.
inline r32 tent(const r32* xm, const r32* xp, r32 R) {
  r32 w = 1;
  for (int a = 0; a < 3; ++a) w *= std::max((r32)1.0 - std::fabs(xm[a] - xp[a]) / R, (r32)0.0);
  return w;
}
}  // namespace

typedef struct efo_scatter_report {
  int64_t active_markers;
  int64_t invalid_markers;
  int64_t active_particle_contributions;
  double marker_force[3];
  double external_force[3];
} efo_scatter_report;

// hibm_mpm.py:4861-4878 _clear_mpm_external_forces_kernel.
EFO_API void efo_clear_external_forces(int particle_count, r32* fext, int64_t* cleared, double* max_abs) {
  *cleared = 0;
  *max_abs = 0.0;
  for (int p = 0; p < particle_count; ++p) {
    r32* f = fext + 3 * p;
    r32 nn = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    if (nn > (r32)0) {
      *cleared += 1;
      *max_abs = std::max(*max_abs, (double)nn);
    }
    f[0] = f[1] = f[2] = 0;
  }
}

// hibm_mpm.py:4899-4959 _scatter_marker_forces_to_mpm_particles_kernel
// (brute force over all particles, as in the reference).
EFO_API void efo_scatter_marker_forces(int marker_count, const r32* xg, const double* Fg, int particle_count,
                                       const r32* xp, float R_in, r32* fext, efo_scatter_report* rep) {
  std::memset(rep, 0, sizeof(*rep));
  const r32 R = (r32)R_in;
  int64_t active = 0, invalid = 0, contrib = 0;
  double mf0 = 0, mf1 = 0, mf2 = 0, ef0 = 0, ef1 = 0, ef2 = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : active, invalid, contrib, mf0, mf1, mf2, ef0, ef1, ef2)
  for (int m = 0; m < marker_count; ++m) {
    const r32* xm = xg + 3 * m;
    const double* Fm = Fg + 3 * m;
    r32 wsum = 0;
    bool valid = finite3(xm) && finite3d(Fm);
    if (valid)
      for (int p = 0; p < particle_count; ++p)
        if (finite3(xp + 3 * p)) wsum += tent(xm, xp + 3 * p, R);
    if (valid && wsum > (r32)1.0e-12) {
      active += 1;
      mf0 += Fm[0];
      mf1 += Fm[1];
      mf2 += Fm[2];
      for (int p = 0; p < particle_count; ++p) {
        r32 w = finite3(xp + 3 * p) ? tent(xm, xp + 3 * p, R) : (r32)0;
        if (w > (r32)0) {
          r32 ratio = w / wsum;
          r32 fc[3];
          for (int a = 0; a < 3; ++a) {
            fc[a] = (r32)(Fm[a] * (double)ratio);
#pragma omp atomic
            fext[3 * p + a] += fc[a];
          }
          ef0 += (double)fc[0];
          ef1 += (double)fc[1];
          ef2 += (double)fc[2];
          contrib += 1;
        }
      }
    } else {
      invalid += 1;
    }
  }
  rep->active_markers = active;
  rep->invalid_markers = invalid;
  rep->active_particle_contributions = contrib;
  rep->marker_force[0] = mf0;
  rep->marker_force[1] = mf1;
  rep->marker_force[2] = mf2;
  rep->external_force[0] = ef0;
  rep->external_force[1] = ef1;
  rep->external_force[2] = ef2;
}

typedef struct efo_feedback_report {
  int64_t updated;
  int64_t invalid;
  int64_t geometry_updated;
  int64_t geometry_invalid;
  double max_displacement;
  double max_speed;
  double max_normal_change;
  double max_area_change;
} efo_feedback_report;

// hibm_mpm.py:5097-5180 _update_surface_feedback_from_mpm_surface_particles_kernel
// (normal/area may be null for the velocity-only variant hibm_mpm.py:5012-5053).
EFO_API void efo_surface_feedback(int marker_count, r32* xg, r32* vg, r32* ng, r32* Ag, int particle_count,
                                  const r32* xp, const r32* vp, const r32* np_, const r32* ap, float R_in,
                                  float dt_in, efo_feedback_report* rep) {
  std::memset(rep, 0, sizeof(*rep));
  const r32 R = (r32)R_in, dt = (r32)dt_in;
  const bool geometry = np_ != nullptr && ap != nullptr;
  int64_t updated = 0, invalid = 0, gupd = 0, ginv = 0;
  double mdisp = 0, mspeed = 0, mnorm = 0, marea = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : updated, invalid, gupd, ginv) \
    reduction(max : mdisp, mspeed, mnorm, marea)
  for (int m = 0; m < marker_count; ++m) {
    r32 xo[3] = {xg[3 * m], xg[3 * m + 1], xg[3 * m + 2]};
    r32 no[3] = {ng[3 * m], ng[3 * m + 1], ng[3 * m + 2]};
    r32 ao = Ag[m];
    r32 vs[3] = {0, 0, 0}, nsum[3] = {0, 0, 0}, asum = 0, wsum = 0, gsum = 0;
    for (int p = 0; p < particle_count; ++p) {
      r32 w = tent(xo, xp + 3 * p, R);
      if (w > (r32)0) {
        for (int a = 0; a < 3; ++a) vs[a] += w * vp[3 * p + a];
        wsum += w;
        if (geometry) {
          const r32* pn = np_ + 3 * p;
          r32 pnn = std::sqrt(pn[0] * pn[0] + pn[1] * pn[1] + pn[2] * pn[2]);
          if (pnn > (r32)1.0e-12 && ap[p] > (r32)0) {
            for (int a = 0; a < 3; ++a) nsum[a] += w * pn[a];
            asum += w * ap[p];
            gsum += w;
          }
        }
      }
    }
    if (wsum > (r32)1.0e-12) {
      r32 nv[3], nx[3];
      for (int a = 0; a < 3; ++a) {
        nv[a] = vs[a] / wsum;
        nx[a] = xo[a] + dt * nv[a];
        xg[3 * m + a] = nx[a];
        vg[3 * m + a] = nv[a];
      }
      updated += 1;
      double dd = 0, sp = 0;
      for (int a = 0; a < 3; ++a) {
        dd += (double)(nx[a] - xo[a]) * (nx[a] - xo[a]);
        sp += (double)nv[a] * nv[a];
      }
      mdisp = std::max(mdisp, std::sqrt(dd));
      mspeed = std::max(mspeed, std::sqrt(sp));
      if (geometry) {
        r32 nn = std::sqrt(nsum[0] * nsum[0] + nsum[1] * nsum[1] + nsum[2] * nsum[2]);
        if (gsum > (r32)1.0e-12 && nn > (r32)1.0e-12) {
          r32 nn3[3] = {nsum[0] / nn, nsum[1] / nn, nsum[2] / nn};
          r32 na = asum / gsum;
          double dn = 0;
          for (int a = 0; a < 3; ++a) {
            ng[3 * m + a] = nn3[a];
            dn += (double)(nn3[a] - no[a]) * (nn3[a] - no[a]);
          }
          Ag[m] = na;
          gupd += 1;
          mnorm = std::max(mnorm, std::sqrt(dn));
          marea = std::max(marea, (double)std::fabs(na - ao));
        } else {
          ginv += 1;
        }
      }
    } else {
      invalid += 1;
      if (geometry) ginv += 1;
    }
  }
  rep->updated = updated;
  rep->invalid = invalid;
  rep->geometry_updated = gupd;
  rep->geometry_invalid = ginv;
  rep->max_displacement = mdisp;
  rep->max_speed = mspeed;
  rep->max_normal_change = mnorm;
  rep->max_area_change = marea;
}
