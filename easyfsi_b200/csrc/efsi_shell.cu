// Triangle Mooney-Rivlin membrane MPM step, B200 path (replaces the fused
// Taichi kernels of simulation_core/mooney_shell_mpm.py: _init_mass_kernel
// :480-540, _step_kernel :860-1003, _step_region_kernel :1005-1177,
// _add_region_area_load_kernel :710-728, _restore_state_kernel :1301-1309).
//
// One Taichi kernel becomes eight launches on one stream, each a flat pass
// over the faces, the particles or the node grid:
//   clear      grid arrays, per-particle forces, the step's accumulators
//   faces      Mooney face law (f64; the reference's is f32) + pressure or region
//              loads, scattered to the three vertices with f32 atomics; the
//              edge-strain maximum in the same launch
//   p2g        body force, out-of-bounds test, trilinear 8-node scatter
//   grid       momentum -> velocity, force, damping
//   g2p        PIC/FLIP blend, position and displacement update, centre sums
//   radial     radial stretch against the in-bounds centres; clears the
//              current-shape normals and area weights
//   normals    per-face area vectors onto the vertices
//   finish     normalises the normals; one thread packs the 37-value report
// The report's sums are reduced per block in f64 and added with one f64
// atomic per block and value (the reference adds every particle's value with
// its own atomic, mostly in f32).  The membrane is small (c4: 20k triangles,
// about 10k vertices, a 36^3 node grid by default), so every pass is a few
// microseconds and the step is launch-latency bound; the caller can capture
// the eight launches in a CUDA graph.  Every buffer comes from the caller;
// the accumulators live in a caller-provided scratch of
// EFSI_SHELL_SCRATCH_DOUBLES doubles.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "efsi_common.cuh"

namespace efsi {
namespace {

// f64 accumulators (slots of the caller's scratch)
enum {
  S_FSQ = 0,
  S_FSUM = 1,  // 3
  S_AREA = 4,
  S_STRETCH = 5,
  S_MASS = 6,
  S_PDISP = 7,    // 3
  S_PVEL = 10,    // 3
  S_SDISP = 13,   // 3
  S_SVEL = 16,    // 3
  S_PMOM = 19,    // 3
  S_GMOM = 22,    // 3
  S_FORCE = 25,   // 3
  S_TMOM = 28,    // 3
  S_MOM2 = 31,
  S_IMP2 = 32,
  S_CSUM = 33,    // 3
  S_RSUM = 36,    // 3
  S_ND = 40
};
// u32 slots after the doubles: counters, and maxima of non-negative floats as bits
enum { U_ACTIVE = 0, U_OOB, U_STRETCH_N, U_PCOUNT, U_SCOUNT, U_CCOUNT, U_MAX_STRETCH, U_MAX_EDGE, U_MAX_SPEED, U_N };
static_assert(S_ND + (U_N + 1) / 2 <= EFSI_SHELL_SCRATCH_DOUBLES, "shell scratch too small");

constexpr int kThreads = 256;
// Vertex and face passes launch 64-thread CTAs: a c4 membrane has about 10k
// vertices, which 256-thread CTAs put on 40 of the 148 SMs, each then bound
// by its own L1 atomic and load latency; 64-thread CTAs spread the same warps
// over every SM.
constexpr int kSmall = 64;

__device__ __forceinline__ unsigned* uslots(double* scratch) { return reinterpret_cast<unsigned*>(scratch + S_ND); }

__device__ __forceinline__ bool finite_small(float v) { return v == v && fabsf(v) < 1.0e30f; }
__device__ __forceinline__ bool safe3(float3 v) { return finite_small(v.x) && finite_small(v.y) && finite_small(v.z); }

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float norm3(float3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ float3 ld3(const float* p, int i) { return f3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
__device__ __forceinline__ void st3(float* p, int i, float3 v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}
__device__ __forceinline__ void atomic_add3(float* p, int i, float3 v) {
  atomicAdd(p + 3 * i, v.x);
  atomicAdd(p + 3 * i + 1, v.y);
  atomicAdd(p + 3 * i + 2, v.z);
}
// atomic max of a non-negative float held as its bit pattern
__device__ __forceinline__ void atomic_max_nonneg(unsigned* slot, float v) {
  if (v == v && v > 0.0f) atomicMax(slot, __float_as_uint(v));
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ unsigned warp_count(bool b) { return __popc(__ballot_sync(0xffffffffu, b)); }

// Adds the block's sums of NV doubles to slots[first + q] with one atomic each.
template <int NV>
__device__ __forceinline__ void block_add(double (&v)[NV], double* slots, const int (&where)[NV]) {
  block_sum<NV>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q)
      if (v[q] != 0.0) atomicAdd(slots + where[q], v[q]);
  }
}

// mooney_shell_mpm.py:744-765: particle node coordinate and its bounds test.
struct Coord {
  float c[3];
  bool oob;
};
__device__ __forceinline__ Coord grid_coord(const efsi_shell_state& s, float3 x) {
  Coord r;
  r.c[0] = (x.x - s.bmin[0]) / s.dx[0];
  r.c[1] = (x.y - s.bmin[1]) / s.dx[1];
  r.c[2] = (x.z - s.bmin[2]) / s.dx[2];
  const int n[3] = {s.nx, s.ny, s.nz};
  r.oob = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (!finite_small(r.c[a])) r.oob = true;
    if (r.c[a] < 0.0f || r.c[a] > (float)(n[a] - 1)) r.oob = true;
  }
  return r;
}

// Base node and fractions of the 2x2x2 trilinear stencil (:767-800).
struct Stencil {
  int base[3];
  float f[3];
};
__device__ __forceinline__ Stencil stencil_of(const efsi_shell_state& s, const Coord& c) {
  Stencil st;
  const int n[3] = {s.nx, s.ny, s.nz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int b = (int)floorf(c.c[a]);
    b = min(max(b, 0), n[a] - 2);
    st.base[a] = b;
    st.f[a] = fminf(fmaxf(c.c[a] - (float)b, 0.0f), 1.0f);
  }
  return st;
}
__device__ __forceinline__ float stencil_weight(const Stencil& st, int ox, int oy, int oz) {
  return (ox ? st.f[0] : 1.0f - st.f[0]) * (oy ? st.f[1] : 1.0f - st.f[1]) * (oz ? st.f[2] : 1.0f - st.f[2]);
}
__device__ __forceinline__ int64_t node_index(const efsi_shell_state& s, const Stencil& st, int ox, int oy, int oz) {
  return ((int64_t)(st.base[0] + ox) * s.ny + (st.base[1] + oy)) * s.nz + (st.base[2] + oz);
}

__device__ __forceinline__ float face_thickness(const efsi_shell_params& p, int region) {
  if (!p.region_loads) return p.thickness;
  if (region == p.primary_region) return p.primary_thickness;
  if (region == p.secondary_region) return p.secondary_thickness;
  return p.thickness;
}

__device__ __forceinline__ double3 d3(double x, double y, double z) { return make_double3(x, y, z); }
__device__ __forceinline__ double3 operator+(double3 a, double3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ double3 operator-(double3 a, double3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double3 operator-(double3 a) { return d3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ double3 operator*(double3 a, double s) { return d3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ double dot3(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double3 cross3(double3 a, double3 b) {
  return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double norm3(double3 a) { return sqrt(dot3(a, a)); }
__device__ __forceinline__ double3 ld3d(const float* p, int i) { return d3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }

// :552-560 _limit_vector_norm, in f64, rounded to f32 for the atomics
__device__ __forceinline__ float3 limit_norm(double3 v, double cap) {
  const double n = norm3(v);
  if (n != n || n > 1.0e30) return make_float3(0.f, 0.f, 0.f);
  const double k = (cap > 0.0 && n > cap) ? cap / n : 1.0;
  return make_float3((float)(v.x * k), (float)(v.y * k), (float)(v.z * k));
}


// ---------------------------------------------------------------------------
// clear: grid (4 arrays, 10 floats per node), per-particle forces, scratch
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_shell_clear(efsi_shell_state s, int preserve_external, double* scratch) {
  const int64_t nn = (int64_t)s.nx * s.ny * s.nz;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t0 < EFSI_SHELL_SCRATCH_DOUBLES) scratch[t0] = 0.0;
  for (int64_t i = t0; i < nn; i += stride) s.grid_mass[i] = 0.0f;
  for (int64_t i = t0; i < 3 * nn; i += stride) {
    s.grid_velocity[i] = 0.0f;
    s.grid_velocity_before[i] = 0.0f;
    s.grid_force[i] = 0.0f;
  }
  const int64_t np3 = 3 * (int64_t)s.particle_count;
  for (int64_t i = t0; i < np3; i += stride) {
    s.internal_force[i] = 0.0f;
    if (!preserve_external) s.external_force[i] = 0.0f;
  }
}

// ---------------------------------------------------------------------------
// faces: Mooney membrane law (:562-646) and external surface loads
// (:648-658 uniform pressure, :667-708 region loads); edges (:542-550)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_shell_faces(efsi_shell_state s, efsi_shell_params p, double* scratch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float edge_strain = 0.0f;
  if (i < s.edge_count) {
    const int ea = s.edges[2 * i], eb = s.edges[2 * i + 1];
    const float rl = norm3(ld3(s.rest_x, eb) - ld3(s.rest_x, ea));
    const float cl = norm3(ld3(s.x, eb) - ld3(s.x, ea));
    if (rl > 1.0e-12f && cl > 1.0e-12f) edge_strain = fabsf(fmaxf(cl / rl, 1.0e-6f) - 1.0f);
  }
  edge_strain = warp_max(edge_strain);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(uslots(scratch) + U_MAX_EDGE, edge_strain);
  if (i >= s.face_count) return;

  const int ia = s.faces[3 * i], ib = s.faces[3 * i + 1], ic = s.faces[3 * i + 2];
  const int region = s.face_region[i];
  const float thickness = face_thickness(p, region);
  // The face law runs in f64: near rest its stress terms are differences of
  // O(1) values (1 - i00 idet) for strains of 1e-6 and below, which f32 (the
  // reference's precision) resolves to about two digits.  Storage and the
  // vertex atomics stay f32.
  const double3 ra = ld3d(s.rest_x, ia), rb = ld3d(s.rest_x, ib), rc = ld3d(s.rest_x, ic);
  const double3 a = ld3d(s.x, ia), b = ld3d(s.x, ib), c = ld3d(s.x, ic);
  const double3 rav = cross3(rb - ra, rc - ra);
  const double3 av = cross3(b - a, c - a);
  const double ravn = norm3(rav);
  const double rarea = 0.5 * ravn;
  const double avn = norm3(av);
  const double area = 0.5 * avn;
  if (rarea > 1.0e-12 && ravn > 1.0e-12) {
    const double3 rn = rav * (1.0 / ravn);
    const double3 e0 = rb - ra;
    const double e0l = norm3(e0);
    if (e0l > 1.0e-12) {
      const double3 t0 = e0 * (1.0 / e0l);
      const double3 t1 = cross3(rn, t0);
      const double3 rac = rc - ra;
      const double xc = dot3(rac, t0), yc = dot3(rac, t1);
      if (fabs(yc) > 1.0e-12) {
        // inverse of the rest edge matrix in the triangle's own frame
        const double inv00 = 1.0 / e0l;
        const double inv01 = -xc / (e0l * yc);
        const double inv11 = 1.0 / yc;
        const double3 g0 = b - a, g1 = c - a;
        const double3 F0 = g0 * inv00;
        const double3 F1 = g0 * inv01 + g1 * inv11;
        const double cap_c = 1.0e6;
        const double c00 = fmin(dot3(F0, F0), cap_c);
        const double c01 = fmin(fmax(dot3(F0, F1), -cap_c), cap_c);
        const double c11 = fmin(dot3(F1, F1), cap_c);
        const double det = fmax(c00 * c11 - c01 * c01, 1.0e-6);
        const double idet = 1.0 / det;
        const double i00 = c11 * idet, i01 = -c01 * idet, i11 = c00 * idet;
        const double tr = c00 + c11;
        const double c1 = p.c1, c2 = p.c2;
        // second Piola-Kirchhoff stress of the incompressible Mooney membrane
        const double s00 = c1 * (1.0 - i00 * idet) + c2 * (det * i00 + idet - tr * idet * i00);
        const double s01 = c1 * (-i01 * idet) + c2 * (det * i01 - tr * idet * i01);
        const double s11 = c1 * (1.0 - i11 * idet) + c2 * (det * i11 + idet - tr * idet * i11);
        const double k2 = (double)p.membrane_force_scale * 2.0;
        const double3 P0 = (F0 * s00 + F1 * s01) * k2;
        const double3 P1 = (F0 * s01 + F1 * s11) * k2;
        const double vol = (double)thickness * rarea;
        const double3 ge0 = (P0 * inv00 + P1 * inv01) * vol;
        const double3 ge1 = (P1 * inv11) * vol;
        const double cap = (double)p.membrane_force_scale * (c1 + c2) * thickness * sqrt(rarea) * 100.0;
        const float3 fa = limit_norm(ge0 + ge1, cap), fb = limit_norm(-ge0, cap), fc = limit_norm(-ge1, cap);
        if (safe3(fa)) atomic_add3(s.internal_force, ia, fa);
        if (safe3(fb)) atomic_add3(s.internal_force, ib, fb);
        if (safe3(fc)) atomic_add3(s.internal_force, ic, fc);
      }
    }
    if (!p.region_loads && p.pressure != 0.0f) {
      const double3 normal = avn > 1.0e-12 ? av * (1.0 / avn) : rn;
      const double3 pfd = normal * ((double)p.pressure * area / 3.0);
      const float3 pf = f3((float)pfd.x, (float)pfd.y, (float)pfd.z);
      if (safe3(pf)) {
        atomic_add3(s.external_force, ia, pf);
        atomic_add3(s.external_force, ib, pf);
        atomic_add3(s.external_force, ic, pf);
      }
    }
  }
  if (p.region_loads) {
    float3 load = f3(0.f, 0.f, 0.f);
    if (region == p.area_load_region)
      load = load + f3(p.primary_area_load[0], p.primary_area_load[1], p.primary_area_load[2]) * (float)rarea;
    if (region == p.primary_region) {
      load = load + f3(p.primary_reaction[0], p.primary_reaction[1], p.primary_reaction[2]) *
                        ((float)rarea / fmaxf(p.primary_area, 1.0e-12f));
    } else if (region == p.secondary_region) {
      load = load + f3(p.secondary_reaction[0], p.secondary_reaction[1], p.secondary_reaction[2]) *
                        ((float)rarea / fmaxf(p.secondary_area, 1.0e-12f));
    }
    if (norm3(load) > 0.0f) {
      const float3 share = load * (1.0f / 3.0f);
      if (safe3(share)) {
        atomic_add3(s.external_force, ia, share);
        atomic_add3(s.external_force, ib, share);
        atomic_add3(s.external_force, ic, share);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// p2g: body force, bounds test, trilinear scatter and the particle sums (:930-959)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_shell_p2g(efsi_shell_state s, efsi_shell_params p, double* scratch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[14] = {0};
  bool oob = false;
  if (i < s.particle_count) {
    const float m = s.mass[i];
    float3 fext = ld3(s.external_force, i) + f3(p.body_acceleration[0], p.body_acceleration[1], p.body_acceleration[2]) * m;
    st3(s.external_force, i, fext);
    const float3 fint = ld3(s.internal_force, i);
    const float3 v = ld3(s.v, i);
    const float3 total = fint + fext;
    const bool fixed = s.fixed[i] != 0;
    const Coord c = grid_coord(s, ld3(s.x, i));
    oob = c.oob;
    if (!oob && !fixed) {
      const Stencil st = stencil_of(s, c);
      const float3 mom = v * m;
#pragma unroll
      for (int o = 0; o < 8; ++o) {
        const int ox = o >> 2, oy = (o >> 1) & 1, oz = o & 1;
        const float w = stencil_weight(st, ox, oy, oz);
        const int64_t n = node_index(s, st, ox, oy, oz);
        atomicAdd(s.grid_mass + n, w * m);
        atomicAdd(s.grid_velocity + 3 * n, w * mom.x);
        atomicAdd(s.grid_velocity + 3 * n + 1, w * mom.y);
        atomicAdd(s.grid_velocity + 3 * n + 2, w * mom.z);
        atomicAdd(s.grid_force + 3 * n, w * total.x);
        atomicAdd(s.grid_force + 3 * n + 1, w * total.y);
        atomicAdd(s.grid_force + 3 * n + 2, w * total.z);
      }
    }
    if (safe3(fint)) {
      acc[0] = fint.x;
      acc[1] = fint.y;
      acc[2] = fint.z;
    }
    acc[3] = (double)fint.x * fint.x + (double)fint.y * fint.y + (double)fint.z * fint.z;
    double pm[3] = {0, 0, 0}, tf[3] = {0, 0, 0};
    if (!fixed) {
      pm[0] = (double)m * v.x;
      pm[1] = (double)m * v.y;
      pm[2] = (double)m * v.z;
      tf[0] = total.x;
      tf[1] = total.y;
      tf[2] = total.z;
    }
    for (int a = 0; a < 3; ++a) {
      acc[4 + a] = pm[a];
      acc[7 + a] = tf[a];
    }
    acc[10] = m;
    acc[11] = s.area[i];
    acc[12] = pm[0] * pm[0] + pm[1] * pm[1] + pm[2] * pm[2];
    const double dt = p.dt;
    acc[13] = dt * dt * (tf[0] * tf[0] + tf[1] * tf[1] + tf[2] * tf[2]);
  }
  const unsigned n_oob = warp_count(i < s.particle_count && oob);
  if ((threadIdx.x & 31) == 0 && n_oob) atomicAdd(uslots(scratch) + U_OOB, n_oob);
  const int where[14] = {S_FSUM,     S_FSUM + 1, S_FSUM + 2,  S_FSQ,       S_PMOM, S_PMOM + 1, S_PMOM + 2,
                         S_FORCE,    S_FORCE + 1, S_FORCE + 2, S_MASS,     S_AREA, S_MOM2,     S_IMP2};
  block_add<14>(acc, scratch, where);
}

// ---------------------------------------------------------------------------
// grid update (:961-976)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_shell_grid(efsi_shell_state s, efsi_shell_params p, double* scratch) {
  const int64_t nn = (int64_t)s.nx * s.ny * s.nz;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double acc[6] = {0};
  bool active = false;
  float speed = 0.0f;
  if (i < nn) {
    const float m = s.grid_mass[i];
    if (m > 1.0e-20f) {
      active = true;
      // velocity = momentum / m, then v += (dt f) / m, divided as the reference does
      const float3 mom = ld3(s.grid_velocity, i);
      const float3 vbd = f3(mom.x / m, mom.y / m, mom.z / m);
      st3(s.grid_velocity_before, i, vbd);
      const float3 fr = ld3(s.grid_force, i);
      const float3 tv = vbd + f3(p.dt * fr.x / m, p.dt * fr.y / m, p.dt * fr.z / m);
      const float3 v = tv * p.velocity_damping;
      st3(s.grid_velocity, i, v);
      acc[0] = (double)m * tv.x;
      acc[1] = (double)m * tv.y;
      acc[2] = (double)m * tv.z;
      acc[3] = (double)m * v.x;
      acc[4] = (double)m * v.y;
      acc[5] = (double)m * v.z;
      speed = norm3(v);
    }
  }
  const unsigned n_act = warp_count(active);
  speed = warp_max(speed);
  if ((threadIdx.x & 31) == 0) {
    if (n_act) atomicAdd(uslots(scratch) + U_ACTIVE, n_act);
    atomic_max_nonneg(uslots(scratch) + U_MAX_SPEED, speed);
  }
  const int where[6] = {S_TMOM, S_TMOM + 1, S_TMOM + 2, S_GMOM, S_GMOM + 1, S_GMOM + 2};
  block_add<6>(acc, scratch, where);
}

// ---------------------------------------------------------------------------
// g2p (:978-1003)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_shell_g2p(efsi_shell_state s, efsi_shell_params p, double* scratch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[18] = {0};
  bool counted = false, prim = false, sec = false;
  float speed = 0.0f;
  if (i < s.particle_count) {
    float3 x = ld3(s.x, i), u = ld3(s.u, i), v = ld3(s.v, i);
    const bool fixed = s.fixed[i] != 0;
    const Coord c = grid_coord(s, x);
    if (!c.oob) {
      const Stencil st = stencil_of(s, c);
      float3 pic = f3(0.f, 0.f, 0.f), dlt = f3(0.f, 0.f, 0.f);
#pragma unroll
      for (int o = 0; o < 8; ++o) {
        const int ox = o >> 2, oy = (o >> 1) & 1, oz = o & 1;
        const float w = stencil_weight(st, ox, oy, oz);
        const int64_t n = node_index(s, st, ox, oy, oz);
        const float3 gv = ld3(s.grid_velocity, n);
        pic = pic + gv * w;
        dlt = dlt + (gv - ld3(s.grid_velocity_before, n)) * w;
      }
      const float3 flip = v + dlt;
      v = pic * (1.0f - p.flip_blend) + flip * p.flip_blend;
      if (!fixed) {
        const float3 dx = v * p.dt;
        x = x + dx;
        u = u + dx;
      } else {
        x = ld3(s.rest_x, i);
        u = f3(0.f, 0.f, 0.f);
        v = f3(0.f, 0.f, 0.f);
      }
    } else if (fixed) {
      x = ld3(s.rest_x, i);
      u = f3(0.f, 0.f, 0.f);
      v = f3(0.f, 0.f, 0.f);
    } else {
      const float3 dx = v * p.dt;
      x = x + dx;
      u = u + dx;
      speed = norm3(v);
    }
    st3(s.x, i, x);
    st3(s.u, i, u);
    st3(s.v, i, v);
    if (!grid_coord(s, x).oob) {
      counted = true;
      const float3 r = ld3(s.rest_x, i);
      acc[0] = x.x;
      acc[1] = x.y;
      acc[2] = x.z;
      acc[3] = r.x;
      acc[4] = r.y;
      acc[5] = r.z;
      const int region = s.vertex_region[i];
      const int slot = region == p.primary_region ? 6 : (region == p.secondary_region ? 12 : -1);
      prim = slot == 6;
      sec = slot == 12;
      if (slot >= 0) {
        acc[slot] = u.x;
        acc[slot + 1] = u.y;
        acc[slot + 2] = u.z;
        acc[slot + 3] = v.x;
        acc[slot + 4] = v.y;
        acc[slot + 5] = v.z;
      }
    }
  }
  const unsigned nc = warp_count(counted), npc = warp_count(prim), nsc = warp_count(sec);
  speed = warp_max(speed);
  if ((threadIdx.x & 31) == 0) {
    unsigned* u = uslots(scratch);
    if (nc) atomicAdd(u + U_CCOUNT, nc);
    if (npc) atomicAdd(u + U_PCOUNT, npc);
    if (nsc) atomicAdd(u + U_SCOUNT, nsc);
    atomic_max_nonneg(u + U_MAX_SPEED, speed);
  }
  const int where[18] = {S_CSUM,  S_CSUM + 1,  S_CSUM + 2,  S_RSUM,  S_RSUM + 1,  S_RSUM + 2,
                                    S_PDISP, S_PDISP + 1, S_PDISP + 2, S_PVEL,  S_PVEL + 1,  S_PVEL + 2,
                                    S_SDISP, S_SDISP + 1, S_SDISP + 2, S_SVEL,  S_SVEL + 1,  S_SVEL + 2};
  block_add<18>(acc, scratch, where);
}

// ---------------------------------------------------------------------------
// radial stretch (:995-1003 of the step); clears normals and area weights (:450-453)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_shell_radial(efsi_shell_state s, double* scratch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  bool counted = false;
  float err = 0.0f;
  if (i < s.particle_count) {
    const unsigned* u = uslots(scratch);
    const double cnt = fmax((double)u[U_CCOUNT], 1.0);
    const float3 x = ld3(s.x, i);
    if (!grid_coord(s, x).oob) {
      const float3 cc = f3((float)(scratch[S_CSUM] / cnt), (float)(scratch[S_CSUM + 1] / cnt), (float)(scratch[S_CSUM + 2] / cnt));
      const float3 rc = f3((float)(scratch[S_RSUM] / cnt), (float)(scratch[S_RSUM + 1] / cnt), (float)(scratch[S_RSUM + 2] / cnt));
      const float rr = norm3(ld3(s.rest_x, i) - rc);
      const float cr = norm3(x - cc);
      const float stretch = cr / fmaxf(rr, 1.0e-12f);
      acc[0] = stretch;
      counted = true;
      err = fabsf(stretch - 1.0f);
    }
    st3(s.normal, i, f3(0.f, 0.f, 0.f));
    s.area[i] = 0.0f;
  }
  const unsigned nc = warp_count(counted);
  err = warp_max(err);
  if ((threadIdx.x & 31) == 0) {
    if (nc) atomicAdd(uslots(scratch) + U_STRETCH_N, nc);
    atomic_max_nonneg(uslots(scratch) + U_MAX_STRETCH, err);
  }
  const int where[1] = {S_STRETCH};
  block_add<1>(acc, scratch, where);
}

__global__ void __launch_bounds__(kThreads) k_shell_clear_normals(efsi_shell_state s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.particle_count) return;
  st3(s.normal, i, f3(0.f, 0.f, 0.f));
  s.area[i] = 0.0f;
}

// :436-447 per-face area vector and a third of the face area onto each vertex
__global__ void __launch_bounds__(kThreads) k_shell_face_normals(efsi_shell_state s) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= s.face_count) return;
  const int ia = s.faces[3 * f], ib = s.faces[3 * f + 1], ic = s.faces[3 * f + 2];
  const float3 a = ld3(s.x, ia);
  const float3 av = cross3(ld3(s.x, ib) - a, ld3(s.x, ic) - a);
  const float n = norm3(av);
  if (n > 1.0e-12f) {
    atomic_add3(s.normal, ia, av);
    atomic_add3(s.normal, ib, av);
    atomic_add3(s.normal, ic, av);
    const float share = 0.5f * n / 3.0f;
    atomicAdd(s.area + ia, share);
    atomicAdd(s.area + ib, share);
    atomicAdd(s.area + ic, share);
  }
}

// :454-461 normalisation; with a scratch, thread 0 also packs the report
// (:337-391 layout, :985-1002 transfer error)
__global__ void __launch_bounds__(kThreads) k_shell_finish(efsi_shell_state s, efsi_shell_params p, const double* scratch,
                                                          double* report) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < s.particle_count) {
    const float3 n = ld3(s.normal, i);
    const float l = norm3(n);
    if (l > 1.0e-12f) st3(s.normal, i, n * (1.0f / l));
  }
  if (i != 0 || !scratch || !report) return;
  const unsigned* u = reinterpret_cast<const unsigned*>(scratch + S_ND);
  double r[37];
  r[0] = scratch[S_FSQ];
  for (int a = 0; a < 3; ++a) r[1 + a] = scratch[S_FSUM + a];
  r[4] = scratch[S_AREA];
  r[5] = scratch[S_STRETCH];
  r[6] = __uint_as_float(u[U_MAX_STRETCH]);
  r[7] = __uint_as_float(u[U_MAX_EDGE]);
  r[8] = __uint_as_float(u[U_MAX_SPEED]);
  r[9] = scratch[S_MASS];
  for (int a = 0; a < 3; ++a) {
    r[10 + a] = scratch[S_PDISP + a];
    r[13 + a] = scratch[S_PVEL + a];
    r[16 + a] = scratch[S_SDISP + a];
    r[19 + a] = scratch[S_SVEL + a];
    r[22 + a] = scratch[S_PMOM + a];
    r[25 + a] = scratch[S_GMOM + a];
    r[28 + a] = scratch[S_FORCE + a];
  }
  const double dt = p.dt;
  double e2 = 0.0, x2 = 0.0;
  for (int a = 0; a < 3; ++a) {
    const double expected = scratch[S_PMOM + a] + dt * scratch[S_FORCE + a];
    const double d = scratch[S_TMOM + a] - expected;
    e2 += d * d;
    x2 += expected * expected;
  }
  const double den = fmax(fmax(sqrt(x2), sqrt(scratch[S_MOM2])), fmax(sqrt(scratch[S_IMP2]), 1.0e-20));
  r[31] = sqrt(e2) / den;
  r[32] = u[U_ACTIVE];
  r[33] = u[U_OOB];
  r[34] = u[U_STRETCH_N];
  r[35] = u[U_PCOUNT];
  r[36] = u[U_SCOUNT];
  for (int k = 0; k < 37; ++k) report[k] = r[k];
}

// :480-540 _init_mass_kernel: per-particle reset
__global__ void __launch_bounds__(kThreads) k_shell_init_particles(efsi_shell_state s, float* mass, int32_t* vregion,
                                                                  int32_t* fixed, float* totals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 4 && totals) totals[i] = 0.0f;
  if (i >= s.particle_count) return;
  st3(s.v, i, f3(0.f, 0.f, 0.f));
  st3(s.u, i, f3(0.f, 0.f, 0.f));
  st3(s.internal_force, i, f3(0.f, 0.f, 0.f));
  st3(s.external_force, i, f3(0.f, 0.f, 0.f));
  st3(s.normal, i, f3(0.f, 0.f, 0.f));
  mass[i] = 0.0f;
  s.area[i] = 0.0f;
  vregion[i] = 2147483647;
  fixed[i] = 0;
}

// :463-478 and :509-539: rest area and mass shares, vertex regions, fixed
// vertices and the two regions' rest areas and masses
__global__ void __launch_bounds__(kThreads) k_shell_init_faces(efsi_shell_state s, float* mass, int32_t* vregion,
                                                              int32_t* fixed, float* totals, float density,
                                                              float thickness, float primary_thickness,
                                                              float secondary_thickness, int primary, int secondary,
                                                              int fixed_region) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= s.face_count) return;
  const int ia = s.faces[3 * f], ib = s.faces[3 * f + 1], ic = s.faces[3 * f + 2];
  const int region = s.face_region[f];
  float t = thickness;
  if (region == primary) t = primary_thickness;
  else if (region == secondary) t = secondary_thickness;
  else if (fixed_region >= 0 && region == fixed_region) t = primary_thickness;
  const float3 ra = ld3(s.rest_x, ia);
  const float area = 0.5f * norm3(cross3(ld3(s.rest_x, ib) - ra, ld3(s.rest_x, ic) - ra));
  const float share = area / 3.0f;
  const float mshare = density * t * share;
  const int v3[3] = {ia, ib, ic};
  for (int k = 0; k < 3; ++k) {
    atomicAdd(s.area + v3[k], share);
    atomicAdd(mass + v3[k], mshare);
    atomicMin(vregion + v3[k], region);
    if (fixed_region >= 0 && region == fixed_region) fixed[v3[k]] = 1;
  }
  if (totals) {
    const float m = density * t * area;
    if (region == primary) {
      atomicAdd(totals + 0, area);
      atomicAdd(totals + 1, m);
    } else if (region == secondary) {
      atomicAdd(totals + 2, area);
      atomicAdd(totals + 3, m);
    }
  }
}

// :710-728 rest-area load on one region's faces, a third per vertex
__global__ void __launch_bounds__(kThreads) k_shell_region_load(efsi_shell_state s, int region, float lx, float ly,
                                                               float lz) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= s.face_count || s.face_region[f] != region) return;
  const int ia = s.faces[3 * f], ib = s.faces[3 * f + 1], ic = s.faces[3 * f + 2];
  const float3 ra = ld3(s.rest_x, ia);
  const float area = 0.5f * norm3(cross3(ld3(s.rest_x, ib) - ra, ld3(s.rest_x, ic) - ra));
  const float3 share = f3(lx, ly, lz) * area * (1.0f / 3.0f);
  if (safe3(share)) {
    atomic_add3(s.external_force, ia, share);
    atomic_add3(s.external_force, ib, share);
    atomic_add3(s.external_force, ic, share);
  }
}

inline unsigned nblk(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + kThreads - 1) / kThreads); }
inline unsigned nblk_small(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + kSmall - 1) / kSmall); }

int check_state(const efsi_shell_state* s) {
  EFSI_ARG_CHECK(s != nullptr, "shell state is NULL");
  EFSI_ARG_CHECK(s->particle_count > 0 && s->face_count > 0 && s->edge_count >= 0, "shell counts must be positive");
  EFSI_ARG_CHECK(s->nx >= 4 && s->ny >= 4 && s->nz >= 4, "grid_nodes must be at least 4 in each direction");
  EFSI_ARG_CHECK((int64_t)s->nx * s->ny * s->nz < ((int64_t)1 << 31), "shell grid too large");
  for (int a = 0; a < 3; ++a) EFSI_ARG_CHECK(std::isfinite(s->dx[a]) && s->dx[a] > 0.0f, "grid spacing must be positive");
  EFSI_ARG_CHECK(s->x && s->u && s->v && s->rest_x && s->mass && s->area && s->normal && s->internal_force &&
                     s->external_force && s->vertex_region && s->fixed && s->faces && s->face_region &&
                     (s->edges || s->edge_count == 0),
                 "shell particle or face buffer is NULL");
  return EFSI_OK;
}

int launch_normals(const efsi_shell_state& s, cudaStream_t st) {
  EFSI_COUNTED k_shell_clear_normals<<<nblk_small(s.particle_count), kSmall, 0, st>>>(s);
  EFSI_COUNTED k_shell_face_normals<<<nblk_small(s.face_count), kSmall, 0, st>>>(s);
  EFSI_COUNTED k_shell_finish<<<nblk_small(s.particle_count), kSmall, 0, st>>>(s, efsi_shell_params{}, nullptr, nullptr);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

}  // namespace
}  // namespace efsi

using namespace efsi;

extern "C" int efsi_shell_init(const efsi_shell_state* state, float* mass, int32_t* vertex_region, int32_t* fixed,
                               float density, float thickness, float primary_thickness, float secondary_thickness,
                               int32_t primary_region, int32_t secondary_region, int32_t fixed_region,
                               float* region_totals, void* stream) {
  EFSI_TRY(check_state(state));
  EFSI_ARG_CHECK(mass && vertex_region && fixed, "shell init output is NULL");
  EFSI_ARG_CHECK(density > 0.0f && thickness > 0.0f, "density and thickness must be positive");
  const efsi_shell_state& s = *state;
  cudaStream_t st = as_stream(stream);
  EFSI_COUNTED k_shell_init_particles<<<nblk(s.particle_count), kThreads, 0, st>>>(s, mass, vertex_region, fixed,
                                                                                   region_totals);
  EFSI_COUNTED k_shell_init_faces<<<nblk(s.face_count), kThreads, 0, st>>>(
      s, mass, vertex_region, fixed, region_totals, density, thickness, primary_thickness, secondary_thickness,
      primary_region, secondary_region, fixed_region);
  EFSI_LAUNCH_CHECK();
  // init ends with the current-shape normals, which rebuild the area weights
  return launch_normals(s, st);
}

extern "C" int efsi_shell_update_normals(const efsi_shell_state* state, void* stream) {
  EFSI_TRY(check_state(state));
  return launch_normals(*state, as_stream(stream));
}

extern "C" int efsi_shell_add_region_area_load(const efsi_shell_state* state, int32_t region_id,
                                               const float* area_load_npm2, void* stream) {
  EFSI_TRY(check_state(state));
  EFSI_ARG_CHECK(area_load_npm2 != nullptr, "area load is NULL");
  const efsi_shell_state& s = *state;
  EFSI_COUNTED k_shell_region_load<<<nblk(s.face_count), kThreads, 0, as_stream(stream)>>>(
      s, region_id, area_load_npm2[0], area_load_npm2[1], area_load_npm2[2]);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

extern "C" int efsi_shell_step(const efsi_shell_state* state, const efsi_shell_params* params, double* scratch,
                               double* report_device, void* stream) {
  EFSI_TRY(check_state(state));
  EFSI_ARG_CHECK(params != nullptr && scratch != nullptr, "shell params or scratch is NULL");
  EFSI_ARG_CHECK(params->flip_blend >= 0.0f && params->flip_blend <= 1.0f, "flip_blend must be in [0, 1]");
  EFSI_ARG_CHECK(state->grid_mass && state->grid_velocity && state->grid_velocity_before && state->grid_force,
                 "shell grid arrays are NULL");
  const efsi_shell_state& s = *state;
  const efsi_shell_params& p = *params;
  cudaStream_t st = as_stream(stream);
  const int64_t nn = (int64_t)s.nx * s.ny * s.nz;
  const bool timed = timing_enabled(KF_SHELL_STEP);
  if (timed) timing_begin(KF_SHELL_STEP, st);
  const int64_t clear_work = std::max<int64_t>(3 * nn, 3 * (int64_t)s.particle_count);
  EFSI_COUNTED k_shell_clear<<<std::min<unsigned>(nblk(clear_work), 148u * 8u), kThreads, 0, st>>>(
      s, p.region_loads ? p.preserve_external_force : 0, scratch);
  EFSI_COUNTED k_shell_faces<<<nblk_small(std::max(s.face_count, s.edge_count)), kSmall, 0, st>>>(s, p, scratch);
  EFSI_COUNTED k_shell_p2g<<<nblk_small(s.particle_count), kSmall, 0, st>>>(s, p, scratch);
  EFSI_COUNTED k_shell_grid<<<nblk(nn), kThreads, 0, st>>>(s, p, scratch);
  EFSI_COUNTED k_shell_g2p<<<nblk_small(s.particle_count), kSmall, 0, st>>>(s, p, scratch);
  EFSI_COUNTED k_shell_radial<<<nblk_small(s.particle_count), kSmall, 0, st>>>(s, scratch);
  EFSI_COUNTED k_shell_face_normals<<<nblk_small(s.face_count), kSmall, 0, st>>>(s);
  EFSI_COUNTED k_shell_finish<<<nblk_small(s.particle_count), kSmall, 0, st>>>(s, p, scratch, report_device);
  EFSI_LAUNCH_CHECK();
  // algorithmic bytes: particles 120 B (x, u, v, rest_x, forces, normal read/written once, mass, area, flags),
  // faces 48 B (indices, region, three vertex reads), nodes 40 B cleared + 40 B touched by the update
  if (timed) timing_end(KF_SHELL_STEP, st, 120.0 * s.particle_count + 48.0 * s.face_count + 80.0 * nn);
  return EFSI_OK;
}
