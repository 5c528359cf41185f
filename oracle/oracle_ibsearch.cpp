// CPU oracle: immersed-boundary node search and in/out classification --
// TEST INFRASTRUCTURE ONLY (see oracle_common.h).
//
// Restates HibmMpmIbNodeSearch (simulation_core/hibm_mpm.py):
//   _closest_point_on_triangle        hibm_mpm.py:5494-5549
//   _oriented_triangle_normal         hibm_mpm.py:5551-5560
//   _barycentric_weights_on_triangle  hibm_mpm.py:5562-5583
//   _nearest_triangle_marker          hibm_mpm.py:5585-5600
//   _search_and_classify_kernel       hibm_mpm.py:5601-5835 (uniform cell centres)
//   _search_and_classify_grid_fields_kernel hibm_mpm.py:5837-6068 (centre arrays)
// as the reference writes it: every node visits every projection triangle
// (or, with none, every marker) in index order and keeps a candidate when its
// distance is strictly smaller than the best so far.  All geometry is in the
// reference's f32 (r32 = float in the mirror build), evaluated left to right
// exactly as the Python expressions read, without contraction.
#include "oracle_common.h"

namespace {

struct V3 {
  r32 x, y, z;
};

inline V3 v3(r32 x, r32 y, r32 z) { return V3{x, y, z}; }
inline V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 scale(V3 a, r32 s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 divide(V3 a, r32 s) { return v3(a.x / s, a.y / s, a.z / s); }
inline V3 neg(V3 a) { return v3(-a.x, -a.y, -a.z); }
inline r32 dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline r32 norm(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 load3(const r32* p, int i) { return v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
inline void store3(r32* p, int64_t i, V3 v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}

// hibm_mpm.py:5494-5549
inline int closest_point_on_triangle(V3 p, V3 a, V3 b, V3 c, V3& closest, V3& face_normal) {
  const V3 ab = sub(b, a), ac = sub(c, a);
  face_normal = cross(ab, ac);
  const r32 nn = norm(face_normal);
  closest = a;
  if (!(nn > (r32)1.0e-12)) return 0;
  face_normal = divide(face_normal, nn);
  const V3 ap = sub(p, a);
  const r32 d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0 && d2 <= 0) {
    closest = a;
    return 1;
  }
  const V3 bp = sub(p, b);
  const r32 d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0 && d4 <= d3) {
    closest = b;
    return 1;
  }
  const r32 vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    const r32 t = d1 / std::max(d1 - d3, (r32)1.0e-30);
    closest = add(a, scale(ab, t));
    return 1;
  }
  const V3 cp = sub(p, c);
  const r32 d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0 && d5 <= d6) {
    closest = c;
    return 1;
  }
  const r32 vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    const r32 t = d2 / std::max(d2 - d6, (r32)1.0e-30);
    closest = add(a, scale(ac, t));
    return 1;
  }
  const r32 va = d3 * d6 - d5 * d4;
  if (va <= 0 && d4 - d3 >= 0 && d5 - d6 >= 0) {
    const r32 t = (d4 - d3) / std::max(d4 - d3 + d5 - d6, (r32)1.0e-30);
    closest = add(b, scale(sub(c, b), t));
    return 1;
  }
  const r32 denom = std::max(va + vb + vc, (r32)1.0e-30);
  const r32 v = vb / denom, w = vc / denom;
  closest = add(add(a, scale(ab, v)), scale(ac, w));
  return 1;
}

// hibm_mpm.py:5551-5560
inline V3 oriented_normal(V3 face_normal, const r32* mn, int ia, int ib, int ic) {
  V3 normal = face_normal;
  V3 avg = add(add(load3(mn, ia), load3(mn, ib)), load3(mn, ic));
  const r32 an = norm(avg);
  if (an > (r32)1.0e-12) {
    avg = divide(avg, an);
    if (dot(normal, avg) < 0) normal = neg(normal);
  }
  return normal;
}

inline r32 clamp01(r32 v) { return std::min(std::max(v, (r32)0), (r32)1); }

// hibm_mpm.py:5562-5583
inline V3 barycentric(V3 p, V3 a, V3 b, V3 c) {
  const V3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
  const r32 d00 = dot(ab, ab), d01 = dot(ab, ac), d11 = dot(ac, ac), d20 = dot(ap, ab), d21 = dot(ap, ac);
  const r32 denom = d00 * d11 - d01 * d01;
  if (!(std::fabs(denom) > (r32)1.0e-30)) return v3(1, 0, 0);
  r32 v = (d11 * d20 - d01 * d21) / denom;
  r32 w = (d00 * d21 - d01 * d20) / denom;
  r32 u = (r32)1 - v - w;
  u = clamp01(u);
  v = clamp01(v);
  w = clamp01(w);
  const r32 total = std::max(u + v + w, (r32)1.0e-30);
  return v3(u / total, v / total, w / total);
}

// hibm_mpm.py:5585-5600
inline int nearest_triangle_marker(V3 p, const r32* mx, int ia, int ib, int ic) {
  int nearest = ia;
  const V3 oa = sub(p, load3(mx, ia));
  r32 best = dot(oa, oa);
  const V3 ob = sub(p, load3(mx, ib));
  const r32 db = dot(ob, ob);
  if (db < best) {
    best = db;
    nearest = ib;
  }
  const V3 oc = sub(p, load3(mx, ic));
  if (dot(oc, oc) < best) nearest = ic;
  return nearest;
}

struct Cand {
  int marker = -1;
  r32 distance = (r32)1.0e30;
  r32 signed_distance = 0;
  V3 boundary{0, 0, 0};
  V3 normal{0, 0, 1};
  int pidx[3] = {-1, -1, -1};
  r32 pw[3] = {0, 0, 0};
};

}  // namespace

// Node positions: centre arrays cx/cy/cz when given (grid-fields variant),
// else bmin + (i + 0.5) * spacing per axis in f32.  Outputs per node (C
// order over nx, ny, nz): kind (0 none, 1 external IB, 2 internal), nearest
// marker, signed distance, boundary point (3), interior fluid point (3),
// projection marker indices (3) and weights (3).  report[4] = near-boundary,
// external IB, internal, invalid-projection counts.
EFO_API void efo_ib_node_search(int nx, int ny, int nz, const r32* cx, const r32* cy, const r32* cz, const r32* bmin,
                                const r32* spacing, const r32* mx, const r32* mn, int marker_count, const int32_t* tri,
                                int tri_count, r32 radius, r32 probe, r32 tol, int classify_far, int32_t* kind,
                                int32_t* nearest_marker, r32* sd, r32* bp, r32* ip, int32_t* pidx, r32* pw,
                                int64_t* report) {
  const int64_t n = (int64_t)nx * ny * nz;
  int64_t near_count = 0, ext_count = 0, int_count = 0, invalid_count = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : near_count, ext_count, int_count, invalid_count)
  for (int64_t c = 0; c < n; ++c) {
    const int i = (int)(c / ((int64_t)ny * nz)), j = (int)((c / nz) % ny), k = (int)(c % nz);
    V3 p;
    if (cx != nullptr) {
      p = v3(cx[i], cy[j], cz[k]);
    } else {
      p = v3(bmin[0] + ((r32)i + (r32)0.5) * spacing[0], bmin[1] + ((r32)j + (r32)0.5) * spacing[1],
             bmin[2] + ((r32)k + (r32)0.5) * spacing[2]);
    }
    kind[c] = 0;
    nearest_marker[c] = -1;
    sd[c] = 0;
    store3(bp, c, v3(0, 0, 0));
    store3(ip, c, v3(0, 0, 0));
    for (int q = 0; q < 3; ++q) {
      pidx[3 * c + q] = -1;
      pw[3 * c + q] = 0;
    }
    Cand nearest, external, global;
    int external_seen = 0, global_external_seen = 0;
    auto consider = [&](int marker, r32 distance, r32 signed_distance, V3 boundary, V3 normal, const int* ix,
                        const r32* w) {
      auto take = [&](Cand& cd) {
        cd.marker = marker;
        cd.distance = distance;
        cd.signed_distance = signed_distance;
        cd.boundary = boundary;
        cd.normal = normal;
        for (int q = 0; q < 3; ++q) {
          cd.pidx[q] = ix[q];
          cd.pw[q] = w[q];
        }
      };
      if (classify_far) {
        if (signed_distance > tol) global_external_seen = 1;
        if (distance < global.distance) take(global);
      }
      if (distance < radius) {
        if (signed_distance > tol) {
          external_seen = 1;
          if (distance < external.distance) take(external);
        }
        if (distance < nearest.distance) take(nearest);
      }
    };
    if (tri_count > 0) {
      for (int t = 0; t < tri_count; ++t) {
        const int ia = tri[3 * t], ib = tri[3 * t + 1], ic = tri[3 * t + 2];
        const V3 a = load3(mx, ia), b = load3(mx, ib), cc = load3(mx, ic);
        V3 closest, fn;
        if (!closest_point_on_triangle(p, a, b, cc, closest, fn)) continue;
        const V3 normal = oriented_normal(fn, mn, ia, ib, ic);
        const V3 offset = sub(p, closest);
        const r32 distance = norm(offset);
        const r32 signed_distance = dot(offset, normal);
        const V3 wv = barycentric(closest, a, b, cc);
        const r32 w[3] = {wv.x, wv.y, wv.z};
        const int ix[3] = {ia, ib, ic};
        consider(nearest_triangle_marker(p, mx, ia, ib, ic), distance, signed_distance, closest, normal, ix, w);
      }
    } else {
      for (int m = 0; m < marker_count; ++m) {
        const V3 xm = load3(mx, m), nm = load3(mn, m);
        const V3 offset = sub(p, xm);
        const int ix[3] = {m, -1, -1};
        const r32 w[3] = {1, 0, 0};
        consider(m, norm(offset), dot(offset, nm), xm, nm, ix, w);
      }
    }
    if (nearest.marker >= 0) {
      near_count += 1;
      const Cand& sel = (external_seen && external.marker >= 0) ? external : nearest;
      nearest_marker[c] = sel.marker;
      sd[c] = sel.signed_distance;
      const r32 normal_distance = dot(sub(p, sel.boundary), sel.normal);
      r32 interior = probe;
      if (normal_distance > tol) interior = normal_distance + probe;
      store3(bp, c, sel.boundary);
      for (int q = 0; q < 3; ++q) {
        pidx[3 * c + q] = sel.pidx[q];
        pw[3 * c + q] = sel.pw[q];
      }
      store3(ip, c, add(sel.boundary, scale(sel.normal, interior)));
      if (std::fabs(sel.signed_distance) <= tol) invalid_count += 1;
      if (external_seen) {
        kind[c] = 1;
        ext_count += 1;
      } else {
        kind[c] = 2;
        int_count += 1;
      }
    } else if (classify_far && global.marker >= 0 && !global_external_seen) {
      kind[c] = 2;
      nearest_marker[c] = global.marker;
      sd[c] = global.signed_distance;
      store3(bp, c, global.boundary);
      for (int q = 0; q < 3; ++q) {
        pidx[3 * c + q] = global.pidx[q];
        pw[3 * c + q] = global.pw[q];
      }
      store3(ip, c, add(global.boundary, scale(global.normal, probe)));
      int_count += 1;
    }
  }
  report[0] = near_count;
  report[1] = ext_count;
  report[2] = int_count;
  report[3] = invalid_count;
}

// hibm_mpm.py:6499-6577 HibmMpmIbBoundaryConditions._build_from_search_kernel:
// per external IB node, the no-slip velocity, Neumann normal and Neumann
// gradient targets interpolated from the projection markers (weights > 0,
// renormalised; the nearest marker's values when no weight is usable); the
// normal is renormalised.  f32 throughout, as the reference's fields.
// Outputs per node: active (0/1), velocity (3), normal (3), gradient;
// report[4] = no-slip rows, Neumann rows, inactive internal nodes, max |v|.
EFO_API void efo_ib_build_boundary_conditions(int64_t n, const int32_t* kind, const int32_t* nearest,
                                              const int32_t* pidx, const r32* pw, const r32* mv, const r32* mn,
                                              const r32* mgrad, int marker_count, int32_t* active, r32* vel,
                                              r32* nrm, r32* grad, double* report) {
  int64_t rows = 0, inactive = 0;
  r32 vmax = 0;
  for (int64_t c = 0; c < n; ++c) {
    active[c] = 0;
    store3(vel, c, v3(0, 0, 0));
    store3(nrm, c, v3(0, 0, 0));
    grad[c] = 0;
    if (kind[c] == 1) {
      const int marker = nearest[c];
      if (!(0 <= marker && marker < marker_count)) continue;
      V3 tv = v3(0, 0, 0), tn = v3(0, 0, 0);
      r32 tg = 0, total = 0;
      for (int q = 0; q < 3; ++q) {
        const int pm = pidx[3 * c + q];
        const r32 w = pw[3 * c + q];
        if (0 <= pm && pm < marker_count && w > 0) {
          tv = add(tv, scale(load3(mv, pm), w));
          tn = add(tn, scale(load3(mn, pm), w));
          tg = tg + w * mgrad[pm];
          total = total + w;
        }
      }
      if (total > (r32)1.0e-12) {
        const r32 inv = (r32)1 / total;
        tv = scale(tv, inv);
        tn = scale(tn, inv);
        tg = tg * inv;
        const r32 nn = norm(tn);
        if (nn > (r32)1.0e-12)
          tn = divide(tn, nn);
        else
          tn = load3(mn, marker);
      } else {
        tv = load3(mv, marker);
        tn = load3(mn, marker);
        tg = mgrad[marker];
      }
      active[c] = 1;
      store3(vel, c, tv);
      store3(nrm, c, tn);
      grad[c] = tg;
      rows += 1;
      vmax = std::max(vmax, std::max(std::max(std::fabs(tv.x), std::fabs(tv.y)), std::fabs(tv.z)));
    } else if (kind[c] == 2) {
      inactive += 1;
    }
  }
  report[0] = (double)rows;
  report[1] = (double)rows;
  report[2] = (double)inactive;
  report[3] = (double)vmax;
}

// ---------------------------------------------------------------------------
// Velocity-Dirichlet reconstructed rows (HibmMpmIbBoundaryConditions,
// hibm_mpm.py:6714-7800), f32 as the reference's fields.
// ---------------------------------------------------------------------------
namespace {

struct VdGrid {
  int n[3];
  const r32* f[3];  // faces, n + 1
  const r32* c[3];  // centres
  const int32_t* obs;
  const r32* vel;   // cell velocity, 3 per cell
  int64_t idx(int i, int j, int k) const { return efo_idx(i, j, k, n[1], n[2]); }
};

// hibm_mpm.py:6714-6743 _axis_grid_coordinate_device
r32 axis_coordinate(r32 value, const r32* faces, const r32* centers, int count) {
  if (value <= centers[0]) {
    const r32 half = std::max(centers[0] - faces[0], (r32)1.0e-18);
    return (r32)-0.5 * (centers[0] - value) / half;
  }
  if (value >= centers[count - 1]) {
    const r32 half = std::max(faces[count] - centers[count - 1], (r32)1.0e-18);
    return (r32)(count - 1) + (r32)0.5 * (value - centers[count - 1]) / half;
  }
  int lower = 0, upper = count - 1;
  while (upper - lower > 1) {
    const int middle = (lower + upper) / 2;
    if (value >= centers[middle])
      lower = middle;
    else
      upper = middle;
  }
  upper = std::min(lower + 1, count - 1);
  const r32 distance = std::max(centers[upper] - centers[lower], (r32)1.0e-18);
  return (r32)lower + (value - centers[lower]) / distance;
}

V3 grid_coordinate(const VdGrid& G, V3 p) {
  return v3(axis_coordinate(p.x, G.f[0], G.c[0], G.n[0]), axis_coordinate(p.y, G.f[1], G.c[1], G.n[1]),
            axis_coordinate(p.z, G.f[2], G.c[2], G.n[2]));
}

int clampi(int v, int lo, int hi) { return std::min(std::max(v, lo), hi); }

// nearest cell of a grid coordinate: clamp(floor(g + 0.5))
void nearest_cell(const VdGrid& G, V3 g, int& i, int& j, int& k) {
  i = clampi((int)std::floor(g.x + (r32)0.5), 0, G.n[0] - 1);
  j = clampi((int)std::floor(g.y + (r32)0.5), 0, G.n[1] - 1);
  k = clampi((int)std::floor(g.z + (r32)0.5), 0, G.n[2] - 1);
}

// hibm_mpm.py:6782-6812 _sample_fluid_velocity_trilinear
V3 sample_velocity(const VdGrid& G, V3 g, r32& fluid_weight) {
  const int i0 = clampi((int)std::floor(g.x), 0, G.n[0] - 2);
  const int j0 = clampi((int)std::floor(g.y), 0, G.n[1] - 2);
  const int k0 = clampi((int)std::floor(g.z), 0, G.n[2] - 2);
  const r32 tx = std::min(std::max(g.x - (r32)i0, (r32)0), (r32)1);
  const r32 ty = std::min(std::max(g.y - (r32)j0, (r32)0), (r32)1);
  const r32 tz = std::min(std::max(g.z - (r32)k0, (r32)0), (r32)1);
  V3 value = v3(0, 0, 0);
  fluid_weight = 0;
  for (int oi = 0; oi < 2; ++oi)
    for (int oj = 0; oj < 2; ++oj)
      for (int ok = 0; ok < 2; ++ok) {
        const r32 wx = oi == 0 ? (r32)1 - tx : tx, wy = oj == 0 ? (r32)1 - ty : ty, wz = ok == 0 ? (r32)1 - tz : tz;
        const r32 w = wx * wy * wz;
        const int64_t c = G.idx(i0 + oi, j0 + oj, k0 + ok);
        if (G.obs[c] == 0) {
          value = add(value, scale(load3(G.vel, (int)c), w));
          fluid_weight = fluid_weight + w;
        }
      }
  if (fluid_weight > (r32)1.0e-12) value = divide(value, fluid_weight);
  return value;
}

// hibm_mpm.py:6846-6902 _walk_interior_velocity_sample: the first of five
// points base + s * step along the normal with any fluid weight.
V3 walk_sample(const VdGrid& G, V3 bp, V3 normal, r32 base, r32 step, r32& weight, r32& distance) {
  weight = 0;
  distance = base;
  for (int s = 0; s < 5; ++s) {
    const r32 cd = base + step * (r32)s;
    r32 w;
    const V3 v = sample_velocity(G, grid_coordinate(G, add(bp, scale(normal, cd))), w);
    if (w > (r32)1.0e-12) {
      weight = w;
      distance = cd;
      return v;
    }
  }
  return v3(0, 0, 0);
}

r32 walk_step(V3 n, r32 wx, r32 wy, r32 wz) {
  const r32 s = std::fabs(n.x) / std::max(wx, (r32)1.0e-12) + std::fabs(n.y) / std::max(wy, (r32)1.0e-12) +
                std::fabs(n.z) / std::max(wz, (r32)1.0e-12);
  return (r32)0.5 / std::max(s, (r32)1.0e-12);
}

r32 max_abs3(V3 v) { return std::max(std::max(std::fabs(v.x), std::fabs(v.y)), std::fabs(v.z)); }

struct VdReport {
  int64_t rows = 0, obstacle = 0, invalid = 0, no_fluid = 0, gap = 0, behind = 0, beyond = 0, narrow = 0,
          relocated = 0, merged = 0;
  r32 vmax = 0, wmin = (r32)1.0e30, wmax = 0;
  void row(r32 alpha, V3 v, bool max_weight = true) {
    rows += 1;
    wmin = std::min(wmin, alpha);
    if (max_weight) wmax = std::max(wmax, alpha);
    vmax = std::max(vmax, max_abs3(v));
  }
};

}  // namespace

// One call of assemble_velocity_dirichlet_reconstructed_boundary_rows
// (hibm_mpm.py:7655-7800): anchor reset and prefill (7551-7616), the row
// reconstruction (6904-7335), the relocation of rows whose node is masked
// (7337-7549) and, with marker_region, the region stamp (7618-7653).  The
// reference's relocation claims target cells with an atomic OR and stamps
// regions from parallel nodes, so their winners depend on thread order; here
// nodes run in C order (first claim wins; for the stamp, the last write).
// report[14]: active rows, inactive obstacle rows (the relocation's blocked
// rows), max |v|, invalid rows, of which no fluid sample / non-positive gap /
// node behind boundary / node beyond interior, narrow-gap rows, relocated,
// merged, blocked, min and max projection weight.
EFO_API void efo_ib_velocity_dirichlet_rows(int nx, int ny, int nz, const r32* fx, const r32* fy, const r32* fz,
                                            const r32* cx, const r32* cy, const r32* cz, const int32_t* active_ib,
                                            const r32* bc_vel, const r32* bc_nrm, const r32* bpts, const r32* ipts,
                                            const int32_t* nearest, const int32_t* obs, const r32* vel,
                                            const int32_t* marker_region, int marker_count, int32_t* vd_active,
                                            r32* vd_value, r32* vd_weight, int32_t* anchor, int32_t* region_out,
                                            double* report) {
  const VdGrid G{{nx, ny, nz}, {fx, fy, fz}, {cx, cy, cz}, obs, vel};
  const int64_t n = (int64_t)nx * ny * nz;
  VdReport R;
  // anchor reset and prefill from the interior probe point
  for (int64_t c = 0; c < n; ++c) {
    anchor[3 * c] = anchor[3 * c + 1] = anchor[3 * c + 2] = -1;
    if (active_ib[c] != 1) continue;
    int i, j, k;
    nearest_cell(G, grid_coordinate(G, load3(ipts, (int)c)), i, j, k);
    if (obs[G.idx(i, j, k)] == 0) {
      anchor[3 * c] = i;
      anchor[3 * c + 1] = j;
      anchor[3 * c + 2] = k;
    }
  }
  // row reconstruction
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const int64_t c = G.idx(i, j, k);
        vd_active[c] = 0;
        store3(vd_value, c, v3(0, 0, 0));
        vd_weight[c] = 0;
        if (active_ib[c] != 1) continue;
        if (obs[c] != 0) {
          R.obstacle += 1;
          continue;
        }
        const V3 bv = load3(bc_vel, (int)c), normal = load3(bc_nrm, (int)c);
        const V3 bp = load3(bpts, (int)c), ip = load3(ipts, (int)c);
        const V3 node = v3(cx[i], cy[j], cz[k]);
        const r32 normal_den = dot(sub(ip, bp), normal);
        const r32 normal_dist = dot(sub(node, bp), normal);
        const r32 wx = fx[i + 1] - fx[i], wy = fy[j + 1] - fy[j], wz = fz[k + 1] - fz[k];
        r32 fw, sample_den;
        const V3 iv = walk_sample(G, bp, normal, normal_den, walk_step(normal, wx, wy, wz), fw, sample_den);
        V3 fb_vel = iv;
        r32 fb_alpha = 0;
        int fai = -1, faj = -1, fak = -1;
        const bool segment = fw > (r32)1.0e-12 && sample_den > (r32)1.0e-12 && normal_dist >= 0 &&
                             normal_dist <= sample_den;
        bool fallback = false;
        if (!segment && fw > (r32)1.0e-12 && sample_den > (r32)1.0e-12 && normal_den > (r32)1.0e-12) {
          const V3 off = sub(node, bp);
          const r32 line = std::sqrt(std::max(dot(off, off), (r32)0));
          if (line > (r32)1.0e-12) {
            const V3 fn = divide(off, line);
            const r32 fstep = walk_step(fn, wx, wy, wz);
            r32 fbw, fb_den;
            fb_vel = walk_sample(G, bp, fn, line + fstep, fstep, fbw, fb_den);
            if (fbw > (r32)1.0e-12 && fb_den > line + (r32)1.0e-12) {
              fb_alpha = std::min(std::max(line / std::max(fb_den, (r32)1.0e-12), (r32)0), (r32)1);
              nearest_cell(G, grid_coordinate(G, add(bp, scale(fn, fb_den))), fai, faj, fak);
              if (obs[G.idx(fai, faj, fak)] == 0) fallback = true;
            }
          }
        }
        if (segment) {
          const r32 alpha = std::min(std::max(normal_dist / sample_den, (r32)0), (r32)1);
          const V3 tv = add(bv, scale(sub(iv, bv), alpha));
          vd_active[c] = 1;
          store3(vd_value, c, tv);
          vd_weight[c] = alpha;
          int ai, aj, ak;
          nearest_cell(G, grid_coordinate(G, add(bp, scale(normal, sample_den))), ai, aj, ak);
          if (obs[G.idx(ai, aj, ak)] == 0) {
            anchor[3 * c] = ai;
            anchor[3 * c + 1] = aj;
            anchor[3 * c + 2] = ak;
          }
          R.row(alpha, tv);
        } else if (fallback) {
          const V3 tv = add(bv, scale(sub(fb_vel, bv), fb_alpha));
          vd_active[c] = 1;
          store3(vd_value, c, tv);
          vd_weight[c] = fb_alpha;
          anchor[3 * c] = fai;
          anchor[3 * c + 1] = faj;
          anchor[3 * c + 2] = fak;
          R.row(fb_alpha, tv);
        } else if (fw <= (r32)1.0e-12 && normal_den > (r32)1.0e-12 && normal_dist >= 0) {
          R.narrow += 1;
          vd_active[c] = 1;
          store3(vd_value, c, bv);
          vd_weight[c] = 0;
          R.row(0, bv, false);
        } else {
          R.invalid += 1;
          if (fw <= (r32)1.0e-12)
            R.no_fluid += 1;
          else if (normal_den <= (r32)1.0e-12)
            R.gap += 1;
          else if (normal_dist < 0)
            R.behind += 1;
          else if (normal_dist > normal_den)
            R.beyond += 1;
          vd_active[c] = 1;
          store3(vd_value, c, bv);
          vd_weight[c] = 0;
          R.row(0, bv, false);
        }
      }
  // relocation of rows whose node is masked (the obstacle count restarts
  // here and counts the rows that found no fluid cell)
  R.obstacle = 0;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const int64_t c = G.idx(i, j, k);
        if (!(active_ib[c] == 1 && obs[c] != 0)) continue;
        const V3 normal = load3(bc_nrm, (int)c), bp = load3(bpts, (int)c), bv = load3(bc_vel, (int)c);
        const V3 node = v3(cx[i], cy[j], cz[k]);
        const r32 side = dot(sub(node, bp), normal);
        const V3 primary = side < 0 ? neg(normal) : normal;
        const r32 node_dist = std::fabs(side);
        int ti = -1, tj = -1, tk = -1;
        r32 tdist = 0, tstep = 0;
        V3 twn = primary;
        const r32 wx = fx[i + 1] - fx[i], wy = fy[j + 1] - fy[j], wz = fz[k + 1] - fz[k];
        for (int s = 0; s < 2; ++s) {
          const V3 wn = s == 0 ? primary : neg(primary);
          const r32 start = s == 0 ? node_dist : (r32)0;
          const r32 step = walk_step(wn, wx, wy, wz);
          for (int q = 0; q < 24 && ti < 0; ++q) {  // HIBM_OWNER_RELOCATION_WALK_STEPS (hibm_mpm.py:23)
            const r32 cd = start + step * (r32)(q + 1);
            int ci, cj, ck;
            nearest_cell(G, grid_coordinate(G, add(bp, scale(wn, cd))), ci, cj, ck);
            if (obs[G.idx(ci, cj, ck)] == 0) {
              const r32 ccd = dot(sub(v3(cx[ci], cy[cj], cz[ck]), bp), wn);
              if (ccd > (r32)1.0e-12) {
                ti = ci;
                tj = cj;
                tk = ck;
                tdist = ccd;
                twn = wn;
                tstep = step;
              }
            }
          }
        }
        if (ti < 0) {
          R.obstacle += 1;
          continue;
        }
        const int64_t t = G.idx(ti, tj, tk);
        if (vd_active[t] != 0) {
          R.merged += 1;
          continue;
        }
        vd_active[t] = 1;
        r32 sw, sd;
        const V3 sv = walk_sample(G, bp, twn, tdist + (r32)2.0 * tstep, tstep, sw, sd);
        V3 tv = bv;
        r32 alpha = 0;
        if (sw > (r32)1.0e-12 && sd > tdist) {
          alpha = std::min(std::max(tdist / sd, (r32)0), (r32)1);
          tv = add(bv, scale(sub(sv, bv), alpha));
        }
        store3(vd_value, t, tv);
        vd_weight[t] = alpha;
        anchor[3 * c] = ti;
        anchor[3 * c + 1] = tj;
        anchor[3 * c + 2] = tk;
        R.relocated += 1;
        R.row(alpha, tv);
      }
  // marker-region stamp
  if (marker_region != nullptr && region_out != nullptr) {
    for (int64_t c = 0; c < n; ++c) {
      if (active_ib[c] != 1) continue;
      const int m = nearest[c];
      if (m < 0 || m >= marker_count) continue;
      const int region = marker_region[m];
      if (vd_active[c] != 0) region_out[c] = region;
      const int ai = anchor[3 * c], aj = anchor[3 * c + 1], ak = anchor[3 * c + 2];
      if (ai >= 0 && ai < nx && aj >= 0 && aj < ny && ak >= 0 && ak < nz && vd_active[G.idx(ai, aj, ak)] != 0)
        region_out[G.idx(ai, aj, ak)] = region;
    }
  }
  const double out[14] = {(double)R.rows,      (double)R.obstacle,  (double)R.vmax,     (double)R.invalid,
                          (double)R.no_fluid,  (double)R.gap,       (double)R.behind,   (double)R.beyond,
                          (double)R.narrow,    (double)R.relocated, (double)R.merged,   (double)R.obstacle,
                          R.rows > 0 ? (double)R.wmin : 0.0, (double)R.wmax};
  for (int q = 0; q < 14; ++q) report[q] = out[q];
}
