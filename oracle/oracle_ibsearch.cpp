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
