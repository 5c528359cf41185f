"""CPU restatement of the triangle Mooney-Rivlin shell MPM -- TEST INFRASTRUCTURE ONLY.

Restates ``TriMooneyShellMpmState`` of simulation_core/mooney_shell_mpm.py in
FP64 numpy: the constructor's mass/area/region set-up (:108-253, :463-540),
the per-face Mooney membrane law (:562-646), the region loads (:660-742), the
trilinear PIC/FLIP step (:744-1003, :1005-1177), the current-shape normals
(:436-461) and the packed report (:1317-1391).  Only the tests use it, as the
checker of the CUDA path; the product never imports it.

Parity is pinned by the reference's own known answers for this class
(tests/test_mooney_shell_mpm.py:443-1670: the equal-biaxial tension formula,
the finite-difference energy gradient, the degenerate triangle, the rest
sphere, body acceleration, out-of-bounds, fixed-region and FLIP cases), which
``tests/test_oracle_shell.py`` runs against this module.  Taichi is not
installed here, so the reference itself cannot be run to make fixtures.
"""

from __future__ import annotations

import numpy as np

_C_CAP = 1.0e6


def unique_undirected_edges(faces: np.ndarray) -> np.ndarray:
    """mooney_shell_mpm.py:53-61: sorted unique (min, max) vertex pairs."""
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    if f.size == 0:
        return np.zeros((0, 2), dtype=np.int32)
    e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], axis=0)
    e = np.sort(e, axis=1)
    return np.unique(e, axis=0).astype(np.int32)


def mesh_bounds_with_padding(vertices: np.ndarray, frac: float):
    """mooney_shell_mpm.py:64-77."""
    lo = np.min(vertices, axis=0).astype(np.float64)
    hi = np.max(vertices, axis=0).astype(np.float64)
    ext = float(np.max(hi - lo))
    if ext <= 0.0:
        ext = 1.0
    pad = max(frac * ext, 1.0e-6 * ext)
    return lo - pad, hi + pad


def _norm(a):
    return np.sqrt(np.sum(a * a, axis=-1))


def mooney_face_forces(rest, cur, faces, c1, c2, scale, thickness):
    """Per-face membrane forces on (a, b, c), mooney_shell_mpm.py:562-639.

    ``thickness`` is a per-face array.  Returns (force[F,3,3], valid[F]) where
    invalid faces (degenerate rest triangle) contribute nothing."""
    ra, rb, rc = rest[faces[:, 0]], rest[faces[:, 1]], rest[faces[:, 2]]
    a, b, c = cur[faces[:, 0]], cur[faces[:, 1]], cur[faces[:, 2]]
    rav = np.cross(rb - ra, rc - ra)
    ravn = _norm(rav)
    rarea = 0.5 * ravn
    e0 = rb - ra
    e0l = _norm(e0)
    ok = (rarea > 1e-12) & (ravn > 1e-12) & (e0l > 1e-12)
    safe_ravn = np.where(ravn > 0, ravn, 1.0)
    safe_e0l = np.where(e0l > 0, e0l, 1.0)
    rn = rav / safe_ravn[:, None]
    t0 = e0 / safe_e0l[:, None]
    t1 = np.cross(rn, t0)
    rac = rc - ra
    xc = np.sum(rac * t0, axis=1)
    yc = np.sum(rac * t1, axis=1)
    ok &= np.abs(yc) > 1e-12
    safe_yc = np.where(np.abs(yc) > 0, yc, 1.0)
    inv00 = 1.0 / safe_e0l
    inv01 = -xc / (safe_e0l * safe_yc)
    inv11 = 1.0 / safe_yc
    g0 = b - a
    g1 = c - a
    f0 = g0 * inv00[:, None]
    f1 = g0 * inv01[:, None] + g1 * inv11[:, None]
    c00 = np.minimum(np.sum(f0 * f0, axis=1), _C_CAP)
    c01 = np.clip(np.sum(f0 * f1, axis=1), -_C_CAP, _C_CAP)
    c11 = np.minimum(np.sum(f1 * f1, axis=1), _C_CAP)
    det = np.maximum(c00 * c11 - c01 * c01, 1e-6)
    idet = 1.0 / det
    i00 = c11 * idet
    i01 = -c01 * idet
    i11 = c00 * idet
    tr = c00 + c11
    s00 = c1 * (1.0 - i00 * idet) + c2 * (det * i00 + idet - tr * idet * i00)
    s01 = c1 * (-i01 * idet) + c2 * (det * i01 - tr * idet * i01)
    s11 = c1 * (1.0 - i11 * idet) + c2 * (det * i11 + idet - tr * idet * i11)
    p0 = scale * 2.0 * (f0 * s00[:, None] + f1 * s01[:, None])
    p1 = scale * 2.0 * (f0 * s01[:, None] + f1 * s11[:, None])
    vol = thickness * rarea
    ge0 = vol[:, None] * (p0 * inv00[:, None] + p1 * inv01[:, None])
    ge1 = vol[:, None] * (p1 * inv11[:, None])
    cap = scale * (c1 + c2) * thickness * np.sqrt(rarea) * 100.0

    def limit(v):
        n = _norm(v)
        out = np.where((n > cap)[:, None] & (cap > 0)[:, None], v * (cap / np.where(n > 0, n, 1.0))[:, None], v)
        bad = ~np.isfinite(n) | (n > 1e30)
        out[bad] = 0.0
        return out

    force = np.zeros((faces.shape[0], 3, 3))
    force[:, 0] = limit(ge0 + ge1)
    force[:, 1] = limit(-ge0)
    force[:, 2] = limit(-ge1)
    force[~ok] = 0.0
    # normal used for the pressure load (rest normal unless the current area is non-degenerate)
    avec = np.cross(b - a, c - a)
    avn = _norm(avec)
    normal = np.where((avn > 1e-12)[:, None], avec / np.where(avn > 0, avn, 1.0)[:, None], rn)
    pressure_ok = (rarea > 1e-12) & (ravn > 1e-12)
    return force, ok, pressure_ok, normal, 0.5 * avn


class OracleTriShell:
    """FP64 restatement of TriMooneyShellMpmState (mooney_shell_mpm.py:105-1391)."""

    def __init__(self, vertices, faces, *, thickness_m, density_kgm3, c1_pa, c2_pa,
                 membrane_force_scale=1.0, grid_nodes=(36, 36, 36), bounds_padding_fraction=0.5,
                 face_region_id=None, primary_region_id, secondary_region_id, fixed_region_id=-1,
                 primary_thickness_m=None, secondary_thickness_m=None, f32_state=True):
        # f32_state mirrors the reference's f32 fields (mooney_shell_mpm.py:179-196):
        # x, u, v and the vertex forces are rounded to f32 where the reference stores them.
        self.f32_state = bool(f32_state)
        v32 = np.asarray(vertices, dtype=np.float32)
        self.faces = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
        self.edges = unique_undirected_edges(self.faces).astype(np.int64)
        self.face_region = (np.zeros(len(self.faces), np.int64) if face_region_id is None
                            else np.asarray(face_region_id, np.int64))
        lo, hi = mesh_bounds_with_padding(v32, bounds_padding_fraction)
        self.bmin = lo.astype(np.float32).astype(np.float64)
        bmax = hi.astype(np.float32).astype(np.float64)
        self.n = np.array(grid_nodes, np.int64)
        self.dx = (bmax - self.bmin) / (self.n - 1)
        self.np_ = v32.shape[0]
        self.thickness = float(thickness_m)
        self.c1, self.c2, self.scale = float(c1_pa), float(c2_pa), float(membrane_force_scale)
        self.primary, self.secondary, self.fixed_region = int(primary_region_id), int(secondary_region_id), int(fixed_region_id)
        self.t_primary = float(thickness_m if primary_thickness_m is None else primary_thickness_m)
        self.t_secondary = float(thickness_m if secondary_thickness_m is None else secondary_thickness_m)
        self.rest_x = v32.astype(np.float64)
        self.x = self.rest_x.copy()
        self.u = np.zeros_like(self.x)
        self.v = np.zeros_like(self.x)
        self.fint = np.zeros_like(self.x)
        self.fext = np.zeros_like(self.x)
        # _init_mass_kernel (:480-540)
        reg = self.face_region
        t = np.full(len(self.faces), self.thickness)
        t[reg == self.primary] = self.t_primary
        sec = (reg == self.secondary) & (reg != self.primary)
        t[sec] = self.t_secondary
        fix = (self.fixed_region >= 0) & (reg == self.fixed_region) & (reg != self.primary) & ~sec
        t[fix] = self.t_primary
        area = self._rest_face_area()
        self.mass = np.zeros(self.np_)
        self.rest_area_w = np.zeros(self.np_)
        for k in range(3):
            np.add.at(self.rest_area_w, self.faces[:, k], area / 3.0)
            np.add.at(self.mass, self.faces[:, k], float(np.float32(density_kgm3)) * t * area / 3.0)
        self.vregion = np.full(self.np_, 2147483647, np.int64)
        self.fixed = np.zeros(self.np_, np.int64)
        for k in range(3):
            np.minimum.at(self.vregion, self.faces[:, k], reg)
            if self.fixed_region >= 0:
                self.fixed[self.faces[reg == self.fixed_region, k]] = 1
        self.primary_area = float(np.sum(area[reg == self.primary]))
        self.secondary_area = float(np.sum(area[sec]))
        self.normal = np.zeros_like(self.x)
        self.area_w = np.zeros(self.np_)
        self.update_normals()
        self.last = None

    def _rest_face_area(self):
        f = self.faces
        r = self.rest_x
        return 0.5 * _norm(np.cross(r[f[:, 1]] - r[f[:, 0]], r[f[:, 2]] - r[f[:, 0]]))

    def update_normals(self):
        """mooney_shell_mpm.py:436-461."""
        f = self.faces
        av = np.cross(self.x[f[:, 1]] - self.x[f[:, 0]], self.x[f[:, 2]] - self.x[f[:, 0]])
        avn = _norm(av)
        keep = avn > 1e-12
        self.normal[:] = 0.0
        self.area_w[:] = 0.0
        for k in range(3):
            np.add.at(self.normal, f[keep, k], av[keep])
            np.add.at(self.area_w, f[keep, k], 0.5 * avn[keep] / 3.0)
        nn = _norm(self.normal)
        ok = nn > 1e-12
        self.normal[ok] /= nn[ok][:, None]

    def add_region_area_load(self, region_id, load):
        """mooney_shell_mpm.py:710-742."""
        area = self._rest_face_area()
        sel = self.face_region == int(region_id)
        share = np.asarray(load, np.float64)[None, :] * area[sel][:, None] / 3.0
        for k in range(3):
            np.add.at(self.fext, self.faces[sel, k], share)

    # -- the step ---------------------------------------------------------------------------
    def _coord(self, x):
        return (x - self.bmin) / self.dx

    def _oob(self, c):
        bad = ~np.all(np.isfinite(c) & (np.abs(c) < 1e30), axis=1)
        return bad | np.any(c < 0.0, axis=1) | np.any(c > (self.n - 1), axis=1)

    def _stencil(self, c):
        base = np.clip(np.floor(c).astype(np.int64), 0, self.n - 2)
        fx = np.clip(c - base, 0.0, 1.0)
        out = []
        for ox in (0, 1):
            for oy in (0, 1):
                for oz in (0, 1):
                    w = ((fx[:, 0] if ox else 1 - fx[:, 0]) * (fx[:, 1] if oy else 1 - fx[:, 1])
                         * (fx[:, 2] if oz else 1 - fx[:, 2]))
                    idx = ((base[:, 0] + ox) * self.n[1] + base[:, 1] + oy) * self.n[2] + base[:, 2] + oz
                    out.append((idx, w))
        return out

    def _store(self, *names):
        if self.f32_state:
            for n in names:
                setattr(self, n, getattr(self, n).astype(np.float32).astype(np.float64))

    def _faces_forces(self, thickness, pressure):
        force, ok, pok, normal, area = mooney_face_forces(
            self.rest_x, self.x, self.faces, self.c1, self.c2, self.scale, thickness)
        for k in range(3):
            np.add.at(self.fint, self.faces[:, k], force[:, k])
        if pressure is not None and pressure != 0.0:
            pf = (pressure * area / 3.0)[:, None] * normal
            pf[~pok] = 0.0
            for k in range(3):
                np.add.at(self.fext, self.faces[:, k], pf)

    def step(self, *, dt_s, pressure_pa, velocity_damping=1.0, flip_blend=0.95, body_acceleration_mps2=(0, 0, 0)):
        """_step_kernel, mooney_shell_mpm.py:860-1003."""
        self.fint[:] = 0.0
        self.fext[:] = 0.0
        self._faces_forces(np.full(len(self.faces), self.thickness), float(np.float32(pressure_pa)))
        return self._transfer(dt_s, velocity_damping, flip_blend, body_acceleration_mps2, self.primary, self.secondary)

    def advance_region_loads(self, *, dt_s, primary_region_id, secondary_region_id, primary_area_load_npm2,
                             primary_interface_reaction_n, secondary_interface_reaction_n,
                             primary_area_load_region_id=None, velocity_damping=1.0, flip_blend=0.95,
                             body_acceleration_mps2=(0, 0, 0), preserve_existing_external_force=False):
        """_step_region_kernel with _compute_region_surface_forces, mooney_shell_mpm.py:667-708, 1005-1177."""
        pid, sid = int(primary_region_id), int(secondary_region_id)
        lid = pid if primary_area_load_region_id is None else int(primary_area_load_region_id)
        self.fint[:] = 0.0
        if not preserve_existing_external_force:
            self.fext[:] = 0.0
        reg = self.face_region
        t = np.full(len(self.faces), self.thickness)
        t[reg == pid] = self.t_primary
        t[(reg == sid) & (reg != pid)] = self.t_secondary
        self._faces_forces(t, None)
        area = self._rest_face_area()
        load = np.zeros((len(self.faces), 3))
        load[reg == lid] += np.asarray(primary_area_load_npm2, np.float64)[None, :] * area[reg == lid][:, None]
        pr = np.asarray(primary_interface_reaction_n, np.float64)
        sr = np.asarray(secondary_interface_reaction_n, np.float64)
        sp = reg == pid
        ss = (reg == sid) & ~sp
        load[sp] += pr[None, :] * (area[sp] / max(self.primary_area, 1e-12))[:, None]
        load[ss] += sr[None, :] * (area[ss] / max(self.secondary_area, 1e-12))[:, None]
        nz = _norm(load) > 0
        for k in range(3):
            np.add.at(self.fext, self.faces[nz, k], load[nz] / 3.0)
        return self._transfer(dt_s, velocity_damping, flip_blend, body_acceleration_mps2, pid, sid)

    def advance_with_external_forces(self, *, dt_s, primary_region_id, secondary_region_id, velocity_damping=1.0,
                                     flip_blend=0.95, body_acceleration_mps2=(0, 0, 0)):
        return self.advance_region_loads(
            dt_s=dt_s, primary_region_id=primary_region_id, secondary_region_id=secondary_region_id,
            primary_area_load_npm2=(0, 0, 0), primary_interface_reaction_n=(0, 0, 0),
            secondary_interface_reaction_n=(0, 0, 0), velocity_damping=velocity_damping,
            flip_blend=flip_blend, body_acceleration_mps2=body_acceleration_mps2,
            preserve_existing_external_force=True)

    def _transfer(self, dt, damping, flip, body, pid, sid):
        dt = float(dt)
        nn = int(np.prod(self.n))
        gm = np.zeros(nn)
        gp = np.zeros((nn, 3))
        gf = np.zeros((nn, 3))
        self._store("fint", "fext")
        # edge strain statistic (:542-550)
        e = self.edges
        rl = _norm(self.rest_x[e[:, 1]] - self.rest_x[e[:, 0]])
        cl = _norm(self.x[e[:, 1]] - self.x[e[:, 0]])
        ok = (rl > 1e-12) & (cl > 1e-12)
        max_edge = float(np.max(np.abs(np.maximum(cl[ok] / rl[ok], 1e-6) - 1.0))) if np.any(ok) else 0.0
        # particle pass (:930-959)
        self.fext += self.mass[:, None] * np.asarray(body, np.float64)[None, :]
        self._store("fext")
        c = self._coord(self.x)
        oob = self._oob(c)
        total = self.fint + self.fext
        dep = ~oob & (self.fixed == 0)
        for idx, w in self._stencil(c[dep]):
            np.add.at(gm, idx, w * self.mass[dep])
            np.add.at(gp, idx, w[:, None] * (self.mass[dep, None] * self.v[dep]))
            np.add.at(gf, idx, w[:, None] * total[dep])
        pm = self.mass[:, None] * self.v
        tf = total.copy()
        pm[self.fixed != 0] = 0.0
        tf[self.fixed != 0] = 0.0
        total_area = float(np.sum(self.area_w))
        fsum = self.fint.sum(axis=0)
        fsq = float(np.sum(self.fint * self.fint))
        pmom = pm.sum(axis=0)
        tforce = tf.sum(axis=0)
        mom2 = float(np.sum(pm * pm))
        imp2 = float(np.sum((dt * tf) ** 2))
        # grid update (:961-976)
        act = gm > 1e-20
        gv = np.zeros((nn, 3))
        gvb = np.zeros((nn, 3))
        gvb[act] = gp[act] / gm[act, None]
        tv = gvb + dt * gf / np.where(act, gm, 1.0)[:, None]
        gv[act] = tv[act] * float(np.float32(damping))
        tmom = (gm[act, None] * tv[act]).sum(axis=0)
        gmom = (gm[act, None] * gv[act]).sum(axis=0)
        max_speed = float(np.max(_norm(gv[act]))) if np.any(act) else 0.0
        # G2P (:978-1003)
        fb = float(np.float32(flip))
        ib = np.nonzero(~oob)[0]
        pic = np.zeros((len(ib), 3))
        dlt = np.zeros((len(ib), 3))
        for idx, w in self._stencil(c[ib]):
            pic += w[:, None] * gv[idx]
            dlt += w[:, None] * (gv[idx] - gvb[idx])
        newv = (1 - fb) * pic + fb * (self.v[ib] + dlt)
        free = self.fixed[ib] == 0
        self.v[ib] = newv
        self.x[ib[free]] += dt * newv[free]
        self.u[ib[free]] += dt * newv[free]
        fx_ = ib[~free]
        fo = np.nonzero(oob & (self.fixed != 0))[0]
        for sel in (fx_, fo):
            self.x[sel] = self.rest_x[sel]
            self.u[sel] = 0.0
            self.v[sel] = 0.0
        mo = np.nonzero(oob & (self.fixed == 0))[0]
        self.x[mo] += dt * self.v[mo]
        self.u[mo] += dt * self.v[mo]
        if len(mo):
            max_speed = max(max_speed, float(np.max(_norm(self.v[mo]))))
        self._store("x", "u", "v")
        ib2 = ~self._oob(self._coord(self.x))
        cnt = int(np.sum(ib2))
        cc = self.x[ib2].sum(axis=0) / max(cnt, 1)
        rc = self.rest_x[ib2].sum(axis=0) / max(cnt, 1)
        rr = _norm(self.rest_x[ib2] - rc)
        cr = _norm(self.x[ib2] - cc)
        st = cr / np.maximum(rr, 1e-12)
        sel_p = ib2 & (self.vregion == pid)
        sel_s = ib2 & (self.vregion == sid) & ~sel_p
        exp = pmom + dt * tforce
        den = max(float(np.linalg.norm(exp)), np.sqrt(mom2), np.sqrt(imp2), 1e-20)
        self.update_normals()
        self.grid_mass = gm
        self.grid_velocity = gv
        self.last = dict(
            active_grid_nodes=int(np.sum(act)), grid_out_of_bounds_particle_count=int(np.sum(oob)),
            stretch_count=int(cnt), mean_radial_stretch=float(np.sum(st)) / max(cnt, 1),
            max_radial_stretch_error=float(np.max(np.abs(st - 1.0))) if cnt else 0.0,
            max_edge_strain=max_edge, max_speed_mps=max_speed, total_mass_kg=float(np.sum(self.mass)),
            total_area_m2=total_area,
            primary_mean_displacement_m=tuple(self.u[sel_p].sum(axis=0) / max(int(sel_p.sum()), 1)),
            primary_mean_velocity_mps=tuple(self.v[sel_p].sum(axis=0) / max(int(sel_p.sum()), 1)),
            secondary_mean_displacement_m=tuple(self.u[sel_s].sum(axis=0) / max(int(sel_s.sum()), 1)),
            secondary_mean_velocity_mps=tuple(self.v[sel_s].sum(axis=0) / max(int(sel_s.sum()), 1)),
            particle_momentum_kg_mps=tuple(pmom), grid_momentum_kg_mps=tuple(gmom), total_force_n=tuple(tforce),
            internal_force_rms_n=float(np.sqrt(fsq / max(self.np_, 1))),
            net_internal_force_relative_error=float(np.linalg.norm(fsum)) / max(np.sqrt(fsq), 1e-20),
            transfer_relative_error=float(np.linalg.norm(tmom - exp)) / den,
        )
        return self.last
