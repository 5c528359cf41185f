"""Known-answer cases of the triangle Mooney membrane MPM, shared by the oracle
tests (CPU) and the drop-in tests (GPU).

Each case restates one of the reference's own tests
(tests/test_mooney_shell_mpm.py, line cited per case) against a ``make``
callable that builds a state with the reference's constructor arguments; the
state exposes ``x``, ``u``, ``v``, ``mass_kg``, ``grid_mass_kg`` and
``internal_force_n`` with ``to_numpy`` / ``from_numpy`` and ``step`` returning
a report with the reference's field names.  ``OracleShellAdapter`` gives the
FP64 oracle that interface.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from easyfsi_b200.geometry import SurfaceMesh, UvSphereResolution, make_plate_mesh, make_uv_sphere
from oracle.oracle_shell import OracleTriShell

TRI = SurfaceMesh(vertices=np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]]),
                  faces=np.array([[0, 1, 2]], dtype=np.int32))
SQUARE = SurfaceMesh(vertices=np.array([[10.0, -4.0, 2.0], [11.0, -4.0, 2.0], [11.0, -3.0, 2.0], [10.0, -3.0, 2.0]]),
                     faces=np.array([[0, 1, 2], [0, 2, 3]], dtype=np.int32))
LAW = dict(thickness_m=0.05, density_kgm3=1.0, c1_pa=20.0, c2_pa=10.0, primary_region_id=1, secondary_region_id=2)


class _View:
    def __init__(self, owner, name):
        self.owner, self.name = owner, name

    def to_numpy(self):
        return np.asarray(getattr(self.owner, self.name), dtype=np.float32).copy()

    def from_numpy(self, a):
        setattr(self.owner, self.name, np.asarray(a, dtype=np.float64).copy())


class OracleShellAdapter:
    """The oracle behind the drop-in's field names (test helper)."""

    _NAMES = dict(x="x", u="u", v="v", mass_kg="mass", internal_force_n="fint", external_force_n="fext",
                  grid_mass_kg="grid_mass", surface_normal="normal", area_weight_m2="area_w")

    def __init__(self, mesh, **kw):
        kw.pop("runtime", None)
        self.o = OracleTriShell(mesh.vertices, mesh.faces, **kw)
        self.bounds_max = tuple(self.o.bmin + self.o.dx * (self.o.n - 1))
        self.dx = tuple(self.o.dx)
        self.o.grid_mass = np.zeros(int(np.prod(self.o.n)))

    def __getattr__(self, name):
        if name in OracleShellAdapter._NAMES:
            return _View(self.o, OracleShellAdapter._NAMES[name])
        raise AttributeError(name)

    def _wrap(self, rep):
        return SimpleNamespace(particle_count=self.o.np_, face_count=len(self.o.faces),
                               edge_count=len(self.o.edges), **rep)

    def step(self, **kw):
        kw.pop("read_report", None)
        return self._wrap(self.o.step(**kw))

    def advance_region_loads(self, **kw):
        kw.pop("read_report", None)
        return self._wrap(self.o.advance_region_loads(**kw))

    def advance_with_external_forces(self, **kw):
        kw.pop("read_report", None)
        return self._wrap(self.o.advance_with_external_forces(**kw))

    def add_region_area_load(self, *, region_id, area_load_npm2):
        self.o.add_region_area_load(region_id, area_load_npm2)


def _energy(rest, cur, thickness, c1, c2):
    """Membrane energy of one triangle (the reference test's helper, test_mooney_shell_mpm.py:13-46)."""
    ra, rb, rc = rest
    ca, cb, cc = cur
    rav = np.cross(rb - ra, rc - ra)
    area = 0.5 * np.linalg.norm(rav)
    n = rav / np.linalg.norm(rav)
    e0 = rb - ra
    t0 = e0 / np.linalg.norm(e0)
    t1 = np.cross(n, t0)
    xc, yc = float(np.dot(rc - ra, t0)), float(np.dot(rc - ra, t1))
    inv = np.array([[1 / np.linalg.norm(e0), -xc / (np.linalg.norm(e0) * yc)], [0.0, 1 / yc]])
    F = np.column_stack((cb - ca, cc - ca)) @ inv
    C = F.T @ F
    det, tr = float(np.linalg.det(C)), float(np.trace(C))
    return thickness * area * (c1 * (tr + 1 / det - 3) + c2 * (det + tr / det - 3))


def _fd_force(rest, cur, thickness, c1, c2, eps=1e-5):
    f = np.zeros_like(cur)
    for v in range(cur.shape[0]):
        for a in range(3):
            p, m = cur.copy(), cur.copy()
            p[v, a] += eps
            m[v, a] -= eps
            f[v, a] = -(_energy(rest, p, thickness, c1, c2) - _energy(rest, m, thickness, c1, c2)) / (2 * eps)
    return f


# -- cases ------------------------------------------------------------------------------------------
def case_equal_biaxial(make):
    """test_mooney_shell_mpm.py:550-592."""
    st = make(TRI, grid_nodes=(12, 12, 12), bounds_padding_fraction=1.0, **LAW)
    s = 1.2
    st.x.from_numpy((TRI.vertices * s).astype(np.float32))
    st.step(dt_s=0.0, pressure_pa=0.0, velocity_damping=1.0)
    f = st.internal_force_n.to_numpy()
    tension = 2.0 * 0.05 * (1.0 - s**-6) * (20.0 + s * s * 10.0)
    np.testing.assert_allclose(f[0], [0.5 * s * tension, 0.5 * s * tension, 0.0], rtol=5.0e-4, atol=1.0e-6)


def case_area_preserving_gradient(make):
    """test_mooney_shell_mpm.py:594-645."""
    st = make(TRI, grid_nodes=(12, 12, 12), bounds_padding_fraction=1.0, **LAW)
    s = 1.35
    cur = np.array([[0.0, 0.0, 0.0], [s, 0.0, 0.0], [0.0, 1.0 / s, 0.0]])
    st.x.from_numpy(cur.astype(np.float32))
    st.step(dt_s=0.0, pressure_pa=0.0, velocity_damping=1.0)
    f = st.internal_force_n.to_numpy()
    want = _fd_force(TRI.vertices, cur, 0.05, 20.0, 10.0)
    assert np.linalg.norm(want) > 1.0e-2
    np.testing.assert_allclose(f, want, rtol=2.0e-3, atol=2.0e-5)
    np.testing.assert_allclose(f.sum(axis=0), np.zeros(3), atol=1.0e-6)


def case_degenerate_triangle(make):
    """test_mooney_shell_mpm.py:647-681."""
    law = dict(LAW, c2_pa=0.0)
    st = make(TRI, grid_nodes=(8, 8, 8), bounds_padding_fraction=1.0, **law)
    cur = TRI.vertices.copy()
    cur[1] = cur[0]
    st.x.from_numpy(cur.astype(np.float32))
    rep = st.step(dt_s=0.0, pressure_pa=0.0, velocity_damping=1.0)
    f = st.internal_force_n.to_numpy()
    assert np.all(np.isfinite(f))
    assert rep.internal_force_rms_n > 1.0e-6
    np.testing.assert_allclose(f.sum(axis=0), np.zeros(3), atol=1.0e-6)


def case_rest_sphere(make):
    """test_mooney_shell_mpm.py:683-704."""
    mesh = make_uv_sphere(UvSphereResolution(latitude_bands=8, longitude_segments=25), 1.0)
    st = make(mesh, grid_nodes=(24, 24, 24), **LAW)
    rep = st.step(dt_s=1.0e-3, pressure_pa=0.0, velocity_damping=1.0)
    assert rep.particle_count == mesh.vertex_count and rep.face_count == mesh.face_count
    assert rep.edge_count > 0
    assert abs(rep.mean_radial_stretch - 1.0) <= 1.0e-6
    assert abs(rep.max_edge_strain) <= 1.0e-6
    assert abs(rep.internal_force_rms_n) <= 1.0e-5
    assert rep.transfer_relative_error < 2.0e-5


def case_translation_invariant_stretch(make, oob=False):
    """test_mooney_shell_mpm.py:706-778 (oob=True: one particle moved out of the grid)."""
    st = make(SQUARE, grid_nodes=(16, 16, 16), bounds_padding_fraction=0.5, **LAW)
    t = np.array([0.2, -0.1, 0.3], dtype=np.float32)
    cur = SQUARE.vertices.astype(np.float32) + t
    if oob:
        cur[0, 0] = float(st.bounds_max[0] + st.dx[0])
    st.x.from_numpy(cur)
    st.u.from_numpy(np.broadcast_to(t, cur.shape).copy())
    rep = st.step(dt_s=0.0, pressure_pa=0.0, velocity_damping=1.0)
    if oob:
        assert rep.grid_out_of_bounds_particle_count == 1
    assert abs(rep.mean_radial_stretch - 1.0) <= 2.0e-6
    assert abs(rep.max_radial_stretch_error) <= 2.0e-6


def case_region_mean_excludes_oob(make):
    """test_mooney_shell_mpm.py:780-838."""
    rest = np.array([[-0.004, -0.004, 0.0], [0.004, -0.004, 0.0], [-0.004, 0.004, 0.0],
                     [0.010, -0.004, 0.0], [0.018, -0.004, 0.0], [0.010, 0.004, 0.0]])
    mesh = SurfaceMesh(vertices=rest, faces=np.array([[0, 1, 2], [3, 4, 5]], dtype=np.int32))
    st = make(mesh, thickness_m=0.003, density_kgm3=1040.0, c1_pa=20.0, c2_pa=10.0,
              face_region_id=np.array([7, 8], dtype=np.int32), primary_region_id=7, secondary_region_id=8,
              grid_nodes=(16, 16, 16), bounds_padding_fraction=1.0)
    cur = rest.astype(np.float32)
    d = np.zeros_like(cur)
    d[0], d[1], d[2] = [2.0, 0, 0], [0.001, 0, 0], [0.003, 0, 0]
    cur += d
    cur[0] = np.array([st.bounds_max[0] + 2.0 * st.dx[0], 0.0, 0.0], dtype=np.float32)
    vel = np.zeros_like(cur)
    vel[0], vel[1], vel[2] = [7.0, 0, 0], [0.02, 0, 0], [0.04, 0, 0]
    st.x.from_numpy(cur)
    st.u.from_numpy(d)
    st.v.from_numpy(vel)
    rep = st.step(dt_s=0.0, pressure_pa=0.0, velocity_damping=1.0)
    np.testing.assert_allclose(rep.primary_mean_displacement_m, st.u.to_numpy()[[1, 2]].mean(axis=0), atol=1.0e-7)
    np.testing.assert_allclose(rep.primary_mean_velocity_mps, st.v.to_numpy()[[1, 2]].mean(axis=0), atol=1.0e-7)
    assert rep.grid_out_of_bounds_particle_count == 1
    assert abs(rep.primary_mean_velocity_mps[0]) < 1.0


def case_oob_no_clamped_deposit(make):
    """test_mooney_shell_mpm.py:840-907."""
    st = make(TRI, grid_nodes=(12, 12, 12), bounds_padding_fraction=0.25, **LAW)
    pos = st.x.to_numpy()
    pos[0, 0] = float(st.bounds_max[0] + st.dx[0])
    st.x.from_numpy(pos.astype(np.float32))
    m = st.mass_kg.to_numpy()
    rep = st.step(dt_s=0.0, pressure_pa=0.0, velocity_damping=1.0)
    assert rep.grid_out_of_bounds_particle_count == 1
    assert abs(float(np.sum(st.grid_mass_kg.to_numpy())) - float(np.sum(m[1:]))) <= max(float(np.sum(m)) * 1e-6, 1e-12)


def case_oob_reentry(make):
    """test_mooney_shell_mpm.py:909-944."""
    st = make(TRI, grid_nodes=(12, 12, 12), bounds_padding_fraction=0.25, **LAW)
    dt = 0.1
    pos = st.x.to_numpy()
    vel = np.zeros_like(pos, dtype=np.float32)
    pos[0, 0] = float(st.bounds_max[0] + 0.5 * st.dx[0])
    vel[0, 0] = float(-2.0 * st.dx[0] / dt)
    st.x.from_numpy(pos.astype(np.float32))
    st.v.from_numpy(vel)
    rep = st.step(dt_s=dt, pressure_pa=0.0, velocity_damping=1.0)
    assert rep.grid_out_of_bounds_particle_count == 1
    assert float(st.x.to_numpy()[0, 0]) <= float(st.bounds_max[0])


def case_pressure_expands(make):
    """test_mooney_shell_mpm.py:946-964."""
    mesh = make_uv_sphere(UvSphereResolution(latitude_bands=8, longitude_segments=25), 1.0)
    st = make(mesh, grid_nodes=(36, 36, 36), **LAW)
    rep = st.step(dt_s=1.0e-3, pressure_pa=2.0, velocity_damping=1.0)
    assert rep.mean_radial_stretch > 1.0 and rep.max_speed_mps > 0.0 and rep.active_grid_nodes > 0
    assert rep.transfer_relative_error < 2.0e-5


def case_body_acceleration(make):
    """test_mooney_shell_mpm.py:966-1009."""
    mesh = SurfaceMesh(vertices=np.array([[0.0, 0.0, 0.0], [0.008, 0.0, 0.0], [0.0, 0.008, 0.0]], dtype=np.float32),
                       faces=np.array([[0, 1, 2]], dtype=np.int32))
    st = make(mesh, thickness_m=0.003, density_kgm3=1040.0, c1_pa=20.0, c2_pa=10.0,
              face_region_id=np.array([7], dtype=np.int32), primary_region_id=7, secondary_region_id=8,
              grid_nodes=(16, 16, 16))
    rep = st.step(dt_s=1.0e-4, pressure_pa=0.0, velocity_damping=1.0, flip_blend=1.0,
                  body_acceleration_mps2=(0.0, -2.0, -9.81))
    assert abs(rep.total_force_n[0]) <= 1.0e-10
    assert abs(rep.total_force_n[1] + 2.0 * rep.total_mass_kg) <= 1.0e-9
    assert abs(rep.total_force_n[2] + 9.81 * rep.total_mass_kg) <= 1.0e-9
    assert rep.primary_mean_velocity_mps[2] < 0.0


ALL_CASES = [case_equal_biaxial, case_area_preserving_gradient, case_degenerate_triangle, case_rest_sphere,
             case_translation_invariant_stretch, lambda make: case_translation_invariant_stretch(make, oob=True),
             case_region_mean_excludes_oob, case_oob_no_clamped_deposit, case_oob_reentry, case_pressure_expands,
             case_body_acceleration]
CASE_IDS = ["equal_biaxial", "area_preserving_gradient", "degenerate_triangle", "rest_sphere",
            "translation_invariant_stretch", "translation_invariant_stretch_oob", "region_mean_excludes_oob",
            "oob_no_clamped_deposit", "oob_reentry", "pressure_expands", "body_acceleration"]


def plate_mesh(nu: int = 40, nv: int = 30, size=(0.4, 0.3)):
    """Plate of 2 nu nv triangles with regions 1 / 2 / 3 (clamped root)."""
    return make_plate_mesh(nu, nv, size)
