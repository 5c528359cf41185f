"""Triangle Mooney membrane MPM on the GPU (csrc/efsi_shell.cu through the
drop-in TriMooneyShellMpmState) against the reference's known answers and the
FP64 oracle (oracle/oracle_shell.py).

Bounds: the kernels store f32 like the reference and evaluate the face law
in f64; the oracle computes in f64 and rounds the state to f32 where the
reference stores it.  The plate starts from a 5% equal-biaxial pre-stretch:
near rest the membrane strains of a pressurised plate (about 1e-6) sit below
the f32 resolution of its positions (about 1e-7 of 0.4 m), and the force of
the reference itself is then rounding noise.  After 20 steps the
displacement u agrees with the oracle to a relative L2 error of 1e-5, the
velocity v to 2e-5 and the membrane force to 5e-4 (one f32 unit of a vertex
position moves a face force by about 6e-5 of its value; the f32 atomics sum
in a run-to-run order); normals and area weights to 1e-5.  Measured on a
B200: u 1.1e-6, v 2.2e-6, membrane force 4.6e-5, external force 5.5e-7,
normals 1.4e-7, area weights 3.4e-7."""

import numpy as np
import pytest
import torch

import shell_cases as sc

pytestmark = pytest.mark.gpu


def _make(mesh, **kw):
    from easyfsi_b200.mooney_shell_mpm import TriMooneyShellMpmState

    return TriMooneyShellMpmState(mesh, **kw)


def _rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


PLATE_LAW = dict(thickness_m=2.0e-3, density_kgm3=1000.0, c1_pa=1.0e5, c2_pa=2.0e4, grid_nodes=(36, 36, 36),
                 primary_region_id=1, secondary_region_id=2, fixed_region_id=3)


@pytest.mark.parametrize("case", sc.ALL_CASES, ids=sc.CASE_IDS)
def test_shell_known_answers_on_gpu(case):
    case(_make)
    torch.cuda.synchronize()


def test_shell_step_matches_oracle_over_20_steps():
    mesh, region = sc.plate_mesh(40, 30)
    gpu = _make(mesh, face_region_id=region, **PLATE_LAW)
    ref = sc.OracleShellAdapter(mesh, face_region_id=region, **PLATE_LAW)
    np.testing.assert_allclose(gpu.mass_kg.to_numpy(), ref.o.mass, rtol=1e-5)
    # 5% equal-biaxial pre-stretch: strains well above the f32 resolution of the positions
    pre = (mesh.vertices * np.array([1.05, 1.05, 1.0])).astype(np.float32)
    gpu.x.from_numpy(pre)
    ref.x.from_numpy(pre)
    assert gpu.fixed_particle.to_numpy().tolist() == ref.o.fixed.tolist()
    assert gpu.vertex_region_id.to_numpy().tolist() == ref.o.vregion.tolist()
    for _ in range(20):
        rg = gpu.step(dt_s=1.0e-4, pressure_pa=50.0, body_acceleration_mps2=(0.0, 0.0, -9.81))
        rr = ref.step(dt_s=1.0e-4, pressure_pa=50.0, body_acceleration_mps2=(0.0, 0.0, -9.81))
    assert np.linalg.norm(ref.o.u) > 1e-6
    errors = {name: _rel(getattr(gpu, name).to_numpy(), getattr(ref.o, attr)) for name, attr in (
        ("u", "u"), ("v", "v"), ("internal_force_n", "fint"), ("external_force_n", "fext"),
        ("surface_normal", "normal"), ("area_weight_m2", "area_w"))}
    print("membrane step vs oracle after 20 steps (relative L2):", errors)
    assert _rel(gpu.u.to_numpy(), ref.o.u) <= 1e-5
    assert _rel(gpu.v.to_numpy(), ref.o.v) <= 2e-5
    assert _rel(gpu.internal_force_n.to_numpy(), ref.o.fint) <= 5e-4
    assert _rel(gpu.external_force_n.to_numpy(), ref.o.fext) <= 5e-6
    assert _rel(gpu.surface_normal.to_numpy(), ref.o.normal) <= 1e-5
    assert _rel(gpu.area_weight_m2.to_numpy(), ref.o.area_w) <= 1e-5
    fixed = ref.o.fixed != 0
    assert np.array_equal(gpu.x.to_numpy()[fixed], mesh.vertices.astype(np.float32)[fixed])
    assert rg.grid_out_of_bounds_particle_count == rr.grid_out_of_bounds_particle_count == 0
    assert abs(rg.active_grid_nodes - rr.active_grid_nodes) <= 2
    assert rg.total_mass_kg == pytest.approx(rr.total_mass_kg, rel=1e-6)
    assert rg.total_area_m2 == pytest.approx(rr.total_area_m2, rel=1e-6)
    assert rg.mean_radial_stretch == pytest.approx(rr.mean_radial_stretch, abs=1e-6)
    assert rg.max_speed_mps == pytest.approx(rr.max_speed_mps, rel=1e-4)
    assert rg.max_edge_strain == pytest.approx(rr.max_edge_strain, abs=1e-6)
    assert _rel(rg.total_force_n, rr.total_force_n) <= 1e-5
    assert _rel(rg.particle_momentum_kg_mps, rr.particle_momentum_kg_mps) <= 1e-4
    assert _rel(rg.grid_momentum_kg_mps, rr.grid_momentum_kg_mps) <= 1e-4
    assert _rel(rg.primary_mean_displacement_m, rr.primary_mean_displacement_m) <= 1e-4
    assert _rel(rg.secondary_mean_velocity_mps, rr.secondary_mean_velocity_mps) <= 1e-4
    assert rg.transfer_relative_error < 1e-4 and rr.transfer_relative_error < 1e-9


def test_shell_region_loads_match_oracle():
    mesh, region = sc.plate_mesh(24, 18)
    gpu = _make(mesh, face_region_id=region, primary_thickness_m=3.0e-3, **PLATE_LAW)
    ref = sc.OracleShellAdapter(mesh, face_region_id=region, primary_thickness_m=3.0e-3, **PLATE_LAW)
    pre = (mesh.vertices * np.array([1.05, 1.05, 1.0])).astype(np.float32)
    gpu.x.from_numpy(pre)
    ref.x.from_numpy(pre)
    args = dict(dt_s=1.0e-4, primary_region_id=1, secondary_region_id=2, primary_area_load_npm2=(0.0, 0.0, 100.0),
                primary_interface_reaction_n=(1.0, 0.0, 2.0), secondary_interface_reaction_n=(0.0, -1.0, 0.5))
    for _ in range(10):
        gpu.advance_region_loads(**args)
        ref.advance_region_loads(**args)
    gpu.add_region_area_load(region_id=2, area_load_npm2=(0.0, 0.0, -50.0))
    ref.add_region_area_load(region_id=2, area_load_npm2=(0.0, 0.0, -50.0))
    for _ in range(10):
        rg = gpu.advance_with_external_forces(dt_s=1.0e-4, primary_region_id=1, secondary_region_id=2)
        rr = ref.advance_with_external_forces(dt_s=1.0e-4, primary_region_id=1, secondary_region_id=2)
    print("membrane region loads vs oracle (relative L2):", {
        "u": _rel(gpu.u.to_numpy(), ref.o.u), "v": _rel(gpu.v.to_numpy(), ref.o.v),
        "external_force_n": _rel(gpu.external_force_n.to_numpy(), ref.o.fext)})
    assert _rel(gpu.u.to_numpy(), ref.o.u) <= 1e-5
    assert _rel(gpu.v.to_numpy(), ref.o.v) <= 2e-5
    assert _rel(gpu.external_force_n.to_numpy(), ref.o.fext) <= 1e-6
    assert _rel(rg.primary_mean_velocity_mps, rr.primary_mean_velocity_mps) <= 1e-4
    assert _rel(rg.total_force_n, rr.total_force_n) <= 1e-5


def test_shell_save_restore_and_skip_report():
    # reference tests/test_mooney_shell_mpm.py:1051-1092 and 1337-1396
    mesh, region = sc.plate_mesh(8, 6)
    st = _make(mesh, face_region_id=region, **PLATE_LAW)
    st.step(dt_s=1.0e-4, pressure_pa=50.0)
    st.save_state()
    x0, u0, v0, n0 = (f.to_numpy() for f in (st.x, st.u, st.v, st.surface_normal))
    assert st.step(dt_s=1.0e-4, pressure_pa=50.0, read_report=False) is None
    assert st.last_report_host_reads == 0
    assert not np.array_equal(st.x.to_numpy(), x0)
    st.restore_state()
    for f, want in ((st.x, x0), (st.u, u0), (st.v, v0)):
        assert np.array_equal(f.to_numpy(), want)
    np.testing.assert_allclose(st.surface_normal.to_numpy(), n0, atol=1e-6)
    assert not st.internal_force_n.to_numpy().any() and not st.external_force_n.to_numpy().any()


def test_shell_argument_errors():
    # reference tests/test_mooney_shell_mpm.py:1305-1335, 1626-1670 and the constructor checks
    with pytest.raises(ValueError, match="flip_blend"):
        _make(sc.TRI, grid_nodes=(8, 8, 8), **sc.LAW).step(dt_s=0.0, pressure_pa=0.0, flip_blend=1.5)
    with pytest.raises(ValueError, match="Mooney constants"):
        _make(sc.TRI, grid_nodes=(8, 8, 8), **dict(sc.LAW, c1_pa=0.0))
    with pytest.raises(ValueError, match="grid_nodes"):
        _make(sc.TRI, grid_nodes=(3, 8, 8), **sc.LAW)
    with pytest.raises(ValueError, match="face_region_id"):
        _make(sc.TRI, grid_nodes=(8, 8, 8), face_region_id=np.zeros(2, np.int32), **sc.LAW)
    st = _make(sc.TRI, grid_nodes=(8, 8, 8), **sc.LAW)
    st.x.from_numpy(np.full((3, 3), 1.0e3, np.float32))
    with pytest.raises(RuntimeError, match="outside the background grid"):
        st.step(dt_s=0.0, pressure_pa=0.0)


def test_marker_forces_drive_the_membrane_as_the_coupled_runner_does():
    """The sharp coupling of the membrane solid (cases/squid_soft_robot.py:8113-8135):
    marker forces F = t A cleared and scattered onto the vertices
    (hibm_mpm.py:4861-5010), then advance_with_external_forces, five times, on
    the GPU and on the oracles.  Bounds as for the plain step."""
    from types import SimpleNamespace

    from easyfsi_b200.hibm_mpm import HibmMpmSurfaceMarkers
    from oracle.oracle import OracleMarkers

    mesh, region = sc.plate_mesh(24, 18)
    gpu = _make(mesh, face_region_id=region, **PLATE_LAW)
    ref = sc.OracleShellAdapter(mesh, face_region_id=region, **PLATE_LAW)
    pre = (mesh.vertices * np.array([1.05, 1.05, 1.0])).astype(np.float32)
    gpu.x.from_numpy(pre)
    ref.x.from_numpy(pre)
    # one marker per face at the rest centroid, normal +z, seeded pressure tractions
    v = mesh.vertices.astype(np.float32)
    tri = v[mesh.faces]
    mx = tri.mean(axis=1).astype(np.float32)
    area = (0.5 * np.linalg.norm(np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]), axis=1)).astype(np.float32)
    normal = np.tile(np.array([0.0, 0.0, 1.0], np.float32), (len(mx), 1))
    p = 40.0 + 10.0 * np.random.default_rng(4002).standard_normal(len(mx))
    traction = -p[:, None] * normal.astype(np.float64)
    radius = 0.03
    markers = HibmMpmSurfaceMarkers(marker_capacity=len(mx))
    markers.load_markers(positions_m=mx, velocities_mps=np.zeros_like(mx), normals=normal, areas_m2=area,
                         region_ids=np.full(len(mx), 7, np.int32))
    markers.set_marker_tractions_pa(traction)
    markers.compute_marker_forces()
    om = OracleMarkers(x=mx, normal=normal, area=area, region=np.full(len(mx), 7, np.int32))
    om.t[:] = traction
    om.compute_forces()
    for _ in range(5):
        markers.clear_mpm_external_forces(gpu.external_force_n, particle_count=gpu.particle_count, read_report=False)
        markers.scatter_marker_forces_to_mpm_particles(gpu.external_force_n, gpu.x, particle_count=gpu.particle_count,
                                                       support_radius_m=radius, read_report=False)
        gpu.advance_with_external_forces(dt_s=1.0e-4, primary_region_id=1, secondary_region_id=2, read_report=False)
        solid = SimpleNamespace(count=ref.o.np_, x=ref.o.x.astype(np.float32),
                                fext=np.zeros((ref.o.np_, 3), np.float32))
        om.scatter(solid, radius)
        ref.o.fext = solid.fext.astype(np.float64)
        ref.advance_with_external_forces(dt_s=1.0e-4, primary_region_id=1, secondary_region_id=2)
    errors = {"u": _rel(gpu.u.to_numpy(), ref.o.u), "v": _rel(gpu.v.to_numpy(), ref.o.v),
              "external_force_n": _rel(gpu.external_force_n.to_numpy(), ref.o.fext)}
    print("membrane driven by marker forces vs oracles (relative L2):", errors)
    assert np.linalg.norm(ref.o.fext) > 0.0
    assert errors["u"] <= 1e-5 and errors["v"] <= 2e-5 and errors["external_force_n"] <= 1e-5
