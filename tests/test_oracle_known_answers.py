"""The reference's own known-answer cases, restated against the CPU oracle.

Each case names the reference test it restates (tests/<file>:<line> in the
reference tree) and keeps that test's inputs and bounds; where the oracle is
exact in f64 the bound is tightened beside the reference's.  These pin the
oracle before it is used as the GPU path's checker.
"""

import math

import numpy as np
import pytest

from easyfsi_b200.grid import CartesianGrid
from easyfsi_b200.scenarios import graded_axis_widths
from oracle import oracle as orc


def _uniform_box(n):
    w = [1.0 / n] * n
    return CartesianGrid(bounds_min_m=(0.0, 0.0, 0.0), cell_widths_x_m=w, cell_widths_y_m=w, cell_widths_z_m=w)


def _fluid(grid, variant="mirror"):
    return orc.OracleFluid(grid, rho=1000.0, mu=1.0e-3, variant=variant)


# test_core_fluid.py:1677 interface diagonal enters operator, diagonal and Jacobi
def test_interface_diagonal_enters_operator_and_jacobi():
    fl = _fluid(_uniform_box(5))
    p = np.ones((5, 5, 5))
    iface = np.zeros((5, 5, 5))
    iface[2, 2, 2] = 7.5
    applied = fl.fv_apply(p, 0, iface=iface)
    diag = fl.fv_diagonal(0, iface=iface)
    base = 6.0 / (0.2 * 0.2)
    assert applied[2, 2, 2] == pytest.approx(7.5, abs=1e-5)
    assert diag[2, 2, 2] == pytest.approx(base + 7.5, abs=3e-5)
    # Jacobi preconditioner z = r / D (fluid.py:4503-4516)
    assert 15.0 / diag[2, 2, 2] == pytest.approx(15.0 / (base + 7.5), abs=1e-6)
    # rows away from the interface: A 1 = 0 on a closed box
    assert np.abs(applied[np.arange(5) != 2]).max() < 1e-9


# test_core_fluid.py:1206 restriction volume-averages the interface diagonal
def test_restriction_volume_averages_interface_diagonal():
    fl = _fluid(_uniform_box(8))
    iface = np.zeros((8, 8, 8))
    iface[2, 2, 2] = 80.0
    out = fl.restrict(np.zeros((8, 8, 8)), iface=iface)
    assert float(out["iface"][1, 1, 1]) == pytest.approx(10.0, abs=1e-5)
    assert float(out["iface"][0, 0, 0]) == pytest.approx(0.0, abs=1e-6)


# test_core_fluid.py:1166 mixed obstacle blocks are blocked on the coarse level
def test_restriction_marks_mixed_obstacle_blocks_blocked():
    fl = _fluid(_uniform_box(8))
    fl.obstacle[1, 1, 1] = 1
    va = np.zeros((8, 8, 8), np.int32)
    va[2, 2, 2] = 1
    vw = np.full((8, 8, 8), 0.5, np.float32)
    out = fl.restrict(np.zeros((8, 8, 8)), vdir_active=va, vdir_weight=vw)
    assert int(out["obstacle"][0, 0, 0]) == 1
    assert int(out["vdir_active"][1, 1, 1]) == 1
    assert int(out["obstacle"].sum()) == 1


# test_core_fluid.py:1242 the coarse smoother reads the coarse interface diagonal
def test_coarse_smoother_uses_the_coarse_interface_diagonal():
    fl = _fluid(_uniform_box(8))
    iface = np.zeros((8, 8, 8))
    iface[1, 1, 1] = 1.0e8
    coarse = fl.restrict(np.zeros((8, 8, 8)), iface=iface)
    rhs = np.zeros((4, 4, 4), np.float32)
    rhs[1, 1, 1] = 1.0
    p = fl.jacobi_sweep_coarse(1, np.zeros((4, 4, 4)), rhs, coarse["iface"], coarse["obstacle"], omega=1.0)
    assert float(p[1, 1, 1]) < -1.0e-3
    assert float(coarse["iface"][0, 0, 0]) == pytest.approx(1.0e8 / 8.0, rel=1e-6)


def _graded_obstacle_grid():
    grid = CartesianGrid(
        bounds_min_m=(0.0, 0.0, 0.0),
        cell_widths_x_m=graded_axis_widths(16, 0.0, 1.0, 0.3, 0.7),
        cell_widths_y_m=graded_axis_widths(14, 0.0, 1.0, 0.3, 0.7),
        cell_widths_z_m=graded_axis_widths(20, 0.0, 1.0, 0.2, 0.8),
    )
    obs = np.zeros(grid.grid_nodes, np.int32)
    obs[6:10, 5:9, 8:13] = 1
    return grid, obs


# test_core_fluid.py:1648 the weighted operator is self-adjoint on a graded obstacle grid
@pytest.mark.parametrize("outlet", [0, 1])
def test_operator_is_self_adjoint_on_graded_obstacle_grid(outlet):
    grid, obs = _graded_obstacle_grid()
    fl = _fluid(grid, variant="fp64")
    fl.obstacle[...] = obs
    rng = np.random.default_rng(17)
    x = rng.normal(size=grid.grid_nodes).astype(np.float32).astype(np.float64)
    y = rng.normal(size=grid.grid_nodes).astype(np.float32).astype(np.float64)
    x[obs == 1] = 0.0
    y[obs == 1] = 0.0
    lhs = fl.weighted_dot(fl.fv_apply(x, outlet), y)
    rhs = fl.weighted_dot(x, fl.fv_apply(y, outlet))
    rel = abs(lhs - rhs) / max(abs(lhs), abs(rhs), 1e-30)
    assert rel < 1.0e-5  # the reference's bound
    assert rel < 1.0e-12  # exact in f64


# test_core_fluid.py:1377 monotone Richardson convergence on a non-uniform grid
def test_nonuniform_operator_converges_monotonically():
    errors = []
    for n in (12, 18, 24):
        q = (np.arange(n, dtype=np.float64) + 0.5) / n
        raw = 1.0 + 0.3 * np.sin(2.0 * np.pi * q)
        widths = tuple(float(v) for v in raw / raw.sum())
        grid = CartesianGrid(bounds_min_m=(0.0, 0.0, 0.0), cell_widths_x_m=widths, cell_widths_y_m=widths,
                             cell_widths_z_m=widths)
        fl = _fluid(grid)
        c = [np.asarray(a, np.float64) for a in (grid.cell_centers_x_m, grid.cell_centers_y_m, grid.cell_centers_z_m)]
        p = (np.sin(np.pi * c[0])[:, None, None] * np.sin(np.pi * c[1])[None, :, None]
             * np.sin(np.pi * c[2])[None, None, :]).astype(np.float32)
        expected = 3.0 * np.pi * np.pi * p.astype(np.float64)
        applied = fl.fv_apply(p.astype(np.float64), 0)
        inner = (slice(2, -2),) * 3
        err = applied[inner] - expected[inner]
        errors.append(float(np.sqrt(np.mean(err * err)) / np.sqrt(np.mean(expected[inner] ** 2))))
    assert errors[1] < errors[0]
    assert errors[2] < errors[1]
    assert errors[2] < 4.0e-3


def _box_particles(counts, lo, hi, density):
    nxp, nyp, nzp = counts
    n = nxp * nyp * nzp
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    p = np.arange(n)
    idx = np.stack([p % nxp, (p // nxp) % nyp, p // (nxp * nyp)], axis=1).astype(np.float32)
    x = (lo + (idx + np.float32(0.5)) * (hi - lo) / np.asarray(counts, np.float32)).astype(np.float32)
    vol = np.float32(np.prod(hi - lo) / n)
    return x, np.full(n, vol, np.float32), np.full(n, np.float32(density) * vol, np.float32)


# test_neo_hookean_mpm.py:102 a uniform velocity transfers conservatively, J stays 1
@pytest.mark.parametrize("variant", ["mirror", "fp64"])
def test_uniform_velocity_transfer_is_conservative(variant):
    x, vol, mass = _box_particles((4, 4, 4), (-0.005,) * 3, (0.005,) * 3, 1100.0)
    s = orc.OracleSolid(capacity=64, grid_nodes=(12, 12, 12), bounds_min=(-0.02,) * 3, bounds_max=(0.02,) * 3,
                        variant=variant)
    s.load(x=x, volume=vol, mass=mass, region=np.full(64, 101, np.int32))
    s.v[:64] = (0.02, -0.01, 0.03)
    e, nu = 1.0e5, 0.45
    mu, lam = e / (2 * (1 + nu)), e * nu / ((1 + nu) * (1 - 2 * nu))
    rep = s.step(dt=1.0e-5, mu=mu, lam=lam)
    assert rep.counts[0] > 0  # active grid nodes
    assert rep.values[11] < 2.0e-5  # transfer relative error
    assert rep.values[13] == pytest.approx(1.0, abs=1e-4)  # max |J|
    assert rep.values[0] > 0.0  # total mass


# test_neo_hookean_mpm.py:38 surface area and normal follow F (Nanson)
def test_surface_geometry_follows_the_deformation_gradient():
    s = orc.OracleSolid(capacity=1, grid_nodes=(12, 12, 12), bounds_min=(-1.0,) * 3, bounds_max=(1.0,) * 3)
    s.load(x=np.array([[1.0 / 3.0, 1.0 / 3.0, 0.0]], np.float32), volume=np.array([1.0e-3], np.float32),
           mass=np.array([1.0], np.float32), region=np.array([1], np.int32),
           normal=np.array([[0.0, 0.0, 1.0]], np.float32), area=np.array([0.5], np.float32))
    s.F[0] = np.array([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.5, 0.0, 1.0]], np.float32)
    s.step(dt=0.0, mu=0.0, lam=0.0, primary=1, secondary=2)
    expected = np.array([-0.5, 0.0, 1.0]) / math.sqrt(1.25)
    assert float(s.area[0]) == pytest.approx(0.5 * math.sqrt(1.25), abs=1e-5)
    np.testing.assert_allclose(s.normal[0], expected, atol=1e-5)


def _one_marker(position, traction, normal, area):
    m = orc.OracleMarkers(x=np.array([position], np.float32), normal=np.array([normal], np.float32),
                          area=np.array([area], np.float32), region=np.array([101], np.int32))
    m.t[0] = traction
    m.compute_forces()
    return m


# test_hibm.py:605 a marker over one particle hands it its whole force
def test_scatter_gives_the_single_particle_the_marker_force():
    m = _one_marker((0.5, 0.5, 0.5), (2.0, -4.0, 6.0), (1.0, 0.0, 0.0), 0.5)
    x, vol, mass = _box_particles((1, 1, 1), (0.0,) * 3, (1.0,) * 3, 1000.0)
    s = orc.OracleSolid(capacity=1, grid_nodes=(4, 4, 4))
    s.load(x=x, volume=vol, mass=mass)
    rep = m.scatter(s, 0.25)
    assert rep.active_markers == 1 and rep.invalid_markers == 0 and rep.active_particle_contributions == 1
    assert tuple(s.fext[0]) == (1.0, -2.0, 3.0)
    assert tuple(rep.marker_force) == (1.0, -2.0, 3.0)
    assert tuple(rep.external_force) == (1.0, -2.0, 3.0)


# test_hibm.py:645 the force is partitioned across the supported particles
def test_scatter_partitions_force_across_supported_particles():
    m = _one_marker((0.5, 0.5, 0.5), (0.0, 0.0, 4.0), (0.0, 0.0, 1.0), 1.0)
    x, vol, mass = _box_particles((2, 1, 1), (0.25, 0.0, 0.0), (0.75, 1.0, 1.0), 1000.0)
    s = orc.OracleSolid(capacity=2, grid_nodes=(4, 4, 4))
    s.load(x=x, volume=vol, mass=mass)
    rep = m.scatter(s, 0.4)
    assert rep.active_markers == 1 and rep.active_particle_contributions == 2
    assert float(s.fext[0, 2]) == pytest.approx(2.0, abs=1e-5)
    assert float(s.fext[1, 2]) == pytest.approx(2.0, abs=1e-5)
    assert rep.external_force[2] == pytest.approx(4.0, abs=1e-5)
    assert rep.external_force[2] - rep.marker_force[2] == pytest.approx(0.0, abs=1e-5)


# test_hibm.py:684 clear-then-scatter replaces a stale external force
def test_clear_then_scatter_replaces_stale_force():
    m = _one_marker((0.5, 0.5, 0.5), (2.0, -4.0, 6.0), (1.0, 0.0, 0.0), 0.5)
    x, vol, mass = _box_particles((1, 1, 1), (0.0,) * 3, (1.0,) * 3, 1000.0)
    s = orc.OracleSolid(capacity=1, grid_nodes=(4, 4, 4))
    s.load(x=x, volume=vol, mass=mass)
    s.fext[0] = (99.0, 0.0, 0.0)
    cleared, largest = m.clear(s)
    assert cleared == 1 and largest == pytest.approx(99.0)
    m.scatter(s, 0.25)
    assert tuple(s.fext[0]) == (1.0, -2.0, 3.0)


# --------------------------------------------------------------------------
# IB node search and classification (hibm_mpm.py:5385-6220), the reference's
# HibmMpmIbNodeSearchTests (tests/test_hibm.py:903-1297) on the oracle.
# --------------------------------------------------------------------------
def _default_sign_tolerance(bmin, bmax, nodes):
    """hibm_mpm.py:5477-5492 for a search box."""
    spacing = [(hi - lo) / n for lo, hi, n in zip(bmin, bmax, nodes)]
    min_spacing = max(min(spacing), 1.0e-12)
    max_extent = max(hi - lo for lo, hi in zip(bmin, bmax))
    max_coord = max(max(abs(v) for v in bmin), max(abs(v) for v in bmax))
    scale = max(max_extent, max_coord, min_spacing, 1.0)
    return max(1.0e-12, 1.0e-6 * min_spacing, 2.0 * 1.1920928955078125e-7 * scale)


def _search(nodes, x, n, *, radius, probe, tol=None, far=False, triangles=None, centers=None,
            bmin=(0.0, 0.0, 0.0), bmax=(1.0, 1.0, 1.0)):
    spacing = [(hi - lo) / k for lo, hi, k in zip(bmin, bmax, nodes)]
    nn = np.asarray(n, np.float64)
    nn = nn / np.linalg.norm(nn, axis=1, keepdims=True)  # load_markers normalises (hibm_mpm.py:553)
    return orc.ib_node_search(
        grid_nodes=nodes, markers_x=np.asarray(x, np.float64), markers_n=nn, triangles=triangles,
        search_radius=radius, interior_probe_distance=probe,
        sign_tolerance=_default_sign_tolerance(bmin, bmax, nodes) if tol is None else tol, classify_far=far,
        centers=centers, bounds_min=bmin, spacing=spacing)


def _report(r, near, ext, internal, invalid=None):
    rep = r["report"]
    assert rep["near_boundary_node_count"] == near
    assert rep["external_ib_node_count"] == ext
    assert rep["internal_node_count"] == internal
    if invalid is not None:
        assert rep["invalid_projection_count"] == invalid


# test_hibm.py:904 plane search classifies external and internal nodes
def test_ib_search_plane_classifies_external_and_internal_nodes():
    r = _search((1, 1, 4), [(0.5, 0.5, 0.5)], [(0.0, 0.0, 1.0)], radius=0.26, probe=0.125)
    _report(r, 2, 1, 1, 0)
    assert r["kind"][0, 0, 2] == 1 and r["kind"][0, 0, 1] == 2
    assert r["nearest_marker"][0, 0, 2] == 0 and r["nearest_marker"][0, 0, 1] == 0
    assert tuple(r["boundary_point"][0, 0, 2]) == (0.5, 0.5, 0.5)
    assert tuple(r["interior_point"][0, 0, 2]) == (0.5, 0.5, 0.75)
    assert r["signed_distance"][0, 0, 2] > 0.0 and r["signed_distance"][0, 0, 1] < 0.0


# test_hibm.py:939 triangle projection finds the closest surface point between markers
def test_ib_search_triangle_projection_between_markers():
    x = [(0.25, 0.25, 0.5), (0.75, 0.25, 0.5), (0.25, 0.75, 0.5)]
    r = _search((8, 8, 8), x, [(0.0, 0.0, 1.0)] * 3, triangles=[(0, 1, 2)], radius=0.08, probe=0.05)
    assert r["report"]["near_boundary_node_count"] >= 1 and r["report"]["external_ib_node_count"] >= 1
    assert r["kind"][2, 2, 4] == 1
    np.testing.assert_allclose(r["boundary_point"][2, 2, 4], (0.3125, 0.3125, 0.5), atol=1e-6)
    assert r["signed_distance"][2, 2, 4] == pytest.approx(0.0625)
    np.testing.assert_allclose(r["interior_point"][2, 2, 4], (0.3125, 0.3125, 0.6125), atol=1e-6)


_CLOSED_X = [(0.25, 0.5, 0.5), (0.75, 0.5, 0.5), (0.5, 0.25, 0.5), (0.5, 0.75, 0.5), (0.5, 0.5, 0.25), (0.5, 0.5, 0.75)]
_CLOSED_N = [(-1.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, -1.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, -1.0), (0.0, 0.0, 1.0)]


# test_hibm.py:987 closed surface search classifies deep internal nodes
def test_ib_search_closed_surface_deep_internal_node():
    r = _search((1, 1, 1), _CLOSED_X, _CLOSED_N, radius=0.1, probe=0.125, far=True)
    _report(r, 0, 0, 1)
    assert r["kind"][0, 0, 0] == 2 and r["nearest_marker"][0, 0, 0] >= 0


# test_hibm.py:1030 closed surface grid-field search classifies deep internal nodes
def test_ib_search_closed_surface_grid_fields_deep_internal_nodes():
    grid = _uniform_box(4)
    centers = (grid.cell_centers_x_m, grid.cell_centers_y_m, grid.cell_centers_z_m)
    r = _search((4, 4, 4), _CLOSED_X, _CLOSED_N, radius=0.08, probe=0.125, far=True, centers=centers)
    assert r["report"]["near_boundary_node_count"] == 0 and r["report"]["internal_node_count"] == 8
    assert r["kind"][1, 1, 1] == 2 and r["kind"][2, 2, 2] == 2 and r["kind"][0, 0, 0] == 0


# test_hibm.py:1088 default sign tolerance flags f32-scale ambiguous nodes
def test_ib_search_default_sign_tolerance_flags_ambiguous_node():
    r = _search((1, 1, 1), [(0.5, 0.5, 0.5 - 5.0e-8)], [(0.0, 0.0, 1.0)], radius=0.01, probe=0.125)
    assert r["report"]["near_boundary_node_count"] == 1 and r["report"]["invalid_projection_count"] == 1
    assert r["kind"][0, 0, 0] == 2 and r["signed_distance"][0, 0, 0] > 0.0


# test_hibm.py:1115 search uses non-uniform fluid cell-centre fields
def test_ib_search_nonuniform_cell_centres():
    grid = CartesianGrid(bounds_min_m=(0.0, 0.0, 0.0), cell_widths_x_m=(0.25,) * 4, cell_widths_y_m=(0.25,) * 4,
                         cell_widths_z_m=(0.1, 0.1, 0.2, 0.6))
    centers = (grid.cell_centers_x_m, grid.cell_centers_y_m, grid.cell_centers_z_m)
    r = _search((4, 4, 4), [(0.625, 0.625, 0.28)], [(0.0, 0.0, 1.0)], radius=0.04, probe=0.05, centers=centers)
    _report(r, 1, 1, 0)
    assert r["kind"][2, 2, 2] == 1 and r["kind"][2, 2, 1] == 0
    assert r["signed_distance"][2, 2, 2] == pytest.approx(0.02, abs=1e-6)
    np.testing.assert_allclose(r["boundary_point"][2, 2, 2], (0.625, 0.625, 0.28), atol=1e-6)
    assert r["interior_point"][2, 2, 2][2] == pytest.approx(0.35, abs=1e-6)


# test_hibm.py:1174 a node is external if any local normal sees it outside
def test_ib_search_external_if_any_local_normal_is_positive():
    r = _search((1, 1, 1), [(0.5, 0.5, 0.55), (0.5, 0.5, 0.45)], [(0.0, 0.0, -1.0), (0.0, 0.0, 1.0)],
                radius=0.08, probe=0.05)
    _report(r, 1, 1, 0)
    assert r["kind"][0, 0, 0] == 1


# test_hibm.py:1201 external search stores the external projection candidate
def test_ib_search_stores_the_external_candidate():
    r = _search((1, 1, 1), [(0.5, 0.5, 0.49), (0.5, 0.5, 0.46)], [(0.0, 0.0, -1.0), (0.0, 0.0, 1.0)],
                radius=0.05, probe=0.05, tol=1.0e-8)
    _report(r, 1, 1, 0)
    assert r["kind"][0, 0, 0] == 1 and r["nearest_marker"][0, 0, 0] == 1
    assert r["signed_distance"][0, 0, 0] > 0.0
    assert r["boundary_point"][0, 0, 0][2] == pytest.approx(0.46, abs=1e-6)
    assert r["interior_point"][0, 0, 0][2] > 0.5


# test_hibm.py:1240 radial marker classifies inside and outside nodes
def test_ib_search_radial_marker_inside_and_outside():
    r = _search((4, 1, 1), [(0.75, 0.5, 0.5)], [(1.0, 0.0, 0.0)], radius=0.14, probe=0.125)
    _report(r, 2, 1, 1)
    assert r["kind"][3, 0, 0] == 1 and r["kind"][2, 0, 0] == 2
    assert r["signed_distance"][3, 0, 0] > 0.0 and r["signed_distance"][2, 0, 0] < 0.0


# test_hibm.py:1270 tangent projection fallback records the invalid count
def test_ib_search_tangent_projection_records_invalid():
    r = _search((1, 1, 1), [(0.5, 0.5, 0.5)], [(0.0, 0.0, 1.0)], radius=0.1, probe=0.125, tol=1.0e-9)
    assert r["report"]["near_boundary_node_count"] == 1 and r["report"]["invalid_projection_count"] == 1
    assert r["nearest_marker"][0, 0, 0] == 0
    assert tuple(r["boundary_point"][0, 0, 0]) == (0.5, 0.5, 0.5)
    assert tuple(r["interior_point"][0, 0, 0]) == (0.5, 0.5, 0.625)


# test_hibm.py:1301 builds external-IB no-slip and pressure-Neumann targets
# (HibmMpmIbBoundaryConditions.build_from_search, hibm_mpm.py:6499-6605)
def test_ib_boundary_targets_from_the_plane_search():
    s = _search((1, 1, 4), [(0.5, 0.5, 0.5)], [(0.0, 0.0, 2.0)], radius=0.26, probe=0.125)
    bc = orc.ib_build_boundary_conditions(s, markers_v=[(1.25, -0.5, 0.75)], markers_n=[(0.0, 0.0, 1.0)],
                                          marker_gradients=[42.0])
    rep = bc["report"]
    assert (rep["no_slip_dirichlet_count"], rep["pressure_neumann_count"], rep["inactive_internal_node_count"]) == (1, 1, 1)
    assert rep["max_abs_velocity_mps"] == pytest.approx(1.25, abs=1e-6)
    assert bc["active"][0, 0, 2] == 1 and bc["active"][0, 0, 1] == 0
    assert tuple(bc["velocity"][0, 0, 2]) == (1.25, -0.5, 0.75)
    assert tuple(bc["normal"][0, 0, 2]) == (0.0, 0.0, 1.0)
    assert bc["gradient"][0, 0, 2] == pytest.approx(42.0)


# test_hibm.py:1345 triangle projection interpolates curved-surface targets
def test_ib_boundary_targets_interpolate_over_the_projection_triangle():
    x = [(0.25, 0.25, 0.5), (0.75, 0.25, 0.5), (0.25, 0.75, 0.5)]
    eye = [(1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0)]
    s = _search((8, 8, 8), x, eye, triangles=[(0, 1, 2)], radius=0.08, probe=0.05)
    bc = orc.ib_build_boundary_conditions(s, markers_v=eye, markers_n=eye, marker_gradients=[100.0, 200.0, 300.0])
    w = np.array((0.75, 0.125, 0.125))
    assert bc["report"]["no_slip_dirichlet_count"] == bc["report"]["pressure_neumann_count"]
    assert bc["active"][2, 2, 4] == 1
    np.testing.assert_allclose(bc["velocity"][2, 2, 4], w, atol=1e-6)
    np.testing.assert_allclose(bc["normal"][2, 2, 4], w / np.linalg.norm(w), atol=1e-6)
    assert bc["gradient"][2, 2, 4] == pytest.approx(137.5, abs=1e-5)


# --------------------------------------------------------------------------
# Interface-coupling operator terms (fluid.py:4345-4456), the reference's
# tests/test_core_fluid.py:1756-1897 on the oracle.
# --------------------------------------------------------------------------
def _slots(shape):
    return [np.zeros(shape, np.int32), np.zeros(shape + (3,), np.int32), np.zeros(shape),
            np.zeros(shape + (15, 3), np.int32), np.zeros(shape + (15,))]


# test_core_fluid.py:1756 interface coupling enters the operator symmetrically
def test_interface_coupling_enters_operator_symmetrically():
    fl = _fluid(_uniform_box(5))
    p = np.ones((5, 5, 5))
    p[2, 2, 2], p[2, 2, 3] = 3.0, 1.0
    base = fl.fv_apply(p, 0)
    diag = np.zeros((5, 5, 5))
    diag[2, 2, 2] = diag[2, 2, 3] = 4.0
    slots = _slots((5, 5, 5))
    slots[0][2, 2, 2] = 1
    slots[1][2, 2, 2] = (2, 2, 3)
    slots[2][2, 2, 2] = 4.0 * 0.2 ** 3
    coupled = fl.fv_apply_coupled(p, 0, iface=diag, slots=slots)
    assert coupled[2, 2, 2] - base[2, 2, 2] == pytest.approx(8.0, abs=1e-5)
    assert coupled[2, 2, 3] - base[2, 2, 3] == pytest.approx(-8.0, abs=1e-5)
    # the same coupling as one explicit row gives the same operator
    rows = (np.array([(2, 2, 2)]), np.array([(2, 2, 3)]), np.array([4.0 * 0.2 ** 3]))
    np.testing.assert_allclose(fl.fv_apply_coupled(p, 0, iface=diag, rows=rows), coupled, rtol=0, atol=1e-12)


# test_core_fluid.py:1792 interface coupling uses the transmissibility on non-uniform cells
def test_interface_coupling_is_self_adjoint_on_nonuniform_cells():
    grid = CartesianGrid(bounds_min_m=(0.0, 0.0, 0.0), cell_widths_x_m=(0.1, 0.2, 0.35, 0.35),
                         cell_widths_y_m=(0.25,) * 4, cell_widths_z_m=(0.25,) * 4)
    fl = _fluid(grid)
    rng = np.random.default_rng(41)
    x = rng.normal(size=grid.grid_nodes).astype(np.float32).astype(np.float64)
    y = rng.normal(size=grid.grid_nodes).astype(np.float32).astype(np.float64)
    t, left, right = 0.375, (1, 2, 2), (2, 2, 2)
    diag = np.zeros(grid.grid_nodes)
    diag[left] = np.float32(t / (0.2 * 0.25 * 0.25))
    diag[right] = np.float32(t / (0.35 * 0.25 * 0.25))
    slots = _slots(grid.grid_nodes)
    slots[0][left] = 1
    slots[1][left] = right
    slots[2][left] = t
    ax = fl.fv_apply_coupled(x, 0, iface=diag, slots=slots)
    ay = fl.fv_apply_coupled(y, 0, iface=diag, slots=slots)
    lhs, rhs = fl.weighted_dot(ax, y), fl.weighted_dot(x, ay)
    assert abs(lhs - rhs) / max(abs(lhs), abs(rhs), 1e-30) < 1.0e-5


# test_core_fluid.py:1839 interface coupling applies multiple owner slots
def test_interface_coupling_applies_multiple_owner_slots():
    fl = _fluid(_uniform_box(5))
    owner, n0, n1 = (2, 2, 2), (2, 2, 3), (2, 3, 2)
    p = np.ones((5, 5, 5))
    p[owner], p[n0], p[n1] = 3.0, 1.0, 2.0
    base = fl.fv_apply(p, 0)
    v = 0.2 ** 3
    c0, c1 = 4.0 * v, 7.0 * v
    diag = np.zeros((5, 5, 5))
    diag[owner], diag[n0], diag[n1] = (c0 + c1) / v, c0 / v, c1 / v
    slots = _slots((5, 5, 5))
    slots[0][owner] = 2
    slots[1][owner] = n0
    slots[2][owner] = c0
    slots[3][owner + (0,)] = n1
    slots[4][owner + (0,)] = c1
    op = fl.fv_apply_coupled(p, 0, iface=diag, slots=slots)
    assert op[owner] - base[owner] == pytest.approx(15.0, abs=5e-5)
    assert op[n0] - base[n0] == pytest.approx(-8.0, abs=5e-5)
    assert op[n1] - base[n1] == pytest.approx(-7.0, abs=5e-5)


# --------------------------------------------------------------------------
# Velocity-Dirichlet reconstructed rows (hibm_mpm.py:6714-7800), the
# reference's tests/test_hibm.py:3337-3753 on the oracle.
# --------------------------------------------------------------------------
def _one_node_rows(node, bv, n, bp, ip, *, obstacle=None, velocity=(0.0, 0.0, 0.0)):
    grid = _uniform_box(4)
    act = np.zeros((4, 4, 4), np.int32)
    act[node] = 1
    fields = {}
    for name, value in (("bc_velocity", bv), ("bc_normal", n), ("boundary_point", bp), ("interior_point", ip)):
        a = np.zeros((4, 4, 4, 3))
        a[node] = value
        fields[name] = a
    obs = np.zeros((4, 4, 4), np.int32) if obstacle is None else obstacle
    return orc.ib_velocity_dirichlet_rows(grid, active_ib=act, obstacle=obs, velocity=velocity, **fields)


# test_hibm.py:3337 no-slip rows reconstruct along the surface normal
def test_vd_rows_reconstruct_along_the_surface_normal():
    s = _search((4, 4, 4), [(0.625, 0.625, 0.5)], [(0.0, 0.0, 1.0)], radius=0.13, probe=0.125)
    bc = orc.ib_build_boundary_conditions(s, markers_v=[(0.0, 0.0, 0.1)], markers_n=[(0.0, 0.0, 1.0)],
                                          marker_gradients=[0.0])
    r = orc.ib_velocity_dirichlet_rows(
        _uniform_box(4), active_ib=bc["active"], bc_velocity=bc["velocity"], bc_normal=bc["normal"],
        boundary_point=s["boundary_point"], interior_point=s["interior_point"], obstacle=np.zeros((4, 4, 4)),
        velocity=(0.0, 0.0, 0.4), nearest_marker=s["nearest_marker"], marker_region=[7])
    rep = r["report"]
    assert rep["active_velocity_dirichlet_rows"] == 1 and rep["invalid_reconstruction_row_count"] == 0
    assert rep["min_projection_weight"] == pytest.approx(0.5, abs=1e-6)
    assert rep["max_projection_weight"] == pytest.approx(0.5, abs=1e-6)
    assert r["active"][2, 2, 2] == 1 and r["region"][2, 2, 2] == 7
    assert r["value"][2, 2, 2][2] == pytest.approx(0.25, abs=1e-6)
    assert r["weight"][2, 2, 2] == pytest.approx(0.5, abs=1e-6)


# test_hibm.py:3411 reconstruction falls back to the nearest marker velocity
def test_vd_rows_zero_gap_falls_back_to_the_boundary_velocity():
    node = (2, 2, 2)
    r = _one_node_rows(node, (0.1, 0.0, 0.0), (1.0, 0.0, 0.0), (0.625,) * 3, (0.625,) * 3)
    rep = r["report"]
    assert rep["active_velocity_dirichlet_rows"] == 1 and rep["invalid_reconstruction_row_count"] == 1
    assert rep["invalid_no_fluid_sample_row_count"] == 0 and rep["invalid_nonpositive_gap_row_count"] == 1
    assert rep["invalid_node_behind_boundary_row_count"] == 0 and rep["invalid_node_beyond_interior_row_count"] == 0
    assert rep["min_projection_weight"] == 0.0 and rep["max_projection_weight"] == 0.0
    assert r["active"][node] == 1 and r["weight"][node] == 0.0
    np.testing.assert_allclose(r["value"][node], (0.1, 0.0, 0.0), atol=1e-7)


# test_hibm.py:3478 a masked node's row relocates to the first fluid cell
def test_vd_rows_relocate_a_masked_node_to_the_first_fluid_cell():
    obs = np.zeros((4, 4, 4), np.int32)
    obs[2, 2, 2] = 1
    r = _one_node_rows((2, 2, 2), (0.2, 0.0, 0.0), (1.0, 0.0, 0.0), (0.5, 0.625, 0.625), (0.875, 0.625, 0.625),
                       obstacle=obs)
    rep = r["report"]
    assert rep["active_velocity_dirichlet_rows"] == 1 and rep["relocated_row_count"] == 1
    assert rep["relocation_blocked_row_count"] == 0 and rep["inactive_obstacle_rows"] == 0
    assert rep["invalid_reconstruction_row_count"] == 0
    assert r["active"][2, 2, 2] == 0 and r["active"][3, 2, 2] == 1
    np.testing.assert_allclose(r["value"][3, 2, 2], (0.08, 0.0, 0.0), atol=1e-6)
    assert r["weight"][3, 2, 2] == pytest.approx(0.6, abs=1e-6)


# test_hibm.py:3540 relocation to the opposite fluid side when the normal side is solid
def test_vd_rows_relocate_to_the_opposite_side():
    obs = np.zeros((4, 4, 4), np.int32)
    obs[2:, :, :] = 1
    r = _one_node_rows((2, 2, 2), (0.2, 0.0, 0.0), (1.0, 0.0, 0.0), (0.5, 0.625, 0.625), (0.875, 0.625, 0.625),
                       obstacle=obs)
    rep = r["report"]
    assert rep["active_velocity_dirichlet_rows"] == 1 and rep["relocated_row_count"] == 1
    assert rep["relocation_blocked_row_count"] == 0
    assert r["active"][2, 2, 2] == 0 and r["active"][1, 2, 2] == 1
    np.testing.assert_allclose(r["value"][1, 2, 2], (0.13333334, 0.0, 0.0), atol=1e-7)


# test_hibm.py:3597 a wall-limited gap is a narrow-gap row
def test_vd_rows_wall_limited_gap_is_a_narrow_gap_row():
    obs = np.zeros((4, 4, 4), np.int32)
    obs[3, :, :] = 1
    node = (2, 2, 2)
    r = _one_node_rows(node, (0.3, 0.0, 0.0), (1.0, 0.0, 0.0), (0.5, 0.625, 0.625), (0.875, 0.625, 0.625),
                       obstacle=obs)
    rep = r["report"]
    assert rep["active_velocity_dirichlet_rows"] == 1 and rep["narrow_gap_boundary_velocity_row_count"] == 1
    assert rep["invalid_reconstruction_row_count"] == 0 and rep["invalid_no_fluid_sample_row_count"] == 0
    assert r["active"][node] == 1 and r["weight"][node] == 0.0
    np.testing.assert_allclose(r["value"][node], (0.3, 0.0, 0.0), atol=1e-7)


# test_hibm.py:3658 fallback for a node beyond the interior segment
def test_vd_rows_fall_back_for_a_node_beyond_the_interior_segment():
    node = (2, 2, 2)
    r = _one_node_rows(node, (0.2, 0.0, 0.0), (1.0, 0.0, 0.0), (0.25, 0.625, 0.625), (0.375, 0.625, 0.625),
                       velocity=(0.4, 0.0, 0.0))
    rep = r["report"]
    assert rep["active_velocity_dirichlet_rows"] == 1 and rep["invalid_reconstruction_row_count"] == 0
    assert r["weight"][node] > 0.0
    np.testing.assert_allclose(r["value"][node], (0.35, 0.0, 0.0), atol=1e-6)


# test_hibm.py:3718 fallback for a node behind the boundary plane
def test_vd_rows_fall_back_for_a_node_behind_the_boundary_plane():
    node = (1, 2, 2)
    r = _one_node_rows(node, (0.2, 0.0, 0.0), (1.0, 0.0, 0.0), (0.5, 0.625, 0.625), (0.625, 0.625, 0.625),
                       velocity=(0.4, 0.0, 0.0))
    rep = r["report"]
    assert rep["active_velocity_dirichlet_rows"] == 1 and rep["invalid_reconstruction_row_count"] == 0
    assert r["weight"][node] == pytest.approx(0.5, abs=1e-6)
    np.testing.assert_allclose(r["value"][node], (0.3, 0.0, 0.0), atol=1e-6)


def _ecoflex_0010():
    """hyperelastic.py:143-165 / :111-140: Ecoflex 00-10, mu from the 100 %
    modulus (8 psi) of a uniaxial neo-Hookean bar, nu = 0.49, 1040 kg/m^3."""
    mu = 8.0 * 6894.757293168361 / (2.0 - 2.0 ** -2)
    nu = 0.49
    e = 2.0 * mu * (1.0 + nu)
    k = e / (3.0 * (1.0 - 2.0 * nu))
    return 1040.0, mu, k - 2.0 * mu / 3.0


# test_neo_hookean_mpm.py:133 a non-cubic grid maps particles with its own axis spacing
def test_mpm_non_cubic_grid_uses_axis_spacing():
    rho, mu, lam = _ecoflex_0010()
    x, vol, mass = _box_particles((2, 2, 2), (-0.002, -0.002, 0.024), (0.002, 0.002, 0.030), rho)
    s = orc.OracleSolid(capacity=8, grid_nodes=(12, 12, 12), bounds_min=(-0.01, -0.01, -0.04),
                        bounds_max=(0.01, 0.01, 0.04))
    s.load(x=x, volume=vol, mass=mass, region=np.ones(8, np.int32))
    s.v[:8] = (0.0, 0.0, 0.01)
    rep = s.step(dt=1.0e-5, mu=mu, lam=lam, primary=1, secondary=2)
    assert rep.counts[0] > 0
    assert rep.values[11] < 2.0e-5
    assert rep.values[13] == pytest.approx(1.0, abs=1e-4)


# test_neo_hookean_mpm.py:163 an external force changes the grid momentum consistently
def test_mpm_external_force_changes_grid_momentum():
    rho, mu, lam = _ecoflex_0010()
    x, vol, mass = _box_particles((2, 2, 2), (-0.004,) * 3, (0.004,) * 3, rho)
    s = orc.OracleSolid(capacity=8, grid_nodes=(12, 12, 12), bounds_min=(-0.02,) * 3, bounds_max=(0.02,) * 3)
    s.load(x=x, volume=vol, mass=mass, region=np.ones(8, np.int32))
    s.fext[:8] = (0.0, 0.0, -1.0e-4)
    rep = s.step(dt=1.0e-5, mu=mu, lam=lam, primary=1, secondary=2)
    assert rep.values[10] < 0.0  # external force z
    assert rep.values[7] < 0.0  # grid momentum z
    assert rep.values[11] < 2.0e-5


# test_neo_hookean_mpm.py:411 a particle next to the boundary deposits no partial stencil
def test_mpm_near_boundary_particle_deposits_nothing():
    rho, mu, lam = _ecoflex_0010()
    x, vol, mass = _box_particles((2, 2, 2), (-0.004,) * 3, (0.004,) * 3, rho)
    dx = 0.04 / 8
    x[0, 0] = np.float32(-0.02 + 0.25 * dx)
    s = orc.OracleSolid(capacity=8, grid_nodes=(8, 8, 8), bounds_min=(-0.02,) * 3, bounds_max=(0.02,) * 3)
    s.load(x=x, volume=vol, mass=mass, region=np.ones(8, np.int32))
    rep = s.step(dt=0.0, mu=mu, lam=lam, primary=1, secondary=2)
    assert rep.counts[1] == 1  # grid out-of-bounds particles
    assert float(np.sum(s.grid_mass, dtype=np.float64)) == pytest.approx(float(np.sum(mass[1:], dtype=np.float64)),
                                                                         abs=1e-8)
    mean_stretch = rep.values[14] / rep.counts[3]
    assert math.isfinite(mean_stretch) and math.isfinite(rep.values[15])
    assert mean_stretch == pytest.approx(1.0, abs=1e-6)
    assert rep.values[15] == pytest.approx(0.0, abs=5e-6)


def _one_particle_with_f(f):
    rho, mu, lam = _ecoflex_0010()
    x, vol, mass = _box_particles((1, 1, 1), (-0.001,) * 3, (0.001,) * 3, rho)
    s = orc.OracleSolid(capacity=1, grid_nodes=(8, 8, 8), bounds_min=(-0.01,) * 3, bounds_max=(0.01,) * 3)
    s.load(x=x, volume=vol, mass=mass, region=np.ones(1, np.int32))
    s.F[0] = np.asarray(f, np.float32)
    return s, s.step(dt=0.0, mu=mu, lam=lam, primary=1, secondary=2)


# test_neo_hookean_mpm.py:543 an inverted deformation gradient triggers the SVD clamp
def test_mpm_inverted_deformation_gradient_is_clamped():
    s, rep = _one_particle_with_f([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, -1.0]])
    assert rep.counts[2] == 1  # deformation clamps
    assert rep.values[13] > 0.0 and abs(rep.values[13] - 1.0) < 1.0e-5


# test_neo_hookean_mpm.py:581 the clamp persists the corrected deformation gradient
def test_mpm_clamp_persists_the_corrected_deformation_gradient():
    s, rep = _one_particle_with_f([[-2.0, 0.0, 0.0], [0.0, 0.5, 0.0], [0.0, 0.0, 0.5]])
    corrected = np.asarray(s.F[0], np.float64).reshape(3, 3)
    assert rep.counts[2] == 1
    assert np.linalg.det(corrected) > 0.0
    sv = np.linalg.svd(corrected, compute_uv=False)
    assert sv.min() >= 1.0e-2 and sv.max() <= 1.0e2


# --------------------------------------------------------------------------
# Divergence and projection (tests/test_fluid.py:28-58 of the reference)
# --------------------------------------------------------------------------
def _divergence_stats(fl, interior_only=False):
    """fluid.py:3494-3522 / 3827-3835: max |div| and RMS over fluid cells."""
    d = np.abs(np.asarray(fl.divergence, np.float64))
    mask = fl.obstacle == 0
    if interior_only:
        inner = np.zeros_like(mask)
        inner[1:-1, 1:-1, 1:-1] = True
        mask &= inner
    vals = d[mask]
    return {"max_abs": float(vals.max(initial=0.0)), "l2": math.sqrt(float((vals * vals).sum()) / max(1, vals.size))}


def _centres(n):
    return (np.arange(n, dtype=np.float32) + np.float32(0.5)) / np.float32(n)


# test_fluid.py:28 a uniform velocity has near-zero divergence
def test_uniform_velocity_has_near_zero_divergence():
    fl = _fluid(_uniform_box(16))
    fl.velocity[...] = (0.2, -0.1, 0.05)
    fl.compute_divergence(0)
    st = _divergence_stats(fl, interior_only=True)
    assert st["max_abs"] < 1.0e-5 and st["l2"] < 1.0e-5


# test_fluid.py:37 a simple shear velocity has near-zero divergence
def test_simple_shear_velocity_has_near_zero_divergence():
    fl = _fluid(_uniform_box(21))
    y = _centres(21)
    fl.velocity[...] = 0.0
    fl.velocity[:, :, :, 0] = (np.float32(75.0) * (y - np.float32(0.5)))[None, :, None]
    fl.compute_divergence(0)
    st = _divergence_stats(fl, interior_only=True)
    assert st["max_abs"] < 1.0e-5 and st["l2"] < 1.0e-5


# test_fluid.py:46 the projection reduces the divergence (the reference's
# default legacy Jacobi solve; here the oracle's MG-PCG, which reduces it further)
def test_projection_reduces_divergence():
    n = 24
    fl = _fluid(_uniform_box(n))
    c = _centres(n)
    two_pi = np.float32(2.0 * math.pi)
    fl.velocity[..., 0] = (np.float32(0.15) * np.sin(two_pi * c))[:, None, None]
    fl.velocity[..., 1] = (np.float32(0.075) * np.sin(two_pi * c))[None, :, None]
    fl.velocity[..., 2] = (np.float32(-0.0375) * np.sin(two_pi * c))[None, None, :]
    fl.compute_divergence(0)
    before = _divergence_stats(fl)
    fl.project(dt=2.0e-3, max_iters=240, tol=1.0e-8)
    fl.compute_divergence(0)
    after = _divergence_stats(fl)
    assert before["l2"] > 0.1
    assert after["l2"] < before["l2"] * 0.45
    assert after["max_abs"] < before["max_abs"] * 0.55


def _cell_volumes(fl):
    w = [np.asarray(m["w"], np.float32).astype(np.float64) for m in fl.metrics[0]]
    return np.einsum("i,j,k->ijk", *w)


def _momentum_change(fl, before):
    """sum rho V du over the fluid cells (the impulse of the body force)."""
    du = np.asarray(fl.velocity, np.float64) - before
    return fl.rho * np.einsum("ijk,ijkc->c", _cell_volumes(fl), du)


# test_fluid.py:85 surface-force spreading conserves action and reaction on the grid
def test_surface_force_spreading_conserves_action_reaction():
    fl = _fluid(_uniform_box(32))
    pos = [(-0.02, 0.0, 0.0), (0.02, 0.0, 0.0), (0.0, -0.02, 0.0), (0.0, 0.02, 0.0)]
    forces = [(0.0, 0.0, -0.25), (0.0, 0.0, -0.5), (0.0, 0.0, -0.75), (0.0, 0.0, -1.0)]
    rep = fl.spread_surface_forces(pos, forces, center=(0.5, 0.5, 0.5), force_sign=-1.0)
    surface, grid = rep[:3], rep[3:]
    assert np.count_nonzero(np.abs(fl.force).sum(axis=-1)) > 0
    assert surface[2] == pytest.approx(-2.5, abs=1e-6)
    assert grid[2] == pytest.approx(-surface[2], abs=abs(surface[2]) * 1e-5)
    # the force densities integrate to the grid force
    np.testing.assert_allclose(np.einsum("ijk,ijkc->c", _cell_volumes(fl), fl.force), grid, rtol=1e-5, atol=1e-9)
    before = np.asarray(fl.velocity, np.float64).copy()
    fl.apply_body_force(2.5e-3)
    assert _momentum_change(fl, before)[2] == pytest.approx(grid[2] * 2.5e-3, rel=1e-5)


# test_fluid.py:139 spreading renormalises around obstacles
def test_surface_force_spreading_renormalises_around_obstacles():
    fl = _fluid(_uniform_box(8))
    fl.obstacle[3, 4, 4] = 1
    c = _centres(8)
    pos = [(0.5 * (c[3] + c[4]), c[4], c[4])]
    rep = fl.spread_surface_forces(pos, [(0.0, 0.0, -2.0)], center=(0.0, 0.0, 0.0), force_sign=-1.0)
    assert np.count_nonzero(np.abs(fl.force).sum(axis=-1)) == 1
    assert rep[5] == pytest.approx(2.0, abs=2e-5)
    before = np.asarray(fl.velocity, np.float64).copy()
    fl.apply_body_force(2.5e-3)
    assert _momentum_change(fl, before)[2] == pytest.approx(rep[5] * 2.5e-3, rel=1e-5)


# --------------------------------------------------------------------------
# FV divergence and pressure gradient next to obstacles (tests/test_core_fluid.py:1038-1146)
# --------------------------------------------------------------------------
def _fluid_with(nodes, obstacle, pressure=None, velocity=None):
    w = [[1.0 / n] * n for n in nodes]
    fl = _fluid(CartesianGrid(bounds_min_m=(0.0, 0.0, 0.0), cell_widths_x_m=w[0], cell_widths_y_m=w[1],
                              cell_widths_z_m=w[2]))
    fl.obstacle[...] = obstacle
    fl.velocity[...] = 0.0 if velocity is None else velocity
    if pressure is not None:
        fl.pressure[...] = pressure
    return fl


# test_core_fluid.py:1038 the divergence has zero flux through obstacle faces
def test_divergence_uses_zero_flux_on_obstacle_faces():
    obs = np.zeros((4, 4, 4), np.int32)
    obs[2, 1, 1] = 1
    vel = np.zeros((4, 4, 4, 3), np.float32)
    vel[1, 1, 1, 0] = 1.25
    fl = _fluid_with((4, 4, 4), obs, velocity=vel)
    fl.compute_divergence(0)
    assert float(fl.divergence[0, 1, 1]) == pytest.approx(5.0, abs=1e-6)
    assert float(fl.divergence[1, 1, 1]) == pytest.approx(-5.0, abs=1e-6)
    assert float(fl.divergence[2, 1, 1]) == pytest.approx(0.0, abs=1e-6)


# test_core_fluid.py:1057 the FV divergence is the pressure gradient's adjoint next to obstacles
def test_divergence_of_the_gradient_is_the_fv_laplacian_next_to_obstacles():
    nodes = (5, 4, 4)
    obs = np.zeros(nodes, np.int32)
    obs[3, 1:3, 1:3] = 1
    i, j, k = np.meshgrid(*[np.arange(n) for n in nodes], indexing="ij")
    p = (0.7 * i - 0.3 * j + 0.11 * k + 0.05 * i * j).astype(np.float32)
    p[obs == 1] = 0.0
    fl = _fluid_with(nodes, obs, pressure=p)
    fl.subtract_pressure_gradient(0.25)
    fl.compute_divergence(0)
    w = [np.asarray(m["w"], np.float32).astype(np.float64) for m in fl.metrics[0]]
    cd = [np.asarray(m["cd"], np.float32).astype(np.float64) for m in fl.metrics[0]]
    expected = np.zeros(nodes)
    for c in zip(*np.nonzero(obs == 0)):
        applied, centre = 0.0, float(p[c])
        for a in range(3):
            for step in (-1, 1):
                q = list(c)
                q[a] += step
                if not 0 <= q[a] < nodes[a] or obs[tuple(q)] != 0:
                    continue
                dist = cd[a][c[a]] if step < 0 else cd[a][c[a] + 1]
                applied += (float(p[tuple(q)]) - centre) / (w[a][c[a]] * dist)
        expected[c] = -0.25 * applied
    active = obs == 0
    np.testing.assert_allclose(np.asarray(fl.divergence)[active], expected[active], rtol=2e-5, atol=1e-5)


# test_core_fluid.py:1124 divergence of the gradient is globally conservative with obstacles
def test_divergence_of_the_gradient_is_globally_conservative():
    nodes = (6, 5, 4)
    obs = np.zeros(nodes, np.int32)
    obs[3, 1:4, 1:3] = 1
    i, j, k = np.meshgrid(*[np.arange(n) for n in nodes], indexing="ij")
    p = (0.17 * i * i - 0.31 * j + 0.13 * k).astype(np.float32)
    p[obs == 1] = 0.0
    fl = _fluid_with(nodes, obs, pressure=p)
    fl.subtract_pressure_gradient(0.4)
    fl.compute_divergence(0)
    cell_volume = 1.0 / (6 * 5 * 4)
    net = float(np.sum(np.asarray(fl.divergence, np.float64)[obs == 0] * cell_volume))
    assert net == pytest.approx(0.0, abs=1e-7)


# test_core_fluid.py:1353 the uniform FV Laplacian converges at second order
def test_uniform_fv_laplacian_converges_at_second_order():
    errors = []
    for n in (16, 32, 64):
        fl = _fluid(_uniform_box(n))
        c = (np.arange(n, dtype=np.float64) + 0.5) / n
        x, y, z = np.meshgrid(c, c, c, indexing="ij")
        p = np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)
        expected = -3.0 * np.pi * np.pi * p
        discrete = -fl.fv_apply(p, 0)  # the operator is -laplacian
        err = (discrete - expected)[1:-1, 1:-1, 1:-1]
        errors.append(float(np.sqrt(np.mean(err * err))))
    assert errors[1] < errors[0] * 0.30
    assert errors[2] < errors[1] * 0.30


# test_core_fluid.py:882 pressure inside an obstacle is Neumann for the projection
def test_obstacle_pressure_does_not_drive_the_fluid():
    obs = np.zeros((8, 8, 8), np.int32)
    obs[4, 4, 4] = 1
    p = np.zeros((8, 8, 8))
    p[4, 4, 4] = 1000.0
    fl = _fluid_with((8, 8, 8), obs, pressure=p)
    fl.project(dt=1.0e-3, max_iters=1)
    assert float(np.linalg.norm(np.asarray(fl.velocity, np.float64), axis=-1).max()) < 1.0e-8


# test_core_fluid.py:927 the projection solves the consistent divergence-gradient system
def test_projection_solves_the_consistent_system():
    n = 24
    fl = _fluid(_uniform_box(n))
    c = _centres(n)
    two_pi = np.float32(2.0 * math.pi)
    fl.velocity[..., 0] = (np.float32(0.15) * np.sin(two_pi * c))[:, None, None]
    fl.velocity[..., 1] = (np.float32(0.075) * np.sin(two_pi * c))[None, :, None]
    fl.velocity[..., 2] = (np.float32(-0.0375) * np.sin(two_pi * c))[None, None, :]
    fl.compute_divergence(0)
    before = _divergence_stats(fl)
    fl.project(dt=2.0e-3, max_iters=480, tol=1.0e-8)
    after = _divergence_stats(fl)
    assert before["l2"] > 0.1
    assert after["l2"] < before["l2"] * 0.05
    assert after["max_abs"] < before["max_abs"] * 0.08


def _nonuniform_fluid(wx, wy, wz):
    return _fluid(CartesianGrid(bounds_min_m=(0.0, 0.0, 0.0), cell_widths_x_m=wx, cell_widths_y_m=wy,
                                cell_widths_z_m=wz))


# test_core_fluid.py:504 the non-uniform divergence and gradient use the grid metrics
def test_nonuniform_divergence_and_gradient_use_grid_metrics():
    fl = _nonuniform_fluid((0.1, 0.2, 0.3, 0.4), (0.25,) * 4, (0.25,) * 4)
    fl.velocity[...] = 0.0
    fl.velocity[1, 1, 1, 0] = 1.0
    fl.velocity[2, 1, 1, 0] = 1.6
    fl.compute_divergence(0)
    assert float(fl.divergence[1, 1, 1]) == pytest.approx(3.0, abs=1e-6)
    fl.velocity[...] = 0.0
    fl.pressure[...] = 0.0
    fl.pressure[0, 1, 1] = 4.0
    fl.pressure[1, 1, 1] = 10.0
    fl.subtract_pressure_gradient(1.0)
    assert float(fl.velocity[1, 1, 1, 0]) == pytest.approx(-40.0, abs=1e-5)


# test_core_fluid.py:541 (body-force part) the impulse integrates over the cell volumes
def test_nonuniform_body_force_impulse_uses_cell_volumes():
    fl = _nonuniform_fluid((0.1, 0.2, 0.3, 0.4), (0.2, 0.2, 0.3, 0.3), (0.1, 0.2, 0.3, 0.4))
    fl.velocity[...] = 0.0
    fl.force = np.zeros((4, 4, 4, 3), np.float32)
    fl.force[0, 0, 0, 0] = 200.0
    fl.force[2, 1, 3, 0] = 300.0
    vol = _cell_volumes(fl)
    before = np.asarray(fl.velocity, np.float64).copy()
    fl.apply_body_force(2.0e-3)
    expected = (200.0 * vol[0, 0, 0] + 300.0 * vol[2, 1, 3]) * 2.0e-3
    assert _momentum_change(fl, before)[0] == pytest.approx(expected, abs=1e-8)


# test_core_fluid.py:593 non-uniform spreading uses the cell volumes
def test_nonuniform_spreading_uses_cell_volumes():
    fl = _nonuniform_fluid((0.1, 0.2, 0.3, 0.4), (0.2, 0.2, 0.3, 0.3), (0.1, 0.2, 0.3, 0.4))
    rep = fl.spread_surface_forces([(0.0, 0.0, 0.0)], [(1.0, -2.0, 3.0)], center=(0.05, 0.1, 0.05), force_sign=-1.0)
    assert np.count_nonzero(np.abs(fl.force).sum(axis=-1)) == 1
    np.testing.assert_allclose(rep[3:], (-1.0, 2.0, -3.0), rtol=1e-6, atol=1e-6)
    before = np.asarray(fl.velocity, np.float64).copy()
    fl.apply_body_force(1.5e-3)
    np.testing.assert_allclose(_momentum_change(fl, before), rep[3:] * 1.5e-3, rtol=1e-6, atol=1e-8)


# test_core_fluid.py:835 the closed-boundary clamp keeps the shifted MAC max faces
def test_closed_boundary_clamp_keeps_the_max_faces():
    fl = _fluid(_uniform_box(4))
    fl.velocity[...] = 0.0
    fl.velocity[0, 1, 1, 0], fl.velocity[-1, 1, 1, 0] = -0.2, 0.3
    fl.velocity[1, 0, 1, 1], fl.velocity[1, -1, 1, 1] = -0.4, 0.5
    fl.velocity[1, 1, 0, 2], fl.velocity[1, 1, -1, 2] = -0.6, 0.7
    fl.apply_closed_boundary(0)
    assert float(fl.velocity[0, 1, 1, 0]) == 0.0 and float(fl.velocity[1, 0, 1, 1]) == 0.0
    assert float(fl.velocity[1, 1, 0, 2]) == 0.0
    assert float(fl.velocity[-1, 1, 1, 0]) == pytest.approx(0.3, abs=1e-7)
    assert float(fl.velocity[1, -1, 1, 1]) == pytest.approx(0.5, abs=1e-7)
    assert float(fl.velocity[1, 1, -1, 2]) == pytest.approx(0.7, abs=1e-7)


# test_core_fluid.py:745 (kernel part) the z-min outlet clamps only backflow
def test_zmin_outlet_clamps_only_backflow():
    fl = _fluid(_uniform_box(8))
    fl.velocity[...] = (0.0, 0.0, 0.05)
    fl.apply_zmin_no_backflow()
    assert float(np.asarray(fl.velocity)[:, :, 0, 2].max()) <= 1.0e-8
    fl.velocity[...] = (0.0, 0.0, -0.05)
    fl.apply_zmin_no_backflow()
    assert float(np.asarray(fl.velocity)[:, :, 0, 2].min()) < -0.049


# test_core_fluid.py:772 the predictor's backtrace ignores velocities inside obstacles
def test_predict_backtrace_ignores_obstacle_velocity():
    fl = orc.OracleFluid(_uniform_box(8), rho=1000.0, mu=0.0)
    fl.obstacle[3, 4, 4] = 1
    fl.velocity[...] = 0.0
    fl.velocity[..., 0] = -4.0
    fl.velocity[3, 4, 4, :] = 0.0
    fl.predict(1.0 / 64.0)
    assert float(fl.velocity[2, 4, 4, 0]) == pytest.approx(-4.0, abs=1e-5)
    np.testing.assert_allclose(fl.velocity[3, 4, 4], (0.0, 0.0, 0.0), atol=1e-7)


# --------------------------------------------------------------------------
# Marker tractions and forces (tests/test_hibm.py:109-410 of the reference)
# --------------------------------------------------------------------------
def _markers_at(positions, normals, areas, regions):
    return orc.OracleMarkers(x=np.asarray(positions, np.float32), normal=np.asarray(normals, np.float32),
                             area=np.asarray(areas, np.float32), region=np.asarray(regions, np.int32))


# test_hibm.py:109 per-marker force from traction and area
def test_marker_force_is_traction_times_area():
    m = _markers_at([(0.0, 0.0, 0.0), (1.0, 0.0, 0.0)], [(0.0, 0.0, 1.0), (0.0, 1.0, 0.0)], [0.5, 0.25], [101, 202])
    m.t[0], m.t[1] = (2.0, 0.0, -4.0), (0.0, 8.0, 0.0)
    m.compute_forces()
    assert tuple(m.F[0]) == (1.0, 0.0, -2.0)
    assert tuple(m.F[1]) == (0.0, 2.0, 0.0)


# test_hibm.py:336 a uniform pressure samples the full stress traction -p n
def test_uniform_pressure_samples_minus_p_n():
    fl = _fluid(_uniform_box(8))
    fl.pressure[...] = 7.0
    m = _markers_at([(0.625, 0.625, 0.5)], [(1.0, 0.0, 0.0)], [0.5], [101])
    rep = m.sample_tractions(fl)
    m.compute_forces()
    assert rep.valid == 1 and rep.invalid == 0
    assert tuple(m.t[0]) == (-7.0, 0.0, 0.0)
    assert tuple(m.F[0]) == (-3.5, 0.0, 0.0)


# test_hibm.py:374 a two-sided thin wall samples the pressure jump, not the centre average
def test_two_sided_wall_samples_the_pressure_jump():
    fl = _fluid(_uniform_box(8))
    fl.pressure[:, :, :4] = 2.0
    fl.pressure[:, :, 4:] = 10.0
    m = _markers_at([(0.625, 0.625, 0.5)], [(0.0, 0.0, 1.0)], [1.0], [101])
    rep = m.sample_tractions(fl, two_sided=1)
    m.compute_forces()
    assert rep.valid == 1 and rep.invalid == 0 and rep.two_sided == 1
    assert tuple(m.t[0]) == (0.0, 0.0, -8.0)
    assert tuple(m.F[0]) == (0.0, 0.0, -8.0)


# --------------------------------------------------------------------------
# z-min outlet reachability (fluid.py:1649-1876), tests/test_core_fluid.py:2243-2472
# --------------------------------------------------------------------------
# test_core_fluid.py:2243 a component cut off from the outlet is counted, not frozen
def test_outlet_reachability_counts_the_cut_off_layers():
    obs = np.zeros((5, 5, 5), np.int32)
    obs[:, :, 2] = 1
    vd = np.zeros((5, 5, 5), np.int32)
    vd[2, 2, 4] = 1
    r = orc.outlet_reachability(obs, velocity_dirichlet_active=vd)
    assert r["unreached"] == 50 and r["converged"]
    assert r["reachable"][:, :, :2].all() and not r["reachable"][:, :, 3:].any()
    assert r["components"] == 1


# test_core_fluid.py:2450 the fill reaches its fixed point along a long serpentine path
def test_outlet_reachability_reaches_the_end_of_a_long_path():
    obs = np.zeros((16, 4, 16), np.int32)
    obs[:, :, 4] = 1
    obs[15, :, 4] = 0
    obs[:, :, 8] = 1
    obs[0, :, 8] = 0
    obs[:, :, 12] = 1
    obs[15, :, 12] = 0
    r = orc.outlet_reachability(obs)
    assert r["unreached"] == 0 and r["converged"]
    assert r["reachable"][8, 1, 15] == 1


# test_core_fluid.py:2307 separate pockets become separate components
def test_outlet_reachability_labels_separate_pockets():
    obs = np.ones((9, 4, 9), np.int32)
    obs[:, :, 0] = 0
    obs[2, 2, 4] = 0
    obs[2, 2, 5] = 0
    obs[6, 2, 6] = 0
    r = orc.outlet_reachability(obs)
    assert r["unreached"] == 3 and r["components"] == 2 and not r["overflow"]
    # components ranked by their smallest linear cell index
    assert r["label"][2, 2, 4] == r["label"][2, 2, 5] == -1
    assert r["label"][6, 2, 6] == -2


def test_outlet_reachability_faces_follow_the_upper_cell():
    """A Dirichlet row closes the faces on its lower sides only
    (fluid.py:1649-1698): the row cell joins through its upper z face."""
    obs = np.zeros((1, 1, 4), np.int32)
    vd = np.zeros((1, 1, 4), np.int32)
    vd[0, 0, 1] = 1
    r = orc.outlet_reachability(obs, velocity_dirichlet_active=vd)
    # k = 0 is seeded; the face (0, 1) is closed by the row at k = 1, so k = 1
    # is reached only from k = 2, which has no way in: nothing above k = 0
    assert r["reachable"][0, 0].tolist() == [1, 0, 0, 0]
    assert r["unreached"] == 3


# --------------------------------------------------------------------------
# Marker surface feedback from the MPM particles (tests/test_hibm.py:726-899)
# --------------------------------------------------------------------------
def _feedback_case(marker_normal, marker_area, px, pv, pn=None, pa=None, box=(1.0, 1.0, 1.0)):
    m = _markers_at([(0.5, 0.5, 0.5)], [marker_normal], [marker_area], [202])
    x, vol, mass = _box_particles((1, 1, 1), (0.0,) * 3, box, 1000.0)
    s = orc.OracleSolid(capacity=1, grid_nodes=(4, 4, 4))
    s.load(x=x, volume=vol, mass=mass, normal=None if pn is None else np.asarray([pn], np.float32),
           area=None if pa is None else np.asarray([pa], np.float32))
    if px is not None:
        s.x[0] = px
    s.v[0] = pv
    return m, s


# test_hibm.py:726 feedback moves the marker by the supporting particles' velocity
def test_feedback_updates_marker_position_and_velocity():
    m, s = _feedback_case((0.0, 0.0, 1.0), 1.0, (0.6, 0.45, 0.7), (1.0, -2.0, 3.0))
    rep = m.feedback(s, 0.5, 0.1, geometry=False)
    assert rep.updated == 1 and rep.invalid == 0
    np.testing.assert_allclose(m.x[0], (0.6, 0.3, 0.8), atol=1e-6)
    np.testing.assert_allclose(m.v[0], (1.0, -2.0, 3.0), atol=1e-6)


# test_hibm.py:770 feedback takes the particles' surface normal and area
def test_feedback_updates_marker_normal_and_area():
    m, s = _feedback_case((0.0, 0.0, 1.0), 0.25, (0.6, 0.45, 0.7), (1.0, -2.0, 3.0), pn=(0.0, 2.0, 0.0), pa=0.75)
    rep = m.feedback(s, 0.5, 0.1, geometry=True)
    assert rep.updated == 1 and rep.invalid == 0 and rep.geometry_updated == 1
    assert tuple(m.n[0]) == (0.0, 1.0, 0.0)
    assert float(m.A[0]) == pytest.approx(0.75, abs=1e-6)
    assert rep.max_area_change == pytest.approx(0.5, abs=1e-6)
    assert rep.max_normal_change > 0.0


# test_hibm.py:817 the marker advances by velocity, not to the particle centroid
def test_feedback_advances_by_velocity_not_to_the_centroid():
    m, s = _feedback_case((0.0, 0.0, 1.0), 0.25, (0.9, 0.5, 0.5), (0.1, 0.0, 0.0), pn=(0.0, 0.0, 1.0), pa=0.25)
    rep = m.feedback(s, 0.5, 0.1, geometry=True)
    assert rep.updated == 1 and rep.invalid == 0
    np.testing.assert_allclose(m.x[0], (0.51, 0.5, 0.5), atol=1e-6)
    np.testing.assert_allclose(m.v[0], (0.1, 0.0, 0.0), atol=1e-6)
    assert rep.max_displacement == pytest.approx(0.01, abs=1e-6)


# test_hibm.py:864 a marker without supporting particles is recorded invalid and kept
def test_feedback_records_unsupported_marker_invalid():
    m, s = _feedback_case((0.0, 1.0, 0.0), 1.0, None, (0.0, 0.0, 0.0), box=(0.2, 0.2, 0.2))
    rep = m.feedback(s, 0.1, 0.1, geometry=False)
    assert rep.updated == 0 and rep.invalid == 1
    assert tuple(m.x[0]) == (0.5, 0.5, 0.5) and tuple(m.v[0]) == (0.0, 0.0, 0.0)


# test_core_fluid.py:1292 the pressure outlet balances an explicit volume source
def test_pressure_outlet_balances_a_volume_source():
    n = 16
    fl = _fluid(_uniform_box(n))
    cell_volume = 1.0 / n ** 3
    total = 2.0e-6
    fl.volume_source[7:9, 7:9, 10:12] = np.float32(total / (8.0 * cell_volume))
    fl.velocity[...] = 0.0
    fl.project_outlet_multigrid(dt=1.0e-3, iterations=8, cycles=8)
    area = (1.0 / n) ** 2
    outlet_flux = float(np.sum(-np.asarray(fl.velocity, np.float64)[:, :, 0, 2]) * area)
    residual = float(np.sum((np.asarray(fl.divergence, np.float64) - np.asarray(fl.volume_source, np.float64))
                            * cell_volume))
    assert outlet_flux == pytest.approx(total, abs=total * 0.08)
    assert residual == pytest.approx(0.0, abs=total * 0.02)


# test_core_fluid.py:1591 (CG part) the non-uniform outlet CG converges and balances the source
def test_nonuniform_outlet_cg_converges_and_balances_the_source():
    widths = tuple(0.02 * (1.0 + 0.15 * ((i % 4) / 3.0)) for i in range(24))
    fl = _nonuniform_fluid(widths, widths, widths)
    assert len(fl.metrics) >= 4
    vol = _cell_volumes(fl)
    total = 2.0e-6
    cells = np.s_[11:13, 11:13, 18:20]
    fl.volume_source[cells] = np.float32(total / float(np.sum(vol[cells])))
    fl.velocity[...] = 0.0
    st = fl.project_outlet_cg(dt=1.0e-3, max_iters=160, tol=1.0e-6)
    assert st.converged and st.iterations < 160
    w = [np.asarray(m["w"], np.float32).astype(np.float64) for m in fl.metrics[0]]
    area = np.outer(w[0], w[1])
    outlet_flux = float(np.sum(-np.asarray(fl.velocity, np.float64)[:, :, 0, 2] * area))
    assert abs(1.0 - outlet_flux / total) < 1.0e-3


# test_core_fluid.py:1548 an obstacle-adjacent volume source is conserved by the fv_jacobi projection
def test_fv_jacobi_obstacle_adjacent_source_is_conserved():
    nodes = (14, 10, 10)
    obs = np.zeros(nodes, np.int32)
    obs[8, 4:6, 5:7] = 1
    fl = _fluid_with(nodes, obs)
    cell_volume = 1.0 / (14 * 10 * 10)
    total = 1.0e-6
    fl.volume_source[7:8, 4:6, 5:7] = np.float32(total / (4.0 * cell_volume))
    fl.project_outlet_jacobi(dt=1.0e-3, iterations=2400)
    area = (1.0 / 14) * (1.0 / 10)
    outlet_flux = float(np.sum(-np.asarray(fl.velocity, np.float64)[:, :, 0, 2]) * area)
    active = obs == 0
    residual = float(np.sum((np.asarray(fl.divergence, np.float64)[active]
                             - np.asarray(fl.volume_source, np.float64)[active]) * cell_volume))
    assert outlet_flux > 0.0
    assert outlet_flux / total == pytest.approx(1.0, abs=0.12)
    assert residual == pytest.approx(0.0, abs=total * 0.01)


# test_core_fluid.py:3713 the BiCGSTAB fallback solves a generic FV rhs
def test_bicgstab_fallback_solves_a_generic_rhs():
    fl = _fluid(_uniform_box(4))
    rhs = np.zeros((4, 4, 4))
    rhs[2, 2, 2] = 1.0
    fl.pressure[...] = 0.0
    b_norm = math.sqrt(max(fl.weighted_dot(rhs, rhs), 0.0))
    st = fl.bicgstab(rhs, outlet=1, max_iters=80, tol=1.0e-8, b_norm=b_norm)
    assert st["converged"] and st["breakdown"] == 0
    assert st["relative_residual"] <= 1.0e-8
    # the recurrence agrees with the true residual of the returned pressure
    res = rhs - fl.fv_apply(np.asarray(fl.pressure), 1)
    assert math.sqrt(fl.weighted_dot(res, res)) / b_norm <= 1.0e-7


# test_core_fluid.py:2277-2342 (the anchoring the reference's outlet solves
# apply to flood-unreached components): two sealed pockets make the outlet
# system singular; with each pocket's mean subtracted where fluid.py:6567-6789
# does it, the PCG converges and leaves each pocket's pressure with zero mean,
# while the same PCG without the anchoring does not converge.
@pytest.mark.parametrize("precond", [0, 1])
def test_anchored_outlet_pcg_converges_on_sealed_pockets(precond):
    n = (12, 10, 16)
    grid = CartesianGrid(bounds_min_m=(0.0, 0.0, 0.0),
                         cell_widths_x_m=graded_axis_widths(n[0], 0.0, 1.0, 0.3, 0.7),
                         cell_widths_y_m=graded_axis_widths(n[1], 0.0, 1.0, 0.3, 0.7),
                         cell_widths_z_m=graded_axis_widths(n[2], 0.0, 1.0, 0.2, 0.8))
    obs = np.zeros(grid.grid_nodes, np.int32)
    for (i0, j0, k0, m) in ((1, 1, 4, 4), (6, 5, 9, 5)):
        obs[i0:i0 + m, j0:j0 + m, k0:k0 + m] = 1
        obs[i0 + 1:i0 + m - 1, j0 + 1:j0 + m - 1, k0 + 1:k0 + m - 1] = 0
    reach = orc.outlet_reachability(obs)
    assert reach["unreached"] == 2 ** 3 + 3 ** 3 and reach["components"] == 2
    label = reach["label"]
    comp = np.where((obs == 0) & (reach["reachable"] == 0) & (label < 0), -label - 1, -1).astype(np.int32)
    div = np.random.default_rng(5).normal(size=grid.grid_nodes).astype(np.float32)
    runs = {}
    for anchored in (True, False):
        ofl = orc.OracleFluid(grid, rho=1000.0, mu=1.0e-3, variant="mirror")
        ofl.obstacle[...] = obs
        ofl.divergence[...] = div
        ofl.pressure[...] = 0.0
        ofl.prepare_rhs(1.0e6)
        st = ofl.pcg_solve(outlet=1, max_iters=300, tol=1e-10, precond=precond, remove_mean=False,
                           components=comp if anchored else None, component_count=2)
        runs[anchored] = (st, ofl.pressure.copy(), ofl)
    st, p, ofl = runs[True]
    assert st.converged and st.unreached_set_mean_projection_count > 0
    assert not runs[False][0].converged
    vol = np.einsum("i,j,k->ijk", *[np.asarray(m["w"], np.float32).astype(np.float64) for m in ofl.metrics[0]])
    for c in range(2):
        on = comp == c
        assert abs((p * vol)[on].sum() / vol[on].sum()) <= 1e-10 * np.abs(p).max()
