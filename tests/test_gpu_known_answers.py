"""The reference's known-answer cases through the drop-in API on the GPU.

Same cases as tests/test_oracle_known_answers.py (which pins the oracle), here
called the way the reference's own tests call its classes; each names the
reference test (tests/<file>:<line> in the reference tree) it restates.
"""

import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _unit_solver(n):
    from easyfsi_b200.fluid import CartesianFluidSolver, FluidDomainSpec

    return CartesianFluidSolver(FluidDomainSpec.unit_box(grid_nodes=(n, n, n), dt_s=1.0e-3))


# test_core_fluid.py:1677
def test_interface_diagonal_enters_operator_diagonal_and_jacobi():
    s = _unit_solver(5)
    diag = np.zeros((5, 5, 5), np.float32)
    diag[2, 2, 2] = 7.5
    res = np.zeros((5, 5, 5), np.float32)
    res[2, 2, 2] = 15.0
    s.pressure_tmp.from_numpy(np.ones((5, 5, 5), np.float32))
    s.pressure_interface_matrix_diagonal.from_numpy(diag)
    s.cg_r.from_numpy(res)
    s._fv_laplacian_apply_kernel(s.pressure_tmp, s.cg_Ad, 0)
    s._fv_diagonal_kernel(s.fv_diag, 0)
    s._apply_jacobi_preconditioner_kernel(s.cg_r, s.cg_z)
    base = 6.0 / (0.2 * 0.2)
    assert s.cg_Ad.to_numpy()[2, 2, 2] == pytest.approx(7.5, abs=1e-5)
    assert s.fv_diag.to_numpy()[2, 2, 2] == pytest.approx(base + 7.5, abs=3e-5)
    assert s.cg_z.to_numpy()[2, 2, 2] == pytest.approx(15.0 / (base + 7.5), abs=1e-6)


def _restrict_level0(s):
    s.compute_divergence()
    s._prepare_fv_multigrid_rhs(1.0)
    s._compute_fv_residual_level(0, pressure_outlet_zmin=False)
    s._mg_restrict_residual_kernel(
        s._mg_residual[0], s._mg_pressure_interface_matrix_diagonal[0], s._mg_obstacle[0],
        s._mg_velocity_dirichlet_boundary_active[0], s._mg_velocity_dirichlet_boundary_projection_weight[0],
        s._mg_cell_width_x_m[0], s._mg_cell_width_y_m[0], s._mg_cell_width_z_m[0],
        s._mg_rhs[1], s._mg_pressure_interface_matrix_diagonal[1], s._mg_pressure[1], s._mg_tmp[1],
        s._mg_residual[1], s._mg_obstacle[1], s._mg_velocity_dirichlet_boundary_active[1],
        s._mg_velocity_dirichlet_boundary_projection_weight[1], 8, 8, 8,
    )


# test_core_fluid.py:1206
def test_restriction_volume_averages_interface_diagonal():
    s = _unit_solver(8)
    diag = np.zeros((8, 8, 8), np.float32)
    diag[2, 2, 2] = 80.0
    s.pressure_interface_matrix_diagonal.from_numpy(diag)
    _restrict_level0(s)
    coarse = s._mg_pressure_interface_matrix_diagonal[1].to_numpy()
    assert float(coarse[1, 1, 1]) == pytest.approx(10.0, abs=1e-5)
    assert float(coarse[0, 0, 0]) == pytest.approx(0.0, abs=1e-6)


# test_core_fluid.py:1166
def test_restriction_marks_mixed_obstacle_blocks_blocked():
    s = _unit_solver(8)
    obs = np.zeros((8, 8, 8), np.int32)
    obs[1, 1, 1] = 1
    s.obstacle.from_numpy(obs)
    s.velocity_dirichlet_boundary_active[2, 2, 2] = 1
    _restrict_level0(s)
    assert int(s._mg_obstacle[1].to_numpy()[0, 0, 0]) == 1
    assert int(s._mg_velocity_dirichlet_boundary_active[1].to_numpy()[1, 1, 1]) == 1


# test_core_fluid.py:1242
def test_coarse_smoother_uses_the_coarse_interface_diagonal():
    s = _unit_solver(8)
    diag = np.zeros((8, 8, 8), np.float32)
    diag[1, 1, 1] = 1.0e8
    s.pressure_interface_matrix_diagonal.from_numpy(diag)
    s._prepare_fv_multigrid_rhs(1.0)
    rhs = np.zeros(s._mg_shapes[1], np.float32)
    rhs[1, 1, 1] = 1.0
    s._mg_rhs[1].from_numpy(rhs)
    s._smooth_fv_pressure_level(1, iterations=1, pressure_outlet_zmin=False, omega=1.0)
    assert float(s._mg_pressure[1].to_numpy()[1, 1, 1]) < -1.0e-3


# test_core_fluid.py:1648
@pytest.mark.parametrize("outlet", [0, 1])
def test_operator_is_self_adjoint_on_graded_obstacle_grid(outlet):
    from easyfsi_b200.fluid import CartesianFluidSolver, FluidDomainSpec
    from easyfsi_b200.grid import CartesianGrid
    from easyfsi_b200.scenarios import graded_axis_widths

    grid = CartesianGrid(
        bounds_min_m=(0.0, 0.0, 0.0),
        cell_widths_x_m=graded_axis_widths(16, 0.0, 1.0, 0.3, 0.7),
        cell_widths_y_m=graded_axis_widths(14, 0.0, 1.0, 0.3, 0.7),
        cell_widths_z_m=graded_axis_widths(20, 0.0, 1.0, 0.2, 0.8),
    )
    obs = np.zeros(grid.grid_nodes, np.int32)
    obs[6:10, 5:9, 8:13] = 1
    s = CartesianFluidSolver(FluidDomainSpec((0, 0, 0), grid.bounds_max_m, None, 1000.0, 1.0e-3, 1.0e-3,
                                             cartesian_grid=grid))
    rng = np.random.default_rng(17)
    x = rng.normal(size=grid.grid_nodes).astype(np.float32)
    y = rng.normal(size=grid.grid_nodes).astype(np.float32)
    x[obs == 1] = 0.0
    y[obs == 1] = 0.0
    s.obstacle.from_numpy(obs)
    s.pressure_tmp.from_numpy(x)
    s.cg_d.from_numpy(y)
    s._fv_laplacian_apply_kernel(s.pressure_tmp, s.cg_r, outlet)
    s._fv_laplacian_apply_kernel(s.cg_d, s.cg_Ad, outlet)
    lhs = float(s._weighted_dot_kernel(s.cg_r, s.cg_d))
    rhs = float(s._weighted_dot_kernel(s.pressure_tmp, s.cg_Ad))
    assert abs(lhs - rhs) / max(abs(lhs), abs(rhs), 1e-30) < 1.0e-12


def _material():
    e, nu = 1.0e5, 0.45
    return e / (2 * (1 + nu)), e * nu / ((1 + nu) * (1 - 2 * nu))


# test_neo_hookean_mpm.py:102
def test_uniform_velocity_transfer_is_conservative():
    from easyfsi_b200.neo_hookean_mpm import NeoHookeanMpmState

    st = NeoHookeanMpmState(particle_capacity=64, bounds_min_m=(-0.02,) * 3, bounds_max_m=(0.02,) * 3,
                            grid_nodes=(12, 12, 12))
    st.initialize_box(particle_counts=(4, 4, 4), box_min_m=(-0.005,) * 3, box_max_m=(0.005,) * 3, density_kgm3=1100.0)
    st.set_uniform_velocity((0.02, -0.01, 0.03))
    mu, lam = _material()
    rep = st.step(dt_s=1.0e-5, mu_pa=mu, lambda_pa=lam, primary_region_id=1, secondary_region_id=2)
    assert rep.particle_count == 64
    assert rep.active_grid_nodes > 0
    assert rep.transfer_relative_error < 2.0e-5
    assert rep.total_mass_kg > 0.0
    assert rep.max_abs_j == pytest.approx(1.0, abs=1e-4)


# test_neo_hookean_mpm.py:38
def test_surface_geometry_follows_the_deformation_gradient():
    from easyfsi_b200.neo_hookean_mpm import NeoHookeanMpmState

    st = NeoHookeanMpmState(particle_capacity=1, bounds_min_m=(-1.0,) * 3, bounds_max_m=(1.0,) * 3, grid_nodes=(12, 12, 12))
    st.load_particles(positions_m=np.array([[1.0 / 3.0, 1.0 / 3.0, 0.0]], np.float32),
                      volumes_m3=np.array([1.0e-3], np.float32), masses_kg=np.array([1.0], np.float32),
                      region_ids=np.array([1], np.int32), normals=np.array([[0.0, 0.0, 1.0]], np.float32),
                      areas_m2=np.array([0.5], np.float32))
    F = st.F.to_numpy()
    F[0] = np.array([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.5, 0.0, 1.0]], np.float32)
    st.F.from_numpy(F)
    st.step(dt_s=0.0, mu_pa=0.0, lambda_pa=0.0, primary_region_id=1, secondary_region_id=2)
    expected = np.array([-0.5, 0.0, 1.0]) / math.sqrt(1.25)
    assert float(st.area_weight_m2.to_numpy()[0]) == pytest.approx(0.5 * math.sqrt(1.25), abs=1e-5)
    np.testing.assert_allclose(st.surface_normal.to_numpy()[0], expected, atol=1e-5)


def _scatter_case(counts, lo, hi, traction, normal, area, radius, stale=None):
    from easyfsi_b200.hibm_mpm import HibmMpmSurfaceMarkers
    from easyfsi_b200.neo_hookean_mpm import NeoHookeanMpmState

    markers = HibmMpmSurfaceMarkers(marker_capacity=1)
    markers.load_markers(positions_m=((0.5, 0.5, 0.5),), velocities_mps=((0.0, 0.0, 0.0),), normals=(normal,),
                         areas_m2=(area,), region_ids=(101,))
    markers.set_marker_tractions_pa((traction,))
    markers.compute_marker_forces()
    n = counts[0] * counts[1] * counts[2]
    solid = NeoHookeanMpmState(particle_capacity=n, bounds_min_m=(0.0,) * 3, bounds_max_m=(1.0,) * 3, grid_nodes=(4, 4, 4))
    solid.initialize_box(particle_counts=counts, box_min_m=lo, box_max_m=hi, density_kgm3=1000.0)
    clear = None
    if stale is not None:
        solid.external_force_n[0] = stale
        clear = markers.clear_mpm_external_forces(solid.external_force_n, particle_count=solid.particle_count)
    rep = markers.scatter_marker_forces_to_mpm_particles(solid.external_force_n, solid.x,
                                                         particle_count=solid.particle_count, support_radius_m=radius)
    return solid, rep, clear


# test_hibm.py:605
def test_scatter_gives_the_single_particle_the_marker_force():
    solid, rep, _ = _scatter_case((1, 1, 1), (0.0,) * 3, (1.0,) * 3, (2.0, -4.0, 6.0), (1.0, 0.0, 0.0), 0.5, 0.25)
    assert rep.active_marker_count == 1 and rep.invalid_marker_count == 0 and rep.active_particle_count == 1
    assert solid.external_force_n[0] == (1.0, -2.0, 3.0)
    assert rep.total_marker_force_n == (1.0, -2.0, 3.0)
    assert rep.total_mpm_external_force_n == (1.0, -2.0, 3.0)
    assert rep.action_reaction_residual_n == pytest.approx(0.0)


# test_hibm.py:645
def test_scatter_partitions_force_across_supported_particles():
    solid, rep, _ = _scatter_case((2, 1, 1), (0.25, 0.0, 0.0), (0.75, 1.0, 1.0), (0.0, 0.0, 4.0), (0.0, 0.0, 1.0), 1.0, 0.4)
    assert rep.active_marker_count == 1 and rep.active_particle_count == 2
    assert solid.external_force_n[0][2] == pytest.approx(2.0, abs=1e-5)
    assert solid.external_force_n[1][2] == pytest.approx(2.0, abs=1e-5)
    assert rep.total_mpm_external_force_n[2] == pytest.approx(4.0, abs=1e-5)
    assert rep.action_reaction_residual_n == pytest.approx(0.0, abs=1e-5)


# test_hibm.py:684
def test_clear_then_scatter_replaces_stale_force():
    solid, rep, clear = _scatter_case((1, 1, 1), (0.0,) * 3, (1.0,) * 3, (2.0, -4.0, 6.0), (1.0, 0.0, 0.0), 0.5, 0.25,
                                      stale=(99.0, 0.0, 0.0))
    assert solid.external_force_n[0] == (1.0, -2.0, 3.0)
    assert rep.total_mpm_external_force_n == (1.0, -2.0, 3.0)


# --------------------------------------------------------------------------
# IB node search (HibmMpmIbNodeSearch, hibm_mpm.py:5385-6220), the reference's
# HibmMpmIbNodeSearchTests through the drop-in classes.
# --------------------------------------------------------------------------
def _markers(positions, normals, triangles=None):
    from easyfsi_b200.hibm_mpm import HibmMpmSurfaceMarkers

    n = len(positions)
    m = HibmMpmSurfaceMarkers(marker_capacity=n, projection_triangle_capacity=len(triangles) if triangles else None)
    m.load_markers(positions_m=positions, velocities_mps=((0.0, 0.0, 0.0),) * n, normals=normals,
                   areas_m2=(1.0,) * n, region_ids=(7,) * n)
    if triangles:
        m.set_projection_triangles(triangles)
    return m


def _node_search(nodes, capacity, bmin=(0.0, 0.0, 0.0), bmax=(1.0, 1.0, 1.0)):
    from easyfsi_b200.hibm_mpm import HibmMpmIbNodeSearch

    return HibmMpmIbNodeSearch(grid_nodes=nodes, bounds_min_m=bmin, bounds_max_m=bmax, marker_capacity=capacity)


_CLOSED_X = ((0.25, 0.5, 0.5), (0.75, 0.5, 0.5), (0.5, 0.25, 0.5), (0.5, 0.75, 0.5), (0.5, 0.5, 0.25), (0.5, 0.5, 0.75))
_CLOSED_N = ((-1.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, -1.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, -1.0), (0.0, 0.0, 1.0))


# test_hibm.py:904
def test_ib_search_plane_classifies_external_and_internal_nodes():
    mk = _markers(((0.5, 0.5, 0.5),), ((0.0, 0.0, 1.0),))
    search = _node_search((1, 1, 4), 1)
    rep = search.search_and_classify(mk, search_radius_m=0.26, interior_probe_distance_m=0.125)
    assert (rep.near_boundary_node_count, rep.external_ib_node_count, rep.internal_node_count,
            rep.invalid_projection_count) == (2, 1, 1, 0)
    assert search.node_kind((0, 0, 2)) == "external_ib" and search.node_kind((0, 0, 1)) == "internal"
    assert search.nearest_marker_index((0, 0, 2)) == 0 and search.nearest_marker_index((0, 0, 1)) == 0
    assert search.boundary_point_m((0, 0, 2)) == (0.5, 0.5, 0.5)
    assert search.interior_fluid_point_m((0, 0, 2)) == (0.5, 0.5, 0.75)
    assert search.signed_distance_m((0, 0, 2)) > 0.0 and search.signed_distance_m((0, 0, 1)) < 0.0


# test_hibm.py:939
def test_ib_search_triangle_projection_between_markers():
    mk = _markers(((0.25, 0.25, 0.5), (0.75, 0.25, 0.5), (0.25, 0.75, 0.5)), ((0.0, 0.0, 1.0),) * 3, [(0, 1, 2)])
    search = _node_search((8, 8, 8), 3)
    rep = search.search_and_classify(mk, search_radius_m=0.08, interior_probe_distance_m=0.05)
    assert rep.near_boundary_node_count >= 1 and rep.external_ib_node_count >= 1
    assert search.node_kind((2, 2, 4)) == "external_ib"
    np.testing.assert_allclose(search.boundary_point_m((2, 2, 4)), (0.3125, 0.3125, 0.5), atol=1e-6)
    assert search.signed_distance_m((2, 2, 4)) == pytest.approx(0.0625)
    np.testing.assert_allclose(search.interior_fluid_point_m((2, 2, 4)), (0.3125, 0.3125, 0.6125), atol=1e-6)


# test_hibm.py:987
def test_ib_search_closed_surface_deep_internal_node():
    search = _node_search((1, 1, 1), 6)
    rep = search.search_and_classify(_markers(_CLOSED_X, _CLOSED_N), search_radius_m=0.1,
                                     interior_probe_distance_m=0.125, classify_far_internal_nodes=True)
    assert (rep.near_boundary_node_count, rep.external_ib_node_count, rep.internal_node_count) == (0, 0, 1)
    assert search.node_kind((0, 0, 0)) == "internal" and search.nearest_marker_index((0, 0, 0)) >= 0


# test_hibm.py:1030
def test_ib_search_closed_surface_grid_fields_deep_internal_nodes():
    fluid = _unit_solver(4)
    search = _node_search(fluid.grid.grid_nodes, 6, fluid.grid.bounds_min_m, fluid.grid.bounds_max_m)
    rep = search.search_and_classify_grid_fields(
        _markers(_CLOSED_X, _CLOSED_N), cell_center_x_m=fluid.cell_center_x_m, cell_center_y_m=fluid.cell_center_y_m,
        cell_center_z_m=fluid.cell_center_z_m, search_radius_m=0.08, interior_probe_distance_m=0.125,
        classify_far_internal_nodes=True)
    assert rep.near_boundary_node_count == 0 and rep.internal_node_count == 8
    assert search.node_kind((1, 1, 1)) == "internal" and search.node_kind((2, 2, 2)) == "internal"
    assert search.node_kind((0, 0, 0)) == "none"


# test_hibm.py:1088
def test_ib_search_default_sign_tolerance_flags_ambiguous_node():
    search = _node_search((1, 1, 1), 1)
    rep = search.search_and_classify(_markers(((0.5, 0.5, 0.5 - 5.0e-8),), ((0.0, 0.0, 1.0),)), search_radius_m=0.01,
                                     interior_probe_distance_m=0.125)
    assert rep.near_boundary_node_count == 1 and rep.invalid_projection_count == 1
    assert search.node_kind((0, 0, 0)) == "internal" and search.signed_distance_m((0, 0, 0)) > 0.0


# test_hibm.py:1115
def test_ib_search_nonuniform_cell_centres():
    from easyfsi_b200.fluid import CartesianFluidSolver, FluidDomainSpec
    from easyfsi_b200.grid import CartesianGrid

    grid = CartesianGrid(bounds_min_m=(0.0, 0.0, 0.0), cell_widths_x_m=(0.25,) * 4, cell_widths_y_m=(0.25,) * 4,
                         cell_widths_z_m=(0.1, 0.1, 0.2, 0.6))
    fluid = CartesianFluidSolver(FluidDomainSpec(bounds_min_m=(0.0, 0.0, 0.0), bounds_max_m=(1.0, 1.0, 1.0),
                                                 grid_nodes=(4, 4, 4), density_kgm3=1000.0, viscosity_pa_s=1.0e-3,
                                                 dt_s=1.0e-3, cartesian_grid=grid))
    search = _node_search(fluid.grid.grid_nodes, 1, fluid.grid.bounds_min_m, fluid.grid.bounds_max_m)
    rep = search.search_and_classify_grid_fields(
        _markers(((0.625, 0.625, 0.28),), ((0.0, 0.0, 1.0),)), cell_center_x_m=fluid.cell_center_x_m,
        cell_center_y_m=fluid.cell_center_y_m, cell_center_z_m=fluid.cell_center_z_m, search_radius_m=0.04,
        interior_probe_distance_m=0.05)
    assert (rep.near_boundary_node_count, rep.external_ib_node_count, rep.internal_node_count) == (1, 1, 0)
    assert search.node_kind((2, 2, 2)) == "external_ib" and search.node_kind((2, 2, 1)) == "none"
    assert search.signed_distance_m((2, 2, 2)) == pytest.approx(0.02, abs=1e-6)
    np.testing.assert_allclose(search.boundary_point_m((2, 2, 2)), (0.625, 0.625, 0.28), atol=1e-6)
    assert search.interior_fluid_point_m((2, 2, 2))[2] == pytest.approx(0.35, abs=1e-6)


# test_hibm.py:1174
def test_ib_search_external_if_any_local_normal_is_positive():
    search = _node_search((1, 1, 1), 2)
    rep = search.search_and_classify(_markers(((0.5, 0.5, 0.55), (0.5, 0.5, 0.45)), ((0.0, 0.0, -1.0), (0.0, 0.0, 1.0))),
                                     search_radius_m=0.08, interior_probe_distance_m=0.05)
    assert (rep.near_boundary_node_count, rep.external_ib_node_count, rep.internal_node_count) == (1, 1, 0)
    assert search.node_kind((0, 0, 0)) == "external_ib"


# test_hibm.py:1201
def test_ib_search_stores_the_external_candidate():
    search = _node_search((1, 1, 1), 2)
    rep = search.search_and_classify(_markers(((0.5, 0.5, 0.49), (0.5, 0.5, 0.46)), ((0.0, 0.0, -1.0), (0.0, 0.0, 1.0))),
                                     search_radius_m=0.05, interior_probe_distance_m=0.05, sign_tolerance_m=1.0e-8)
    assert (rep.near_boundary_node_count, rep.external_ib_node_count, rep.internal_node_count) == (1, 1, 0)
    assert search.node_kind((0, 0, 0)) == "external_ib" and search.nearest_marker_index((0, 0, 0)) == 1
    assert search.signed_distance_m((0, 0, 0)) > 0.0
    assert search.boundary_point_m((0, 0, 0))[2] == pytest.approx(0.46, abs=1e-6)
    assert search.interior_fluid_point_m((0, 0, 0))[2] > 0.5


# test_hibm.py:1240
def test_ib_search_radial_marker_inside_and_outside():
    search = _node_search((4, 1, 1), 1)
    rep = search.search_and_classify(_markers(((0.75, 0.5, 0.5),), ((1.0, 0.0, 0.0),)), search_radius_m=0.14,
                                     interior_probe_distance_m=0.125)
    assert (rep.near_boundary_node_count, rep.external_ib_node_count, rep.internal_node_count) == (2, 1, 1)
    assert search.node_kind((3, 0, 0)) == "external_ib" and search.node_kind((2, 0, 0)) == "internal"
    assert search.signed_distance_m((3, 0, 0)) > 0.0 and search.signed_distance_m((2, 0, 0)) < 0.0


# test_hibm.py:1270
def test_ib_search_tangent_projection_records_invalid():
    search = _node_search((1, 1, 1), 1)
    rep = search.search_and_classify(_markers(((0.5, 0.5, 0.5),), ((0.0, 0.0, 1.0),)), search_radius_m=0.1,
                                     interior_probe_distance_m=0.125, sign_tolerance_m=1.0e-9)
    assert rep.near_boundary_node_count == 1 and rep.invalid_projection_count == 1
    assert search.nearest_marker_index((0, 0, 0)) == 0
    assert search.boundary_point_m((0, 0, 0)) == (0.5, 0.5, 0.5)
    assert search.interior_fluid_point_m((0, 0, 0)) == (0.5, 0.5, 0.625)


def test_ib_search_rejects_bad_arguments():
    """hibm_mpm.py:6069-6094 argument errors."""
    mk = _markers(((0.5, 0.5, 0.5),), ((0.0, 0.0, 1.0),))
    search = _node_search((2, 2, 2), 1)
    for kwargs in ({"search_radius_m": 0.0, "interior_probe_distance_m": 0.1},
                   {"search_radius_m": math.inf, "interior_probe_distance_m": 0.1},
                   {"search_radius_m": 0.1, "interior_probe_distance_m": -1.0},
                   {"search_radius_m": 0.1, "interior_probe_distance_m": 0.1, "sign_tolerance_m": -1.0}):
        with pytest.raises(ValueError):
            search.search_and_classify(mk, **kwargs)


# --------------------------------------------------------------------------
# IB boundary conditions and velocity-Dirichlet rows (HibmMpmIbBoundaryConditions,
# hibm_mpm.py:6222-7800) through the drop-in classes.  The oracle side of the
# same cases passes in tests/test_oracle_known_answers.py.
# --------------------------------------------------------------------------
def _boundary(nodes, capacity):
    from easyfsi_b200.hibm_mpm import HibmMpmIbBoundaryConditions

    return HibmMpmIbBoundaryConditions(grid_nodes=nodes, marker_capacity=capacity)


def _vd_rows(boundary, fluid, search, **kw):
    return boundary.assemble_velocity_dirichlet_reconstructed_boundary_rows(
        fluid.velocity_dirichlet_boundary_active, fluid.velocity_dirichlet_boundary_value_mps,
        fluid.velocity_dirichlet_boundary_projection_weight, fluid.obstacle, fluid.velocity, search,
        cell_face_x_m=fluid.cell_face_x_m, cell_face_y_m=fluid.cell_face_y_m, cell_face_z_m=fluid.cell_face_z_m,
        cell_center_x_m=fluid.cell_center_x_m, cell_center_y_m=fluid.cell_center_y_m,
        cell_center_z_m=fluid.cell_center_z_m, grid_nodes=fluid.grid.grid_nodes, **kw)


def _one_node(node, bv, n, bp, ip, obstacle=None, velocity=None):
    fluid = _unit_solver(4)
    search = _node_search((4, 4, 4), 1)
    boundary = _boundary((4, 4, 4), 1)
    boundary.active_ib_node[node] = 1
    boundary.velocity_dirichlet_mps_field[node] = bv
    boundary.pressure_neumann_normal_field[node] = n
    search.node_boundary_point_m[node] = bp
    search.node_interior_fluid_point_m[node] = ip
    if obstacle is not None:
        fluid.obstacle.from_numpy(obstacle)
    if velocity is not None:
        fluid.velocity.tensor[...] = torch.tensor(velocity, dtype=torch.float32, device=fluid.velocity.tensor.device)
    return fluid, _vd_rows(boundary, fluid, search)


# test_hibm.py:1301
def test_ib_boundary_targets_from_the_plane_search():
    mk = _markers(((0.5, 0.5, 0.5),), ((0.0, 0.0, 2.0),))
    mk.v_gamma_mps[0] = (1.25, -0.5, 0.75)
    search = _node_search((1, 1, 4), 1)
    search.search_and_classify(mk, search_radius_m=0.26, interior_probe_distance_m=0.125)
    boundary = _boundary((1, 1, 4), 1)
    rep = boundary.build_from_search(search, mk, marker_pressure_neumann_gradient_pa_per_m=(42.0,))
    assert (rep.no_slip_dirichlet_count, rep.pressure_neumann_count, rep.inactive_internal_node_count) == (1, 1, 1)
    assert rep.max_abs_velocity_mps == pytest.approx(1.25, abs=1e-6)
    assert boundary.is_active((0, 0, 2)) and not boundary.is_active((0, 0, 1))
    assert boundary.velocity_dirichlet_mps((0, 0, 2)) == (1.25, -0.5, 0.75)
    assert boundary.pressure_neumann_normal((0, 0, 2)) == (0.0, 0.0, 1.0)
    assert boundary.pressure_neumann_gradient_pa_per_m((0, 0, 2)) == pytest.approx(42.0)


# test_hibm.py:3337
def test_vd_rows_reconstruct_along_the_surface_normal():
    mk = _markers(((0.625, 0.625, 0.5),), ((0.0, 0.0, 1.0),))
    mk.v_gamma_mps[0] = (0.0, 0.0, 0.1)
    search = _node_search((4, 4, 4), 1)
    search.search_and_classify(mk, search_radius_m=0.13, interior_probe_distance_m=0.125)
    boundary = _boundary((4, 4, 4), 1)
    boundary.build_from_search(search, mk, marker_pressure_neumann_gradient_pa_per_m=(0.0,))
    fluid = _unit_solver(4)
    fluid.velocity.tensor[...] = torch.tensor((0.0, 0.0, 0.4), device=fluid.velocity.tensor.device)
    rep = _vd_rows(boundary, fluid, search,
                   velocity_dirichlet_marker_region_id=fluid.velocity_dirichlet_boundary_marker_region_id,
                   marker_region_id=mk.region_id)
    assert rep.active_velocity_dirichlet_rows == 1 and rep.invalid_reconstruction_row_count == 0
    assert rep.min_projection_weight == pytest.approx(0.5, abs=1e-6)
    assert rep.max_projection_weight == pytest.approx(0.5, abs=1e-6)
    assert fluid.velocity_dirichlet_boundary_active[2, 2, 2] == 1
    assert int(fluid.velocity_dirichlet_boundary_marker_region_id[2, 2, 2]) == 7
    assert fluid.velocity_dirichlet_boundary_value_mps[2, 2, 2][2] == pytest.approx(0.25, abs=1e-6)
    assert fluid.velocity_dirichlet_boundary_projection_weight[2, 2, 2] == pytest.approx(0.5, abs=1e-6)


# test_hibm.py:3478
def test_vd_rows_relocate_a_masked_node_to_the_first_fluid_cell():
    obs = np.zeros((4, 4, 4), np.int32)
    obs[2, 2, 2] = 1
    fluid, rep = _one_node((2, 2, 2), (0.2, 0.0, 0.0), (1.0, 0.0, 0.0), (0.5, 0.625, 0.625), (0.875, 0.625, 0.625),
                           obstacle=obs)
    assert rep.active_velocity_dirichlet_rows == 1 and rep.relocated_row_count == 1
    assert rep.relocation_blocked_row_count == 0 and rep.inactive_obstacle_rows == 0
    assert fluid.velocity_dirichlet_boundary_active[2, 2, 2] == 0
    assert fluid.velocity_dirichlet_boundary_active[3, 2, 2] == 1
    np.testing.assert_allclose(fluid.velocity_dirichlet_boundary_value_mps[3, 2, 2], (0.08, 0.0, 0.0), atol=1e-6)
    assert fluid.velocity_dirichlet_boundary_projection_weight[3, 2, 2] == pytest.approx(0.6, abs=1e-6)


# test_hibm.py:3540
def test_vd_rows_relocate_to_the_opposite_side():
    obs = np.zeros((4, 4, 4), np.int32)
    obs[2:, :, :] = 1
    fluid, rep = _one_node((2, 2, 2), (0.2, 0.0, 0.0), (1.0, 0.0, 0.0), (0.5, 0.625, 0.625), (0.875, 0.625, 0.625),
                           obstacle=obs)
    assert rep.active_velocity_dirichlet_rows == 1 and rep.relocated_row_count == 1
    assert fluid.velocity_dirichlet_boundary_active[1, 2, 2] == 1
    np.testing.assert_allclose(fluid.velocity_dirichlet_boundary_value_mps[1, 2, 2], (0.13333334, 0.0, 0.0),
                               atol=1e-7)


# test_hibm.py:3597
def test_vd_rows_wall_limited_gap_is_a_narrow_gap_row():
    obs = np.zeros((4, 4, 4), np.int32)
    obs[3, :, :] = 1
    fluid, rep = _one_node((2, 2, 2), (0.3, 0.0, 0.0), (1.0, 0.0, 0.0), (0.5, 0.625, 0.625), (0.875, 0.625, 0.625),
                           obstacle=obs)
    assert rep.active_velocity_dirichlet_rows == 1 and rep.narrow_gap_boundary_velocity_row_count == 1
    assert rep.invalid_reconstruction_row_count == 0
    np.testing.assert_allclose(fluid.velocity_dirichlet_boundary_value_mps[2, 2, 2], (0.3, 0.0, 0.0), atol=1e-7)


# test_hibm.py:3658 and 3718
@pytest.mark.parametrize("node,bp,ip,value,weight", [
    ((2, 2, 2), (0.25, 0.625, 0.625), (0.375, 0.625, 0.625), 0.35, None),
    ((1, 2, 2), (0.5, 0.625, 0.625), (0.625, 0.625, 0.625), 0.3, 0.5),
])
def test_vd_rows_fall_back_along_the_line_of_sight(node, bp, ip, value, weight):
    fluid, rep = _one_node(node, (0.2, 0.0, 0.0), (1.0, 0.0, 0.0), bp, ip, velocity=(0.4, 0.0, 0.0))
    assert rep.active_velocity_dirichlet_rows == 1 and rep.invalid_reconstruction_row_count == 0
    np.testing.assert_allclose(fluid.velocity_dirichlet_boundary_value_mps[node], (value, 0.0, 0.0), atol=1e-6)
    if weight is not None:
        assert fluid.velocity_dirichlet_boundary_projection_weight[node] == pytest.approx(weight, abs=1e-6)


# --------------------------------------------------------------------------
# z-min outlet reachability (fluid.py:1771-1876) through the drop-in solver;
# the oracle side passes in tests/test_oracle_known_answers.py.
# --------------------------------------------------------------------------
def _box_solver(nodes):
    from easyfsi_b200.fluid import CartesianFluidSolver, FluidDomainSpec

    return CartesianFluidSolver(FluidDomainSpec.unit_box(grid_nodes=nodes, dt_s=1.0e-3))


# test_core_fluid.py:2243
def test_outlet_reachability_counts_the_cut_off_layers():
    s = _box_solver((5, 5, 5))
    obs = np.zeros((5, 5, 5), np.int32)
    obs[:, :, 2] = 1
    s.obstacle.from_numpy(obs)
    s.velocity_dirichlet_boundary_active[2, 2, 4] = 1
    assert s.mark_hibm_pressure_outlet_disconnected_nonprojectable_cells(pressure_outlet_zmin=True) == 50
    assert s.last_hibm_pressure_unreached_cell_count == 50 and s.last_hibm_pressure_reachability_converged
    assert (s.obstacle.to_numpy()[:, :, 3:] == 0).all()
    # the unreached layers are anchored (their mean subtracted) in the solve
    report = s.project(iterations=200, pressure_outlet_zmin=True, pressure_solver="fv_cg", cg_tolerance=1.0e-6)
    assert report["cg_converged_all"] and int(report["cg_unreached_set_mean_projection_count"]) >= 1


# test_core_fluid.py:2450
def test_outlet_reachability_reaches_the_end_of_a_long_path():
    s = _box_solver((16, 4, 16))
    obs = np.zeros((16, 4, 16), np.int32)
    obs[:, :, 4] = 1
    obs[15, :, 4] = 0
    obs[:, :, 8] = 1
    obs[0, :, 8] = 0
    obs[:, :, 12] = 1
    obs[15, :, 12] = 0
    s.obstacle.from_numpy(obs)
    assert s.mark_hibm_pressure_outlet_disconnected_nonprojectable_cells(pressure_outlet_zmin=True) == 0
    assert int(s.hibm_pressure_outlet_reachable[8, 1, 15]) == 1


# test_core_fluid.py:2307 (reachability part)
def test_outlet_reachability_labels_separate_pockets():
    s = _box_solver((9, 4, 9))
    obs = np.ones((9, 4, 9), np.int32)
    obs[:, :, 0] = 0
    obs[2, 2, 4] = 0
    obs[2, 2, 5] = 0
    obs[6, 2, 6] = 0
    s.obstacle.from_numpy(obs)
    assert s.mark_hibm_pressure_outlet_disconnected_nonprojectable_cells(pressure_outlet_zmin=True) == 3
    assert s.last_hibm_pressure_unreached_component_count == 2
    assert not s.last_hibm_pressure_unreached_component_overflow
    labels = s.hibm_pressure_unreached_component_label.to_numpy()
    assert labels[2, 2, 4] == labels[2, 2, 5] == -1 and labels[6, 2, 6] == -2


# test_core_fluid.py:3713 the BiCGSTAB fallback solves a generic FV rhs
def test_bicgstab_fallback_solves_a_generic_rhs():
    s = _box_solver((4, 4, 4))
    rhs = np.zeros((4, 4, 4))
    rhs[2, 2, 2] = 1.0
    s.cg_rhs.from_numpy(rhs)
    b_norm = float(np.sqrt(max(s._weighted_dot_kernel(s.cg_rhs, s.cg_rhs), 0.0)))
    s._continue_pressure_poisson_fv_bicgstab(start_iteration=0, max_iters=80, b_norm=b_norm, outlet=1,
                                             tolerance=1.0e-8, anchor_unreached=False, remove_nullspace_mean=False)
    assert s.last_cg_converged, s.last_cg_breakdown
    assert s.last_cg_relative_residual <= 1.0e-8
    assert "bicgstab_fallback" in s.last_cg_restart_policy


# test_core_fluid.py:3259 negative curvature sets the device breakdown code
# (the same device alpha / beta steps the PCG's finishers run)
def test_fv_cg_negative_curvature_sets_device_breakdown_code():
    s = _unit_solver(4)
    s.cg_rz[None] = 1.0
    s.cg_rz_new[None] = 1.0
    s.cg_dAd[None] = 0.0
    s._cg_compute_alpha_kernel()
    assert int(s.cg_breakdown_code[None]) == 1
    assert float(s.cg_alpha[None]) == 0.0
    assert float(s.cg_breakdown_dAd[None]) == 0.0
    s._cg_compute_beta_kernel(0)
    assert int(s.cg_breakdown_code[None]) == 1


def test_fv_cg_alpha_and_flexible_beta_steps():
    s = _unit_solver(4)
    s.cg_breakdown_code[None] = 0
    s.cg_rz[None] = 2.0
    s.cg_dAd[None] = 8.0
    s._cg_compute_alpha_kernel()
    assert float(s.cg_alpha[None]) == 0.25 and int(s.cg_breakdown_code[None]) == 0
    # flexible (Polak-Ribiere) beta is clamped at zero; Fletcher-Reeves is rz_new / rz
    s.cg_rz_new[None] = 3.0
    s.cg_beta_numerator[None] = -1.0
    s._cg_compute_beta_kernel(1)
    assert float(s.cg_beta[None]) == 0.0 and int(s.cg_breakdown_code[None]) == 0
    s.cg_beta_numerator[None] = 1.0
    s._cg_compute_beta_kernel(1)
    assert float(s.cg_beta[None]) == 0.5
    s._cg_compute_beta_kernel(0)
    assert float(s.cg_beta[None]) == 1.5
    # rz_new <= 0 is breakdown code 2; a negative dAd keeps the first offending value
    s.cg_rz_new[None] = 0.0
    s._cg_compute_beta_kernel(0)
    assert int(s.cg_breakdown_code[None]) == 2 and float(s.cg_beta[None]) == 0.0
    s.cg_breakdown_code[None] = 0
    s.cg_dAd[None] = -3.0
    s._cg_compute_alpha_kernel()
    s.cg_dAd[None] = -5.0
    s._cg_compute_alpha_kernel()
    assert int(s.cg_breakdown_code[None]) == 1 and float(s.cg_breakdown_dAd[None]) == -3.0


# --------------------------------------------------------------------------
# Interface-coupling terms of the FV operator (fluid.py:4345-4456) through the
# drop-in solver; the oracle side passes in tests/test_oracle_known_answers.py.
# --------------------------------------------------------------------------
# test_core_fluid.py:1756
def test_fv_cg_interface_coupling_enters_operator_symmetrically():
    s = _unit_solver(5)
    pressure = np.ones((5, 5, 5), np.float32)
    pressure[2, 2, 2] = 3.0
    pressure[2, 2, 3] = 1.0
    s.pressure_tmp.from_numpy(pressure)
    s._fv_laplacian_apply_kernel(s.pressure_tmp, s.cg_r, 0)
    base = s.cg_r.to_numpy()
    diagonal = np.zeros((5, 5, 5), np.float32)
    diagonal[2, 2, 2] = 4.0
    diagonal[2, 2, 3] = 4.0
    s.pressure_interface_matrix_diagonal.from_numpy(diagonal)
    s.pressure_interface_coupling_active[2, 2, 2] = 1
    s.pressure_interface_coupling_neighbor[2, 2, 2] = (2, 2, 3)
    s.pressure_interface_coupling_coefficient[2, 2, 2] = 4.0 * 0.2 * 0.2 * 0.2
    s._fv_laplacian_apply_kernel(s.pressure_tmp, s.cg_Ad, 0)
    coupled = s.cg_Ad.to_numpy()
    assert coupled[2, 2, 2] - base[2, 2, 2] == pytest.approx(8.0, abs=1e-5)
    assert coupled[2, 2, 3] - base[2, 2, 3] == pytest.approx(-8.0, abs=1e-5)


# test_core_fluid.py:1793
def test_fv_cg_interface_coupling_uses_transmissibility_on_nonuniform_cells():
    from easyfsi_b200.fluid import CartesianFluidSolver, FluidDomainSpec
    from easyfsi_b200.grid import CartesianGrid

    grid = CartesianGrid(bounds_min_m=(0.0, 0.0, 0.0), cell_widths_x_m=(0.1, 0.2, 0.35, 0.35),
                         cell_widths_y_m=(0.25,) * 4, cell_widths_z_m=(0.25,) * 4)
    s = CartesianFluidSolver(FluidDomainSpec(grid.bounds_min_m, grid.bounds_max_m, None, 1000.0, 1.0e-3, 1.0e-3,
                                             cartesian_grid=grid))
    rng = np.random.default_rng(41)
    x = rng.normal(size=grid.grid_nodes).astype(np.float32)
    y = rng.normal(size=grid.grid_nodes).astype(np.float32)
    t, left, right = 0.375, (1, 2, 2), (2, 2, 2)
    diagonal = np.zeros(grid.grid_nodes, np.float32)
    diagonal[left] = t / (0.2 * 0.25 * 0.25)
    diagonal[right] = t / (0.35 * 0.25 * 0.25)
    s.pressure_interface_matrix_diagonal.from_numpy(diagonal)
    s.pressure_interface_coupling_active[left] = 1
    s.pressure_interface_coupling_neighbor[left] = right
    s.pressure_interface_coupling_coefficient[left] = t
    s.pressure_tmp.from_numpy(x)
    s.cg_d.from_numpy(y)
    s._fv_laplacian_apply_kernel(s.pressure_tmp, s.cg_r, 0)
    s._fv_laplacian_apply_kernel(s.cg_d, s.cg_Ad, 0)
    lhs = float(s._weighted_dot_kernel(s.cg_r, s.cg_d))
    rhs = float(s._weighted_dot_kernel(s.pressure_tmp, s.cg_Ad))
    assert abs(lhs - rhs) / max(abs(lhs), abs(rhs), 1e-30) < 1e-5


# test_core_fluid.py:1836
def test_fv_cg_interface_coupling_applies_multiple_owner_slots():
    s = _unit_solver(5)
    pressure = np.ones((5, 5, 5), np.float32)
    owner, n0, n1 = (2, 2, 2), (2, 2, 3), (2, 3, 2)
    pressure[owner] = 3.0
    pressure[n0] = 1.0
    pressure[n1] = 2.0
    s.pressure_tmp.from_numpy(pressure)
    s._fv_laplacian_apply_kernel(s.pressure_tmp, s.cg_r, 0)
    base = s.cg_r.to_numpy()
    v = 0.2**3
    c0, c1 = 4.0 * v, 7.0 * v
    diagonal = np.zeros((5, 5, 5), np.float32)
    diagonal[owner] = (c0 + c1) / v
    diagonal[n0] = c0 / v
    diagonal[n1] = c1 / v
    s.pressure_interface_matrix_diagonal.from_numpy(diagonal)
    s.pressure_interface_coupling_active[owner] = 2
    s.pressure_interface_coupling_neighbor[owner] = n0
    s.pressure_interface_coupling_coefficient[owner] = c0
    s.pressure_interface_coupling_extra_neighbor[owner[0], owner[1], owner[2], 0] = n1
    s.pressure_interface_coupling_extra_coefficient[owner[0], owner[1], owner[2], 0] = c1
    s._fv_laplacian_apply_kernel(s.pressure_tmp, s.cg_Ad, 0)
    op = s.cg_Ad.to_numpy()
    assert op[owner] - base[owner] == pytest.approx(15.0, abs=5e-5)
    assert op[n0] - base[n0] == pytest.approx(-8.0, abs=5e-5)
    assert op[n1] - base[n1] == pytest.approx(-7.0, abs=5e-5)


def _sealed_cells_solver(cells, sources=None):
    """(9, 4, 9) unit box, solid except the z-min layer (the outlet) and the
    given sealed cells; optional volume sources on them."""
    from easyfsi_b200.fluid import CartesianFluidSolver, FluidDomainSpec

    s = CartesianFluidSolver(FluidDomainSpec.unit_box(grid_nodes=(9, 4, 9), dt_s=1.0e-3))
    obs = np.ones((9, 4, 9), np.int32)
    obs[:, :, 0] = 0
    for c in cells:
        obs[c] = 0
    s.obstacle.from_numpy(obs)
    if sources:
        src = np.zeros((9, 4, 9), np.float32)
        for c, v in sources.items():
            src[c] = v
        s.volume_source_s.from_numpy(src)
    return s


# test_core_fluid.py:2277
def test_fv_cg_anchors_pressure_mean_over_outlet_unreached_set():
    from easyfsi_b200.fluid import CartesianFluidSolver, FluidDomainSpec

    s = CartesianFluidSolver(FluidDomainSpec.unit_box(grid_nodes=(5, 5, 5), dt_s=1.0e-3))
    obs = np.zeros((5, 5, 5), np.int32)
    obs[:, :, 2] = 1
    s.obstacle.from_numpy(obs)
    assert s.mark_hibm_pressure_outlet_disconnected_nonprojectable_cells(pressure_outlet_zmin=True) == 50
    vel = np.zeros((5, 5, 5, 3), np.float32)
    vel[2, 2, 4, 0] = 0.4
    s.velocity.from_numpy(vel)
    report = s.project(iterations=200, pressure_outlet_zmin=True, pressure_solver="fv_cg", cg_tolerance=1.0e-6)
    assert report["cg_converged_all"]
    assert int(report["cg_unreached_set_mean_projection_count"]) >= 1


# test_core_fluid.py:2306
def test_fv_cg_anchors_multiple_disconnected_components_independently():
    s = _sealed_cells_solver([(2, 2, 4), (2, 2, 5), (6, 2, 6)],
                             {(2, 2, 4): 1.0, (2, 2, 5): 3.0, (6, 2, 6): -2.0})
    assert s.mark_hibm_pressure_outlet_disconnected_nonprojectable_cells(pressure_outlet_zmin=True) == 3
    assert s.last_hibm_pressure_unreached_component_count == 2
    assert not s.last_hibm_pressure_unreached_component_overflow
    report = s.project(iterations=200, pressure_outlet_zmin=True, pressure_solver="fv_cg", cg_tolerance=1.0e-6)
    assert report["cg_converged_all"]
    assert int(report["cg_unreached_component_count"]) == 2
    assert int(report["cg_unreached_set_mean_projection_count"]) >= 1


# test_core_fluid.py:2344
def test_fv_cg_reports_unreached_component_rhs_incompatibility():
    s = _sealed_cells_solver([(2, 2, 4), (2, 2, 5), (6, 2, 6)],
                             {(2, 2, 4): 1.0, (2, 2, 5): 3.0, (6, 2, 6): -2.0})
    assert s.mark_hibm_pressure_outlet_disconnected_nonprojectable_cells(pressure_outlet_zmin=True) == 3
    report = s.project(iterations=200, pressure_outlet_zmin=True, pressure_solver="fv_cg", cg_tolerance=1.0e-6)
    assert report["cg_converged_all"]
    assert not report["pressure_solve_failed"]
    assert report["pressure_projection_physical_failure"]
    assert report["pressure_projection_physical_failure_reason"] == "unreached_component_rhs_incompatible"
    assert int(report["hibm_unreached_incompatible_component_count"]) == 2
    assert float(report["hibm_unreached_component_rhs_mean_max_abs"]) > 0.0


# test_core_fluid.py:2386
def test_fv_cg_raises_on_unreached_component_rhs_incompatibility():
    s = _sealed_cells_solver([(2, 2, 4), (2, 2, 5)], {(2, 2, 4): 1.0, (2, 2, 5): 3.0})
    assert s.mark_hibm_pressure_outlet_disconnected_nonprojectable_cells(pressure_outlet_zmin=True) == 2
    with pytest.raises(RuntimeError, match="unreached component RHS is incompatible"):
        s.project(iterations=200, pressure_outlet_zmin=True, pressure_solver="fv_cg", cg_tolerance=1.0e-6,
                  pressure_solve_failure_policy="raise")


# test_core_fluid.py:2415
def test_final_divergence_report_excludes_anchored_unreached_cells():
    s = _sealed_cells_solver([(2, 2, 4), (2, 2, 5), (6, 2, 6)],
                             {(2, 2, 4): 1.0, (2, 2, 5): 3.0, (6, 2, 6): -2.0})
    assert s.mark_hibm_pressure_outlet_disconnected_nonprojectable_cells(pressure_outlet_zmin=True) == 3
    residual = s.divergence_residual_stats(interior_only=True)
    _raw, final, _int_raw, final_int = s.final_divergence_report_stats(pressure_outlet_zmin=True)
    assert residual["l2"] == pytest.approx(0.0, abs=1e-12)
    assert final["l2"] == pytest.approx(0.0, abs=1e-12)
    assert final_int["l2"] == pytest.approx(0.0, abs=1e-12)
    assert int(s.last_unreached_divergence_stats["count"]) == 3
    assert float(s.last_unreached_divergence_stats["l2"]) > 1.0
