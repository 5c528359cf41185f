"""The reference's known-answer cases through the drop-in API on the GPU.

Same cases as tests/test_oracle_known_answers.py (which pins the oracle), here
called the way the reference's own tests call its classes; each names the
reference test (tests/<file>:<line> in the reference tree) it restates.
"""

import math

import numpy as np
import pytest

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
