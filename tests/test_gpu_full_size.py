"""The c2 workload at full size (128 x 128 x 256 graded grid, ~201k particles,
8066 markers) through the drop-in API, checked by properties that hold at any
size: the pressure solve reaches its true-residual tolerance and removes the
divergence, the MPM transfer conserves momentum with det F ~ 1, and the marker
force spreading conserves force (action = reaction).  The oracle checks the
same kernels element by element on smaller grids (test_gpu_parity.py).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    from easyfsi_b200.scenarios import CONFIGS, CoupledScene

    return CoupledScene(CONFIGS["c2"])


def test_c2_projection_reaches_tolerance_and_removes_divergence(scene):
    cfg, fl = scene.cfg, scene.fluid
    fl.predict(cfg.dt_s)
    fl.compute_divergence()
    before = fl.divergence_stats()["l2"]
    fl.project(iterations=cfg.cg_max_iterations, dt_s=cfg.dt_s, pressure_solver="fv_cg",
               cg_tolerance=cfg.cg_tolerance, cg_preconditioner="fv_multigrid", read_report=False)
    assert fl.last_cg_converged
    assert fl.last_cg_used_multigrid
    assert fl.last_cg_relative_residual <= cfg.cg_tolerance * (1.0 + 1e-6)
    assert 0 < fl.last_cg_iterations < cfg.cg_max_iterations
    fl.compute_divergence()
    after = fl.divergence_stats()["l2"]
    # velocity is f32 (as in the reference), so what remains is f32 rounding
    # of the face velocities (~1e-7 |u| / h); the reference's own test asks
    # for a reduction to 0.45 (tests/test_fluid.py:46-57)
    assert before > 0.0
    assert after <= 1.0e-2 * before


def test_c2_marker_forces_spread_conservatively(scene):
    fl, mk, so = scene.fluid, scene.markers, scene.solid
    mk.sample_fluid_stress_to_marker_tractions(
        fl.velocity, fl.pressure, fl.obstacle,
        fl.cell_face_x_m, fl.cell_face_y_m, fl.cell_face_z_m,
        fl.cell_center_x_m, fl.cell_center_y_m, fl.cell_center_z_m,
        fl.cell_width_x_m, fl.cell_width_y_m, fl.cell_width_z_m,
        fl.grid.grid_nodes, viscosity_pa_s=0.0, two_sided_pressure=False, read_report=False,
    )
    mk.compute_marker_forces()
    mk.clear_mpm_external_forces(so.external_force_n, particle_count=so.particle_count, read_report=False)
    rep = mk.scatter_marker_forces_to_mpm_particles(
        so.external_force_n, so.x, particle_count=so.particle_count, support_radius_m=scene.radius
    )
    assert rep.active_marker_count > 0 and rep.invalid_marker_count == 0
    total = np.asarray(rep.total_marker_force_n)
    spread = so.external_force_n.to_numpy()[: so.particle_count].astype(np.float64).sum(axis=0)
    scale = max(np.abs(total).max(), 1e-30)
    assert np.abs(np.asarray(rep.total_mpm_external_force_n) - total).max() <= 1e-5 * scale
    assert np.abs(spread - total).max() <= 1e-4 * scale


def test_c2_mpm_substep_conserves_momentum(scene):
    from easyfsi_b200.scenarios import PRIMARY_REGION_ID, SECONDARY_REGION_ID

    cfg, so = scene.cfg, scene.solid
    rep = so.step(dt_s=cfg.dt_s / cfg.solid_substeps, mu_pa=scene.mu_pa, lambda_pa=scene.lambda_pa,
                  primary_region_id=PRIMARY_REGION_ID, secondary_region_id=SECONDARY_REGION_ID)
    assert rep.particle_count == so.particle_count
    assert rep.active_grid_nodes > 0
    assert rep.transfer_relative_error < 2.0e-5
    assert rep.max_abs_j == pytest.approx(1.0, abs=1e-3)


def test_c2_mixed_precision_vcycle_solves_to_the_same_tolerance(scene):
    """fv_multigrid_mixed at full size: the FP64 outer CG reaches the same
    true-residual tolerance, in about as many iterations, and the pressure
    stays close to the FP64 V-cycle's solution of the same system."""
    cfg, fl = scene.cfg, scene.fluid
    fl.predict(cfg.dt_s)
    fl.compute_divergence()
    out = {}
    for name in ("fv_multigrid", "fv_multigrid_mixed"):
        fl.pressure.tensor.zero_()
        fl._solve_pressure_poisson_fv_cg(iterations=cfg.cg_max_iterations, rhs_scale=cfg.density_kgm3 / cfg.dt_s,
                                         pressure_outlet_zmin=False, tolerance=cfg.cg_tolerance, preconditioner=name)
        assert fl.last_cg_converged and fl.last_cg_used_multigrid
        assert fl.last_cg_relative_residual <= cfg.cg_tolerance * (1.0 + 1e-6)
        out[name] = (fl.last_cg_iterations, fl.pressure.to_numpy().astype(np.float64))
    (it32, a), (it64, b) = out["fv_multigrid_mixed"], out["fv_multigrid"]
    assert it32 <= it64 + 5
    # the FP32 V-cycle ran: the FP64 one is deterministic and would repeat b bit for bit
    assert not np.array_equal(a, b)
    # both stop at relative residual 1e-8: the solutions agree to the
    # condition number times that
    assert np.linalg.norm((a - b).ravel()) <= 1e-3 * np.linalg.norm(b.ravel())


def test_c3_plain_and_mixed_steps_match_the_fp64_oracle():
    """The c3 workload (256^3 graded grid, two spheres, ~505k particles):
    one coupled step with the FP64 V-cycle and one with the FP32 level-0
    V-cycle (fv_multigrid_mixed) on the GPU, and one on the FP64 build of the
    oracle, all from the same projected initial velocity.  Per-field relative
    L2 against the FP64 oracle: velocity, particle position and F <= 1e-6 (the
    GPU stores them in f32, as the reference does).  The pressure differs in
    its smoothest modes, which a relative residual of 1e-8 fixes only to the
    residual times the condition number (measured 6.5e-3; the velocity it
    corrects agrees to 2.6e-7), and the particle velocity follows it through
    the marker tractions (4.8e-3): both <= 2e-2.  The FP32 V-cycle's step
    agrees with the FP64 V-cycle's to 1e-6 in every field."""
    from easyfsi_b200.scenarios import CONFIGS, CoupledScene
    from oracle import oracle as orc

    cfg = CONFIGS["c3"]
    plain = CoupledScene(cfg)
    u0 = plain.fluid.velocity.to_numpy()
    mixed = CoupledScene(cfg, initial_velocity=u0, project_initial=False)
    mixed.preconditioner = "fv_multigrid_mixed"
    ref = orc.OracleScene(cfg, variant="fp64", initial_velocity=u0, project_initial=False)
    plain.step()
    mixed.step()
    ref.step()
    n = plain.solid.particle_count

    def rel(a, b):
        a = np.asarray(a, np.float64).ravel()
        b = np.asarray(b, np.float64).ravel()
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    out = {}
    for name, sc in (("fv_multigrid", plain), ("fv_multigrid_mixed", mixed)):
        out[name] = {
            "cg_iterations": int(sc.last_cg_iterations),
            "pressure": rel(sc.fluid.pressure.to_numpy(), ref.fluid.pressure),
            "velocity": rel(sc.fluid.velocity.to_numpy(), ref.fluid.velocity),
            "x": rel(sc.solid.x.to_numpy()[:n], ref.solid.x[:n]),
            "F": rel(sc.solid.F.to_numpy()[:n], ref.solid.F[:n]),
            "v": rel(sc.solid.v.to_numpy()[:n], ref.solid.v[:n]),
        }
    print("c3, one coupled step, relative L2 against the FP64 oracle "
          f"(oracle CG iterations {ref.last_stats.iterations}):", out)
    for name, e in out.items():
        for k in ("velocity", "x", "F"):
            assert e[k] <= 1e-6, (name, k, e[k])
        assert e["v"] <= 2e-2, (name, e["v"])
        assert e["pressure"] <= 2e-2, (name, e["pressure"])
    assert rel(mixed.fluid.pressure.to_numpy(), plain.fluid.pressure.to_numpy()) <= 1e-6
    assert rel(mixed.fluid.velocity.to_numpy(), plain.fluid.velocity.to_numpy()) <= 1e-6
    assert rel(mixed.solid.v.to_numpy()[:n], plain.solid.v.to_numpy()[:n]) <= 1e-6
