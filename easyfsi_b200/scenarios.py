"""Seeded synthetic coupled-FSI workloads and the coupled step.

The workloads stand in for the reference's benchmark configurations (no
dataset is involved): a closed unit box of water with a random divergence-free
initial velocity and one (or two) immersed neo-Hookean bodies, sampled by MPM
particles (8 per MPM cell, jittered) and wrapped by surface markers.

* ``c1``: uniform 64^3 fluid grid, sphere r = 0.15 at (0.5, 0.5, 0.35),
  E = 1e5 Pa, nu = 0.45, rho_s = 1100, dt = 1e-4 (about 30k particles);
* ``c2``: graded 128 x 128 x 256 grid refined 4x inside
  [0.3, 0.7]^2 x [0.2, 0.8] and growing by 1.05 per cell outward, ellipsoid with
  semi-axes (0.12, 0.08, 0.2), E = 5e4 Pa, dt = 5e-5 (about 200k particles);
* ``c3``: 256^3 with the same grading law, two spheres r = 0.1 with
  E = 2e4 / 2e5 Pa, dt = 2e-5 (about 500k particles);
* ``c5`` (``batched_configs``): 32 independent instances, uniform grids of
  48^3, 64^3, 96^3 or 128^3 cells (seeded per instance), each with one sphere
  of seeded radius in [0.08, 0.18] and Young's modulus log-uniform in
  [1e4, 1e6] Pa, 8 particles per cell, dt = 1e-4.

One coupled step (``CoupledScene.step``) is: predict -> project (flexible
MG-PCG to relative residual 1e-8) -> marker pressure tractions -> marker forces
-> clear + spread onto the MPM particles -> MPM substep(s) -> surface feedback,
the sequence of the reference's marker-MPM runner
(simulation_core/benchmarking/solid_mpm_fsi_runner.py:50-89) with the fluid
advanced every step as in the sharp HIBM step (hibm_mpm.py:10533-10616).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .geometry import UvSphereResolution, make_uv_sphere
from .grid import CartesianGrid
from .hyperelastic import lame_parameters

PRIMARY_REGION_ID = 101
SECONDARY_REGION_ID = 202


@dataclass(frozen=True)
class Body:
    center: tuple[float, float, float]
    semi_axes: tuple[float, float, float]
    youngs_modulus_pa: float
    region_id: int


@dataclass(frozen=True)
class ScenarioConfig:
    name: str
    grid_nodes: tuple[int, int, int]
    graded: bool
    refine_box: tuple[tuple[float, float, float], tuple[float, float, float]] | None
    mpm_nodes: tuple[int, int, int]
    bodies: tuple[Body, ...]
    dt_s: float
    steps: int
    velocity_seed: int
    particle_seed: int
    marker_resolution: tuple[int, int]
    density_kgm3: float = 1000.0
    viscosity_pa_s: float = 1.0e-3
    solid_density_kgm3: float = 1100.0
    poisson_ratio: float = 0.45
    amplitude_mps: float = 0.1
    max_wavenumber: int = 4
    cg_tolerance: float = 1.0e-8
    cg_max_iterations: int = 400
    solid_substeps: int = 1
    support_radius_cells: float = 1.5
    extra: dict = field(default_factory=dict)


CONFIGS = {
    "c1": ScenarioConfig(
        name="c1_uniform64_sphere",
        grid_nodes=(64, 64, 64),
        graded=False,
        refine_box=None,
        mpm_nodes=(64, 64, 64),
        bodies=(Body((0.5, 0.5, 0.35), (0.15, 0.15, 0.15), 1.0e5, PRIMARY_REGION_ID),),
        dt_s=1.0e-4,
        steps=20,
        velocity_seed=1001,
        particle_seed=1002,
        marker_resolution=(32, 64),
    ),
    "c2": ScenarioConfig(
        name="c2_graded128x128x256_ellipsoid",
        grid_nodes=(128, 128, 256),
        graded=True,
        refine_box=((0.3, 0.3, 0.2), (0.7, 0.7, 0.8)),
        mpm_nodes=(116, 116, 232),
        bodies=(Body((0.5, 0.5, 0.5), (0.12, 0.08, 0.2), 5.0e4, PRIMARY_REGION_ID),),
        dt_s=5.0e-5,
        steps=100,
        velocity_seed=2001,
        particle_seed=2002,
        marker_resolution=(64, 128),
    ),
    "c3": ScenarioConfig(
        name="c3_graded256_two_spheres",
        grid_nodes=(256, 256, 256),
        graded=True,
        refine_box=((0.3, 0.3, 0.2), (0.7, 0.7, 0.8)),
        mpm_nodes=(196, 196, 196),
        bodies=(
            Body((0.5, 0.5, 0.35), (0.1, 0.1, 0.1), 2.0e4, PRIMARY_REGION_ID),
            Body((0.5, 0.5, 0.65), (0.1, 0.1, 0.1), 2.0e5, SECONDARY_REGION_ID),
        ),
        dt_s=2.0e-5,
        steps=50,
        velocity_seed=3001,
        particle_seed=3002,
        marker_resolution=(48, 96),
    ),
}


BATCH_GRID_SIZES = (48, 64, 96, 128)


def batched_configs(count: int = 32, seed: int = 5000, sizes: tuple[int, ...] = BATCH_GRID_SIZES) -> list[ScenarioConfig]:
    """The uneven batch of independent instances: instance i draws, from
    seed + i, its uniform grid size (one of `sizes`, the same along every
    axis and for the MPM grid), a sphere radius in [0.08, 0.18] and a Young's
    modulus log-uniform in [1e4, 1e6] Pa; the sphere sits at
    (0.5, 0.5, 0.4), dt = 1e-4."""
    out = []
    for i in range(count):
        rng = np.random.default_rng(seed + i)
        n = int(rng.choice(np.asarray(sizes)))
        radius = float(rng.uniform(0.08, 0.18))
        youngs = float(10.0 ** rng.uniform(4.0, 6.0))
        out.append(
            ScenarioConfig(
                name=f"c5_{i:02d}_uniform{n}_r{radius:.3f}",
                grid_nodes=(n, n, n),
                graded=False,
                refine_box=None,
                mpm_nodes=(n, n, n),
                bodies=(Body((0.5, 0.5, 0.4), (radius, radius, radius), youngs, PRIMARY_REGION_ID),),
                dt_s=1.0e-4,
                steps=50,
                velocity_seed=seed + 100 + i,
                particle_seed=seed + 200 + i,
                marker_resolution=(24, 48),
            )
        )
    return out


def tiny_config(n: int = 12, mpm: int = 12, seed: int = 7) -> ScenarioConfig:
    """A small graded case for parity tests (finishes in seconds on the oracle)."""
    return ScenarioConfig(
        name=f"tiny{n}",
        grid_nodes=(n, n, n + 4),
        graded=True,
        refine_box=((0.3, 0.3, 0.25), (0.7, 0.7, 0.75)),
        mpm_nodes=(mpm, mpm, mpm),
        bodies=(Body((0.5, 0.5, 0.5), (0.22, 0.2, 0.25), 5.0e4, PRIMARY_REGION_ID),),
        dt_s=5.0e-4,
        steps=3,
        velocity_seed=seed,
        particle_seed=seed + 1,
        marker_resolution=(8, 16),
    )


# ---------------------------------------------------------------------------
# graded axes with an exact cell count
# ---------------------------------------------------------------------------


def graded_axis_widths(n: int, lo: float, hi: float, a: float, b: float, ratio: float = 1.05, refine: float = 4.0):
    """``n`` cell widths on [lo, hi]: uniform width h on [a, b], growing by
    ``ratio`` per cell away from it up to ``refine * h``.  h is chosen so the
    continuous cell count equals n; the integer counts are then distributed
    and each side is rescaled to its exact length."""
    s_left, s_right, inner = a - lo, hi - b, b - a

    def side_profile(h: float, length: float) -> tuple[float, list[float]]:
        widths, total, k = [], 0.0, 1
        while total < length and length > 0.0:
            w = h * min(ratio**k, refine)
            widths.append(w)
            total += w
            k += 1
        if not widths:
            return 0.0, []
        excess = total - length
        frac = len(widths) - excess / widths[-1]
        return frac, widths

    def count(h: float) -> float:
        return inner / h + side_profile(h, s_left)[0] + side_profile(h, s_right)[0]

    h_lo, h_hi = (hi - lo) / (n * refine * 4.0), (hi - lo) / max(n / 4.0, 1.0)
    for _ in range(200):
        h = 0.5 * (h_lo + h_hi)
        if count(h) > n:
            h_lo = h
        else:
            h_hi = h
    h = 0.5 * (h_lo + h_hi)
    fl, fr = side_profile(h, s_left)[0], side_profile(h, s_right)[0]
    m = max(1, int(round(inner / h)))
    rest = n - m
    cl = int(round(rest * fl / max(fl + fr, 1e-30))) if fl + fr > 0 else 0
    cr = rest - cl

    def side(c: int, length: float) -> list[float]:
        if c <= 0:
            return []
        w = [h * min(ratio ** (k + 1), refine) for k in range(c)]
        scale = length / sum(w)
        return [v * scale for v in w]

    left = list(reversed(side(cl, s_left)))
    right = side(cr, s_right)
    widths = left + [inner / m] * m + right
    assert len(widths) == n
    return tuple(widths)


def build_grid(cfg: ScenarioConfig) -> CartesianGrid:
    if not cfg.graded:
        return CartesianGrid.uniform(bounds_min_m=(0.0, 0.0, 0.0), bounds_max_m=(1.0, 1.0, 1.0), grid_nodes=cfg.grid_nodes)
    (a0, a1, a2), (b0, b1, b2) = cfg.refine_box
    return CartesianGrid(
        bounds_min_m=(0.0, 0.0, 0.0),
        cell_widths_x_m=graded_axis_widths(cfg.grid_nodes[0], 0.0, 1.0, a0, b0),
        cell_widths_y_m=graded_axis_widths(cfg.grid_nodes[1], 0.0, 1.0, a1, b1),
        cell_widths_z_m=graded_axis_widths(cfg.grid_nodes[2], 0.0, 1.0, a2, b2),
    )


# ---------------------------------------------------------------------------
# initial state
# ---------------------------------------------------------------------------


def _inside(body: Body, pts: np.ndarray) -> np.ndarray:
    c = np.asarray(body.center)
    s = np.asarray(body.semi_axes)
    return (((pts - c) / s) ** 2).sum(axis=-1) <= 1.0


def fourier_velocity(grid: CartesianGrid, seed: int, amplitude: float, kmax: int) -> np.ndarray:
    """Random Fourier-mode velocity, 0 < |k| <= kmax, scaled to max |u| = amplitude.
    Component d is evaluated on the min-side face of each cell (the reference's
    face-velocity storage).  The sum over modes of cc cos(phase) + cs sin(phase)
    is the real part of sum C[k] e^(i pi k.x) with C = cc - i cs; e^(i pi k.x)
    factors by axis, so the sum is three small tensor contractions."""
    rng = np.random.default_rng(seed)
    modes = [(kx, ky, kz) for kx in range(-kmax, kmax + 1) for ky in range(-kmax, kmax + 1) for kz in range(-kmax, kmax + 1)
             if 0 < kx * kx + ky * ky + kz * kz <= kmax * kmax]
    coef_c = rng.normal(size=(len(modes), 3))
    coef_s = rng.normal(size=(len(modes), 3))
    faces = [np.asarray(grid.axis_faces(a)[:-1]) for a in range(3)]
    centers = [np.asarray(grid.axis_centers(a)) for a in range(3)]
    nx, ny, nz = grid.grid_nodes
    ks = np.arange(-kmax, kmax + 1, dtype=np.float64)
    u = np.zeros((nx, ny, nz, 3), dtype=np.float64)
    for d in range(3):
        coords = [faces[a] if a == d else centers[a] for a in range(3)]
        C = np.zeros((2 * kmax + 1,) * 3, dtype=np.complex128)
        for (kx, ky, kz), cc, cs in zip(modes, coef_c, coef_s):
            C[kx + kmax, ky + kmax, kz + kmax] = cc[d] - 1j * cs[d]
        ex, ey, ez = (np.exp(1j * math.pi * np.outer(ks, np.asarray(c, dtype=np.float64))) for c in coords)
        t = np.tensordot(C, ez, axes=([2], [0]))           # (a, b, k)
        t = np.tensordot(t, ey, axes=([1], [0]))           # (a, k, j)
        acc = np.tensordot(ex, t, axes=([0], [0]))         # (i, k, j)
        u[..., d] = acc.real.transpose(0, 2, 1)
    u *= amplitude / max(np.abs(u).max(), 1e-30)
    return u.astype(np.float32)


def obstacle_mask(grid: CartesianGrid, bodies) -> np.ndarray:
    X, Y, Z = np.meshgrid(*[np.asarray(grid.axis_centers(a)) for a in range(3)], indexing="ij")
    pts = np.stack([X, Y, Z], axis=-1)
    obs = np.zeros(grid.grid_nodes, dtype=np.int32)
    for body in bodies:
        obs[_inside(body, pts)] = 1
    return obs


def particles(cfg: ScenarioConfig):
    """8 jittered particles per MPM cell inside each body."""
    rng = np.random.default_rng(cfg.particle_seed)
    n = np.asarray(cfg.mpm_nodes)
    dx = 1.0 / n
    out_x, out_vol, out_region, out_E, out_normal, out_area = [], [], [], [], [], []
    for body in cfg.bodies:
        c, s = np.asarray(body.center), np.asarray(body.semi_axes)
        lo = np.maximum(np.floor((c - s) / dx).astype(int) - 1, 0)
        hi = np.minimum(np.ceil((c + s) / dx).astype(int) + 1, n)
        ii, jj, kk = np.meshgrid(*[np.arange(lo[a], hi[a]) for a in range(3)], indexing="ij")
        cells = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1)
        centers = (cells + 0.5) * dx
        cells = cells[_inside(body, centers)]
        sub = np.array([[a, b, d] for a in (0, 1) for b in (0, 1) for d in (0, 1)], dtype=np.float64)
        pts = (cells[:, None, :] + 0.25 + 0.5 * sub[None, :, :]) * dx
        pts = pts.reshape(-1, 3)
        pts = pts + (rng.uniform(-0.125, 0.125, size=pts.shape) * dx)
        vol = np.full(pts.shape[0], np.prod(dx) / 8.0)
        # surface layer: particles within one MPM cell of the surface carry the
        # normal and an equal share of the surface area.
        q = (pts - c) / s
        r = np.sqrt((q * q).sum(axis=1))
        grad = q / s
        nrm = grad / np.maximum(np.linalg.norm(grad, axis=1, keepdims=True), 1e-30)
        depth = (1.0 - r) * np.min(s)
        shell = depth < dx.max()
        p_ = 1.6075
        a_, b_, c_ = s
        surface_area = 4.0 * math.pi * (((a_ * b_) ** p_ + (a_ * c_) ** p_ + (b_ * c_) ** p_) / 3.0) ** (1.0 / p_)
        area = np.where(shell, surface_area / max(int(shell.sum()), 1), 0.0)
        out_x.append(pts)
        out_vol.append(vol)
        out_region.append(np.full(pts.shape[0], body.region_id, dtype=np.int32))
        out_E.append(np.full(pts.shape[0], body.youngs_modulus_pa))
        out_normal.append(np.where(shell[:, None], nrm, 0.0))
        out_area.append(area)
    x = np.concatenate(out_x).astype(np.float32)
    vol = np.concatenate(out_vol).astype(np.float32)
    return {
        "x": x,
        "volume": vol,
        "mass": (vol * np.float32(cfg.solid_density_kgm3)).astype(np.float32),
        "region": np.concatenate(out_region),
        "E": np.concatenate(out_E),
        "normal": np.concatenate(out_normal).astype(np.float32),
        "area": np.concatenate(out_area).astype(np.float32),
    }


def markers(cfg: ScenarioConfig):
    lat, lon = cfg.marker_resolution
    xs, ns, As, rs = [], [], [], []
    for body in cfg.bodies:
        mesh = make_uv_sphere(UvSphereResolution(lat, lon), 1.0)
        s = np.asarray(body.semi_axes)
        v = mesh.vertices * s + np.asarray(body.center)
        f = mesh.faces
        fa = 0.5 * np.linalg.norm(np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]]), axis=1)
        area = np.zeros(v.shape[0])
        for corner in range(3):
            np.add.at(area, f[:, corner], fa / 3.0)
        g = (v - np.asarray(body.center)) / (s * s)
        n = g / np.linalg.norm(g, axis=1, keepdims=True)
        xs.append(v)
        ns.append(n)
        As.append(area)
        rs.append(np.full(v.shape[0], body.region_id, dtype=np.int32))
    return {
        "x": np.concatenate(xs).astype(np.float32),
        "normal": np.concatenate(ns).astype(np.float32),
        "area": np.concatenate(As).astype(np.float32),
        "region": np.concatenate(rs),
    }


def support_radius(cfg: ScenarioConfig) -> float:
    return cfg.support_radius_cells / min(cfg.mpm_nodes)


def material(cfg: ScenarioConfig) -> tuple[float, float]:
    """Lame parameters of the (first) body."""
    return lame_parameters(cfg.bodies[0].youngs_modulus_pa, cfg.poisson_ratio)


# ---------------------------------------------------------------------------
# the coupled step on the B200 path
# ---------------------------------------------------------------------------


class CoupledScene:
    """Fluid + MPM solid + markers of one workload, advanced on the GPU."""

    def __init__(self, cfg: ScenarioConfig, *, initial_velocity: np.ndarray | None = None, project_initial: bool = True):
        from .fluid import CartesianFluidSolver, FluidDomainSpec
        from .hibm_mpm import HibmMpmSurfaceMarkers
        from .neo_hookean_mpm import NeoHookeanMpmState

        self.cfg = cfg
        self.grid = build_grid(cfg)
        spec = FluidDomainSpec(
            bounds_min_m=(0.0, 0.0, 0.0),
            bounds_max_m=self.grid.bounds_max_m,
            grid_nodes=None,
            density_kgm3=cfg.density_kgm3,
            viscosity_pa_s=cfg.viscosity_pa_s,
            dt_s=cfg.dt_s,
            cartesian_grid=self.grid,
        )
        self.fluid = CartesianFluidSolver(spec)
        self.fluid.obstacle.from_numpy(obstacle_mask(self.grid, cfg.bodies))
        u0 = initial_velocity if initial_velocity is not None else fourier_velocity(
            self.grid, cfg.velocity_seed, cfg.amplitude_mps, cfg.max_wavenumber
        )
        self.fluid.velocity.from_numpy(u0)
        if project_initial:
            self.fluid.project(
                iterations=cfg.cg_max_iterations, pressure_solver="fv_cg", cg_tolerance=cfg.cg_tolerance,
                cg_preconditioner="fv_multigrid", read_report=False,
            )
            self.fluid.pressure.tensor.zero_()
        part = particles(cfg)
        self.solid = NeoHookeanMpmState(
            particle_capacity=part["x"].shape[0], bounds_min_m=(0.0, 0.0, 0.0), bounds_max_m=(1.0, 1.0, 1.0), grid_nodes=cfg.mpm_nodes
        )
        self.solid.load_particles(
            positions_m=part["x"], volumes_m3=part["volume"], masses_kg=part["mass"], region_ids=part["region"],
            normals=part["normal"], areas_m2=part["area"],
        )
        mk = markers(cfg)
        self.markers = HibmMpmSurfaceMarkers(marker_capacity=mk["x"].shape[0])
        self.markers.load_markers(
            positions_m=mk["x"].tolist(), velocities_mps=np.zeros_like(mk["x"]).tolist(), normals=mk["normal"].tolist(),
            areas_m2=mk["area"].tolist(), region_ids=mk["region"].tolist(),
        )
        self.mu_pa, self.lambda_pa = material(cfg)
        self.radius = support_radius(cfg)
        self.last_cg_iterations = 0
        # "fv_multigrid" (the reference's) or "fv_multigrid_mixed" (FP32 level-0 V-cycle)
        self.preconditioner = "fv_multigrid"
        # overlap_solid: the marker forces, scatter, MPM substep and feedback of
        # a step run on a side stream beside the next step's fluid work
        # (finish() joins them); off, the step runs in order on one stream
        self.overlap_solid = False
        self._side = None
        self._solid_pending = False

    def step(self) -> None:
        cfg, fluid, solid, mk = self.cfg, self.fluid, self.solid, self.markers
        fluid.predict(cfg.dt_s)
        fluid.project(
            iterations=cfg.cg_max_iterations, dt_s=cfg.dt_s, pressure_solver="fv_cg", cg_tolerance=cfg.cg_tolerance,
            cg_preconditioner=self.preconditioner, read_report=False,
        )
        self.last_cg_iterations = fluid.last_cg_iterations
        self.finish()  # the previous step's solid part has moved the markers
        mk.sample_fluid_stress_to_marker_tractions(
            fluid.velocity, fluid.pressure, fluid.obstacle,
            fluid.cell_face_x_m, fluid.cell_face_y_m, fluid.cell_face_z_m,
            fluid.cell_center_x_m, fluid.cell_center_y_m, fluid.cell_center_z_m,
            fluid.cell_width_x_m, fluid.cell_width_y_m, fluid.cell_width_z_m,
            fluid.grid.grid_nodes, viscosity_pa_s=0.0, two_sided_pressure=False, read_report=False,
        )
        if not self.overlap_solid:
            self._solid_part()
            return
        # The rest of the step reads and writes only markers and particles, and
        # the next step's predict and projection only the fluid: it runs on a
        # side stream beside them and is joined before the next tractions.
        import torch

        if self._side is None:
            self._side = torch.cuda.Stream()
        self._side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(self._side):
            self._solid_part()
        self._solid_pending = True

    def finish(self) -> None:
        """Joins the solid part of the last step (``overlap_solid``) into the
        current stream; the particle and marker state is final after it."""
        if self._solid_pending:
            import torch

            torch.cuda.current_stream().wait_stream(self._side)
            self._solid_pending = False

    def _solid_part(self) -> None:
        cfg, solid, mk = self.cfg, self.solid, self.markers
        mk.compute_marker_forces()
        mk.clear_mpm_external_forces(solid.external_force_n, particle_count=solid.particle_count, read_report=False)
        mk.scatter_marker_forces_to_mpm_particles(
            solid.external_force_n, solid.x, particle_count=solid.particle_count, support_radius_m=self.radius, read_report=False
        )
        dt_sub = cfg.dt_s / cfg.solid_substeps
        for _ in range(cfg.solid_substeps):
            solid.step(
                dt_s=dt_sub, mu_pa=self.mu_pa, lambda_pa=self.lambda_pa, primary_region_id=PRIMARY_REGION_ID,
                secondary_region_id=SECONDARY_REGION_ID, read_report=False,
            )
        mk.update_surface_feedback_from_mpm_surface_particles(
            solid.x, solid.v, solid.surface_normal, solid.area_weight_m2, particle_count=solid.particle_count,
            support_radius_m=self.radius, dt_s=cfg.dt_s, read_report=False,
        )
