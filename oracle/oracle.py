"""Python binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``liboracle_mirror.so`` (the reference's f32/f64 precision mix) or
``liboracle_fp64.so`` (all FP64) built from the C++ restatement in this
directory, and exposes numpy-level wrappers plus ``OracleScene``, the coupled
step of the reference's marker-MPM runner on host arrays.  Only the tests,
``__graft_entry__.smoke`` and the CPU legs of ``bench.py`` use this module; the
product path never imports it.
"""

from __future__ import annotations

import ctypes
import subprocess
from ctypes import POINTER, Structure, byref, c_double, c_float, c_int, c_int32, c_int64, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIBS: dict[str, ctypes.CDLL] = {}


def build(force: bool = False) -> None:
    """Compile both oracle variants with the Makefile in this directory."""
    args = ["make", "-C", str(HERE)]
    if force:
        args.append("-B")
    subprocess.run(args, check=True, capture_output=True)


def load(variant: str = "mirror") -> ctypes.CDLL:
    if variant not in ("mirror", "fp64"):
        raise ValueError("variant must be 'mirror' or 'fp64'")
    if variant not in _LIBS:
        path = HERE / f"liboracle_{variant}.so"
        if not path.exists():
            build()
        _LIBS[variant] = ctypes.CDLL(str(path))
    return _LIBS[variant]


def r32_dtype(variant: str):
    return np.float32 if variant == "mirror" else np.float64


class Level(Structure):
    _fields_ = [("nx", c_int32), ("ny", c_int32), ("nz", c_int32)] + [
        (n, c_void_p) for n in ("wx", "wy", "wz", "cdx", "cdy", "cdz")
    ]


class Grid(Structure):
    _fields_ = [("l0", Level)] + [(n, c_void_p) for n in ("fx", "fy", "fz", "cx", "cy", "cz")]


class CgStats(Structure):
    _fields_ = [
        ("iterations", c_int32),
        ("converged", c_int32),
        ("breakdown_code", c_int32),
        ("breakdown_reason", c_int32),
        ("host_residual_checks", c_int32),
        ("restart_count", c_int32),
        ("mean_projection_count", c_int32),
        ("used_mg", c_int32),
        ("initial_relative_residual", c_double),
        ("relative_residual", c_double),
        ("breakdown_dAd", c_double),
        ("b_norm", c_double),
        ("unreached_set_mean_projection_count", c_int32),
    ]


class MpmState(Structure):
    _fields_ = [
        ("particle_count", c_int32),
        ("nx", c_int32),
        ("ny", c_int32),
        ("nz", c_int32),
        ("bmin", c_double * 3),
        ("dx", c_double * 3),
    ] + [(n, c_void_p) for n in (
        "x", "v", "C", "F", "mass", "volume", "fext", "fixed", "region", "rest_x", "normal", "area",
        "rest_normal", "rest_area", "grid_mass", "grid_vel", "grid_force")]


class MpmReport(Structure):
    _fields_ = [("values", c_double * 28), ("counts", c_int64 * 6)]


class TractionReport(Structure):
    _fields_ = [("valid", c_int64), ("invalid", c_int64), ("two_sided", c_int64), ("one_sided", c_int64), ("max_abs_traction", c_double)]


class ScatterReport(Structure):
    _fields_ = [("active_markers", c_int64), ("invalid_markers", c_int64), ("active_particle_contributions", c_int64),
                ("marker_force", c_double * 3), ("external_force", c_double * 3)]


class FeedbackReport(Structure):
    _fields_ = [("updated", c_int64), ("invalid", c_int64), ("geometry_updated", c_int64), ("geometry_invalid", c_int64),
                ("max_displacement", c_double), ("max_speed", c_double), ("max_normal_change", c_double),
                ("max_area_change", c_double)]


def _p(a: np.ndarray | None):
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("oracle arrays must be C-contiguous")
    return c_void_p(a.ctypes.data)


# ---------------------------------------------------------------------------
# host grid metrics (same order of operations as the reference: running sums)
# ---------------------------------------------------------------------------


def axis_metrics(origin: float, widths) -> dict[str, np.ndarray]:
    widths = [float(w) for w in widths]
    faces = [float(origin)]
    centers = []
    face = float(origin)
    for w in widths:
        centers.append(face + 0.5 * w)
        face += w
        faces.append(faces[-1] + w)
    dist = [widths[0]] + [centers[n] - centers[n - 1] for n in range(1, len(centers))]
    return {"w": np.asarray(widths), "faces": np.asarray(faces), "centers": np.asarray(centers), "cd": np.asarray(dist)}


def multigrid_levels(grid) -> list[list[dict]]:
    """Per-level per-axis metrics (fluid.py:692-729, 1161-1199)."""
    shape = grid.grid_nodes
    shapes = [tuple(shape)]
    cur = shapes[0]
    while min(cur) > 3:
        nxt = tuple(max(2, (n + 1) // 2) for n in cur)
        if nxt == cur:
            break
        shapes.append(nxt)
        cur = nxt
    axes = [list(grid.cell_widths_x_m), list(grid.cell_widths_y_m), list(grid.cell_widths_z_m)]
    levels = []
    for _ in shapes:
        levels.append([axis_metrics(grid.bounds_min_m[a], axes[a]) for a in range(3)])
        axes = [[sum(w[n : min(n + 2, len(w))]) for n in range(0, len(w), 2)] for w in axes]
    return levels


class OracleFluid:
    """Fluid state on host arrays (reference layouts) driven by the oracle."""

    def __init__(self, grid, *, rho: float, mu: float, variant: str = "mirror"):
        self.lib = load(variant)
        self.variant = variant
        self.rt = r32_dtype(variant)
        self.grid = grid
        self.nx, self.ny, self.nz = grid.grid_nodes
        self.rho, self.mu = float(rho), float(mu)
        self.uniform = bool(grid.is_uniform)
        self.metrics = multigrid_levels(grid)
        self._arrays = []
        self.levels = (Level * len(self.metrics))()
        for level, axes in enumerate(self.metrics):
            L = self.levels[level]
            L.nx, L.ny, L.nz = (len(a["w"]) for a in axes)
            for a, name in enumerate("xyz"):
                w = np.ascontiguousarray(axes[a]["w"].astype(np.float32).astype(self.rt))
                cd = np.ascontiguousarray(axes[a]["cd"].astype(np.float32).astype(self.rt))
                self._arrays += [w, cd]
                setattr(L, "w" + name, _p(w))
                setattr(L, "cd" + name, _p(cd))
        m0 = self.metrics[0]
        self.axes_f = []
        for a in range(3):
            fa = np.ascontiguousarray(m0[a]["faces"].astype(np.float32).astype(self.rt))
            ce = np.ascontiguousarray(m0[a]["centers"].astype(np.float32).astype(self.rt))
            self.axes_f.append((fa, ce))
        self.gridstruct = Grid()
        self.gridstruct.l0 = self.levels[0]
        self.gridstruct.fx, self.gridstruct.fy, self.gridstruct.fz = (_p(self.axes_f[a][0]) for a in range(3))
        self.gridstruct.cx, self.gridstruct.cy, self.gridstruct.cz = (_p(self.axes_f[a][1]) for a in range(3))
        shape = (self.nx, self.ny, self.nz)
        self.velocity = np.zeros(shape + (3,), dtype=self.rt)
        self.velocity_prev = np.zeros_like(self.velocity)
        self.pressure = np.zeros(shape, dtype=np.float64)
        self.divergence = np.zeros(shape, dtype=self.rt)
        self.volume_source = np.zeros(shape, dtype=self.rt)
        self.obstacle = np.zeros(shape, dtype=np.int32)
        self.rhs0 = np.zeros(shape, dtype=np.float64)
        self.last_stats = CgStats()

    # single kernels -------------------------------------------------------
    def compute_divergence(self, outlet: int = 0) -> None:
        self.lib.efo_compute_divergence(byref(self.levels[0]), _p(self.obstacle), _p(self.velocity), c_int(outlet), _p(self.divergence))

    def prepare_rhs(self, rhs_scale: float) -> None:
        self.lib.efo_mg_prepare_level0(byref(self.levels[0]), _p(self.obstacle), _p(self.divergence), _p(self.volume_source), None,
                                       c_float(rhs_scale), _p(self.rhs0))

    def fv_apply(self, p: np.ndarray, outlet: int = 0, vdir_active=None, vdir_weight=None, iface=None) -> np.ndarray:
        out = np.zeros_like(p, dtype=np.float64)
        p = np.ascontiguousarray(p, dtype=np.float64)
        self.lib.efo_fv_apply(byref(self.levels[0]), _p(self.obstacle), _p(vdir_active), _p(vdir_weight), _p(iface), _p(p), _p(out), c_int(outlet))
        return out

    def fv_apply_coupled(self, p: np.ndarray, outlet: int = 0, iface=None, *, slots=None, rows=None) -> np.ndarray:
        """The FV operator plus the interface-coupling terms (fluid.py:4345-4456):
        ``slots = (active, neighbor, coefficient, extra_neighbor,
        extra_coefficient)`` per cell, or ``rows = (owner, neighbor,
        transmissibility)``, which take precedence when non-empty."""
        out = self.fv_apply(p, outlet, iface=iface)
        p = np.ascontiguousarray(p, dtype=np.float64)
        shape = (self.nx, self.ny, self.nz)
        if slots is None:
            slots = (np.zeros(shape, np.int32), np.zeros(shape + (3,), np.int32), np.zeros(shape),
                     np.zeros(shape + (15, 3), np.int32), np.zeros(shape + (15,)))
        active, nb, coef, xnb, xcoef = (np.ascontiguousarray(a, dt) for a, dt in zip(
            slots, (np.int32, np.int32, np.float64, np.int32, np.float64)))
        n_extra = int(xcoef.shape[-1])
        if rows is None or len(rows[2]) == 0:
            owner = nbr = np.zeros((1, 3), np.int32)
            trans = np.zeros(1)
            count = 0
        else:
            owner, nbr = (np.ascontiguousarray(a, np.int32).reshape(-1, 3) for a in rows[:2])
            trans = np.ascontiguousarray(rows[2], np.float64)
            count = len(trans)
        self.lib.efo_fv_interface_coupling(byref(self.levels[0]), _p(self.obstacle), _p(p), _p(out), _p(active),
                                           _p(nb), _p(coef), _p(xnb), _p(xcoef), c_int(n_extra), c_int(count),
                                           _p(owner), _p(nbr), _p(trans))
        return out

    def bicgstab(self, rhs, *, outlet: int, max_iters: int, tol: float, b_norm: float,
                 remove_mean: bool = False) -> dict:
        """fluid.py:6264-6533: the BiCGSTAB fallback on the level-0 system
        A p = rhs from the current pressure (efo_bicgstab)."""
        rhs = np.ascontiguousarray(rhs, np.float64)
        stats = np.zeros(4, np.int64)
        rel = c_double(0.0)
        self.lib.efo_bicgstab(byref(self.levels[0]), _p(self.obstacle), _p(rhs), _p(self.pressure), c_int(outlet),
                              c_int(max_iters), c_double(tol), c_double(b_norm), c_int(1 if remove_mean else 0),
                              _p(stats), byref(rel))
        return {"iterations": int(stats[0]), "converged": bool(stats[1]), "restarts": int(stats[2]),
                "breakdown": int(stats[3]), "relative_residual": rel.value}

    def multigrid_solve(self, *, outlet: int, iterations: int, cycles: int) -> None:
        """fluid.py fv_multigrid solve of the prepared rhs (efo_fv_multigrid_solve)."""
        self.lib.efo_fv_multigrid_solve(c_int(len(self.levels)), self.levels, _p(self.obstacle), None, None, None,
                                        _p(self.rhs0), _p(self.pressure), c_int(outlet), c_int(iterations),
                                        c_int(cycles), c_int(1 if self.uniform else 0))

    def project_outlet_multigrid(self, *, dt: float, iterations: int, cycles: int) -> None:
        """project(pressure_outlet_zmin=True, reset_pressure=True,
        pressure_solver="fv_multigrid") without Dirichlet rows (fluid.py:7190-7260):
        boundary conditions, divergence, rhs with the volume source, the MG
        solve, the gradient correction and the boundary conditions again."""
        self._project_outlet(dt, lambda: self.multigrid_solve(outlet=1, iterations=iterations, cycles=cycles))

    def project_outlet_jacobi(self, *, dt: float, iterations: int) -> None:
        """The same with pressure_solver="fv_jacobi": damped Jacobi sweeps
        (omega 0.8) of the level-0 system, the one-level case of
        efo_fv_multigrid_solve (fluid.py:5862-5900)."""
        def solve():
            self.lib.efo_fv_multigrid_solve(c_int(1), self.levels, _p(self.obstacle), None, None, None,
                                            _p(self.rhs0), _p(self.pressure), c_int(1), c_int(iterations), c_int(1),
                                            c_int(1 if self.uniform else 0))
        self._project_outlet(dt, solve)

    def project_outlet_cg(self, *, dt: float, max_iters: int, tol: float, precond: int = 1) -> CgStats:
        """The same with pressure_solver="fv_cg" (flexible PCG, outlet rows,
        no mean projection)."""
        out = []
        self._project_outlet(dt, lambda: out.append(
            self.pcg_solve(outlet=1, max_iters=max_iters, tol=tol, precond=precond, remove_mean=False)))
        return out[0]

    def _project_outlet(self, dt: float, solve) -> None:
        self.apply_closed_boundary(1)
        self.apply_zmin_no_backflow()
        self.compute_divergence(1)
        self.pressure[...] = 0.0
        self.prepare_rhs(self.rho / dt)
        solve()
        self.subtract_pressure_gradient(dt / self.rho, 1)
        self.apply_closed_boundary(1)
        self.apply_zmin_no_backflow()
        self.compute_divergence(1)

    def apply_closed_boundary(self, outlet: int = 0) -> None:
        """fluid.py:5529-5536: the normal velocity on the min faces is zeroed (z-min kept with the outlet)."""
        self.lib.efo_apply_closed_boundary(byref(self.levels[0]), c_int(outlet), _p(self.velocity))

    def apply_zmin_no_backflow(self) -> None:
        """fluid.py:5762-5766: no inflow through the z-min outlet."""
        self.lib.efo_apply_zmin_no_backflow(byref(self.levels[0]), _p(self.obstacle), _p(self.velocity))

    def subtract_pressure_gradient(self, dt_over_rho: float, outlet: int = 0) -> None:
        """fluid.py:5538-5582 _subtract_pressure_gradient_kernel on the current
        pressure (no Dirichlet rows)."""
        self.lib.efo_subtract_pressure_gradient(byref(self.levels[0]), _p(self.obstacle), None, None, None,
                                                _p(self.pressure), c_float(dt_over_rho), c_int(outlet),
                                                _p(self.velocity))

    def spread_surface_forces(self, positions, forces, *, center=(0.0, 0.0, 0.0), force_sign: float = -1.0):
        """fluid.py:3196-3273: surface forces spread trilinearly onto the fluid
        cells as force densities (renormalised over the fluid corners).
        Returns the report: surface force sum (3), grid force sum (3)."""
        pos = np.ascontiguousarray(positions, self.rt).reshape(-1, 3)
        f = np.ascontiguousarray(forces, self.rt).reshape(-1, 3)
        self.force = np.zeros((self.nx, self.ny, self.nz, 3), self.rt)
        report = np.zeros(6)
        self.lib.efo_spread_surface_forces(byref(self.gridstruct), _p(self.obstacle), _p(pos), _p(f), c_int(len(pos)),
                                           c_float(center[0]), c_float(center[1]), c_float(center[2]),
                                           c_float(force_sign), _p(self.force), _p(report))
        return report

    def apply_body_force(self, dt: float) -> None:
        """fluid.py:3301-3328: u += f dt / rho on the fluid cells."""
        self.lib.efo_apply_body_force(byref(self.levels[0]), _p(self.obstacle), _p(self.force), c_float(dt),
                                      c_float(self.rho), _p(self.velocity))

    def fv_diagonal(self, outlet: int = 0, vdir_active=None, vdir_weight=None, iface=None) -> np.ndarray:
        out = np.zeros((self.nx, self.ny, self.nz), dtype=np.float64)
        self.lib.efo_fv_diagonal(byref(self.levels[0]), _p(self.obstacle), _p(vdir_active), _p(vdir_weight), _p(iface), _p(out), c_int(outlet))
        return out

    def weighted_dot(self, a: np.ndarray, b: np.ndarray) -> float:
        self.lib.efo_weighted_dot.restype = c_double
        return float(self.lib.efo_weighted_dot(byref(self.levels[0]), _p(self.obstacle), _p(np.ascontiguousarray(a, dtype=np.float64)),
                                               _p(np.ascontiguousarray(b, dtype=np.float64))))

    def restrict(self, res: np.ndarray, iface=None, vdir_active=None, vdir_weight=None):
        """Level 0 -> 1 restriction of a fine residual (fluid.py:5310-5388):
        coarse rhs, interface diagonal, obstacle, Dirichlet flag and weight."""
        C = self.levels[1]
        shape = (C.nx, C.ny, C.nz)
        crhs = np.zeros(shape, self.rt)
        ciface = np.zeros(shape, self.rt)
        cobs = np.zeros(shape, np.int32)
        cva = np.zeros(shape, np.int32)
        cvw = np.zeros(shape, self.rt)
        self.lib.efo_mg_restrict_f64(byref(self.levels[0]), _p(np.ascontiguousarray(res, dtype=np.float64)), _p(iface),
                                     _p(self.obstacle), _p(vdir_active), _p(vdir_weight), byref(C), _p(crhs), _p(ciface),
                                     _p(cobs), _p(cva), _p(cvw))
        return {"rhs": crhs, "iface": ciface, "obstacle": cobs, "vdir_active": cva, "vdir_weight": cvw}

    def jacobi_sweep_coarse(self, level: int, p, rhs, iface, obstacle, omega: float, outlet: int = 0) -> np.ndarray:
        """One damped-Jacobi sweep (fluid.py:4224-4273) on a coarse (f32) level."""
        L = self.levels[level]
        out = np.zeros((L.nx, L.ny, L.nz), self.rt)
        args = [np.ascontiguousarray(a, dtype=self.rt) for a in (p, rhs, iface)]
        self.lib.efo_jacobi_sweep_r32(byref(L), *(_p(a) for a in args), _p(np.ascontiguousarray(obstacle, dtype=np.int32)),
                                      None, None, _p(out), c_int(outlet), c_double(omega))
        return out

    def vcycle(self, r: np.ndarray, outlet: int = 0, pre: int = 2, coarse: int = 24, post: int = 2) -> np.ndarray:
        z = np.zeros_like(r, dtype=np.float64)
        self.lib.efo_mg_vcycle(c_int(len(self.metrics)), self.levels, _p(self.obstacle), None, None, None,
                               _p(np.ascontiguousarray(r, dtype=np.float64)), _p(z), c_int(outlet), c_int(pre), c_int(coarse),
                               c_int(post), c_int(1 if self.uniform else 0))
        return z

    def pcg_solve(self, *, outlet: int, max_iters: int, tol: float, precond: int, remove_mean: bool,
                  components=None, component_count: int = 0) -> CgStats:
        """The flexible PCG; with an outlet, `components` (int32 per cell, -1
        outside the anchored set) and `component_count` anchor the unreached
        components as fluid.py:6582-6789 does."""
        st = CgStats()
        comp = None if components is None else np.ascontiguousarray(components, dtype=np.int32)
        self.lib.efo_fv_pcg_solve_anchored(c_int(len(self.metrics)), self.levels, _p(self.obstacle), None, None, None,
                                           _p(self.rhs0), _p(self.pressure), c_int(outlet), c_int(max_iters),
                                           c_double(tol), c_int(precond), c_int(1 if remove_mean else 0),
                                           c_int(1 if self.uniform else 0), c_int(0), None if comp is None else _p(comp),
                                           c_int(int(component_count) if comp is not None else 0), byref(st))
        self.last_stats = st
        return st

    def predict(self, dt: float, rk2: bool = False) -> None:
        """fluid.py:2447-2527: semi-Lagrangian predictor (Euler backtrace, or
        the RK2 midpoint with ``rk2``) plus explicit viscosity."""
        self.velocity_prev[...] = self.velocity
        self.lib.efo_predict(byref(self.gridstruct), _p(self.obstacle), _p(self.velocity_prev), c_float(dt),
                             c_float(self.mu / self.rho), c_int(1 if rk2 else 0), _p(self.velocity))

    def apply_velocity_dirichlet_rows(self, active, value) -> None:
        """fluid.py:2549-2593: velocity = row value on active fluid cells."""
        self.lib.efo_apply_velocity_dirichlet_rows(ctypes.c_int64(self.obstacle.size), _p(self.obstacle),
                                                   _p(np.ascontiguousarray(active, np.int32)),
                                                   _p(np.ascontiguousarray(value, self.rt)), _p(self.velocity))

    def project(self, *, dt: float, max_iters: int = 400, tol: float = 1.0e-8, precond: int = 1) -> CgStats:
        """Plain closed-box fv_cg projection (fluid.py:6889-7340 without Dirichlet rows)."""
        self.compute_divergence(0)
        self.prepare_rhs(self.rho / dt)
        st = self.pcg_solve(outlet=0, max_iters=max_iters, tol=tol, precond=precond, remove_mean=True)
        if not st.converged:
            self.pressure[...] = 0.0
        self.lib.efo_subtract_pressure_gradient(byref(self.levels[0]), _p(self.obstacle), None, None, None, _p(self.pressure),
                                                c_float(dt / self.rho), c_int(0), _p(self.velocity))
        self.compute_divergence(0)
        self.lib.efo_apply_closed_boundary(byref(self.levels[0]), c_int(0), _p(self.velocity))
        return st


class OracleSolid:
    def __init__(self, *, capacity: int, grid_nodes, bounds_min=(0.0, 0.0, 0.0), bounds_max=(1.0, 1.0, 1.0), variant="mirror"):
        self.lib = load(variant)
        self.rt = r32_dtype(variant)
        self.nodes = tuple(int(n) for n in grid_nodes)
        self.bmin = tuple(float(v) for v in bounds_min)
        self.dx = tuple((float(bounds_max[a]) - self.bmin[a]) / self.nodes[a] for a in range(3))
        P = int(capacity)
        rt = self.rt
        self.count = 0
        self.x = np.zeros((P, 3), rt)
        self.v = np.zeros((P, 3), rt)
        self.C = np.zeros((P, 3, 3), rt)
        self.F = np.tile(np.eye(3, dtype=rt), (P, 1, 1))
        self.mass = np.zeros(P, rt)
        self.volume = np.zeros(P, rt)
        self.fext = np.zeros((P, 3), rt)
        self.fixed = np.zeros(P, np.int32)
        self.region = np.zeros(P, np.int32)
        self.rest_x = np.zeros((P, 3), rt)
        self.normal = np.zeros((P, 3), rt)
        self.area = np.zeros(P, rt)
        self.rest_normal = np.zeros((P, 3), rt)
        self.rest_area = np.zeros(P, rt)
        self.grid_mass = np.zeros(self.nodes, rt)
        self.grid_vel = np.zeros(self.nodes + (3,), rt)
        self.grid_force = np.zeros(self.nodes + (3,), rt)

    def load(self, *, x, volume, mass, region=None, normal=None, area=None, fixed=None) -> None:
        n = x.shape[0]
        self.count = n
        self.x[:n] = x
        self.rest_x[:n] = x
        self.volume[:n] = volume
        self.mass[:n] = mass
        if region is not None:
            self.region[:n] = region
        if normal is not None:
            self.normal[:n] = normal
            self.rest_normal[:n] = normal
        if area is not None:
            self.area[:n] = area
            self.rest_area[:n] = area
        if fixed is not None:
            self.fixed[:n] = fixed

    def step(self, *, dt: float, mu: float, lam: float, damping: float = 1.0, primary: int = 101, secondary: int = 202):
        s = MpmState()
        s.particle_count = self.count
        s.nx, s.ny, s.nz = self.nodes
        for a in range(3):
            s.bmin[a] = float(np.float32(self.bmin[a]))
            s.dx[a] = float(np.float32(self.dx[a]))
        for name in ("x", "v", "C", "F", "mass", "volume", "fext", "fixed", "region", "rest_x", "normal", "area",
                     "rest_normal", "rest_area", "grid_mass", "grid_vel", "grid_force"):
            setattr(s, name, _p(getattr(self, name)))
        rep = MpmReport()
        self.lib.efo_mpm_step(byref(s), c_float(dt), c_float(mu), c_float(lam), c_float(damping), c_int(primary), c_int(secondary), byref(rep))
        return rep


class OracleMarkers:
    def __init__(self, *, x, normal, area, region, variant="mirror"):
        self.lib = load(variant)
        rt = r32_dtype(variant)
        self.count = x.shape[0]
        self.x = np.ascontiguousarray(x, dtype=rt)
        self.v = np.zeros_like(self.x)
        self.n = np.ascontiguousarray(normal, dtype=rt)
        self.A = np.ascontiguousarray(area, dtype=rt)
        self.region = np.ascontiguousarray(region, dtype=np.int32)
        self.t = np.zeros((self.count, 3), np.float64)
        self.F = np.zeros((self.count, 3), np.float64)
        self.valid = np.zeros(self.count, np.int32)

    def sample_tractions(self, fluid: OracleFluid, *, two_sided: int = 0, one_sided_region: int = -1, one_sided_ref: float = 0.0):
        rep = TractionReport()
        self.lib.efo_sample_pressure_tractions(byref(fluid.gridstruct), _p(fluid.obstacle), _p(fluid.pressure), c_int(self.count),
                                               _p(self.x), _p(self.n), _p(self.region), c_int(two_sided), c_int(one_sided_region),
                                               c_float(one_sided_ref), _p(self.t), _p(self.valid), byref(rep))
        return rep

    def compute_forces(self) -> None:
        self.lib.efo_compute_marker_forces(c_int(self.count), _p(self.t), _p(self.A), _p(self.F))

    def clear(self, solid: OracleSolid):
        cleared, mx = c_int64(0), c_double(0.0)
        self.lib.efo_clear_external_forces(c_int(solid.count), _p(solid.fext), byref(cleared), byref(mx))
        return cleared.value, mx.value

    def scatter(self, solid: OracleSolid, radius: float):
        rep = ScatterReport()
        self.lib.efo_scatter_marker_forces(c_int(self.count), _p(self.x), _p(self.F), c_int(solid.count), _p(solid.x),
                                           c_float(radius), _p(solid.fext), byref(rep))
        return rep

    def feedback(self, solid: OracleSolid, radius: float, dt: float, geometry: bool = True):
        rep = FeedbackReport()
        self.lib.efo_surface_feedback(c_int(self.count), _p(self.x), _p(self.v), _p(self.n), _p(self.A), c_int(solid.count),
                                      _p(solid.x), _p(solid.v), _p(solid.normal) if geometry else None,
                                      _p(solid.area) if geometry else None, c_float(radius), c_float(dt), byref(rep))
        return rep


def ib_node_search(*, grid_nodes, markers_x, markers_n, triangles=None, search_radius: float,
                   interior_probe_distance: float, sign_tolerance: float, classify_far: bool = False,
                   centers=None, bounds_min=None, spacing=None, variant: str = "mirror") -> dict:
    """Immersed-boundary node search and classification of every node
    (oracle_ibsearch.cpp; hibm_mpm.py:5603-6068).  Node positions are the
    centre arrays ``centers = (cx, cy, cz)`` when given, else ``bounds_min +
    (i + 0.5) * spacing``.  Returns the per-node fields and the four report
    counts."""
    lib = load(variant)
    rt = r32_dtype(variant)
    nx, ny, nz = (int(v) for v in grid_nodes)
    mx = np.ascontiguousarray(markers_x, dtype=rt).reshape(-1, 3)
    mn = np.ascontiguousarray(markers_n, dtype=rt).reshape(-1, 3)
    tri = np.zeros((0, 3), np.int32) if triangles is None else np.ascontiguousarray(triangles, dtype=np.int32).reshape(-1, 3)
    if centers is not None:
        cx, cy, cz = (np.ascontiguousarray(c, dtype=rt) for c in centers)
        bmin = sp = None
    else:
        cx = cy = cz = None
        bmin = np.ascontiguousarray(bounds_min, dtype=rt)
        sp = np.ascontiguousarray(spacing, dtype=rt)
    shape = (nx, ny, nz)
    out = {
        "kind": np.zeros(shape, np.int32),
        "nearest_marker": np.zeros(shape, np.int32),
        "signed_distance": np.zeros(shape, rt),
        "boundary_point": np.zeros(shape + (3,), rt),
        "interior_point": np.zeros(shape + (3,), rt),
        "projection_indices": np.zeros(shape + (3,), np.int32),
        "projection_weights": np.zeros(shape + (3,), rt),
    }
    report = np.zeros(4, np.int64)
    real = c_float if rt == np.float32 else c_double
    lib.efo_ib_node_search(
        c_int(nx), c_int(ny), c_int(nz), _p(cx), _p(cy), _p(cz), _p(bmin), _p(sp), _p(mx), _p(mn), c_int(mx.shape[0]),
        _p(tri), c_int(tri.shape[0]), real(search_radius), real(interior_probe_distance), real(sign_tolerance),
        c_int(1 if classify_far else 0), _p(out["kind"]), _p(out["nearest_marker"]), _p(out["signed_distance"]),
        _p(out["boundary_point"]), _p(out["interior_point"]), _p(out["projection_indices"]),
        _p(out["projection_weights"]), _p(report),
    )
    out["report"] = dict(zip(("near_boundary_node_count", "external_ib_node_count", "internal_node_count",
                              "invalid_projection_count"), (int(v) for v in report)))
    return out


def ib_build_boundary_conditions(search: dict, *, markers_v, markers_n, marker_gradients,
                                 variant: str = "mirror") -> dict:
    """hibm_mpm.py:6499-6577 on the fields of ``ib_node_search``: per-node
    no-slip velocity, Neumann normal and gradient targets of the external IB
    nodes, and the report (no-slip rows, Neumann rows, inactive internal
    nodes, max |v|)."""
    lib = load(variant)
    rt = r32_dtype(variant)
    kind = np.ascontiguousarray(search["kind"], np.int32)
    shape = kind.shape
    n = int(kind.size)
    mv = np.ascontiguousarray(markers_v, dtype=rt).reshape(-1, 3)
    mn = np.ascontiguousarray(markers_n, dtype=rt).reshape(-1, 3)
    mg = np.ascontiguousarray(marker_gradients, dtype=rt).reshape(-1)
    out = {
        "active": np.zeros(shape, np.int32),
        "velocity": np.zeros(shape + (3,), rt),
        "normal": np.zeros(shape + (3,), rt),
        "gradient": np.zeros(shape, rt),
    }
    report = np.zeros(4, np.float64)
    lib.efo_ib_build_boundary_conditions(
        c_int64(n), _p(kind), _p(np.ascontiguousarray(search["nearest_marker"], np.int32)),
        _p(np.ascontiguousarray(search["projection_indices"], np.int32)),
        _p(np.ascontiguousarray(search["projection_weights"], rt)), _p(mv), _p(mn), _p(mg), c_int(mv.shape[0]),
        _p(out["active"]), _p(out["velocity"]), _p(out["normal"]), _p(out["gradient"]), _p(report))
    out["report"] = {"no_slip_dirichlet_count": int(report[0]), "pressure_neumann_count": int(report[1]),
                     "inactive_internal_node_count": int(report[2]), "max_abs_velocity_mps": float(report[3])}
    return out


def outlet_reachability(obstacle, *, velocity_dirichlet_active=None, barrier=None, variant: str = "mirror") -> dict:
    """z-min outlet pressure reachability and the unreached components
    (fluid.py:1649-1876, 4764-4910): per-cell reachable flags, component
    labels (-(rank + 1) for unreached cells, 1 << 30 elsewhere), the unreached
    count, component count, sweep count and convergence flags."""
    lib = load(variant)
    obs = np.ascontiguousarray(obstacle, np.int32)
    nx, ny, nz = obs.shape
    vd = None if velocity_dirichlet_active is None else np.ascontiguousarray(velocity_dirichlet_active, np.int32)
    br = None if barrier is None else np.ascontiguousarray(barrier, np.int32)
    reach = np.zeros(obs.shape, np.int32)
    label = np.zeros(obs.shape, np.int32)
    info = np.zeros(5, np.int64)
    lib.efo_outlet_reachability.restype = c_int64
    unreached = lib.efo_outlet_reachability(c_int(nx), c_int(ny), c_int(nz), _p(obs), _p(vd), _p(br), _p(reach),
                                            _p(label), _p(info))
    return {"reachable": reach, "label": label, "unreached": int(unreached), "components": int(info[0]),
            "sweeps": int(info[1]), "converged": bool(info[2]), "labels_converged": bool(info[3]),
            "overflow": bool(info[4])}


VD_REPORT_KEYS = (
    "active_velocity_dirichlet_rows", "inactive_obstacle_rows", "max_abs_velocity_mps",
    "invalid_reconstruction_row_count", "invalid_no_fluid_sample_row_count", "invalid_nonpositive_gap_row_count",
    "invalid_node_behind_boundary_row_count", "invalid_node_beyond_interior_row_count",
    "narrow_gap_boundary_velocity_row_count", "relocated_row_count", "relocation_merged_row_count",
    "relocation_blocked_row_count", "min_projection_weight", "max_projection_weight",
)


def ib_velocity_dirichlet_rows(grid, *, active_ib, bc_velocity, bc_normal, boundary_point, interior_point,
                               obstacle, velocity, nearest_marker=None, marker_region=None, region_out=None,
                               variant: str = "mirror") -> dict:
    """assemble_velocity_dirichlet_reconstructed_boundary_rows
    (hibm_mpm.py:7655-7800) on host arrays: ``grid`` is a CartesianGrid
    (faces and centres as the fluid's f32 fields); the boundary fields come
    from ``ib_build_boundary_conditions`` and the points from
    ``ib_node_search``.  ``region_out`` (int32 per node) is stamped in place
    when ``marker_region`` is given."""
    lib = load(variant)
    rt = r32_dtype(variant)
    nx, ny, nz = grid.grid_nodes
    shape = (nx, ny, nz)
    faces = [np.ascontiguousarray(grid.axis_faces(a), rt) for a in range(3)]
    centres = [np.ascontiguousarray(grid.axis_centers(a), rt) for a in range(3)]
    f32 = lambda a, extra=(): np.ascontiguousarray(np.broadcast_to(np.asarray(a, rt), shape + extra))  # noqa: E731
    i32 = lambda a, extra=(): np.ascontiguousarray(np.broadcast_to(np.asarray(a, np.int32), shape + extra))  # noqa: E731
    act, obs = i32(active_ib), i32(obstacle)
    bv, bn, bp, ip, vel = (f32(a, (3,)) for a in (bc_velocity, bc_normal, boundary_point, interior_point, velocity))
    near = i32(-1 if nearest_marker is None else nearest_marker)
    regions = None if marker_region is None else np.ascontiguousarray(marker_region, np.int32)
    out = {
        "active": np.zeros(shape, np.int32),
        "value": np.zeros(shape + (3,), rt),
        "weight": np.zeros(shape, rt),
        "anchor": np.zeros(shape + (3,), np.int32),
    }
    if regions is not None and region_out is None:
        region_out = np.zeros(shape, np.int32)
    report = np.zeros(14, np.float64)
    lib.efo_ib_velocity_dirichlet_rows(
        c_int(nx), c_int(ny), c_int(nz), *(_p(a) for a in faces), *(_p(a) for a in centres), _p(act), _p(bv), _p(bn),
        _p(bp), _p(ip), _p(near), _p(obs), _p(vel), _p(regions), c_int(0 if regions is None else len(regions)),
        _p(out["active"]), _p(out["value"]), _p(out["weight"]), _p(out["anchor"]),
        _p(region_out) if regions is not None else None, _p(report))
    out["region"] = region_out
    out["report"] = {k: (float(v) if k in ("max_abs_velocity_mps", "min_projection_weight", "max_projection_weight")
                         else int(v)) for k, v in zip(VD_REPORT_KEYS, report)}
    return out


class OracleScene:
    """The coupled step of easyfsi_b200.scenarios.CoupledScene on host arrays."""

    def __init__(self, cfg, *, variant: str = "mirror", initial_velocity=None, project_initial: bool = True):
        from easyfsi_b200 import scenarios as sc

        self.cfg = cfg
        self.grid = sc.build_grid(cfg)
        self.fluid = OracleFluid(self.grid, rho=cfg.density_kgm3, mu=cfg.viscosity_pa_s, variant=variant)
        self.fluid.obstacle[...] = sc.obstacle_mask(self.grid, cfg.bodies)
        u0 = initial_velocity if initial_velocity is not None else sc.fourier_velocity(
            self.grid, cfg.velocity_seed, cfg.amplitude_mps, cfg.max_wavenumber)
        self.fluid.velocity[...] = u0
        if project_initial:
            self.fluid.project(dt=cfg.dt_s, max_iters=cfg.cg_max_iterations, tol=cfg.cg_tolerance)
            self.fluid.pressure[...] = 0.0
        part = sc.particles(cfg)
        self.solid = OracleSolid(capacity=part["x"].shape[0], grid_nodes=cfg.mpm_nodes, variant=variant)
        self.solid.load(x=part["x"], volume=part["volume"], mass=part["mass"], region=part["region"], normal=part["normal"],
                        area=part["area"])
        mk = sc.markers(cfg)
        self.markers = OracleMarkers(x=mk["x"], normal=mk["normal"], area=mk["area"], region=mk["region"], variant=variant)
        self.mu, self.lam = sc.material(cfg)
        self.radius = sc.support_radius(cfg)
        self.last_stats = None

    def step(self) -> None:
        cfg = self.cfg
        self.fluid.predict(cfg.dt_s)
        self.last_stats = self.fluid.project(dt=cfg.dt_s, max_iters=cfg.cg_max_iterations, tol=cfg.cg_tolerance)
        self.markers.sample_tractions(self.fluid, two_sided=0)
        self.markers.compute_forces()
        self.markers.clear(self.solid)
        self.markers.scatter(self.solid, self.radius)
        for _ in range(cfg.solid_substeps):
            self.solid.step(dt=cfg.dt_s / cfg.solid_substeps, mu=self.mu, lam=self.lam)
        self.markers.feedback(self.solid, self.radius, cfg.dt_s, geometry=True)
