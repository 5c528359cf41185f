"""HIBM surface markers, B200 path (drop-in for the marker part of
simulation_core/hibm_mpm.py, class HibmMpmSurfaceMarkers :279).

Provides the coupled-step members of the reference class with their
signatures: ``load_markers`` (:553), ``set_marker_tractions_pa`` (:893),
``compute_marker_forces`` (:908), the pressure-only fast path of
``sample_fluid_stress_to_marker_tractions`` (:3710 -> :2253),
``aggregate_region_forces`` (:5291), ``clear_mpm_external_forces`` (:4880),
``scatter_marker_forces_to_mpm_particles`` (:4961) and the two surface-feedback
updates (:5055, :5182).  Every method accepts an extra ``read_report=False``
keyword that skips the host read of its report (the report is then ``None``).

Projection triangles (``set_projection_triangles`` :590), the IB node search
(class ``HibmMpmIbNodeSearch`` :5385) and the boundary-condition targets and
velocity-Dirichlet rows built from it (class ``HibmMpmIbBoundaryConditions``
:6222, without its pressure-Neumann rows) are provided too.  The viscous /
closure stress sampler of the reference is outside the hot path and not
provided.
"""

from __future__ import annotations

import math
from ctypes import byref, c_float, c_void_p
from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from .field import Field
from .runtime import TaichiRuntimeConfig, current_stream_handle, f32, f64, i32, init_runtime


def _vector3(value, *, name: str) -> tuple[float, float, float]:
    if len(value) != 3:
        raise ValueError(f"{name} must contain exactly 3 components")
    out = tuple(float(v) for v in value)
    if not all(math.isfinite(v) for v in out):
        raise ValueError(f"{name} must contain finite values")
    return out  # type: ignore[return-value]


def _normalize_vector3(value, *, name: str) -> tuple[float, float, float]:
    v = _vector3(value, name=name)
    n = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    if n <= 1.0e-12:
        raise ValueError(f"{name} must be non-zero")
    return (v[0] / n, v[1] / n, v[2] / n)


@dataclass(frozen=True)
class HibmMpmFluidStressSampleReport:
    valid_marker_count: int
    invalid_marker_count: int
    max_abs_traction_pa: float
    two_sided_pressure_marker_count: int = 0
    one_sided_pressure_marker_count: int = 0


@dataclass(frozen=True)
class HibmMpmSurfaceMarkerForceReport:
    primary_marker_force_n: tuple[float, float, float]
    secondary_marker_force_n: tuple[float, float, float]
    total_marker_force_n: tuple[float, float, float]
    primary_marker_count: int
    secondary_marker_count: int
    total_marker_count: int
    fluid_reaction_force_n: tuple[float, float, float]
    action_reaction_residual_n: float
    primary_stress_valid_marker_count: int = 0
    primary_stress_invalid_marker_count: int = 0
    secondary_stress_valid_marker_count: int = 0
    secondary_stress_invalid_marker_count: int = 0
    primary_marker_force_norm_sum_n: float = 0.0
    secondary_marker_force_norm_sum_n: float = 0.0
    total_marker_force_norm_sum_n: float = 0.0
    primary_marker_force_norm_max_n: float = 0.0
    secondary_marker_force_norm_max_n: float = 0.0
    total_marker_force_norm_max_n: float = 0.0


@dataclass(frozen=True)
class HibmMpmExternalForceClearReport:
    cleared_particle_count: int
    max_abs_external_force_before_n: float


@dataclass(frozen=True)
class HibmMpmMpmForceScatterReport:
    active_marker_count: int
    invalid_marker_count: int
    active_particle_count: int
    total_marker_force_n: tuple[float, float, float]
    total_mpm_external_force_n: tuple[float, float, float]
    action_reaction_residual_n: float


@dataclass(frozen=True)
class HibmMpmSurfaceUpdateReport:
    updated_marker_count: int
    invalid_marker_count: int
    max_marker_displacement_m: float
    max_marker_speed_mps: float
    geometry_updated_marker_count: int = 0
    geometry_invalid_marker_count: int = 0
    max_marker_normal_change: float = 0.0
    max_marker_area_change_m2: float = 0.0


def _tensor(field_or_tensor) -> torch.Tensor:
    return field_or_tensor.tensor if isinstance(field_or_tensor, Field) else field_or_tensor


class HibmMpmSurfaceMarkers:
    def __init__(self, marker_capacity: int, projection_triangle_capacity: int | None = None, runtime: TaichiRuntimeConfig | None = None) -> None:
        self.device = init_runtime(runtime)
        if int(marker_capacity) <= 0:
            raise ValueError("marker_capacity must be positive")
        self.marker_capacity = int(marker_capacity)
        if projection_triangle_capacity is None:
            projection_triangle_capacity = self.marker_capacity
        if int(projection_triangle_capacity) <= 0:
            raise ValueError("projection_triangle_capacity must be positive")
        self.projection_triangle_capacity = int(projection_triangle_capacity)
        self.marker_count = 0
        self.projection_triangle_count = 0
        cap, dev = self.marker_capacity, self.device
        self.x_gamma_m = Field((cap,), f32, n=3, device=dev)
        self.v_gamma_mps = Field((cap,), f32, n=3, device=dev)
        self.n_gamma = Field((cap,), f32, n=3, device=dev)
        self.A_gamma_m2 = Field((cap,), f32, device=dev)
        self.region_id = Field((cap,), i32, device=dev)
        self.t_gamma_pa = Field((cap,), f64, n=3, device=dev)
        self._stress_pressure_valid = Field((cap,), i32, device=dev)
        self.F_gamma_n = Field((cap,), f64, n=3, device=dev)
        self.projection_triangle_indices = Field((self.projection_triangle_capacity,), i32, n=3, device=dev)
        self._report = torch.zeros(16, dtype=torch.float64, device=dev)
        self._bins: dict = {}

    def __del__(self):
        for plan in getattr(self, "_bins", {}).values():
            try:
                _native.load().efsi_bin_plan_destroy(plan[0])
            except Exception:
                pass

    # ------------------------------------------------------------------
    def load_markers(self, *, positions_m, velocities_mps, normals, areas_m2, region_ids) -> None:
        count = len(positions_m)
        if count > self.marker_capacity:
            raise ValueError("marker count exceeds marker_capacity")
        if not (len(velocities_mps) == len(normals) == len(areas_m2) == len(region_ids) == count):
            raise ValueError("marker inputs must have matching lengths")
        pos = np.zeros((self.marker_capacity, 3), dtype=np.float32)
        vel = np.zeros_like(pos)
        nor = np.zeros_like(pos)
        area = np.zeros(self.marker_capacity, dtype=np.float32)
        reg = np.zeros(self.marker_capacity, dtype=np.int32)
        for m in range(count):
            pos[m] = _vector3(positions_m[m], name="positions_m")
            vel[m] = _vector3(velocities_mps[m], name="velocities_mps")
            nor[m] = _normalize_vector3(normals[m], name="normals")
            a = float(areas_m2[m])
            if not math.isfinite(a) or a < 0.0:
                raise ValueError("areas_m2 must contain finite non-negative values")
            area[m] = a
            reg[m] = int(region_ids[m])
        self.marker_count = int(count)
        self.projection_triangle_count = 0
        self.x_gamma_m.from_numpy(pos)
        self.v_gamma_mps.from_numpy(vel)
        self.n_gamma.from_numpy(nor)
        self.A_gamma_m2.from_numpy(area)
        self.region_id.from_numpy(reg)
        self.t_gamma_pa.tensor.zero_()
        self.F_gamma_n.tensor.zero_()

    def set_projection_triangles(self, triangle_indices) -> int:
        """hibm_mpm.py:590-615: marker-index triangles used by the IB node
        search's closest-point projection."""
        count = len(triangle_indices)
        if count > self.projection_triangle_capacity:
            raise ValueError("projection triangle count exceeds projection_triangle_capacity")
        marker_count = int(self.marker_count)
        tri = np.zeros((self.projection_triangle_capacity, 3), dtype=np.int32)
        for t, triangle in enumerate(triangle_indices):
            if len(triangle) != 3:
                raise ValueError("projection triangles must contain three indices")
            ia, ib, ic = (int(triangle[0]), int(triangle[1]), int(triangle[2]))
            if min(ia, ib, ic) < 0 or max(ia, ib, ic) >= marker_count:
                raise ValueError("projection triangle index out of marker range")
            tri[t] = (ia, ib, ic)
        self.projection_triangle_indices.from_numpy(tri)
        self.projection_triangle_count = int(count)
        return self.projection_triangle_count

    def set_marker_tractions_pa(self, tractions_pa) -> None:
        if len(tractions_pa) != self.marker_count:
            raise ValueError("tractions_pa must match marker_count")
        t = np.zeros((self.marker_capacity, 3), dtype=np.float64)
        for m in range(self.marker_count):
            t[m] = _vector3(tractions_pa[m], name="tractions_pa")
        self.t_gamma_pa.from_numpy(t)

    def compute_marker_forces(self) -> None:
        _native.call(
            "efsi_compute_marker_forces",
            int(self.marker_count),
            self.t_gamma_pa.ptr(),
            self.A_gamma_m2.ptr(),
            self.F_gamma_n.ptr(),
            c_void_p(current_stream_handle()),
        )

    # ------------------------------------------------------------------
    def sample_fluid_stress_to_marker_tractions(
        self,
        velocity_field,
        pressure_field,
        obstacle_field,
        cell_face_x_m,
        cell_face_y_m,
        cell_face_z_m,
        cell_center_x_m,
        cell_center_y_m,
        cell_center_z_m,
        cell_width_x_m,
        cell_width_y_m,
        cell_width_z_m,
        grid_nodes,
        *,
        viscosity_pa_s: float,
        two_sided_pressure: bool = False,
        far_pressure_region_id: int = -1,
        far_pressure_pa: float = 0.0,
        far_pressure_side_normal_sign: float = 0.0,
        far_pressure_inside_probe_max_multiplier: float = 3.0,
        two_sided_probe_max_multiplier: float = 3.0,
        one_sided_pressure_region_id: int = -1,
        one_sided_reference_pressure_pa: float = 0.0,
        one_sided_probe_max_multiplier: float = 3.0,
        use_pressure_anchor_fallback: bool = False,
        node_anchor_cell=None,
        sampling_obstacle_field=None,
        read_report: bool = True,
    ) -> HibmMpmFluidStressSampleReport | None:
        nodes = tuple(int(v) for v in grid_nodes)
        if len(nodes) != 3 or any(v < 2 for v in nodes):
            raise ValueError("grid_nodes must contain three values >= 2")
        viscosity = float(viscosity_pa_s)
        if not math.isfinite(viscosity) or viscosity < 0.0:
            raise ValueError("viscosity_pa_s must be a finite non-negative number")
        if not math.isfinite(float(far_pressure_pa)):
            raise ValueError("far_pressure_pa must be a finite number")
        if float(far_pressure_side_normal_sign) not in (-1.0, 0.0, 1.0):
            raise ValueError("far_pressure_side_normal_sign must be -1.0, 0.0, or 1.0")
        for value, name in (
            (far_pressure_inside_probe_max_multiplier, "far_pressure_inside_probe_max_multiplier"),
            (two_sided_probe_max_multiplier, "two_sided_probe_max_multiplier"),
            (one_sided_probe_max_multiplier, "one_sided_probe_max_multiplier"),
        ):
            if not math.isfinite(float(value)) or float(value) < 3.0:
                raise ValueError(f"{name} must be finite and >= 3.0")
        if not math.isfinite(float(one_sided_reference_pressure_pa)):
            raise ValueError("one_sided_reference_pressure_pa must be a finite number")
        fast_path = (
            viscosity == 0.0
            and int(far_pressure_region_id) < 0
            and not bool(use_pressure_anchor_fallback)
            and node_anchor_cell is None
            and sampling_obstacle_field is None
        )
        if not fast_path:
            raise NotImplementedError(
                "only the pressure-only traction sampler (hibm_mpm.py:2253) is on the B200 hot path"
            )
        p = _tensor(pressure_field)
        if p.dtype != torch.float64:
            p = p.to(torch.float64)
        p = p.contiguous()
        axes = _native.GridAxes(
            _tensor(cell_face_x_m).data_ptr(),
            _tensor(cell_face_y_m).data_ptr(),
            _tensor(cell_face_z_m).data_ptr(),
            _tensor(cell_center_x_m).data_ptr(),
            _tensor(cell_center_y_m).data_ptr(),
            _tensor(cell_center_z_m).data_ptr(),
        )
        rep = self._report
        _native.call(
            "efsi_sample_pressure_tractions",
            nodes[0],
            nodes[1],
            nodes[2],
            byref(axes),
            c_void_p(_tensor(cell_width_x_m).data_ptr()),
            c_void_p(_tensor(cell_width_y_m).data_ptr()),
            c_void_p(_tensor(cell_width_z_m).data_ptr()),
            c_void_p(_tensor(obstacle_field).data_ptr()),
            c_void_p(p.data_ptr()),
            int(self.marker_count),
            self.x_gamma_m.ptr(),
            self.n_gamma.ptr(),
            self.region_id.ptr(),
            1 if two_sided_pressure else 0,
            int(one_sided_pressure_region_id),
            float(one_sided_reference_pressure_pa),
            self.t_gamma_pa.ptr(),
            self._stress_pressure_valid.ptr(),
            c_void_p(rep.data_ptr()),
            c_void_p(current_stream_handle()),
        )
        if not read_report:
            return None
        r = rep[:5].cpu().tolist()
        return HibmMpmFluidStressSampleReport(
            valid_marker_count=int(r[0]),
            invalid_marker_count=int(r[1]),
            max_abs_traction_pa=float(r[4]),
            two_sided_pressure_marker_count=int(r[2]),
            one_sided_pressure_marker_count=int(r[3]),
        )

    def aggregate_region_forces(self, *, primary_region_id: int, secondary_region_id: int) -> HibmMpmSurfaceMarkerForceReport:
        n = int(self.marker_count)
        F = self.F_gamma_n.tensor[:n]
        reg = self.region_id.tensor[:n]
        valid = self._stress_pressure_valid.tensor[:n] != 0
        norms = F.norm(dim=1)

        def part(mask):
            if mask is None:
                mask = torch.ones(n, dtype=torch.bool, device=F.device)
            return torch.cat(
                [
                    torch.where(mask[:, None], F, 0.0).sum(dim=0),
                    torch.where(mask, norms, 0.0).sum()[None],
                    torch.where(mask, norms, 0.0).max()[None] if n else torch.zeros(1, dtype=F.dtype, device=F.device),
                    mask.sum()[None].to(F.dtype),
                    (mask & valid).sum()[None].to(F.dtype),
                    (mask & ~valid).sum()[None].to(F.dtype),
                ]
            )

        pm, sm = reg == int(primary_region_id), reg == int(secondary_region_id)
        vals = torch.stack([part(pm), part(sm), part(None)]).cpu().numpy()
        p, s, t = vals
        total = tuple(float(v) for v in t[:3])
        reaction = tuple(-v for v in total)
        resid = math.sqrt(sum((a + b) * (a + b) for a, b in zip(total, reaction)))
        return HibmMpmSurfaceMarkerForceReport(
            primary_marker_force_n=tuple(float(v) for v in p[:3]),
            secondary_marker_force_n=tuple(float(v) for v in s[:3]),
            total_marker_force_n=total,
            primary_marker_count=int(p[5]),
            secondary_marker_count=int(s[5]),
            total_marker_count=int(t[5]),
            fluid_reaction_force_n=reaction,
            action_reaction_residual_n=resid,
            primary_stress_valid_marker_count=int(p[6]),
            primary_stress_invalid_marker_count=int(p[7]),
            secondary_stress_valid_marker_count=int(s[6]),
            secondary_stress_invalid_marker_count=int(s[7]),
            primary_marker_force_norm_sum_n=float(p[3]),
            secondary_marker_force_norm_sum_n=float(s[3]),
            total_marker_force_norm_sum_n=float(t[3]),
            primary_marker_force_norm_max_n=float(p[4]),
            secondary_marker_force_norm_max_n=float(s[4]),
            total_marker_force_norm_max_n=float(t[4]),
        )

    # ------------------------------------------------------------------
    def clear_mpm_external_forces(self, external_force_n, *, particle_count: int, read_report: bool = True):
        particles = int(particle_count)
        if particles <= 0:
            raise ValueError("particle_count must be positive")
        rep = self._report
        _native.call(
            "efsi_clear_external_forces",
            particles,
            c_void_p(_tensor(external_force_n).data_ptr()),
            c_void_p(rep.data_ptr()) if read_report else None,
            c_void_p(current_stream_handle()),
        )
        if not read_report:
            return None
        r = rep[:2].cpu().tolist()
        return HibmMpmExternalForceClearReport(cleared_particle_count=int(r[0]), max_abs_external_force_before_n=float(r[1]))

    def _bin_plan(self, particle_x: torch.Tensor, particle_count: int, support_radius: float):
        key = (int(particle_x.shape[0]), float(support_radius))
        plan = self._bins.get(key)
        if plan is None:
            pts = particle_x[:particle_count]
            mk = self.x_gamma_m.tensor[: max(int(self.marker_count), 1)]
            allp = torch.cat([pts, mk], dim=0)
            finite = torch.isfinite(allp).all(dim=1)
            allp = allp[finite] if bool(finite.any()) else torch.zeros(1, 3, device=allp.device)
            lo = allp.min(dim=0).values.cpu().numpy().astype(np.float64)
            hi = allp.max(dim=0).values.cpu().numpy().astype(np.float64)
            pad = np.maximum(0.5 * (hi - lo), 4.0 * support_radius)
            lo, hi = lo - pad, hi + pad
            bmin = (c_float * 3)(*[float(v) for v in lo])
            bmax = (c_float * 3)(*[float(v) for v in hi])
            handle = c_void_p()
            _native.call("efsi_bin_plan_create", key[0], bmin, bmax, float(support_radius), byref(handle))
            plan = (handle,)
            self._bins[key] = plan
        _native.call(
            "efsi_bin_particles", plan[0], c_void_p(particle_x.data_ptr()), int(particle_count), c_void_p(current_stream_handle())
        )
        return plan[0]

    def scatter_marker_forces_to_mpm_particles(
        self, external_force_n, particle_position_m, *, particle_count: int, support_radius_m: float, read_report: bool = True
    ) -> HibmMpmMpmForceScatterReport | None:
        particles = int(particle_count)
        if particles <= 0:
            raise ValueError("particle_count must be positive")
        radius = float(support_radius_m)
        if not math.isfinite(radius) or radius <= 0.0:
            raise ValueError("support_radius_m must be a finite positive number")
        xp = _tensor(particle_position_m)
        plan = self._bin_plan(xp, particles, radius)
        rep = self._report
        _native.call(
            "efsi_scatter_marker_forces",
            plan,
            int(self.marker_count),
            self.x_gamma_m.ptr(),
            self.F_gamma_n.ptr(),
            c_void_p(xp.data_ptr()),
            c_void_p(_tensor(external_force_n).data_ptr()),
            c_void_p(rep.data_ptr()),
            c_void_p(current_stream_handle()),
        )
        if not read_report:
            return None
        r = rep[:9].cpu().tolist()
        marker = tuple(float(v) for v in r[3:6])
        ext = tuple(float(v) for v in r[6:9])
        resid = math.sqrt(sum((a - b) * (a - b) for a, b in zip(marker, ext)))
        return HibmMpmMpmForceScatterReport(
            active_marker_count=int(r[0]),
            invalid_marker_count=int(r[1]),
            active_particle_count=int(r[2]),
            total_marker_force_n=marker,
            total_mpm_external_force_n=ext,
            action_reaction_residual_n=resid,
        )

    def _feedback(self, xp, vp, np_, ap, particle_count, support_radius_m, dt_s, read_report):
        particles = int(particle_count)
        if particles <= 0:
            raise ValueError("particle_count must be positive")
        radius = float(support_radius_m)
        if not math.isfinite(radius) or radius <= 0.0:
            raise ValueError("support_radius_m must be a finite positive number")
        dt = float(dt_s)
        if not math.isfinite(dt) or dt <= 0.0:
            raise ValueError("dt_s must be a finite positive number")
        xp = _tensor(xp)
        plan = self._bin_plan(xp, particles, radius)
        rep = self._report
        _native.call(
            "efsi_surface_feedback",
            plan,
            int(self.marker_count),
            self.x_gamma_m.ptr(),
            self.v_gamma_mps.ptr(),
            self.n_gamma.ptr(),
            self.A_gamma_m2.ptr(),
            c_void_p(xp.data_ptr()),
            c_void_p(_tensor(vp).data_ptr()),
            None if np_ is None else c_void_p(_tensor(np_).data_ptr()),
            None if ap is None else c_void_p(_tensor(ap).data_ptr()),
            dt,
            c_void_p(rep.data_ptr()),
            c_void_p(current_stream_handle()),
        )
        if not read_report:
            return None
        r = rep[:8].cpu().tolist()
        return HibmMpmSurfaceUpdateReport(
            updated_marker_count=int(r[0]),
            invalid_marker_count=int(r[1]),
            max_marker_displacement_m=float(r[4]),
            max_marker_speed_mps=float(r[5]),
            geometry_updated_marker_count=int(r[2]),
            geometry_invalid_marker_count=int(r[3]),
            max_marker_normal_change=float(r[6]),
            max_marker_area_change_m2=float(r[7]),
        )

    def update_surface_feedback_from_mpm_particles(
        self, particle_position_m, particle_velocity_mps, *, particle_count: int, support_radius_m: float, dt_s: float, read_report: bool = True
    ):
        return self._feedback(particle_position_m, particle_velocity_mps, None, None, particle_count, support_radius_m, dt_s, read_report)

    def update_surface_feedback_from_mpm_surface_particles(
        self,
        particle_position_m,
        particle_velocity_mps,
        particle_normal,
        particle_area_m2,
        *,
        particle_count: int,
        support_radius_m: float,
        dt_s: float,
        read_report: bool = True,
    ):
        return self._feedback(
            particle_position_m, particle_velocity_mps, particle_normal, particle_area_m2, particle_count, support_radius_m, dt_s, read_report
        )

    # ------------------------------------------------------------------
    @staticmethod
    def _vector_value_tuple(field: Field, index: int) -> tuple[float, float, float]:
        v = field[int(index)]
        return (float(v[0]), float(v[1]), float(v[2]))

    def marker_force_n(self, marker_index: int):
        return self._vector_value_tuple(self.F_gamma_n, marker_index)

    def marker_traction_pa(self, marker_index: int):
        return self._vector_value_tuple(self.t_gamma_pa, marker_index)

    def marker_normal(self, marker_index: int):
        return self._vector_value_tuple(self.n_gamma, marker_index)

    def marker_velocity_mps(self, marker_index: int):
        return self._vector_value_tuple(self.v_gamma_mps, marker_index)

    def marker_region_id(self, marker_index: int) -> int:
        return int(self.region_id[int(marker_index)])


@dataclass(frozen=True)
class HibmMpmIbNodeSearchReport:
    near_boundary_node_count: int
    external_ib_node_count: int
    internal_node_count: int
    invalid_projection_count: int


class HibmMpmIbNodeSearch:
    """Immersed-boundary node search and in/out classification (drop-in for
    simulation_core/hibm_mpm.py:5385 HibmMpmIbNodeSearch).

    Every node finds the nearest projection triangle (or marker) within the
    search radius, records its boundary point, projection weights and the
    interior fluid probe point, and is classified external IB (some candidate
    sees it outside), internal, or none; with ``classify_far_internal_nodes``
    a node outside the radius of every candidate is internal when no
    candidate at all sees it outside.  The search runs in
    ``efsi_ib_node_search`` (binned triangles on the device); the fields and
    report counts are the reference's.
    """

    _NODE_NONE = 0
    _NODE_EXTERNAL_IB = 1
    _NODE_INTERNAL = 2
    _F32_EPSILON = 1.1920928955078125e-7

    def __init__(self, *, grid_nodes, bounds_min_m, bounds_max_m, marker_capacity: int,
                 runtime: TaichiRuntimeConfig | None = None) -> None:
        self.device = init_runtime(runtime)
        nodes = tuple(int(v) for v in grid_nodes)
        if len(nodes) != 3 or any(v <= 0 for v in nodes):
            raise ValueError("grid_nodes must contain three positive integers")
        bounds_min = _vector3(bounds_min_m, name="bounds_min_m")
        bounds_max = _vector3(bounds_max_m, name="bounds_max_m")
        if any(hi <= lo for lo, hi in zip(bounds_min, bounds_max)):
            raise ValueError("bounds_max_m must be greater than bounds_min_m")
        if int(marker_capacity) <= 0:
            raise ValueError("marker_capacity must be positive")
        self.grid_nodes = nodes
        self.bounds_min_m = bounds_min
        self.bounds_max_m = bounds_max
        self.spacing_m = tuple((hi - lo) / float(n) for lo, hi, n in zip(bounds_min, bounds_max, nodes))
        self.marker_capacity = int(marker_capacity)
        dev = self.device
        self.node_kind_code = Field(nodes, i32, device=dev)
        self.nearest_marker = Field(nodes, i32, device=dev)
        self.node_signed_distance_m = Field(nodes, f32, device=dev)
        self.node_boundary_point_m = Field(nodes, f32, n=3, device=dev)
        self.node_interior_fluid_point_m = Field(nodes, f32, n=3, device=dev)
        self.node_projection_marker_indices = Field(nodes, i32, n=3, device=dev)
        self.node_projection_marker_weights = Field(nodes, f32, n=3, device=dev)
        self.node_anchor_cell = Field(nodes, i32, n=3, device=dev)
        self._report = torch.zeros(4, dtype=torch.int32, device=dev)
        handle = c_void_p()
        _native.call("efsi_ib_search_plan_create", byref(handle))
        self._plan = handle
        self.reset_node_anchor_cells()

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None:
            try:
                _native.load().efsi_ib_search_plan_destroy(plan)
            except Exception:
                pass

    def reset_node_anchor_cells(self) -> None:
        """hibm_mpm.py:5463-5475: every node's anchor cell to (-1, -1, -1)."""
        n = int(np.prod(self.grid_nodes))
        _native.call("efsi_ib_reset_anchor_cells", self.node_anchor_cell.ptr(), n, current_stream_handle())

    def _default_sign_tolerance_m(self) -> float:
        """hibm_mpm.py:5477-5492."""
        min_spacing = max(min(self.spacing_m), 1.0e-12)
        max_extent = max(hi - lo for lo, hi in zip(self.bounds_min_m, self.bounds_max_m))
        max_coordinate = max(max(abs(v) for v in self.bounds_min_m), max(abs(v) for v in self.bounds_max_m))
        coordinate_scale = max(max_extent, max_coordinate, min_spacing, 1.0)
        return max(1.0e-12, 1.0e-6 * min_spacing, 2.0 * self._F32_EPSILON * coordinate_scale)

    def _validate_search_inputs(self, markers, *, search_radius_m, interior_probe_distance_m, sign_tolerance_m):
        """hibm_mpm.py:6069-6094."""
        if int(markers.marker_count) > self.marker_capacity:
            raise ValueError("markers.marker_count exceeds marker_capacity")
        radius = float(search_radius_m)
        if not math.isfinite(radius) or radius <= 0.0:
            raise ValueError("search_radius_m must be a finite positive number")
        probe = float(interior_probe_distance_m)
        if not math.isfinite(probe) or probe <= 0.0:
            raise ValueError("interior_probe_distance_m must be a finite positive number")
        tol = self._default_sign_tolerance_m() if sign_tolerance_m is None else float(sign_tolerance_m)
        if not math.isfinite(tol) or tol < 0.0:
            raise ValueError("sign_tolerance_m must be a finite non-negative number")
        return radius, probe, tol

    def _run(self, markers, centres, radius, probe, tol, classify_far) -> HibmMpmIbNodeSearchReport:
        prm = _native.IbSearchParams()
        prm.nx, prm.ny, prm.nz = self.grid_nodes
        prm.marker_count = int(markers.marker_count)
        prm.triangle_count = int(getattr(markers, "projection_triangle_count", 0))
        prm.classify_far_internal_nodes = 1 if classify_far else 0
        prm.search_radius_m = radius
        prm.interior_probe_distance_m = probe
        prm.sign_tolerance_m = tol
        keep = []
        if centres is not None:
            axes = []
            for c, count in zip(centres, self.grid_nodes):
                t = (c.tensor if isinstance(c, Field) else torch.as_tensor(c))
                t = t.to(device=self.device, dtype=torch.float32).contiguous()
                if t.numel() < count:
                    raise ValueError("cell centre fields must cover grid_nodes")
                keep.append(t)
                axes.append(t.data_ptr())
            prm.cell_center_x_m, prm.cell_center_y_m, prm.cell_center_z_m = axes
        for a in range(3):
            prm.bounds_min_m[a] = self.bounds_min_m[a]
            prm.spacing_m[a] = self.spacing_m[a]
            prm.box_min_m[a] = self.bounds_min_m[a]
            prm.box_max_m[a] = self.bounds_max_m[a]
        prm.marker_x = markers.x_gamma_m.ptr()
        prm.marker_n = markers.n_gamma.ptr()
        prm.triangles = markers.projection_triangle_indices.ptr() if prm.triangle_count > 0 else None
        out = _native.IbSearchFields()
        out.node_kind = self.node_kind_code.ptr()
        out.nearest_marker = self.nearest_marker.ptr()
        out.signed_distance_m = self.node_signed_distance_m.ptr()
        out.boundary_point_m = self.node_boundary_point_m.ptr()
        out.interior_fluid_point_m = self.node_interior_fluid_point_m.ptr()
        out.projection_marker_indices = self.node_projection_marker_indices.ptr()
        out.projection_marker_weights = self.node_projection_marker_weights.ptr()
        out.report = self._report.data_ptr()
        _native.call("efsi_ib_node_search", self._plan, byref(prm), byref(out), current_stream_handle())
        counts = [int(v) for v in self._report.cpu()]
        del keep
        return HibmMpmIbNodeSearchReport(*counts)

    def search_and_classify(self, markers, *, search_radius_m: float, interior_probe_distance_m: float,
                            sign_tolerance_m: float | None = None,
                            classify_far_internal_nodes: bool = False) -> HibmMpmIbNodeSearchReport:
        """hibm_mpm.py:6096-6133: nodes at the uniform cell centres of the
        search box."""
        radius, probe, tol = self._validate_search_inputs(
            markers, search_radius_m=search_radius_m, interior_probe_distance_m=interior_probe_distance_m,
            sign_tolerance_m=sign_tolerance_m)
        return self._run(markers, None, radius, probe, tol, classify_far_internal_nodes)

    def search_and_classify_grid_fields(self, markers, *, cell_center_x_m, cell_center_y_m, cell_center_z_m,
                                        search_radius_m: float, interior_probe_distance_m: float,
                                        sign_tolerance_m: float | None = None,
                                        classify_far_internal_nodes: bool = False) -> HibmMpmIbNodeSearchReport:
        """hibm_mpm.py:6135-6170: nodes at the fluid's (graded) cell centres."""
        radius, probe, tol = self._validate_search_inputs(
            markers, search_radius_m=search_radius_m, interior_probe_distance_m=interior_probe_distance_m,
            sign_tolerance_m=sign_tolerance_m)
        return self._run(markers, (cell_center_x_m, cell_center_y_m, cell_center_z_m), radius, probe, tol,
                         classify_far_internal_nodes)

    def node_kind(self, node_index) -> str:
        code = int(self.node_kind_code[self._node_index(node_index)])
        if code == self._NODE_EXTERNAL_IB:
            return "external_ib"
        if code == self._NODE_INTERNAL:
            return "internal"
        return "none"

    def nearest_marker_index(self, node_index) -> int:
        return int(self.nearest_marker[self._node_index(node_index)])

    def signed_distance_m(self, node_index) -> float:
        return float(self.node_signed_distance_m[self._node_index(node_index)])

    def boundary_point_m(self, node_index) -> tuple[float, float, float]:
        return tuple(float(v) for v in self.node_boundary_point_m[self._node_index(node_index)])

    def interior_fluid_point_m(self, node_index) -> tuple[float, float, float]:
        return tuple(float(v) for v in self.node_interior_fluid_point_m[self._node_index(node_index)])

    def _node_index(self, node_index) -> tuple[int, int, int]:
        index = tuple(int(v) for v in node_index)
        if len(index) != 3 or any(v < 0 or v >= n for v, n in zip(index, self.grid_nodes)):
            raise IndexError("node_index out of range")
        return index


@dataclass(frozen=True)
class HibmMpmIbBoundaryConditionReport:
    no_slip_dirichlet_count: int
    pressure_neumann_count: int
    inactive_internal_node_count: int
    max_abs_velocity_mps: float = 0.0


@dataclass(frozen=True)
class HibmMpmVelocityDirichletBoundaryReport:
    active_velocity_dirichlet_rows: int
    inactive_obstacle_rows: int
    max_abs_velocity_mps: float
    invalid_reconstruction_row_count: int = 0
    invalid_no_fluid_sample_row_count: int = 0
    invalid_nonpositive_gap_row_count: int = 0
    invalid_node_behind_boundary_row_count: int = 0
    invalid_node_beyond_interior_row_count: int = 0
    narrow_gap_boundary_velocity_row_count: int = 0
    relocated_row_count: int = 0
    relocation_merged_row_count: int = 0
    relocation_blocked_row_count: int = 0
    min_projection_weight: float = 0.0
    max_projection_weight: float = 0.0


class HibmMpmIbBoundaryConditions:
    """External-IB boundary conditions from the node search (drop-in for
    simulation_core/hibm_mpm.py:6222 HibmMpmIbBoundaryConditions, the
    build-from-search and velocity-Dirichlet row members).

    ``build_from_search`` interpolates each external IB node's no-slip
    velocity, Neumann normal and Neumann gradient from its projection markers
    (``efsi_ib_build_boundary_conditions``); the two row assemblies write the
    fluid's velocity-Dirichlet row fields (``efsi_ib_velocity_dirichlet_rows``):
    the target velocity itself, or the reconstruction along the surface normal
    with its fallbacks and the relocation of rows whose node is masked.  The
    pressure-Neumann row assembly of the reference class is not provided.
    """

    _NODE_EXTERNAL_IB = HibmMpmIbNodeSearch._NODE_EXTERNAL_IB
    _NODE_INTERNAL = HibmMpmIbNodeSearch._NODE_INTERNAL

    def __init__(self, *, grid_nodes, marker_capacity: int, runtime: TaichiRuntimeConfig | None = None) -> None:
        self.device = init_runtime(runtime)
        nodes = tuple(int(v) for v in grid_nodes)
        if len(nodes) != 3 or any(v <= 0 for v in nodes):
            raise ValueError("grid_nodes must contain three positive integers")
        if int(marker_capacity) <= 0:
            raise ValueError("marker_capacity must be positive")
        self.grid_nodes = nodes
        self.marker_capacity = int(marker_capacity)
        dev = self.device
        self.active_ib_node = Field(nodes, i32, device=dev)
        self.velocity_dirichlet_mps_field = Field(nodes, f32, n=3, device=dev)
        self.pressure_neumann_normal_field = Field(nodes, f32, n=3, device=dev)
        self.pressure_neumann_gradient_field = Field(nodes, f32, device=dev)
        self.marker_pressure_neumann_gradient_field = Field((self.marker_capacity,), f32, device=dev)
        self._bc_report = torch.zeros(4, dtype=torch.int32, device=dev)
        self._vd_report = torch.zeros(13, dtype=torch.int32, device=dev)
        handle = c_void_p()
        _native.call("efsi_ib_search_plan_create", byref(handle))
        self._plan = handle

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None:
            try:
                _native.load().efsi_ib_search_plan_destroy(plan)
            except Exception:
                pass

    def _validate_search_and_markers(self, search, markers) -> None:
        """hibm_mpm.py:6636-6647."""
        if tuple(search.grid_nodes) != self.grid_nodes:
            raise ValueError("search.grid_nodes must match boundary grid_nodes")
        if int(markers.marker_count) > self.marker_capacity:
            raise ValueError("markers.marker_count exceeds marker_capacity")
        if int(search.marker_capacity) > self.marker_capacity:
            raise ValueError("search.marker_capacity exceeds marker_capacity")

    def build_from_search(self, search, markers, *,
                          marker_pressure_neumann_gradient_pa_per_m) -> HibmMpmIbBoundaryConditionReport:
        """hibm_mpm.py:6579-6605."""
        self._validate_search_and_markers(search, markers)
        if len(marker_pressure_neumann_gradient_pa_per_m) != markers.marker_count:
            raise ValueError("marker_pressure_neumann_gradient_pa_per_m must match marker_count")
        grad = np.zeros(self.marker_capacity, dtype=np.float32)
        for m, g in enumerate(marker_pressure_neumann_gradient_pa_per_m):
            v = float(g)
            if not math.isfinite(v):
                raise ValueError("marker_pressure_neumann_gradient_pa_per_m must be finite")
            grad[m] = v
        self.marker_pressure_neumann_gradient_field.from_numpy(grad)
        return self.build_from_search_device_fields(
            search, markers, marker_pressure_neumann_gradient_pa_per_m_field=self.marker_pressure_neumann_gradient_field)

    def build_from_search_device_fields(self, search, markers, *,
                                        marker_pressure_neumann_gradient_pa_per_m_field
                                        ) -> HibmMpmIbBoundaryConditionReport:
        """hibm_mpm.py:6607-6634 over the search's fields."""
        self._validate_search_and_markers(search, markers)
        grad = _tensor(marker_pressure_neumann_gradient_pa_per_m_field)
        _native.call(
            "efsi_ib_build_boundary_conditions", int(np.prod(self.grid_nodes)), search.node_kind_code.ptr(),
            search.nearest_marker.ptr(), search.node_projection_marker_indices.ptr(),
            search.node_projection_marker_weights.ptr(), markers.v_gamma_mps.ptr(), markers.n_gamma.ptr(),
            grad.data_ptr(), int(markers.marker_count), self.active_ib_node.ptr(),
            self.velocity_dirichlet_mps_field.ptr(), self.pressure_neumann_normal_field.ptr(),
            self.pressure_neumann_gradient_field.ptr(), self._bc_report.data_ptr(), current_stream_handle())
        rep = self._bc_report.cpu()
        return HibmMpmIbBoundaryConditionReport(int(rep[0]), int(rep[1]), int(rep[2]),
                                                float(rep[3:4].view(torch.float32)[0]))

    def _vd_call(self, prm, fields, reconstruct: int, written) -> torch.Tensor:
        _native.call("efsi_ib_velocity_dirichlet_rows", self._plan, byref(prm), byref(fields), reconstruct,
                     current_stream_handle())
        # the kernels write through raw pointers: bump the fields' versions so
        # the fluid rebuilds its stencil masks from the new rows
        for field in written:
            _tensor(field).add_(0)
        return self._vd_report.cpu()

    def assemble_velocity_dirichlet_boundary_rows(self, velocity_dirichlet_active, velocity_dirichlet_value_mps,
                                                  obstacle_field) -> HibmMpmVelocityDirichletBoundaryReport:
        """hibm_mpm.py:6690-6712: the target velocity on every unmasked active IB node."""
        prm = _native.IbVdParams()
        prm.nx, prm.ny, prm.nz = self.grid_nodes
        prm.active_ib_node = self.active_ib_node.ptr()
        prm.target_velocity = self.velocity_dirichlet_mps_field.ptr()
        prm.obstacle = _tensor(obstacle_field).data_ptr()
        out = _native.IbVdFields()
        out.active = _tensor(velocity_dirichlet_active).data_ptr()
        out.value_mps = _tensor(velocity_dirichlet_value_mps).data_ptr()
        out.report = self._vd_report.data_ptr()
        rep = self._vd_call(prm, out, 0, (velocity_dirichlet_active, velocity_dirichlet_value_mps))
        return HibmMpmVelocityDirichletBoundaryReport(int(rep[0]), int(rep[1]), float(rep[10:11].view(torch.float32)[0]))

    def assemble_velocity_dirichlet_reconstructed_boundary_rows(
        self, velocity_dirichlet_active, velocity_dirichlet_value_mps, velocity_dirichlet_projection_weight,
        obstacle_field, velocity_field, search, *, cell_face_x_m, cell_face_y_m, cell_face_z_m, cell_center_x_m,
        cell_center_y_m, cell_center_z_m, grid_nodes, velocity_dirichlet_marker_region_id=None, marker_region_id=None,
    ) -> HibmMpmVelocityDirichletBoundaryReport:
        """hibm_mpm.py:7655-7800: anchor prefill, row reconstruction along the
        surface normal (with the line-of-sight fallback, narrow-gap and invalid
        rows), relocation of rows whose node is masked, and the region stamp
        when both region fields are given."""
        if tuple(search.grid_nodes) != self.grid_nodes:
            raise ValueError("search.grid_nodes must match boundary grid_nodes")
        nodes = tuple(int(v) for v in grid_nodes)
        if len(nodes) != 3 or any(v < 2 for v in nodes):
            raise ValueError("grid_nodes must contain three values >= 2")
        if nodes != self.grid_nodes:
            raise ValueError("grid_nodes must match boundary grid_nodes")
        if (velocity_dirichlet_marker_region_id is None) != (marker_region_id is None):
            raise ValueError("velocity_dirichlet_marker_region_id and marker_region_id must be provided together")
        region_out = None
        if velocity_dirichlet_marker_region_id is not None:
            region_out = _tensor(velocity_dirichlet_marker_region_id)
            if tuple(region_out.shape) != tuple(_tensor(velocity_dirichlet_active).shape):
                raise ValueError("velocity_dirichlet_marker_region_id shape must match velocity_dirichlet_active")
        keep = []

        def f32_ptr(field, count):
            t = _tensor(field).to(device=self.device, dtype=torch.float32).contiguous()
            if t.numel() < count:
                raise ValueError("grid axis fields must cover grid_nodes")
            keep.append(t)
            return t.data_ptr()

        prm = _native.IbVdParams()
        prm.nx, prm.ny, prm.nz = nodes
        prm.face_x_m, prm.face_y_m, prm.face_z_m = (f32_ptr(f, n + 1) for f, n in zip(
            (cell_face_x_m, cell_face_y_m, cell_face_z_m), nodes))
        prm.center_x_m, prm.center_y_m, prm.center_z_m = (f32_ptr(f, n) for f, n in zip(
            (cell_center_x_m, cell_center_y_m, cell_center_z_m), nodes))
        prm.active_ib_node = self.active_ib_node.ptr()
        prm.target_velocity = self.velocity_dirichlet_mps_field.ptr()
        prm.target_normal = self.pressure_neumann_normal_field.ptr()
        prm.boundary_point_m = search.node_boundary_point_m.ptr()
        prm.interior_fluid_point_m = search.node_interior_fluid_point_m.ptr()
        prm.nearest_marker = search.nearest_marker.ptr()
        prm.obstacle = _tensor(obstacle_field).data_ptr()
        prm.velocity = _tensor(velocity_field).data_ptr()
        if marker_region_id is not None:
            regions = _tensor(marker_region_id).to(device=self.device, dtype=torch.int32).contiguous()
            keep.append(regions)
            prm.marker_region_id = regions.data_ptr()
            prm.marker_count = int(regions.shape[0])
        out = _native.IbVdFields()
        out.active = _tensor(velocity_dirichlet_active).data_ptr()
        out.value_mps = _tensor(velocity_dirichlet_value_mps).data_ptr()
        out.projection_weight = _tensor(velocity_dirichlet_projection_weight).data_ptr()
        out.anchor_cell = search.node_anchor_cell.ptr()
        out.marker_region_id = region_out.data_ptr() if region_out is not None else None
        out.report = self._vd_report.data_ptr()
        rep = self._vd_call(prm, out, 1, (velocity_dirichlet_active, velocity_dirichlet_value_mps,
                                          velocity_dirichlet_projection_weight))
        del keep
        counts = [int(v) for v in rep[:10]]
        vmax, wmin, wmax = (float(v) for v in rep[10:13].view(torch.float32))
        return HibmMpmVelocityDirichletBoundaryReport(
            active_velocity_dirichlet_rows=counts[0], inactive_obstacle_rows=counts[1], max_abs_velocity_mps=vmax,
            invalid_reconstruction_row_count=counts[2], invalid_no_fluid_sample_row_count=counts[3],
            invalid_nonpositive_gap_row_count=counts[4], invalid_node_behind_boundary_row_count=counts[5],
            invalid_node_beyond_interior_row_count=counts[6], narrow_gap_boundary_velocity_row_count=counts[7],
            relocated_row_count=counts[8], relocation_merged_row_count=counts[9],
            relocation_blocked_row_count=counts[1], min_projection_weight=wmin if counts[0] > 0 else 0.0,
            max_projection_weight=wmax)

    def is_active(self, node_index) -> bool:
        return bool(int(self.active_ib_node[self._node_index(node_index)]))

    def velocity_dirichlet_mps(self, node_index) -> tuple[float, float, float]:
        return tuple(float(v) for v in self.velocity_dirichlet_mps_field[self._node_index(node_index)])

    def pressure_neumann_normal(self, node_index) -> tuple[float, float, float]:
        return tuple(float(v) for v in self.pressure_neumann_normal_field[self._node_index(node_index)])

    def pressure_neumann_gradient_pa_per_m(self, node_index) -> float:
        return float(self.pressure_neumann_gradient_field[self._node_index(node_index)])

    def _node_index(self, node_index) -> tuple[int, int, int]:
        index = tuple(int(v) for v in node_index)
        if len(index) != 3 or any(v < 0 or v >= n for v, n in zip(index, self.grid_nodes)):
            raise IndexError("node_index out of range")
        return index
