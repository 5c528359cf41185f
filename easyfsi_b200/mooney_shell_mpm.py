"""Triangle Mooney-Rivlin membrane MPM on the B200 (drop-in for
simulation_core/mooney_shell_mpm.py ``TriMooneyShellMpmState``, :105-1391).

The class keeps the reference's constructor arguments, validation errors,
fields (``x``, ``rest_x``, ``u``, ``v``, ``internal_force_n``,
``external_force_n``, ``surface_normal``, ``area_weight_m2``, ...), step
entry points (``step``, ``advance_region_loads``,
``advance_with_external_forces``, ``add_region_area_load``,
``save_state`` / ``restore_state``) and the 37-value packed report.  Every
step runs as the CUDA kernels of ``csrc/efsi_shell.cu`` through the C ABI
(``efsi_shell_step``); there is no host fallback.
"""

from __future__ import annotations

from ctypes import byref, c_float, c_void_p
from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from .field import Field
from .geometry import SurfaceMesh
from .runtime import TaichiRuntimeConfig, current_stream_handle, f32, f64, i32, init_runtime


@dataclass(frozen=True)
class TriMooneyShellMpmReport:
    """Field list of mooney_shell_mpm.py:26-50."""

    particle_count: int
    face_count: int
    edge_count: int
    active_grid_nodes: int
    grid_out_of_bounds_particle_count: int
    particle_spacing_m: float
    grid_spacing_m: tuple[float, float, float]
    mean_radial_stretch: float
    max_radial_stretch_error: float
    max_edge_strain: float
    max_speed_mps: float
    total_mass_kg: float
    total_area_m2: float
    primary_mean_displacement_m: tuple[float, float, float]
    primary_mean_velocity_mps: tuple[float, float, float]
    secondary_mean_displacement_m: tuple[float, float, float]
    secondary_mean_velocity_mps: tuple[float, float, float]
    particle_momentum_kg_mps: tuple[float, float, float]
    grid_momentum_kg_mps: tuple[float, float, float]
    total_force_n: tuple[float, float, float]
    internal_force_rms_n: float
    net_internal_force_relative_error: float
    transfer_relative_error: float


def _unique_undirected_edges(faces: np.ndarray) -> np.ndarray:
    """Sorted unique (min, max) vertex pairs of the triangles (mooney_shell_mpm.py:53-61)."""
    f = np.asarray(faces, dtype=np.int64).reshape(-1, 3)
    if f.size == 0:
        return np.zeros((0, 2), dtype=np.int32)
    pairs = np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], axis=0), axis=1)
    return np.unique(pairs, axis=0).astype(np.int32)


def _mesh_bounds_with_padding(vertices: np.ndarray, bounds_padding_fraction: float):
    """Mesh box grown by a fraction of its largest extent (mooney_shell_mpm.py:64-77)."""
    lo = np.min(vertices, axis=0)
    hi = np.max(vertices, axis=0)
    extent = float(np.max(hi - lo))
    if extent <= 0.0:
        extent = 1.0
    pad = max(bounds_padding_fraction * extent, 1.0e-6 * extent)
    return tuple(float(v) for v in lo - pad), tuple(float(v) for v in hi + pad)


def _validate_flip_blend(flip_blend: float) -> float:
    value = float(flip_blend)
    if not 0.0 <= value <= 1.0:
        raise ValueError("flip_blend must be in [0, 1]")
    return value


def _vector3(value, name: str) -> tuple[float, float, float]:
    if len(value) != 3:
        raise ValueError(f"{name} must contain exactly 3 components")
    return (float(value[0]), float(value[1]), float(value[2]))


def _raise_if_all_particles_out_of_bounds(particle_count: int, out_of_bounds: int) -> None:
    if particle_count > 0 and out_of_bounds == particle_count:
        raise RuntimeError(
            f"all {particle_count} MPM particles are outside the background grid; "
            "the solid has left the simulation domain"
        )


class TriMooneyShellMpmState:
    """Mooney membrane MPM on an explicit triangle surface mesh (mooney_shell_mpm.py:105)."""

    def __init__(
        self,
        mesh: SurfaceMesh,
        *,
        thickness_m: float,
        density_kgm3: float,
        c1_pa: float,
        c2_pa: float,
        membrane_force_scale: float = 1.0,
        grid_nodes: tuple[int, int, int] = (36, 36, 36),
        bounds_padding_fraction: float = 0.5,
        face_region_id: np.ndarray | None = None,
        primary_region_id: int,
        secondary_region_id: int,
        fixed_region_id: int = -1,
        primary_thickness_m: float | None = None,
        secondary_thickness_m: float | None = None,
        runtime: TaichiRuntimeConfig | None = None,
    ):
        self.device = init_runtime(runtime)
        vertex_count = int(np.asarray(mesh.vertices).shape[0])
        # argument checks and messages of mooney_shell_mpm.py:127-142
        if vertex_count <= 0:
            raise ValueError("mesh must contain at least one vertex")
        if mesh.face_count <= 0:
            raise ValueError("mesh must contain at least one triangle")
        if thickness_m <= 0.0:
            raise ValueError("thickness_m must be positive")
        if density_kgm3 <= 0.0:
            raise ValueError("density_kgm3 must be positive")
        if c1_pa <= 0.0 or c2_pa < 0.0:
            raise ValueError("Mooney constants must be non-negative with c1 > 0")
        if membrane_force_scale <= 0.0:
            raise ValueError("membrane_force_scale must be positive")
        if min(grid_nodes) < 4:
            raise ValueError("grid_nodes must be at least 4 in each direction")
        if bounds_padding_fraction <= 0.0:
            raise ValueError("bounds_padding_fraction must be positive")

        vertices = np.asarray(mesh.vertices, dtype=np.float32)
        faces = np.asarray(mesh.faces, dtype=np.int32)
        if faces.size and (faces.min() < 0 or faces.max() >= vertex_count):
            raise ValueError("mesh faces must index existing vertices")
        edges = _unique_undirected_edges(faces)
        regions = np.zeros(mesh.face_count, dtype=np.int32)
        if face_region_id is not None:
            regions = np.asarray(face_region_id, dtype=np.int32)
            if regions.shape != (mesh.face_count,):
                raise ValueError("face_region_id must have shape (face_count,)")
        bounds_min, bounds_max = _mesh_bounds_with_padding(vertices, bounds_padding_fraction)

        self.particle_count = vertex_count
        self.face_count = int(mesh.face_count)
        self.edge_count = int(edges.shape[0])
        self.thickness_m = float(thickness_m)
        self.density_kgm3 = float(density_kgm3)
        self.c1_pa = float(c1_pa)
        self.c2_pa = float(c2_pa)
        self.membrane_force_scale = float(membrane_force_scale)
        self.primary_region_id = int(primary_region_id)
        self.secondary_region_id = int(secondary_region_id)
        self.fixed_region_id = int(fixed_region_id)
        self.primary_thickness_m = float(thickness_m if primary_thickness_m is None else primary_thickness_m)
        self.secondary_thickness_m = float(thickness_m if secondary_thickness_m is None else secondary_thickness_m)
        self.grid_nodes = tuple(int(v) for v in grid_nodes)
        self.nx, self.ny, self.nz = self.grid_nodes
        self.bounds_min = bounds_min
        self.bounds_max = bounds_max
        self.dx = tuple((self.bounds_max[a] - self.bounds_min[a]) / (self.grid_nodes[a] - 1) for a in range(3))

        dev = self.device
        n = self.particle_count

        def vec(count=n):
            return Field((count,), f32, n=3, device=dev)

        self.x = vec()
        self.rest_x = vec()
        self.u = vec()
        self.v = vec()
        self.saved_x = vec()
        self.saved_u = vec()
        self.saved_v = vec()
        self.mass_kg = Field((n,), f32, device=dev)
        self.area_weight_m2 = Field((n,), f32, device=dev)
        self.surface_normal = vec()
        self.internal_force_n = vec()
        self.external_force_n = vec()
        self.vertex_region_id = Field((n,), i32, device=dev)
        self.fixed_particle = Field((n,), i32, device=dev)
        self.rest_center_m = Field((), f32, n=3, device=dev)
        self.face_indices = Field((self.face_count,), i32, n=3, device=dev)
        self.face_region_id = Field((self.face_count,), i32, device=dev)
        self.edge_indices = Field((max(self.edge_count, 1),), i32, n=2, device=dev)
        self.grid_mass_kg = Field(self.grid_nodes, f32, device=dev)
        self.grid_velocity_mps = Field(self.grid_nodes, f32, n=3, device=dev)
        self.grid_velocity_before_force_mps = Field(self.grid_nodes, f32, n=3, device=dev)
        self.grid_force_n = Field(self.grid_nodes, f32, n=3, device=dev)
        self.report_host_snapshot = Field((37,), f64, device=dev)
        self.primary_area_m2 = Field((), f32, device=dev)
        self.secondary_area_m2 = Field((), f32, device=dev)
        self.primary_mass_kg = Field((), f32, device=dev)
        self.secondary_mass_kg = Field((), f32, device=dev)
        self.last_report_host_reads = 0
        self._scratch = torch.zeros(_native.SHELL_SCRATCH_DOUBLES, dtype=torch.float64, device=dev)
        self._region_totals = torch.zeros(4, dtype=torch.float32, device=dev)

        self.x.from_numpy(vertices)
        self.rest_x.from_numpy(vertices)
        self.saved_x.from_numpy(vertices)
        self.face_indices.from_numpy(faces)
        self.face_region_id.from_numpy(regions)
        if self.edge_count > 0:
            self.edge_indices.from_numpy(edges)
        _native.call(
            "efsi_shell_init",
            byref(self._state_struct()),
            c_void_p(self.mass_kg.ptr()),
            c_void_p(self.vertex_region_id.ptr()),
            c_void_p(self.fixed_particle.ptr()),
            float(density_kgm3),
            self.thickness_m,
            self.primary_thickness_m,
            self.secondary_thickness_m,
            self.primary_region_id,
            self.secondary_region_id,
            self.fixed_region_id,
            c_void_p(self._region_totals.data_ptr()),
            c_void_p(current_stream_handle()),
        )
        self.primary_area_m2.tensor.copy_(self._region_totals[0])
        self.primary_mass_kg.tensor.copy_(self._region_totals[1])
        self.secondary_area_m2.tensor.copy_(self._region_totals[2])
        self.secondary_mass_kg.tensor.copy_(self._region_totals[3])
        # the two region areas scale the interface reactions of every region step
        self._primary_area = float(self._region_totals[0].item())
        self._secondary_area = float(self._region_totals[2].item())
        self._update_rest_center()

    # -- set-up helpers -------------------------------------------------------------------
    def _update_rest_center(self) -> None:
        """mooney_shell_mpm.py:255-267: mean of the rest positions."""
        self.rest_center_m.tensor.copy_(self.rest_x.tensor.mean(dim=0))

    def _state_struct(self) -> _native.ShellState:
        s = _native.ShellState()
        s.particle_count, s.face_count, s.edge_count = self.particle_count, self.face_count, self.edge_count
        s.nx, s.ny, s.nz = self.nx, self.ny, self.nz
        for a in range(3):
            s.bmin[a] = self.bounds_min[a]
            s.dx[a] = self.dx[a]
        s.x, s.u, s.v = self.x.ptr(), self.u.ptr(), self.v.ptr()
        s.rest_x, s.mass = self.rest_x.ptr(), self.mass_kg.ptr()
        s.area, s.normal = self.area_weight_m2.ptr(), self.surface_normal.ptr()
        s.internal_force, s.external_force = self.internal_force_n.ptr(), self.external_force_n.ptr()
        s.vertex_region, s.fixed = self.vertex_region_id.ptr(), self.fixed_particle.ptr()
        s.faces, s.face_region = self.face_indices.ptr(), self.face_region_id.ptr()
        s.edges = self.edge_indices.ptr()
        s.grid_mass, s.grid_velocity = self.grid_mass_kg.ptr(), self.grid_velocity_mps.ptr()
        s.grid_velocity_before, s.grid_force = self.grid_velocity_before_force_mps.ptr(), self.grid_force_n.ptr()
        return s

    def _params(self, *, dt_s, velocity_damping, flip_blend, body_acceleration, pressure_pa=0.0,
                region_loads=0, preserve=0, primary_region_id=None, secondary_region_id=None,
                area_load_region_id=None, area_load=(0.0, 0.0, 0.0), primary_reaction=(0.0, 0.0, 0.0),
                secondary_reaction=(0.0, 0.0, 0.0)) -> _native.ShellParams:
        p = _native.ShellParams()
        p.dt, p.pressure = float(dt_s), float(pressure_pa)
        p.velocity_damping, p.flip_blend = float(velocity_damping), float(flip_blend)
        p.c1, p.c2, p.membrane_force_scale = self.c1_pa, self.c2_pa, self.membrane_force_scale
        p.thickness, p.primary_thickness, p.secondary_thickness = (
            self.thickness_m, self.primary_thickness_m, self.secondary_thickness_m)
        p.region_loads, p.preserve_external_force = int(region_loads), int(preserve)
        p.primary_region = self.primary_region_id if primary_region_id is None else int(primary_region_id)
        p.secondary_region = self.secondary_region_id if secondary_region_id is None else int(secondary_region_id)
        p.area_load_region = p.primary_region if area_load_region_id is None else int(area_load_region_id)
        for a in range(3):
            p.body_acceleration[a] = body_acceleration[a]
            p.primary_area_load[a] = area_load[a]
            p.primary_reaction[a] = primary_reaction[a]
            p.secondary_reaction[a] = secondary_reaction[a]
        p.primary_area, p.secondary_area = self._primary_area, self._secondary_area
        return p

    def _run(self, params: _native.ShellParams, read_report: bool):
        _native.call(
            "efsi_shell_step",
            byref(self._state_struct()),
            byref(params),
            c_void_p(self._scratch.data_ptr()),
            c_void_p(self.report_host_snapshot.ptr()),
            c_void_p(current_stream_handle()),
        )
        if not read_report:
            self.last_report_host_reads = 0
            return None
        return self.report()

    # -- public API (mooney_shell_mpm.py:730-742, 1179-1315) -----------------------------------
    def add_region_area_load(self, *, region_id: int, area_load_npm2: tuple[float, float, float]) -> None:
        load = (c_float * 3)(*_vector3(area_load_npm2, "area_load_npm2"))
        _native.call("efsi_shell_add_region_area_load", byref(self._state_struct()), int(region_id), load,
                     c_void_p(current_stream_handle()))

    def step(self, *, dt_s: float, pressure_pa: float, velocity_damping: float = 1.0, flip_blend: float = 0.95,
             body_acceleration_mps2: tuple[float, float, float] = (0.0, 0.0, 0.0),
             read_report: bool = True) -> TriMooneyShellMpmReport | None:
        body = _vector3(body_acceleration_mps2, "body_acceleration_mps2")
        params = self._params(dt_s=dt_s, pressure_pa=pressure_pa, velocity_damping=velocity_damping,
                              flip_blend=_validate_flip_blend(flip_blend), body_acceleration=body)
        return self._run(params, read_report)

    def advance_region_loads(self, *, dt_s: float, primary_region_id: int, secondary_region_id: int,
                             primary_area_load_npm2: tuple[float, float, float],
                             primary_interface_reaction_n: tuple[float, float, float],
                             secondary_interface_reaction_n: tuple[float, float, float],
                             primary_area_load_region_id: int | None = None, velocity_damping: float = 1.0,
                             flip_blend: float = 0.95,
                             body_acceleration_mps2: tuple[float, float, float] = (0.0, 0.0, 0.0),
                             read_report: bool = True) -> TriMooneyShellMpmReport | None:
        """Advance two region-specific external loads without case-specific axes."""
        load = _vector3(primary_area_load_npm2, "primary_area_load_npm2")
        prim = _vector3(primary_interface_reaction_n, "primary_interface_reaction_n")
        sec = _vector3(secondary_interface_reaction_n, "secondary_interface_reaction_n")
        body = _vector3(body_acceleration_mps2, "body_acceleration_mps2")
        params = self._params(dt_s=dt_s, velocity_damping=velocity_damping,
                              flip_blend=_validate_flip_blend(flip_blend), body_acceleration=body, region_loads=1,
                              preserve=0, primary_region_id=primary_region_id,
                              secondary_region_id=secondary_region_id,
                              area_load_region_id=(int(primary_region_id) if primary_area_load_region_id is None
                                                   else int(primary_area_load_region_id)),
                              area_load=load, primary_reaction=prim, secondary_reaction=sec)
        return self._run(params, read_report)

    def advance_with_external_forces(self, *, dt_s: float, primary_region_id: int, secondary_region_id: int,
                                     velocity_damping: float = 1.0, flip_blend: float = 0.95,
                                     body_acceleration_mps2: tuple[float, float, float] = (0.0, 0.0, 0.0),
                                     read_report: bool = True) -> TriMooneyShellMpmReport | None:
        """Advance shell dynamics using preloaded external_force_n as MPM load."""
        body = _vector3(body_acceleration_mps2, "body_acceleration_mps2")
        params = self._params(dt_s=dt_s, velocity_damping=velocity_damping,
                              flip_blend=_validate_flip_blend(flip_blend), body_acceleration=body, region_loads=1,
                              preserve=1, primary_region_id=primary_region_id,
                              secondary_region_id=secondary_region_id, area_load_region_id=int(primary_region_id))
        return self._run(params, read_report)

    def save_state(self) -> None:
        """mooney_shell_mpm.py:1294-1299."""
        self.saved_x.copy_from(self.x)
        self.saved_u.copy_from(self.u)
        self.saved_v.copy_from(self.v)

    def restore_state(self) -> None:
        """mooney_shell_mpm.py:1301-1309: positions back, forces cleared, normals rebuilt."""
        self.x.copy_from(self.saved_x)
        self.u.copy_from(self.saved_u)
        self.v.copy_from(self.saved_v)
        self.internal_force_n.tensor.zero_()
        self.external_force_n.tensor.zero_()
        _native.call("efsi_shell_update_normals", byref(self._state_struct()), c_void_p(current_stream_handle()))

    def report(self) -> TriMooneyShellMpmReport:
        """mooney_shell_mpm.py:1317-1391: one host read of the packed snapshot."""
        snapshot = self.report_host_snapshot.to_numpy()
        values = snapshot[:32]
        counts = snapshot[32:37]
        self.last_report_host_reads = 1
        _raise_if_all_particles_out_of_bounds(int(self.particle_count), int(counts[1]))
        force_l2 = float(values[0]) ** 0.5
        total_area = float(values[4])
        spacing = (total_area / self.particle_count) ** 0.5 if total_area > 0.0 and self.particle_count > 0 else 0.0
        pc = max(int(counts[3]), 1)
        sc = max(int(counts[4]), 1)

        def v3(k, d=1):
            return (float(values[k]) / d, float(values[k + 1]) / d, float(values[k + 2]) / d)

        return TriMooneyShellMpmReport(
            particle_count=self.particle_count,
            face_count=self.face_count,
            edge_count=self.edge_count,
            active_grid_nodes=int(counts[0]),
            grid_out_of_bounds_particle_count=int(counts[1]),
            particle_spacing_m=spacing,
            grid_spacing_m=self.dx,
            mean_radial_stretch=float(values[5]) / max(int(counts[2]), 1),
            max_radial_stretch_error=float(values[6]),
            max_edge_strain=float(values[7]),
            max_speed_mps=float(values[8]),
            total_mass_kg=float(values[9]),
            total_area_m2=total_area,
            primary_mean_displacement_m=v3(10, pc),
            primary_mean_velocity_mps=v3(13, pc),
            secondary_mean_displacement_m=v3(16, sc),
            secondary_mean_velocity_mps=v3(19, sc),
            particle_momentum_kg_mps=v3(22),
            grid_momentum_kg_mps=v3(25),
            total_force_n=v3(28),
            internal_force_rms_n=(force_l2 * force_l2 / max(self.particle_count, 1)) ** 0.5,
            net_internal_force_relative_error=(
                (float(values[1]) ** 2 + float(values[2]) ** 2 + float(values[3]) ** 2) ** 0.5 / max(force_l2, 1.0e-20)
            ),
            transfer_relative_error=float(values[31]),
        )
