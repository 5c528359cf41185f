"""Neo-Hookean MLS/APIC-MPM state, B200 path (drop-in for
simulation_core/neo_hookean_mpm.py).

Same constructor, public fields (``x, v, C, F, mass_kg, volume_m3,
external_force_n, ...``) and ``step`` / ``report`` semantics as the reference
(neo_hookean_mpm.py:57-1066).  ``step`` runs the binned P2G / grid update / G2P
substep of ``efsi_mpm_step`` on the device.
"""

from __future__ import annotations

from ctypes import byref, c_void_p
from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from .field import Field
from .runtime import TaichiRuntimeConfig, current_stream_handle, f32, i32, init_runtime

MIN_DEFORMATION_SINGULAR_VALUE = 1.0e-2
MAX_DEFORMATION_SINGULAR_VALUE = 1.0e2


def _vector3(value, name: str) -> tuple[float, float, float]:
    if len(value) != 3:
        raise ValueError(f"{name} must contain exactly 3 components")
    return (float(value[0]), float(value[1]), float(value[2]))


def _raise_if_all_particles_out_of_bounds(particle_count: int, oob: int) -> None:
    # neo_hookean_mpm.py:18-26
    if particle_count > 0 and oob == particle_count:
        raise RuntimeError(
            f"all {particle_count} MPM particles are outside the background grid; the solid has left the simulation domain"
        )


@dataclass(frozen=True)
class NeoHookeanMpmReport:
    particle_count: int
    active_grid_nodes: int
    grid_out_of_bounds_particle_count: int
    particle_spacing_m: float
    grid_spacing_m: tuple[float, float, float]
    total_mass_kg: float
    total_volume_m3: float
    primary_mean_displacement_m: tuple[float, float, float]
    primary_mean_velocity_mps: tuple[float, float, float]
    secondary_mean_displacement_m: tuple[float, float, float]
    secondary_mean_velocity_mps: tuple[float, float, float]
    particle_momentum_kg_mps: tuple[float, float, float]
    grid_momentum_kg_mps: tuple[float, float, float]
    external_force_n: tuple[float, float, float]
    transfer_relative_error: float
    max_speed_mps: float
    max_abs_j: float
    deformation_clamp_count: int
    mean_radial_stretch: float
    max_radial_stretch_error: float


class NeoHookeanMpmState:
    """GPU Neo-Hookean APIC/MLS-MPM particle state (neo_hookean_mpm.py:53)."""

    def __init__(self, particle_capacity: int, bounds_min_m, bounds_max_m, grid_nodes, runtime: TaichiRuntimeConfig | None = None):
        self.device = init_runtime(runtime)
        if particle_capacity <= 0:
            raise ValueError("particle_capacity must be positive")
        if min(grid_nodes) < 4:
            raise ValueError("grid_nodes must be at least 4 in each direction")
        self.particle_capacity = int(particle_capacity)
        self.particle_count = 0
        self.grid_nodes = tuple(int(v) for v in grid_nodes)
        self.nx, self.ny, self.nz = self.grid_nodes
        self.bounds_min = tuple(float(v) for v in bounds_min_m)
        self.bounds_max = tuple(float(v) for v in bounds_max_m)
        self.dx = tuple((self.bounds_max[a] - self.bounds_min[a]) / self.grid_nodes[a] for a in range(3))
        if min(self.dx) <= 0.0:
            raise ValueError("bounds must define a positive grid spacing")
        cap = self.particle_capacity
        dev = self.device

        def vec(n=cap):
            return Field((n,), f32, n=3, device=dev)

        def mat():
            return Field((cap,), f32, n=3, m=3, device=dev)

        def sca(dtype=f32, n=cap):
            return Field((n,), dtype, device=dev)

        self.x = vec()
        self.rest_x = vec()
        self.v = vec()
        self.C = mat()
        self.F = mat()
        self.saved_x = vec()
        self.saved_v = vec()
        self.saved_C = mat()
        self.saved_F = mat()
        self.mass_kg = sca()
        self.volume_m3 = sca()
        self.area_weight_m2 = sca()
        self.rest_area_weight_m2 = sca()
        self.region_id = sca(i32)
        self.fixed_particle = sca(i32)
        self.surface_normal = vec()
        self.rest_surface_normal = vec()
        self.external_force_n = vec()
        self.rest_center_m = Field((), f32, n=3, device=dev)
        self.grid_mass_kg = Field(self.grid_nodes, f32, device=dev)
        self.grid_velocity_mps = Field(self.grid_nodes, f32, n=3, device=dev)
        self.grid_force_n = Field(self.grid_nodes, f32, n=3, device=dev)
        self.report_host_snapshot = Field((34,), f32, device=dev)
        self.primary_mass_kg = Field((), f32, device=dev)
        self.secondary_mass_kg = Field((), f32, device=dev)
        self.last_report_host_reads = 0
        self._report_dev = torch.zeros(34, dtype=torch.float64, device=dev)
        handle = c_void_p()
        _native.call("efsi_mpm_plan_create", cap, self.nx, self.ny, self.nz, byref(handle))
        self._plan = handle
        self.F.tensor.copy_(torch.eye(3, dtype=torch.float32).expand(cap, 3, 3))

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value:
            try:
                _native.load().efsi_mpm_plan_destroy(plan)
            except Exception:
                pass
            self._plan = None

    # ------------------------------------------------------------------
    # initialisation helpers (neo_hookean_mpm.py:140-357)
    # ------------------------------------------------------------------
    def _update_rest_center(self) -> None:
        n = int(self.particle_count)
        if n > 0:
            self.rest_center_m.tensor.copy_(self.rest_x.tensor[:n].sum(dim=0) / float(n))
        else:
            self.rest_center_m.tensor.zero_()

    def initialize_box(self, *, particle_counts, box_min_m, box_max_m, density_kgm3: float) -> None:
        nxp, nyp, nzp = (int(v) for v in particle_counts)
        if min(nxp, nyp, nzp) <= 0:
            raise ValueError("particle_counts must be positive")
        count = nxp * nyp * nzp
        if count > self.particle_capacity:
            raise ValueError("particle count exceeds capacity")
        self.particle_count = count
        lo = np.asarray(box_min_m, dtype=np.float32)
        hi = np.asarray(box_max_m, dtype=np.float32)
        volume = np.float32((hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]))
        pvol = np.float32(volume / np.float32(max(count, 1)))
        p = np.arange(count)
        ix, iy, iz = p % nxp, (p // nxp) % nyp, p // (nxp * nyp)
        pos = np.stack(
            [
                lo[0] + (ix.astype(np.float32) + np.float32(0.5)) * (hi[0] - lo[0]) / np.float32(nxp),
                lo[1] + (iy.astype(np.float32) + np.float32(0.5)) * (hi[1] - lo[1]) / np.float32(nyp),
                lo[2] + (iz.astype(np.float32) + np.float32(0.5)) * (hi[2] - lo[2]) / np.float32(nzp),
            ],
            axis=1,
        ).astype(np.float32)
        self.load_particles(
            positions_m=pos,
            volumes_m3=np.full(count, pvol, dtype=np.float32),
            masses_kg=np.full(count, np.float32(density_kgm3) * pvol, dtype=np.float32),
        )

    def load_particles(self, *, positions_m, volumes_m3, masses_kg, region_ids=None, fixed=None, normals=None, areas_m2=None) -> None:
        """Bulk particle upload (positions at rest, zero v / C, F = I)."""
        pos = np.asarray(positions_m, dtype=np.float32).reshape(-1, 3)
        count = pos.shape[0]
        if count > self.particle_capacity:
            raise ValueError("particle count exceeds capacity")
        self.particle_count = count
        cap = self.particle_capacity
        dev = self.device

        def put(field: Field, values):
            t = torch.zeros(field.tensor.shape, dtype=field.dtype)
            if values is not None:
                t[:count] = torch.as_tensor(np.asarray(values)).to(field.dtype).reshape(t[:count].shape)
            field.tensor.copy_(t.to(dev))

        put(self.x, pos)
        put(self.rest_x, pos)
        self.v.tensor.zero_()
        self.C.tensor.zero_()
        self.F.tensor.copy_(torch.eye(3, dtype=torch.float32, device=dev).expand(cap, 3, 3))
        put(self.volume_m3, np.asarray(volumes_m3, dtype=np.float32))
        put(self.mass_kg, np.asarray(masses_kg, dtype=np.float32))
        put(self.region_id, None if region_ids is None else np.asarray(region_ids, dtype=np.int32))
        put(self.fixed_particle, None if fixed is None else np.asarray(fixed, dtype=np.int32))
        put(self.surface_normal, None if normals is None else np.asarray(normals, dtype=np.float32))
        put(self.rest_surface_normal, None if normals is None else np.asarray(normals, dtype=np.float32))
        put(self.area_weight_m2, None if areas_m2 is None else np.asarray(areas_m2, dtype=np.float32))
        put(self.rest_area_weight_m2, None if areas_m2 is None else np.asarray(areas_m2, dtype=np.float32))
        self.external_force_n.tensor.zero_()
        self._update_rest_center()

    def set_uniform_velocity(self, velocity_mps) -> None:
        n = int(self.particle_count)
        self.v.tensor[:n] = torch.tensor([float(c) for c in velocity_mps], dtype=torch.float32, device=self.device)

    def set_uniform_external_force(self, force_n) -> None:
        n = int(self.particle_count)
        self.external_force_n.tensor[:n] = torch.tensor([float(c) for c in force_n], dtype=torch.float32, device=self.device)

    def set_region_normal_pressure(self, *, region_id: int, pressure_pa: float) -> None:
        if self.particle_count <= 0:
            raise ValueError("initialize particles before setting loads")
        n = int(self.particle_count)
        sel = (self.region_id.tensor[:n] == int(region_id)).unsqueeze(1)
        load = -np.float32(pressure_pa) * self.area_weight_m2.tensor[:n, None] * self.surface_normal.tensor[:n]
        self.external_force_n.tensor[:n] = torch.where(sel, load, torch.zeros_like(load))

    # ------------------------------------------------------------------
    # substep (neo_hookean_mpm.py:961-986)
    # ------------------------------------------------------------------
    def _state_struct(self) -> _native.MpmState:
        s = _native.MpmState()
        s.particle_count = int(self.particle_count)
        s.nx, s.ny, s.nz = self.grid_nodes
        for a in range(3):
            s.bmin[a] = float(np.float32(self.bounds_min[a]))
            s.dx[a] = float(np.float32(self.dx[a]))
        s.x = self.x.ptr()
        s.v = self.v.ptr()
        s.C = self.C.ptr()
        s.F = self.F.ptr()
        s.mass = self.mass_kg.ptr()
        s.volume = self.volume_m3.ptr()
        s.fext = self.external_force_n.ptr()
        s.fixed = self.fixed_particle.ptr()
        s.region = self.region_id.ptr()
        s.rest_x = self.rest_x.ptr()
        s.normal = self.surface_normal.ptr()
        s.area = self.area_weight_m2.ptr()
        s.rest_normal = self.rest_surface_normal.ptr()
        s.rest_area = self.rest_area_weight_m2.ptr()
        s.grid_mass = self.grid_mass_kg.ptr()
        s.grid_velocity = self.grid_velocity_mps.ptr()
        s.grid_force = self.grid_force_n.ptr()
        return s

    def step(
        self,
        *,
        dt_s: float,
        mu_pa: float,
        lambda_pa: float,
        primary_region_id: int,
        secondary_region_id: int,
        velocity_damping: float = 1.0,
        read_report: bool = True,
    ) -> NeoHookeanMpmReport | None:
        if self.particle_count <= 0:
            raise ValueError("initialize particles before stepping")
        state = self._state_struct()
        _native.call(
            "efsi_mpm_step",
            self._plan,
            byref(state),
            float(dt_s),
            float(mu_pa),
            float(lambda_pa),
            float(velocity_damping),
            int(primary_region_id),
            int(secondary_region_id),
            c_void_p(self._report_dev.data_ptr()),
            c_void_p(current_stream_handle()),
        )
        self.report_host_snapshot.tensor.copy_(self._report_dev.to(torch.float32))
        if not read_report:
            self.last_report_host_reads = 0
            return None
        return self.report()

    # ------------------------------------------------------------------
    # snapshots and report (neo_hookean_mpm.py:988-1066)
    # ------------------------------------------------------------------
    def save_state(self) -> None:
        if self.particle_count <= 0:
            raise ValueError("initialize particles before saving state")
        n = int(self.particle_count)
        for src, dst in ((self.x, self.saved_x), (self.v, self.saved_v), (self.C, self.saved_C), (self.F, self.saved_F)):
            dst.tensor[:n].copy_(src.tensor[:n])

    def restore_state(self) -> None:
        if self.particle_count <= 0:
            raise ValueError("initialize particles before restoring state")
        n = int(self.particle_count)
        for src, dst in ((self.saved_x, self.x), (self.saved_v, self.v), (self.saved_C, self.C), (self.saved_F, self.F)):
            dst.tensor[:n].copy_(src.tensor[:n])
        self._refresh_surface_geometry(n)
        self.external_force_n.tensor[:n].zero_()

    def _refresh_surface_geometry(self, n: int) -> None:
        # Nanson update of area / normal from F (neo_hookean_mpm.py:674-685).
        F = self.F.tensor[:n]
        rn = self.rest_surface_normal.tensor[:n]
        ra = self.rest_area_weight_m2.tensor[:n]
        J = torch.linalg.det(F)
        cof = torch.linalg.inv(F).transpose(1, 2) * J[:, None, None]
        av = torch.einsum("pij,pj->pi", cof, rn)
        sc = av.norm(dim=1)
        ok = (ra > 0) & (rn.norm(dim=1) > 1e-12) & (J > 1e-12) & (sc > 1e-12)
        self.surface_normal.tensor[:n] = torch.where(ok[:, None], av / sc.clamp_min(1e-30)[:, None], self.surface_normal.tensor[:n])
        self.area_weight_m2.tensor[:n] = torch.where(ok, ra * sc, self.area_weight_m2.tensor[:n])

    def report(self) -> NeoHookeanMpmReport:
        snapshot = self.report_host_snapshot.to_numpy()
        values = snapshot[:28].astype(np.float64)
        counts = snapshot[28:34]
        self.last_report_host_reads = 1
        _raise_if_all_particles_out_of_bounds(int(self.particle_count), int(counts[1]))
        total_volume = float(values[1])
        spacing = (total_volume / self.particle_count) ** (1.0 / 3.0) if total_volume > 0.0 and self.particle_count > 0 else 0.0
        pc = max(int(counts[4]), 1)
        sc = max(int(counts[5]), 1)
        rc = max(int(counts[3]), 1)
        return NeoHookeanMpmReport(
            particle_count=int(self.particle_count),
            active_grid_nodes=int(counts[0]),
            grid_out_of_bounds_particle_count=int(counts[1]),
            particle_spacing_m=spacing,
            grid_spacing_m=self.dx,
            total_mass_kg=float(values[0]),
            total_volume_m3=total_volume,
            primary_mean_displacement_m=tuple(float(values[16 + a]) / pc for a in range(3)),
            primary_mean_velocity_mps=tuple(float(values[19 + a]) / pc for a in range(3)),
            secondary_mean_displacement_m=tuple(float(values[22 + a]) / sc for a in range(3)),
            secondary_mean_velocity_mps=tuple(float(values[25 + a]) / sc for a in range(3)),
            particle_momentum_kg_mps=tuple(float(values[2 + a]) for a in range(3)),
            grid_momentum_kg_mps=tuple(float(values[5 + a]) for a in range(3)),
            external_force_n=tuple(float(values[8 + a]) for a in range(3)),
            transfer_relative_error=float(values[11]),
            max_speed_mps=float(values[12]),
            max_abs_j=float(values[13]),
            deformation_clamp_count=int(counts[2]),
            mean_radial_stretch=float(values[14]) / rc,
            max_radial_stretch_error=float(values[15]),
        )
