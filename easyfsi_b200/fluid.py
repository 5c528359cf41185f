"""Cartesian fluid solver, B200 path (drop-in for simulation_core/fluid.py).

``CartesianFluidSolver`` keeps the reference's constructor, public fields and
the methods on the coupled-step hot path with their Python signatures:
``predict`` (fluid.py:2515), ``compute_divergence`` (:3488), ``project``
(:6889), ``spread_surface_forces`` (:3275), ``apply_body_force`` (:3330),
``save_state`` / ``restore_state`` (:2266), plus the private kernels the
reference's tests drive directly (``_fv_laplacian_apply_kernel``,
``_weighted_dot_kernel``, ``_mg_restrict_residual_kernel``, ...).  Fields are
torch CUDA tensors behind the ``Field`` adapter; every numerical operation is a
call into the sm_100a library through the C ABI (``easyfsi_b200._native``).

Out of scope (the HIBM sharp-interface machinery outside the hot path):
interface row-list / slot couplings, outlet reachability and component
anchoring, viscous constraint blending and local divergence cleanup.  Their
fields exist where the plain path reads them; their kernels are not provided.
"""

from __future__ import annotations

import ctypes
import math
from ctypes import byref, c_double, c_void_p
from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from .field import Field
from .grid import (
    CartesianGrid,
    FluidDomainSpec,
    GradedGridSpec,
    RefinementRegion,
    build_graded_grid,
    coarsen_axis_widths,
    multigrid_axis_widths,
    multigrid_shapes,
)
from .runtime import TaichiRuntimeConfig, current_stream_handle, f32, f64, i32, init_runtime

__all__ = [
    "CG_PRECONDITIONER_CHOICES",
    "CartesianFluidSolver",
    "CartesianGrid",
    "FluidDomainSpec",
    "ForceSpreadingReport",
    "FluidImpulseReport",
    "GradedGridSpec",
    "RefinementRegion",
    "VelocityDirichletBoundaryReport",
    "build_graded_grid",
]

# "fv_multigrid_mixed" (no reference counterpart): the fv_multigrid V-cycle
# with FP32 storage and arithmetic on level 0, inside the same FP64 flexible CG
# (true residual, inner products and scalars in FP64).
PRESSURE_INTERFACE_COUPLING_SLOT_COUNT = 16  # pressure_interface.py:10: one slot plus 15 extra per owner cell
CG_PRECONDITIONER_CHOICES = ("auto", "jacobi", "fv_multigrid", "fv_multigrid_light", "fv_multigrid_mixed", "learned",
                             "learned_no_fallback")
_PRECOND_CODE = {"jacobi": 0, "fv_multigrid": 1, "fv_multigrid_light": 2, "fv_multigrid_mixed": 3, "learned": 4,
                 "learned_no_fallback": 5}
_BREAKDOWN_TEXT = {
    0: "",
    1: "initial residual/preconditioner dot is not positive finite",
    2: "device-side CG scalar update failed",
    3: "restarted residual/preconditioner dot is not positive finite",
}


@dataclass(frozen=True)
class ForceSpreadingReport:
    surface_force_n: tuple[float, float, float]
    grid_force_n: tuple[float, float, float]
    action_reaction_relative_error: float
    active_grid_cells: int


@dataclass(frozen=True)
class FluidImpulseReport:
    grid_impulse_n_s: tuple[float, float, float]
    momentum_delta_n_s: tuple[float, float, float]
    impulse_relative_error: float
    active_velocity_cells: int


@dataclass(frozen=True)
class VelocityDirichletBoundaryReport:
    active_cells: int
    max_delta_mps: float
    mean_delta_mps: float
    momentum_delta_n_s: tuple[float, float, float] = (0.0, 0.0, 0.0)


def _stream():
    return c_void_p(current_stream_handle())


def _ptr(field_or_tensor):
    t = field_or_tensor.tensor if isinstance(field_or_tensor, Field) else field_or_tensor
    if not t.is_contiguous():
        raise RuntimeError("non-contiguous storage cannot cross the C ABI")
    return c_void_p(t.data_ptr())


class CartesianFluidSolver:
    """Cell-centred 3D Cartesian fluid state for coupled FSI simulations (fluid.py:684)."""

    DEFAULT_MULTIGRID_CYCLES = 12
    DEFAULT_NONUNIFORM_MULTIGRID_CYCLES = 24

    _build_multigrid_shapes = staticmethod(multigrid_shapes)
    _coarsen_axis_widths = staticmethod(coarsen_axis_widths)
    _build_multigrid_axis_widths = staticmethod(multigrid_axis_widths)

    def default_multigrid_cycles(self) -> int:
        return self.DEFAULT_MULTIGRID_CYCLES if self.grid.is_uniform else self.DEFAULT_NONUNIFORM_MULTIGRID_CYCLES

    def __init__(self, spec: FluidDomainSpec, runtime: TaichiRuntimeConfig | None = None):
        self.device = init_runtime(runtime)
        self.spec = spec
        self.grid = spec.cartesian_grid
        self.nx, self.ny, self.nz = self.grid.grid_nodes
        if self.grid.is_uniform:
            self.dx, self.dy, self.dz = self.grid.uniform_spacing_m
        else:
            self.dx, self.dy, self.dz = (
                min(self.grid.cell_widths_x_m),
                min(self.grid.cell_widths_y_m),
                min(self.grid.cell_widths_z_m),
            )
        self.bounds_min = tuple(float(v) for v in self.grid.bounds_min_m)
        self.bounds_max = tuple(float(v) for v in self.grid.bounds_max_m)
        self.rho = float(spec.density_kgm3)
        self.mu = float(spec.viscosity_pa_s)
        self.dt = float(spec.dt_s)
        shape = self.grid.grid_nodes
        dev = self.device

        def scalar(dtype, shp=shape):
            return Field(shp, dtype, device=dev)

        def vector(dtype, shp=shape):
            return Field(shp, dtype, n=3, device=dev)

        self.velocity = vector(f32)
        self.velocity_prev = vector(f32)
        self.saved_velocity = vector(f32)
        self.pressure = scalar(f64)
        self.saved_pressure = scalar(f64)
        self.fsi_pressure = scalar(f64)
        self.pressure_tmp = scalar(f64)
        self.pressure_accum = scalar(f64)
        self.divergence = scalar(f32)
        self.pressure_interface_projection_divergence_s = scalar(f64)
        self.volume_source_s = scalar(f32)
        self.pressure_interface_matrix_diagonal = scalar(f64)
        self.pressure_interface_matrix_rhs = scalar(f64)
        # interface couplings (fluid.py:772-811): per-cell slots and an
        # explicit row list; the 15 extra slots per cell and the row arrays
        # (capacity nx * ny * nz) are created on first access
        self.pressure_interface_coupling_active = scalar(i32)
        self.pressure_interface_coupling_neighbor = vector(i32)
        self.pressure_interface_coupling_coefficient = scalar(f64)
        self.pressure_interface_row_capacity = int(np.prod(shape))
        self.pressure_interface_row_count = Field((), i32, device=dev)
        self.obstacle = scalar(i32)
        self.force = vector(f32)
        self.velocity_dirichlet_boundary_active = scalar(i32)
        self.velocity_dirichlet_boundary_value_mps = vector(f32)
        self.velocity_dirichlet_boundary_projection_weight = scalar(f32)
        self.velocity_dirichlet_boundary_marker_region_id = scalar(i32)
        self.fv_diag = scalar(f64)
        self.cg_r = scalar(f64)
        self.cg_rhs = scalar(f64)
        self.cg_z = scalar(f64)
        self.cg_d = scalar(f64)
        self.cg_Ad = scalar(f64)
        self.cg_r_old = scalar(f64)
        self.cg_mg_rhs = scalar(f64)
        self.cg_mg_residual = scalar(f64)
        for name in ("cg_rz", "cg_rz_new", "cg_dAd", "cg_rr", "cg_beta_numerator", "cg_alpha", "cg_beta"):
            setattr(self, name, Field((), f64, device=dev))
        self.cg_breakdown_code = Field((), i32, device=dev)
        self.cg_breakdown_dAd = Field((), f64, device=dev)

        # Axis metric fields, f32 on the device like the reference (fluid.py:1013-1024).
        g = self.grid
        for axis, name in enumerate("xyz"):
            n = shape[axis]
            setattr(self, f"cell_width_{name}_m", self._axis_field(g._widths(axis)))
            setattr(self, f"cell_face_{name}_m", self._axis_field(g.axis_faces(axis)))
            setattr(self, f"cell_center_{name}_m", self._axis_field(g.axis_centers(axis)))
            setattr(self, f"center_distance_{name}_m", self._axis_field(g.axis_center_distances(axis)))
            assert getattr(self, f"cell_width_{name}_m").shape == (n,)

        # Multigrid hierarchy (fluid.py:1026-1075).
        self._mg_shapes = multigrid_shapes(shape)
        self._mg_axis_widths_m = multigrid_axis_widths(self.grid, self._mg_shapes)
        self._mg_cell_width_x_m = [self.cell_width_x_m]
        self._mg_cell_width_y_m = [self.cell_width_y_m]
        self._mg_cell_width_z_m = [self.cell_width_z_m]
        self._mg_center_distance_x_m = [self.center_distance_x_m]
        self._mg_center_distance_y_m = [self.center_distance_y_m]
        self._mg_center_distance_z_m = [self.center_distance_z_m]
        for level, widths in enumerate(self._mg_axis_widths_m[1:], start=1):
            for axis, name in enumerate("xyz"):
                centers = CartesianGrid._axis_centers(self.bounds_min[axis], widths[axis])
                getattr(self, f"_mg_cell_width_{name}_m").append(self._axis_field(widths[axis]))
                getattr(self, f"_mg_center_distance_{name}_m").append(
                    self._axis_field(CartesianGrid._axis_center_distances(centers, widths[axis]))
                )
        self._mg_pressure = [self.pressure]
        self._mg_tmp = [self.pressure_tmp]
        self._mg_obstacle = [self.obstacle]
        self._mg_velocity_dirichlet_boundary_active = [self.velocity_dirichlet_boundary_active]
        self._mg_velocity_dirichlet_boundary_projection_weight = [self.velocity_dirichlet_boundary_projection_weight]
        self._mg_pressure_interface_matrix_diagonal = [self.pressure_interface_matrix_diagonal]
        self._mg_rhs = [scalar(f64)]
        self._mg_residual = [scalar(f64)]
        self._pcg_mg_rhs = [self.cg_mg_rhs]
        self._pcg_mg_residual = [self.cg_mg_residual]
        self._pcg_mg_pressure = [self.cg_z]
        self._pcg_mg_tmp = [self.cg_Ad]
        for lshape in self._mg_shapes[1:]:
            self._mg_rhs.append(scalar(f32, lshape))
            self._mg_residual.append(scalar(f32, lshape))
            self._mg_pressure.append(scalar(f32, lshape))
            self._mg_tmp.append(scalar(f32, lshape))
            self._mg_obstacle.append(scalar(i32, lshape))
            self._mg_velocity_dirichlet_boundary_active.append(scalar(i32, lshape))
            self._mg_velocity_dirichlet_boundary_projection_weight.append(scalar(f32, lshape))
            self._mg_pressure_interface_matrix_diagonal.append(scalar(f32, lshape))
            self._pcg_mg_rhs.append(scalar(f32, lshape))
            self._pcg_mg_residual.append(scalar(f32, lshape))
            self._pcg_mg_pressure.append(scalar(f32, lshape))
            self._pcg_mg_tmp.append(scalar(f32, lshape))

        # Native plan: level metric views + f64 face tables + work vectors.
        self._level_descs = (_native.LevelDesc * len(self._mg_shapes))()
        for level, lshape in enumerate(self._mg_shapes):
            d = self._level_descs[level]
            d.nx, d.ny, d.nz = lshape
            d.wx = self._mg_cell_width_x_m[level].ptr()
            d.wy = self._mg_cell_width_y_m[level].ptr()
            d.wz = self._mg_cell_width_z_m[level].ptr()
            d.cdx = self._mg_center_distance_x_m[level].ptr()
            d.cdy = self._mg_center_distance_y_m[level].ptr()
            d.cdz = self._mg_center_distance_z_m[level].ptr()
        torch.cuda.synchronize(self.device)
        handle = c_void_p()
        _native.call(
            "efsi_fv_plan_create", self._level_descs, len(self._mg_shapes), 1 if self.grid.is_uniform else 0, byref(handle)
        )
        self._plan = handle
        self._axes = _native.GridAxes(
            self.cell_face_x_m.ptr(),
            self.cell_face_y_m.ptr(),
            self.cell_face_z_m.ptr(),
            self.cell_center_x_m.ptr(),
            self.cell_center_y_m.ptr(),
            self.cell_center_z_m.ptr(),
        )
        self._report = torch.zeros(16, dtype=torch.float64, device=dev)
        self._vdir_active = False
        self._iface_active = False

        self.last_cg_iterations = 0
        self.last_cg_initial_relative_residual = math.inf
        self.last_cg_relative_residual = math.inf
        self.last_cg_converged = False
        self.last_cg_breakdown = ""
        self.last_cg_host_residual_checks = 0
        self.last_cg_mean_host_reads = 0
        self.last_cg_mean_projection_count = 0
        self.last_cg_unreached_set_mean_projection_count = 0
        self.last_cg_restart_count = 0
        self.last_cg_restart_count_measured = False
        self.last_cg_restart_policy = ""
        self.last_cg_breakdown_dAd = 0.0
        self.last_cg_used_multigrid = False
        # steps captured into CUDA graphs (runtime.StepGraph): PCG solves run
        # their device-side loop and the predictor copies instead of exchanging
        # its buffers
        self.device_loop_solves = False
        self._hibm_pressure_unreached_count = 0
        self._hibm_pressure_unreached_component_count = 0
        self.last_hibm_unreached_incompatible_component_count = 0
        self.last_hibm_unreached_component_rhs_mean_max_abs = 0.0
        self.last_hibm_unreached_component_rhs_integral_max_abs = 0.0
        self.last_hibm_unreached_cells_with_interface_diagonal = 0
        self.last_hibm_unreached_cells_with_interface_coupling = 0
        self.last_hibm_unreached_components_with_interface_hits = 0
        self.last_unreached_divergence_raw_stats = {"max_abs": 0.0, "l2": 0.0, "count": 0}
        self.last_unreached_divergence_stats = {"max_abs": 0.0, "l2": 0.0, "count": 0}
        self.last_divergence_report_host_reads = 0
        self._reset_project_cg_stats()
        self.clear()

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value:
            try:
                _native.load().efsi_fv_plan_destroy(plan)
            except Exception:
                pass
            self._plan = None
        reach = getattr(self, "_reach_plan", None)
        if reach is not None and reach.value:
            try:
                _native.load().efsi_reach_plan_destroy(reach)
            except Exception:
                pass
            self._reach_plan = None

    # ------------------------------------------------------------------
    # helpers
    # ------------------------------------------------------------------
    def _axis_field(self, values) -> Field:
        field = Field((len(values),), f32, device=self.device)
        field.tensor.copy_(torch.tensor([float(v) for v in values], dtype=torch.float32))
        return field

    def _cell_volume_f32(self) -> torch.Tensor:
        return (
            self.cell_width_x_m.tensor[:, None, None]
            * self.cell_width_y_m.tensor[None, :, None]
            * self.cell_width_z_m.tensor[None, None, :]
        )

    _LAZY_COUPLING_FIELDS = ("pressure_interface_coupling_extra_neighbor",
                             "pressure_interface_coupling_extra_coefficient", "pressure_interface_row_owner",
                             "pressure_interface_row_neighbor", "pressure_interface_row_transmissibility")

    def __getattr__(self, name):
        # the large coupling arrays of the reference (fluid.py:783-811) exist
        # from their first access on
        if name in CartesianFluidSolver._LAZY_COUPLING_FIELDS:
            dev = self.__dict__["device"]
            shape = tuple(self.grid.grid_nodes)
            cap = self.pressure_interface_row_capacity
            extra = shape + (PRESSURE_INTERFACE_COUPLING_SLOT_COUNT - 1,)
            made = {
                "pressure_interface_coupling_extra_neighbor": lambda: Field(extra, i32, n=3, device=dev),
                "pressure_interface_coupling_extra_coefficient": lambda: Field(extra, f64, device=dev),
                "pressure_interface_row_owner": lambda: Field((cap,), i32, n=3, device=dev),
                "pressure_interface_row_neighbor": lambda: Field((cap,), i32, n=3, device=dev),
                "pressure_interface_row_transmissibility": lambda: Field((cap,), f64, device=dev),
            }[name]()
            self.__dict__[name] = made
            return made
        raise AttributeError(f"{type(self).__name__!s} has no attribute {name!r}")

    def _structure_key(self):
        fields = [
            self.obstacle,
            self.velocity_dirichlet_boundary_active,
            self.velocity_dirichlet_boundary_projection_weight,
            self.pressure_interface_matrix_diagonal,
            self.pressure_interface_coupling_active,
            self.pressure_interface_coupling_neighbor,
            self.pressure_interface_coupling_coefficient,
            self.pressure_interface_row_count,
        ]
        fields += [self.__dict__[n] for n in CartesianFluidSolver._LAZY_COUPLING_FIELDS if n in self.__dict__]
        fields += [self.cell_width_x_m, self.cell_width_y_m, self.cell_width_z_m]
        return tuple((f.tensor.data_ptr(), f.tensor._version) for f in fields)

    def _interface_coupling_rows(self):
        """fluid.py:4345-4456: the couplings as (owner, neighbour, T) pairs in
        the reference's visiting order -- the row list when its count is
        positive, else the per-cell slots in cell order -- kept where both
        cells are fluid and T > 0; returned as CSR rows per receiving cell
        (entries in visiting order, coef = T / V_receiver with V the f32
        product of the widths).  None when there are none."""
        nx, ny, nz = self.grid.grid_nodes
        obs = self.obstacle.tensor.reshape(-1)
        row_count = int(self.pressure_interface_row_count[None])
        if row_count > 0:
            limit = min(row_count, self.pressure_interface_row_capacity)
            own = self.pressure_interface_row_owner.tensor[:limit].to(torch.int64)
            nbr = self.pressure_interface_row_neighbor.tensor[:limit].to(torch.int64)
            trans = self.pressure_interface_row_transmissibility.tensor[:limit]
            inside = ((own >= 0) & (own < torch.tensor([nx, ny, nz], device=own.device))).all(dim=1)
            inside &= ((nbr >= 0) & (nbr < torch.tensor([nx, ny, nz], device=own.device))).all(dim=1)
        else:
            act = self.pressure_interface_coupling_active.tensor.reshape(-1)
            if not bool((act > 0).any()):
                return None
            have_extra = "pressure_interface_coupling_extra_neighbor" in self.__dict__
            n_slots = PRESSURE_INTERFACE_COUPLING_SLOT_COUNT if have_extra else 1
            cells = torch.nonzero((act > 0) & (obs == 0)).reshape(-1)
            slots = torch.clamp(act[cells], max=n_slots).to(torch.int64)
            nb0 = self.pressure_interface_coupling_neighbor.tensor.reshape(-1, 3)[cells].to(torch.int64)
            tr0 = self.pressure_interface_coupling_coefficient.tensor.reshape(-1)[cells]
            if have_extra:
                xnb = self.pressure_interface_coupling_extra_neighbor.tensor.reshape(-1, n_slots - 1, 3)[cells]
                xtr = self.pressure_interface_coupling_extra_coefficient.tensor.reshape(-1, n_slots - 1)[cells]
                nbr = torch.cat([nb0[:, None, :], xnb.to(torch.int64)], dim=1).reshape(-1, 3)
                trans = torch.cat([tr0[:, None], xtr], dim=1).reshape(-1)
            else:
                nbr, trans = nb0, tr0
            valid_slot = (torch.arange(n_slots, device=cells.device)[None, :] < slots[:, None]).reshape(-1)
            own_lin = cells.repeat_interleave(n_slots)
            own = torch.stack([own_lin // (ny * nz), (own_lin // nz) % ny, own_lin % nz], dim=1)
            inside = valid_slot & ((nbr >= 0) & (nbr < torch.tensor([nx, ny, nz], device=nbr.device))).all(dim=1)
        own_c = torch.where(inside[:, None], own, torch.zeros_like(own))
        nbr_c = torch.where(inside[:, None], nbr, torch.zeros_like(nbr))
        o_lin = (own_c[:, 0] * ny + own_c[:, 1]) * nz + own_c[:, 2]
        n_lin = (nbr_c[:, 0] * ny + nbr_c[:, 1]) * nz + nbr_c[:, 2]
        keep = inside & (obs[o_lin] == 0) & (obs[n_lin] == 0) & (trans > 0.0)
        o_lin, n_lin, trans = o_lin[keep], n_lin[keep], trans[keep]
        own_c, nbr_c = own_c[keep], nbr_c[keep]
        if o_lin.numel() == 0:
            return None
        w = [getattr(self, f"cell_width_{a}_m").tensor for a in "xyz"]

        def volume(ijk):
            v = (w[0][ijk[:, 0]] * w[1][ijk[:, 1]]) * w[2][ijk[:, 2]]  # f32 product, as the reference
            return torch.clamp(v, min=1.0e-30).to(torch.float64)

        # two entries per coupling, owner's first, in visiting order
        recv = torch.stack([o_lin, n_lin], dim=1).reshape(-1)
        src = torch.stack([n_lin, o_lin], dim=1).reshape(-1)
        coef = torch.stack([trans / volume(own_c), trans / volume(nbr_c)], dim=1).reshape(-1)
        order = torch.sort(recv, stable=True).indices
        recv, src, coef = recv[order], src[order], coef[order]
        rows, counts = torch.unique_consecutive(recv, return_counts=True)
        ptr = torch.zeros(rows.numel() + 1, dtype=torch.int64, device=rows.device)
        ptr[1:] = torch.cumsum(counts, dim=0)
        return (rows.to(torch.int32).contiguous(), ptr.to(torch.int32).contiguous(), src.to(torch.int32).contiguous(),
                coef.to(torch.float64).contiguous())

    def _refresh_structure(self) -> None:
        """Rebuild every level's stencil masks from obstacle / Dirichlet rows /
        interface diagonal when one of them changed since the last build (torch
        version counters; one host read decides which optional terms are live)."""
        key = self._structure_key()
        if key == getattr(self, "_structure_cache", None):
            return
        flags = torch.stack(
            [
                (self.velocity_dirichlet_boundary_active.tensor != 0).any(),
                (self.pressure_interface_matrix_diagonal.tensor != 0).any(),
            ]
        ).cpu()
        self._vdir_active = bool(flags[0])
        self._iface_active = bool(flags[1])
        _native.call(
            "efsi_fv_set_masks",
            self._plan,
            self.obstacle.ptr(),
            self.velocity_dirichlet_boundary_active.ptr() if self._vdir_active else None,
            self.velocity_dirichlet_boundary_projection_weight.ptr() if self._vdir_active else None,
            self.pressure_interface_matrix_diagonal.ptr() if self._iface_active else None,
            _stream(),
        )
        csr = self._interface_coupling_rows()
        if csr is None:
            if getattr(self, "_coupling_rows_installed", 0):
                _native.call("efsi_fv_set_interface_coupling", self._plan, 0, None, None, None, None, _stream())
            self._coupling_rows_installed = 0
        else:
            rows, ptr, src, coef = csr
            _native.call("efsi_fv_set_interface_coupling", self._plan, int(rows.numel()), rows.data_ptr(),
                         ptr.data_ptr(), src.data_ptr(), coef.data_ptr(), _stream())
            self._coupling_rows_installed = int(rows.numel())
        self._structure_cache = key

    _BICGSTAB_BREAKDOWN_TEXT = {
        1: "BiCGSTAB shadow residual dot is not finite",
        2: "BiCGSTAB recurrence scalar is not finite",
        3: "BiCGSTAB beta is not finite",
        4: "BiCGSTAB alpha denominator is not finite",
        5: "BiCGSTAB alpha is not finite",
        6: "BiCGSTAB omega denominator is not finite",
        7: "BiCGSTAB omega is not finite",
        8: "BiCGSTAB fallback did not converge",
    }

    def set_learned_preconditioner(self, network) -> None:
        """Attaches a trained ``easyfsi_b200.learned.UNetPreconditioner`` as
        ``cg_preconditioner="learned"`` (no counterpart in the reference):
        inside the flexible PCG the network is the coarse correction of a
        two-level preconditioner (two damped-Jacobi sweeps, the network's
        correction at its energy-minimising scale, two sweeps), with the
        multigrid V-cycle taking over when a 16-iteration block does not halve
        the residual (``"learned_no_fallback"`` runs it alone).  ``None``
        detaches it."""
        self._refresh_structure()
        handle = None if network is None else network.handle
        _native.call("efsi_fv_set_learned_preconditioner", self._plan, handle, _stream())
        self._learned_network = network

    def autotune(self, reps: int = 10) -> list[dict]:
        """Tile autotuner of the V-cycle (``efsi_fv_autotune``; no reference
        counterpart): times a unit of each level's work (level 0: the PCG's
        direction SpMV and a whole V-cycle; a coarse level: its sweep and
        restriction) under every candidate launch shape and keeps the
        fastest.  Returns, per tuned level, the blocks-per-SM multiple picked
        (0: tiled / per-cell kernels) and the time of its unit in
        microseconds."""
        self._refresh_structure()
        n = 16
        choice = (ctypes.c_int32 * n)()
        best = (ctypes.c_double * n)()
        _native.call("efsi_fv_autotune", self._plan, int(reps), choice, best, n, _stream())
        return [{"level": l, "blocks_per_sm": int(choice[l]), "us": float(best[l])} for l in range(n) if choice[l] >= 0]

    def read_device_pcg_stats(self) -> None:
        """After a captured step ran: the statistics of its device-side PCG loop
        (``efsi_fv_pcg_device_stats``) into ``last_cg_*``."""
        stats = _native.CgStats()
        _native.call("efsi_fv_pcg_device_stats", self._plan, byref(stats), _stream())
        self.last_cg_iterations = int(stats.iterations)
        self.last_cg_initial_relative_residual = float(stats.initial_relative_residual)
        self.last_cg_relative_residual = float(stats.relative_residual)
        self.last_cg_converged = bool(stats.converged)
        self.last_cg_breakdown_dAd = float(stats.breakdown_dAd)
        self.last_cg_used_multigrid = bool(stats.used_mg)
        self.last_cg_used_graphs = True
        self._last_cg_breakdown_code = int(stats.breakdown_code)
        self._device_stats_pending = False

    _CG_SCALAR_FIELDS = (("rz", "cg_rz"), ("rz_new", "cg_rz_new"), ("dAd", "cg_dAd"),
                         ("beta_numerator", "cg_beta_numerator"), ("alpha", "cg_alpha"), ("beta", "cg_beta"),
                         ("breakdown_dAd", "cg_breakdown_dAd"), ("breakdown_code", "cg_breakdown_code"))

    def _run_cg_scalar_step(self, name: str, *args) -> None:
        """Runs one of the PCG's device scalar steps on the solver's 0-D
        ``cg_*`` fields: they are written to the plan's device scalars, the
        step runs there (the same device code as the PCG finishers) and the
        results are written back to the fields."""
        vals = _native.CgScalarValues()
        for key, field in self._CG_SCALAR_FIELDS:
            value = getattr(self, field)[None]
            setattr(vals, key, int(value) if key == "breakdown_code" else float(value))
        _native.call("efsi_cg_scalars_write", self._plan, byref(vals), _stream())
        _native.call(name, self._plan, *args, _stream())
        _native.call("efsi_cg_scalars_read", self._plan, byref(vals), _stream())
        for key, field in self._CG_SCALAR_FIELDS:
            getattr(self, field)[None] = getattr(vals, key)

    def _cg_compute_alpha_kernel(self) -> None:
        """fluid.py:4567-4574: alpha = rz / dAd, or breakdown code 1 when dAd <= 0."""
        self._run_cg_scalar_step("efsi_cg_compute_alpha")

    def _cg_compute_beta_kernel(self, use_mg_preconditioner: int) -> None:
        """fluid.py:4590-4601: the flexible / Fletcher-Reeves beta, or
        breakdown code 2 when rz <= 1e-300 or rz_new <= 0."""
        self._run_cg_scalar_step("efsi_cg_compute_beta", 1 if use_mg_preconditioner else 0)

    def _continue_pressure_poisson_fv_bicgstab(self, *, start_iteration: int, max_iters: int, b_norm: float,
                                               outlet: int, tolerance: float, anchor_unreached: bool,
                                               remove_nullspace_mean: bool) -> None:
        """fluid.py:6264-6533: the BiCGSTAB fallback on ``cg_rhs`` from the
        current pressure (``efsi_fv_bicgstab``).  With ``anchor_unreached`` the
        library subtracts the unreached components' means where the reference
        does (the components installed by the reachability marking)."""
        if anchor_unreached and not outlet:
            raise ValueError("the unreached-component anchoring applies to outlet solves only")
        self._refresh_structure()
        self.last_cg_restart_policy = "periodic_exact_residual+bicgstab_fallback"
        self.last_cg_breakdown = ""
        stats = (ctypes.c_int64 * 4)()
        rel = c_double(0.0)
        _native.call("efsi_fv_bicgstab", self._plan, self.cg_rhs.ptr(), self.pressure.ptr(), 1 if outlet else 0,
                     max(1, int(max_iters)), max(0.0, float(tolerance)), float(b_norm),
                     1 if remove_nullspace_mean else 0, stats, byref(rel), current_stream_handle())
        self.last_cg_iterations = int(start_iteration) + int(stats[0])
        self.last_cg_converged = bool(stats[1])
        self.last_cg_restart_count = int(getattr(self, "last_cg_restart_count", 0)) + int(stats[2])
        self.last_cg_relative_residual = float(rel.value)
        self.last_cg_breakdown = self._BICGSTAB_BREAKDOWN_TEXT.get(int(stats[3]), "")

    def mark_hibm_pressure_outlet_disconnected_nonprojectable_cells(
        self, *, pressure_outlet_zmin: bool = False, node_kind_code=None, barrier_node_code: int = 0,
        use_existing_reachability_barrier: bool = False,
    ) -> int:
        """fluid.py:1771-1876: z-min outlet pressure reachability of the fluid
        cells, and the unreached cells' components (labels -(rank + 1) in
        ``hibm_pressure_unreached_component_label``).  Unreached cells are
        neither masked nor changed.  ``efsi_outlet_reachability`` computes both
        from the connected components of the open faces (hook and pointer-jump
        rounds; ``last_hibm_pressure_reachability_sweeps`` is 1); the
        reference's opt-in checksum reuse is not provided.  The components
        are handed to the library, which anchors them in outlet solves."""
        if getattr(self, "hibm_pressure_outlet_reachable", None) is None:
            shape = self.obstacle.shape
            self.hibm_pressure_outlet_reachable = Field(shape, i32, device=self.device)
            self.hibm_pressure_unreached_component_label = Field(shape, i32, device=self.device)
            self.hibm_pressure_reachability_barrier = Field(shape, i32, device=self.device)
            handle = c_void_p()
            _native.call("efsi_reach_plan_create", byref(handle))
            self._reach_plan = handle
        self.last_hibm_pressure_reachability_reused = False
        self.last_hibm_pressure_component_labels_converged = True
        self.last_hibm_unreached_cells_with_interface_diagonal = 0
        self.last_hibm_unreached_cells_with_interface_coupling = 0
        self.last_hibm_unreached_components_with_interface_hits = 0
        self.last_hibm_pressure_unreached_component_overflow = False
        if not pressure_outlet_zmin:
            if not use_existing_reachability_barrier:
                self.hibm_pressure_reachability_barrier.tensor.zero_()
            self.last_hibm_pressure_unreached_cell_count = 0
            self.last_hibm_pressure_reachability_converged = True
            self.last_hibm_pressure_reachability_sweeps = 0
            self._hibm_pressure_unreached_count = 0
            self.last_hibm_pressure_unreached_component_count = 0
            self._hibm_pressure_unreached_component_count = 0
            self._install_unreached_components(0)
            return 0
        kind_ptr = None
        update = 0 if use_existing_reachability_barrier else 1
        if update and node_kind_code is not None:
            kind = node_kind_code.tensor if isinstance(node_kind_code, Field) else torch.as_tensor(node_kind_code)
            if tuple(kind.shape) != tuple(self.obstacle.shape):
                raise ValueError(
                    f"node_kind_code shape {tuple(kind.shape)} does not match the fluid cell grid "
                    f"{tuple(self.obstacle.shape)}"
                )
            kind = kind.to(device=self.device, dtype=torch.int32).contiguous()
            kind_ptr = kind.data_ptr()
        rep = _native.ReachReport()
        _native.call(
            "efsi_outlet_reachability", self._reach_plan, *self.obstacle.shape, self.obstacle.ptr(),
            self.velocity_dirichlet_boundary_active.ptr(), self.hibm_pressure_reachability_barrier.ptr(), kind_ptr,
            int(barrier_node_code), update, self.hibm_pressure_outlet_reachable.ptr(),
            self.hibm_pressure_unreached_component_label.ptr(), byref(rep), current_stream_handle())
        unreached = int(rep.unreached_cells)
        self.last_hibm_pressure_unreached_cell_count = unreached
        self.last_hibm_pressure_reachability_converged = True
        self.last_hibm_pressure_reachability_sweeps = 1
        self._hibm_pressure_unreached_count = unreached
        self.last_hibm_pressure_unreached_component_count = int(rep.components)
        self._hibm_pressure_unreached_component_count = int(rep.components)
        self.last_hibm_pressure_unreached_component_overflow = bool(rep.overflow)
        self._install_unreached_components(unreached)
        return unreached

    def _unreached_mask(self) -> torch.Tensor:
        """fluid.py:4733-4737: fluid, no reachability barrier, not reached."""
        return ((self.obstacle.tensor == 0) & (self.hibm_pressure_reachability_barrier.tensor == 0)
                & (self.hibm_pressure_outlet_reachable.tensor == 0))

    def _install_unreached_components(self, unreached: int) -> None:
        """Hands the anchored components of outlet solves to the library
        (``efsi_fv_set_unreached_components``): the ranked components
        -(rank + 1) of ``hibm_pressure_unreached_component_label`` when there
        are any, else the whole unreached set as one (fluid.py:4965-4981)."""
        if getattr(self, "_plan", None) is None:
            return
        if int(unreached) <= 0 or getattr(self, "hibm_pressure_outlet_reachable", None) is None:
            _native.call("efsi_fv_set_unreached_components", self._plan, None, 0, _stream())
            return
        mask = self._unreached_mask()
        count = int(self._hibm_pressure_unreached_component_count)
        if count > 0:
            label = self.hibm_pressure_unreached_component_label.tensor
            comp = -label - 1
            comp = torch.where(mask & (label < 0) & (comp < count), comp, torch.full_like(comp, -1))
            ncomp = count
        else:
            comp = torch.where(mask, torch.zeros_like(self.obstacle.tensor), torch.full_like(self.obstacle.tensor, -1))
            ncomp = 1
        comp = comp.to(torch.int32).contiguous()
        _native.call("efsi_fv_set_unreached_components", self._plan, c_void_p(comp.data_ptr()), ncomp, _stream())

    def _record_unreached_interface_hit_diagnostics(self) -> None:
        """fluid.py:5037-5222: unreached cells whose row the interface terms
        touch -- a positive interface diagonal, or a valid coupling (row list,
        else the per-cell slots) of which the cell is owner or neighbour --
        and the ranked components that hold such cells."""
        unreached = self._unreached_mask().reshape(-1)
        label = self.hibm_pressure_unreached_component_label.tensor.reshape(-1)
        count = int(self._hibm_pressure_unreached_component_count)
        diag = unreached & (self.pressure_interface_matrix_diagonal.tensor.reshape(-1) > 0.0)
        cell_hit = torch.zeros_like(unreached)
        csr = self._interface_coupling_rows()
        if csr is not None:
            rows = csr[0].to(torch.int64)
            cell_hit[rows] = unreached[rows]
        flagged = label[diag | cell_hit].to(torch.int64)
        comp = -flagged - 1
        comp = comp[(flagged < 0) & (comp < count)]
        self.last_hibm_unreached_cells_with_interface_diagonal = int(diag.sum())
        self.last_hibm_unreached_cells_with_interface_coupling = int(cell_hit.sum())
        self.last_hibm_unreached_components_with_interface_hits = int(torch.unique(comp).numel())

    def _measure_and_subtract_unreached_rhs_means(self, field: Field, *, mean_abs_tolerance: float = 1.0e-12) -> int:
        """fluid.py:4985-5020 and 4965-4981 on the level-0 rhs: each ranked
        component's volume-weighted integral and mean (the incompatibility
        measure: components whose |mean| exceeds the tolerance), then the
        components' means subtracted.  Returns the incompatible count."""
        sums = (c_double * 256)()
        vols = (c_double * 256)()
        _native.call("efsi_fv_subtract_unreached_means", self._plan, field.ptr(), sums, vols, _stream())
        count = int(self._hibm_pressure_unreached_component_count)
        incompatible, max_mean, max_integral = 0, 0.0, 0.0
        tol = max(0.0, float(mean_abs_tolerance))
        for c in range(count):
            volume, integral = float(vols[c]), float(sums[c])
            max_integral = max(max_integral, abs(integral))
            if volume <= 0.0:
                continue
            mean = abs(integral / volume)
            max_mean = max(max_mean, mean)
            if mean > tol:
                incompatible += 1
        self.last_hibm_unreached_incompatible_component_count = incompatible
        self.last_hibm_unreached_component_rhs_mean_max_abs = max_mean
        self.last_hibm_unreached_component_rhs_integral_max_abs = max_integral
        return incompatible

    def _as_f64(self, field: Field) -> torch.Tensor:
        return field.tensor if field.dtype == f64 else field.tensor.to(torch.float64).contiguous()

    # ------------------------------------------------------------------
    # state management (fluid.py:442-566, 2221-2295)
    # ------------------------------------------------------------------
    def clear(self) -> None:
        for value in self.__dict__.values():
            if isinstance(value, Field) and value.shape == tuple(self.grid.grid_nodes):
                value.tensor.zero_()
        self.velocity_dirichlet_boundary_marker_region_id.fill(-1)
        for lst in (self._mg_rhs, self._mg_residual, self._mg_pressure, self._mg_tmp):
            for fld in lst:
                fld.tensor.zero_()

    def save_state(self) -> None:
        self.saved_velocity.tensor.copy_(self.velocity.tensor)
        self.saved_pressure.tensor.copy_(self.pressure.tensor)

    def restore_state(self) -> None:
        self.velocity.tensor.copy_(self.saved_velocity.tensor)
        self.velocity_prev.tensor.copy_(self.saved_velocity.tensor)
        self.pressure.tensor.copy_(self.saved_pressure.tensor)
        self.pressure_tmp.tensor.copy_(self.saved_pressure.tensor)
        self.pressure_accum.tensor.copy_(self.saved_pressure.tensor)
        for fld in (
            self.volume_source_s,
            self.pressure_interface_projection_divergence_s,
            self.pressure_interface_matrix_diagonal,
            self.pressure_interface_matrix_rhs,
            self.force,
            self.velocity_dirichlet_boundary_active,
            self.velocity_dirichlet_boundary_value_mps,
            self.velocity_dirichlet_boundary_projection_weight,
        ):
            fld.tensor.zero_()
        self._hibm_pressure_unreached_count = 0
        self._install_unreached_components(0)

    def clear_force(self) -> None:
        self.force.tensor.zero_()

    def clear_volume_source(self) -> None:
        self.volume_source_s.tensor.zero_()

    def _clear_pressure_kernel(self) -> None:
        self.pressure.tensor.zero_()
        self.pressure_tmp.tensor.zero_()
        self.pressure_accum.tensor.zero_()

    def clear_pressure(self) -> None:
        self._clear_pressure_kernel()

    def snapshot_pressure(self) -> None:
        self.fsi_pressure.tensor.copy_(self.pressure.tensor)

    def clear_velocity_dirichlet_boundary_rows(self) -> None:
        self.velocity_dirichlet_boundary_active.tensor.zero_()
        self.velocity_dirichlet_boundary_value_mps.tensor.zero_()
        self.velocity_dirichlet_boundary_projection_weight.tensor.zero_()

    def clear_pressure_interface_matrix_terms(self) -> None:
        self.pressure_interface_matrix_diagonal.tensor.zero_()
        self.pressure_interface_matrix_rhs.tensor.zero_()
        self.pressure_interface_projection_divergence_s.tensor.zero_()

    # ------------------------------------------------------------------
    # predictor (fluid.py:2378-2527)
    # ------------------------------------------------------------------
    def _copy_velocity_to_prev_kernel(self) -> None:
        self.velocity_prev.tensor.copy_(self.velocity.tensor)

    def _predict_kernel(self, dt_s: float, nu_m2_s: float, advection_scheme_code: int) -> None:
        self._refresh_structure()
        _native.call(
            "efsi_predict",
            self._plan,
            byref(self._axes),
            self.velocity_prev.ptr(),
            float(dt_s),
            float(nu_m2_s),
            int(advection_scheme_code),
            self.velocity.ptr(),
            _stream(),
        )

    def predict(self, dt_s: float | None = None, *, advection_scheme: str = "euler") -> None:
        step_dt_s = self.dt if dt_s is None else float(dt_s)
        if step_dt_s <= 0.0:
            raise ValueError("dt_s must be positive")
        scheme = str(advection_scheme).lower()
        if scheme not in {"euler", "rk2"}:
            raise ValueError(f"unsupported advection_scheme: {advection_scheme!r}")
        # velocity_prev <- velocity: by exchanging the two buffers (the
        # predictor overwrites every cell of velocity), or, when steps are
        # captured into CUDA graphs (device_loop_solves), by a device copy, so
        # that every replay reads and writes the same buffers
        if getattr(self, "device_loop_solves", False):
            self.velocity_prev.tensor.copy_(self.velocity.tensor)
        else:
            self.velocity.tensor, self.velocity_prev.tensor = self.velocity_prev.tensor, self.velocity.tensor
        self._predict_kernel(step_dt_s, self.mu / self.rho, 1 if scheme == "rk2" else 0)

    # ------------------------------------------------------------------
    # divergence and its statistics (fluid.py:3451-3565, 3827-3848)
    # ------------------------------------------------------------------
    def _compute_divergence_kernel(self, pressure_outlet_zmin: int) -> None:
        _native.call(
            "efsi_compute_divergence", self._plan, self.velocity.ptr(), int(pressure_outlet_zmin), self.divergence.ptr(), _stream()
        )

    def compute_divergence(self, *, pressure_outlet_zmin: bool = False) -> None:
        self._refresh_structure()
        self._compute_divergence_kernel(1 if pressure_outlet_zmin else 0)

    def _div_stats(self, mode: int, interior_only: bool) -> dict[str, float]:
        out = (c_double * 3)()
        _native.call(
            "efsi_divergence_stats",
            self._plan,
            self.divergence.ptr(),
            self.pressure_interface_projection_divergence_s.ptr(),
            self.volume_source_s.ptr(),
            int(mode),
            1 if interior_only else 0,
            out,
            _stream(),
        )
        self.last_divergence_report_host_reads += 1
        count = max(1, int(out[2]))
        return {"max_abs": float(out[0]), "l2": math.sqrt(float(out[1]) / count)}

    def divergence_stats(self, *, interior_only: bool = False) -> dict[str, float]:
        return self._div_stats(0, interior_only)

    def divergence_residual_stats(self, *, interior_only: bool = False) -> dict[str, float]:
        """fluid.py:3837-3848: outlet-unreached cells are left out while any exist."""
        if int(self._hibm_pressure_unreached_count) > 0:
            slots = self._final_report_slots(pressure_outlet_zmin=False)
            return {k: slots[3 if interior_only else 1][k] for k in ("max_abs", "l2")}
        return self._div_stats(1, interior_only)

    def _final_report_slots(self, *, pressure_outlet_zmin: bool) -> list[dict]:
        """The 18 slots of ``efsi_divergence_final_report`` decoded as the
        reference's _decode_divergence_report_snapshot (fluid.py:3850-3858)."""
        self._refresh_structure()
        out = (c_double * 54)()
        reach = None
        if int(self._hibm_pressure_unreached_count) > 0 and getattr(self, "hibm_pressure_outlet_reachable", None) is not None:
            reach = self.hibm_pressure_outlet_reachable.ptr()
        _native.call("efsi_divergence_final_report", self._plan, self.divergence.ptr(),
                     self.pressure_interface_projection_divergence_s.ptr(), self.volume_source_s.ptr(),
                     self.velocity_dirichlet_boundary_active.ptr(), reach, 1 if pressure_outlet_zmin else 0, out,
                     _stream())
        self.last_divergence_report_host_reads += 1
        slots = []
        for q in range(18):
            count = int(out[3 * q + 2])
            slots.append({"max_abs": float(out[3 * q]), "l2": math.sqrt(float(out[3 * q + 1]) / max(1, count)),
                          "count": count})
        return slots

    def final_divergence_report_stats(self, *, pressure_outlet_zmin: bool = False):
        """fluid.py:3870-3896: (raw, residual, interior raw, interior residual)
        over the reached fluid cells; the unreached cells' stats land in
        ``last_unreached_divergence_raw_stats`` / ``last_unreached_divergence_stats``."""
        slots = self._final_report_slots(pressure_outlet_zmin=pressure_outlet_zmin)
        self.last_unreached_divergence_raw_stats = slots[16]
        self.last_unreached_divergence_stats = slots[17]
        return slots[0], slots[1], slots[2], slots[3]

    def final_and_dirichlet_partition_report_stats(self, *, pressure_outlet_zmin: bool = False):
        """fluid.py:3898-3990: the final stats followed by the velocity-Dirichlet
        near / far and pressure-correctable / fixed partitions (raw, residual
        each, then the interior correctable / fixed ones)."""
        slots = self._final_report_slots(pressure_outlet_zmin=pressure_outlet_zmin)
        self.last_unreached_divergence_raw_stats = slots[16]
        self.last_unreached_divergence_stats = slots[17]
        return tuple(slots[:16])

    # ------------------------------------------------------------------
    # FV operator and pressure-solver kernels (fluid.py:4080-4726, 5228-6262)
    # ------------------------------------------------------------------
    def _fv_laplacian_apply_kernel(self, pressure: Field, output: Field, pressure_outlet_zmin: int) -> None:
        self._refresh_structure()
        src = self._as_f64(pressure)
        dst = output.tensor if output.dtype == f64 else torch.empty_like(src)
        _native.call("efsi_fv_apply", self._plan, _ptr(src), _ptr(dst), int(pressure_outlet_zmin), _stream())
        if dst is not output.tensor:
            output.tensor.copy_(dst)

    def _fv_diagonal_kernel(self, diagonal: Field, pressure_outlet_zmin: int) -> None:
        self._refresh_structure()
        _native.call("efsi_fv_diagonal", self._plan, diagonal.ptr(), int(pressure_outlet_zmin), _stream())

    def _apply_jacobi_preconditioner_kernel(self, residual: Field, preconditioned: Field) -> None:
        self._refresh_structure()
        _native.call(
            "efsi_apply_jacobi_preconditioner",
            self._plan,
            self.fv_diag.ptr(),
            _ptr(self._as_f64(residual)),
            preconditioned.ptr(),
            _stream(),
        )

    def _weighted_dot_kernel(self, a: Field, b: Field) -> float:
        self._refresh_structure()
        out = c_double(0.0)
        _native.call("efsi_weighted_dot", self._plan, _ptr(self._as_f64(a)), _ptr(self._as_f64(b)), byref(out), _stream())
        return float(out.value)

    def _weighted_dot_to_field_kernel(self, a: Field, b: Field, out: Field) -> None:
        out[None] = self._weighted_dot_kernel(a, b)

    def _prepare_fv_multigrid_rhs(self, rhs_scale: float) -> None:
        self._refresh_structure()
        _native.call(
            "efsi_mg_prepare_level0",
            self._plan,
            self.divergence.ptr(),
            self.volume_source_s.ptr(),
            self.pressure_interface_matrix_rhs.ptr(),
            float(rhs_scale),
            self._mg_rhs[0].ptr(),
            _stream(),
        )
        # the multigrid work fields start from zero (fluid.py:5228-5260): one
        # library launch clears them all
        if getattr(self, "_mg_zero_list", None) is None:
            fields = [self._mg_residual[0]]
            for level in range(1, len(self._mg_shapes)):
                for lst in (self._mg_pressure, self._mg_tmp, self._mg_rhs, self._mg_residual,
                            self._mg_pressure_interface_matrix_diagonal):
                    fields.append(lst[level])
            fields = fields[:64]
            ptrs = (c_void_p * len(fields))(*[f.ptr() for f in fields])
            sizes = (ctypes.c_int64 * len(fields))(*[f.tensor.numel() * f.tensor.element_size() for f in fields])
            self._mg_zero_list = (len(fields), ptrs, sizes)
        n, ptrs, sizes = self._mg_zero_list
        _native.call("efsi_zero_buffers", n, ptrs, sizes, _stream())

    def _smooth_fv_pressure_level(self, level: int, *, iterations: int, pressure_outlet_zmin: bool, omega: float) -> None:
        self._refresh_structure()
        p = self._mg_pressure[level]
        tmp = self._mg_tmp[level]
        for _ in range(max(0, int(iterations))):
            _native.call(
                "efsi_fv_jacobi_sweep",
                self._plan,
                int(level),
                p.ptr(),
                self._mg_rhs[level].ptr(),
                tmp.ptr(),
                1 if pressure_outlet_zmin else 0,
                float(omega),
                _stream(),
            )
            p.tensor.copy_(tmp.tensor)

    def _compute_fv_residual_level(self, level: int, *, pressure_outlet_zmin: bool) -> None:
        self._refresh_structure()
        _native.call(
            "efsi_fv_residual",
            self._plan,
            int(level),
            self._mg_pressure[level].ptr(),
            self._mg_rhs[level].ptr(),
            self._mg_residual[level].ptr(),
            1 if pressure_outlet_zmin else 0,
            _stream(),
        )

    def _level_of(self, field: Field, lists) -> int:
        for lst in lists:
            for level, fld in enumerate(lst):
                if fld is field:
                    return level
        for level, lshape in enumerate(self._mg_shapes):
            if tuple(lshape) == tuple(field.shape):
                return level
        raise ValueError("field does not belong to a multigrid level of this solver")

    def _mg_restrict_residual_kernel(
        self,
        fine_residual,
        fine_pressure_interface_matrix_diagonal,
        fine_obstacle,
        fine_velocity_dirichlet_boundary_active,
        fine_velocity_dirichlet_boundary_projection_weight,
        fine_cell_width_x_m,
        fine_cell_width_y_m,
        fine_cell_width_z_m,
        coarse_rhs,
        coarse_pressure_interface_matrix_diagonal,
        coarse_pressure,
        coarse_tmp,
        coarse_residual,
        coarse_obstacle,
        coarse_velocity_dirichlet_boundary_active,
        coarse_velocity_dirichlet_boundary_projection_weight,
        fine_nx,
        fine_ny,
        fine_nz,
    ) -> None:
        level = self._level_of(fine_residual, (self._mg_residual, self._pcg_mg_residual))
        self._refresh_structure()
        _native.call(
            "efsi_mg_restrict",
            self._plan,
            int(level),
            fine_residual.ptr(),
            coarse_rhs.ptr(),
            coarse_pressure_interface_matrix_diagonal.ptr(),
            coarse_obstacle.ptr(),
            coarse_velocity_dirichlet_boundary_active.ptr(),
            coarse_velocity_dirichlet_boundary_projection_weight.ptr(),
            _stream(),
        )
        coarse_pressure.tensor.zero_()
        coarse_tmp.tensor.zero_()
        coarse_residual.tensor.zero_()

    def _mg_prolongate_add_kernel(
        self, fine_pressure, fine_obstacle, coarse_pressure, coarse_nx, coarse_ny, coarse_nz, correction_scale
    ) -> None:
        level = self._level_of(fine_pressure, (self._mg_pressure, self._pcg_mg_pressure))
        self._refresh_structure()
        _native.call(
            "efsi_mg_prolong", self._plan, int(level), fine_pressure.ptr(), coarse_pressure.ptr(), float(correction_scale), _stream()
        )

    def _apply_fv_multigrid_preconditioner(
        self,
        residual: Field,
        *,
        pressure_outlet_zmin: bool,
        pre_smooth_iterations: int = 2,
        coarse_smooth_iterations: int = 24,
        post_smooth_iterations: int = 2,
    ) -> None:
        self._refresh_structure()
        _native.call(
            "efsi_mg_vcycle",
            self._plan,
            _ptr(self._as_f64(residual)),
            self.cg_z.ptr(),
            1 if pressure_outlet_zmin else 0,
            int(pre_smooth_iterations),
            int(coarse_smooth_iterations),
            int(post_smooth_iterations),
            _stream(),
        )

    def _subtract_pressure_gradient_kernel(self, dt_over_rho: float, pressure_outlet_zmin: int) -> None:
        self._refresh_structure()
        vd = self._vdir_active
        _native.call(
            "efsi_subtract_pressure_gradient",
            self._plan,
            self.pressure.ptr(),
            self.velocity_dirichlet_boundary_active.ptr() if vd else None,
            self.velocity_dirichlet_boundary_projection_weight.ptr() if vd else None,
            self.velocity_dirichlet_boundary_value_mps.ptr() if vd else None,
            float(dt_over_rho),
            int(pressure_outlet_zmin),
            self.velocity.ptr(),
            _stream(),
        )

    def _apply_closed_boundary_no_normal_flow_kernel(self, pressure_outlet_zmin: int) -> None:
        self._refresh_structure()
        _native.call("efsi_apply_closed_boundary", self._plan, int(pressure_outlet_zmin), self.velocity.ptr(), _stream())

    def _apply_zmin_no_backflow_kernel(self) -> None:
        _native.call("efsi_apply_zmin_no_backflow", self._plan, self.velocity.ptr(), _stream())

    def apply_velocity_dirichlet_boundary_rows(self, *, read_report: bool = True) -> VelocityDirichletBoundaryReport | None:
        self._refresh_structure()
        if not self._vdir_active:
            return VelocityDirichletBoundaryReport(0, 0.0, 0.0) if read_report else None
        rep = self._report
        _native.call(
            "efsi_apply_velocity_dirichlet_rows",
            self._plan,
            self.velocity_dirichlet_boundary_active.ptr(),
            self.velocity_dirichlet_boundary_value_mps.ptr(),
            float(self.rho),
            self.velocity.ptr(),
            _ptr(rep) if read_report else None,
            _stream(),
        )
        if not read_report:
            return None
        r = rep[:6].cpu().tolist()
        cells = int(r[0])
        return VelocityDirichletBoundaryReport(
            active_cells=cells,
            max_delta_mps=float(r[2]),
            mean_delta_mps=float(r[1]) / cells if cells > 0 else 0.0,
            momentum_delta_n_s=(float(r[3]), float(r[4]), float(r[5])),
        )

    # ------------------------------------------------------------------
    # pressure solvers (fluid.py:5842-6811)
    # ------------------------------------------------------------------
    def _solve_pressure_poisson(self, *, iterations, rhs_scale, inv_dx2, inv_dy2, inv_dz2, pressure_outlet_zmin) -> None:
        self._refresh_structure()
        _native.call(
            "efsi_legacy_jacobi_solve",
            self._plan,
            self.divergence.ptr(),
            self.volume_source_s.ptr(),
            float(rhs_scale),
            float(inv_dx2),
            float(inv_dy2),
            float(inv_dz2),
            1 if pressure_outlet_zmin else 0,
            int(iterations),
            self.pressure.ptr(),
            self.pressure_tmp.ptr(),
            _stream(),
        )

    def _solve_pressure_poisson_fv_jacobi(self, *, iterations, rhs_scale, pressure_outlet_zmin) -> None:
        self._prepare_fv_multigrid_rhs(rhs_scale)
        _native.call(
            "efsi_fv_jacobi_solve",
            self._plan,
            self._mg_rhs[0].ptr(),
            self.pressure.ptr(),
            1 if pressure_outlet_zmin else 0,
            int(iterations),
            _stream(),
        )

    def _solve_pressure_poisson_fv_multigrid(self, *, iterations, rhs_scale, pressure_outlet_zmin, multigrid_cycles) -> None:
        self._prepare_fv_multigrid_rhs(rhs_scale)
        cycles = int(multigrid_cycles) if multigrid_cycles is not None else self.default_multigrid_cycles()
        if cycles <= 0:
            raise ValueError("multigrid_cycles must be positive")
        _native.call(
            "efsi_fv_multigrid_solve",
            self._plan,
            self._mg_rhs[0].ptr(),
            self.pressure.ptr(),
            1 if pressure_outlet_zmin else 0,
            int(iterations),
            cycles,
            _stream(),
        )

    def _solve_pressure_poisson_fv_cg(
        self,
        *,
        iterations: int,
        rhs_scale: float,
        pressure_outlet_zmin: bool,
        tolerance: float,
        preconditioner: str = "auto",
        remove_nullspace_mean: bool = True,
        pressure_interface_matrix_active: bool = False,
        use_graphs: bool = True,
    ) -> None:
        name = str(preconditioner)
        if name not in CG_PRECONDITIONER_CHOICES:
            raise ValueError(f"unsupported cg_preconditioner: {preconditioner!r}")
        if name == "auto":
            name = "jacobi" if self.grid.is_uniform else "fv_multigrid"
        # fluid.py:6567-6588: an outlet solve with flood-unreached cells anchors
        # each unreached component by subtracting its volume-weighted mean
        anchor_unreached = bool(pressure_outlet_zmin) and int(self._hibm_pressure_unreached_count) > 0
        self.last_hibm_unreached_cells_with_interface_diagonal = 0
        self.last_hibm_unreached_cells_with_interface_coupling = 0
        self.last_hibm_unreached_components_with_interface_hits = 0
        if anchor_unreached:
            self._record_unreached_interface_hit_diagnostics()
        self._prepare_fv_multigrid_rhs(rhs_scale)
        if anchor_unreached:
            self._measure_and_subtract_unreached_rhs_means(self._mg_rhs[0])
        else:
            self.last_hibm_unreached_incompatible_component_count = 0
            self.last_hibm_unreached_component_rhs_mean_max_abs = 0.0
            self.last_hibm_unreached_component_rhs_integral_max_abs = 0.0
        # device-side loop (no host reads) when the solver is set up for
        # captured steps; the learned preconditioner's fallback is a host decision
        device = bool(getattr(self, "device_loop_solves", False)) and name not in ("learned", "learned_no_fallback")
        params = _native.PcgParams(
            max(1, int(iterations)),
            _PRECOND_CODE[name],
            1 if remove_nullspace_mean else 0,
            1 if pressure_outlet_zmin else 0,
            1 if pressure_interface_matrix_active else 0,
            1 if use_graphs else 0,
            max(0.0, float(tolerance)),
            1 if device else 0,
        )
        stats = _native.CgStats()
        _native.call(
            "efsi_fv_pcg_solve", self._plan, self._mg_rhs[0].ptr(), self.pressure.ptr(), byref(params), byref(stats), _stream()
        )
        self._device_stats_pending = int(stats.converged) == -1
        if self._device_stats_pending:
            # inside a step-graph capture: the statistics exist once the graph ran
            # (read_device_pcg_stats)
            return
        self.last_cg_iterations = int(stats.iterations)
        self.last_cg_initial_relative_residual = float(stats.initial_relative_residual)
        self.last_cg_relative_residual = float(stats.relative_residual)
        self.last_cg_converged = bool(stats.converged)
        self.last_cg_breakdown = _BREAKDOWN_TEXT.get(int(stats.breakdown_reason), "")
        self.last_cg_host_residual_checks = int(stats.host_residual_checks)
        self.last_cg_mean_host_reads = 0
        self.last_cg_mean_projection_count = int(stats.mean_projection_count)
        self.last_cg_unreached_set_mean_projection_count = int(stats.unreached_set_mean_projection_count)
        self.last_cg_restart_count = int(stats.restart_count)
        self.last_cg_restart_count_measured = True
        self.last_cg_restart_policy = "periodic_exact_residual"
        self.last_cg_breakdown_dAd = float(stats.breakdown_dAd)
        self.last_cg_used_multigrid = bool(stats.used_mg)
        self.last_cg_used_graphs = bool(stats.used_graphs)
        self.last_cg_learned_iterations = int(stats.learned_iterations)
        self.last_cg_learned_relative_residual = float(stats.learned_relative_residual)
        if use_graphs and not stats.used_graphs:
            self.last_cg_graph_error = _native.load().efsi_fv_graph_error(self._plan).decode(errors="replace")
        self._last_cg_breakdown_code = int(stats.breakdown_code)
        if (pressure_interface_matrix_active and not stats.converged and int(stats.breakdown_reason) == 0
                and int(self.pressure_interface_row_count[None]) > 0):
            # fluid.py:6799-6811: with row-list couplings, an exhausted CG loop
            # continues as BiCGSTAB on the same system from its pressure
            _native.call("efsi_fv_copy_rhs", self._plan, self.cg_rhs.ptr(), _stream())
            self._continue_pressure_poisson_fv_bicgstab(
                start_iteration=max(1, int(iterations)), max_iters=max(1, int(iterations)), b_norm=float(stats.b_norm),
                outlet=1 if pressure_outlet_zmin else 0, tolerance=max(0.0, float(tolerance)),
                anchor_unreached=anchor_unreached, remove_nullspace_mean=bool(remove_nullspace_mean))
        if stats.b_norm <= 1.0e-30:
            self.pressure_tmp.tensor.zero_()
            self.pressure_accum.tensor.zero_()

    def _solve_pressure_poisson_with_solver(
        self,
        *,
        iterations,
        rhs_scale,
        inv_dx2,
        inv_dy2,
        inv_dz2,
        pressure_outlet_zmin,
        pressure_solver,
        multigrid_cycles,
        cg_tolerance,
        cg_preconditioner="auto",
        remove_nullspace_mean=True,
        pressure_interface_matrix_active=False,
    ) -> None:
        if pressure_solver in {"jacobi", "compact_jacobi"}:
            self._solve_pressure_poisson(
                iterations=int(iterations),
                rhs_scale=float(rhs_scale),
                inv_dx2=float(inv_dx2),
                inv_dy2=float(inv_dy2),
                inv_dz2=float(inv_dz2),
                pressure_outlet_zmin=bool(pressure_outlet_zmin),
            )
        elif pressure_solver == "fv_jacobi":
            self._solve_pressure_poisson_fv_jacobi(
                iterations=int(iterations), rhs_scale=float(rhs_scale), pressure_outlet_zmin=bool(pressure_outlet_zmin)
            )
        elif pressure_solver == "fv_multigrid":
            self._solve_pressure_poisson_fv_multigrid(
                iterations=int(iterations),
                rhs_scale=float(rhs_scale),
                pressure_outlet_zmin=bool(pressure_outlet_zmin),
                multigrid_cycles=multigrid_cycles,
            )
        elif pressure_solver == "fv_cg":
            self._solve_pressure_poisson_fv_cg(
                iterations=int(iterations),
                rhs_scale=float(rhs_scale),
                pressure_outlet_zmin=bool(pressure_outlet_zmin),
                tolerance=float(cg_tolerance),
                preconditioner=str(cg_preconditioner),
                remove_nullspace_mean=bool(remove_nullspace_mean),
                pressure_interface_matrix_active=bool(pressure_interface_matrix_active),
            )
        else:
            raise ValueError(f"unsupported pressure_solver: {pressure_solver!r}")

    # ------------------------------------------------------------------
    # projection (fluid.py:6889-7613)
    # ------------------------------------------------------------------
    def _reset_project_cg_stats(self) -> None:
        self.last_project_cg_project_calls = 0
        self.last_project_cg_iterations_total = 0
        self.last_project_cg_iterations_max = 0
        self.last_project_cg_host_residual_checks = 0
        self.last_project_cg_mean_host_reads = 0
        self.last_project_cg_mean_projection_count = 0
        self.last_project_cg_unreached_set_mean_projection_count = 0
        self.last_project_cg_restart_count = 0
        self.last_project_cg_restart_count_measured = False
        self.last_project_cg_restart_policy = ""
        self.last_project_cg_initial_relative_residual_max = 0.0
        self.last_project_cg_relative_residual_max = 0.0
        self.last_project_cg_converged_all = True
        self.last_project_cg_breakdown_count = 0
        self.last_project_cg_breakdown_code = 0
        self.last_project_cg_breakdown_dAd = 0.0
        self.last_project_cg_breakdown = ""

    def pressure_interface_matrix_terms_report(self) -> dict[str, float]:
        """fluid.py:2864-3118 _pressure_interface_matrix_terms_report_kernel:
        integrals of the interface diagonal and rhs over the cells, the row
        list (or, without one, the per-cell slots) checked as couplings --
        both cells inside and fluid, T > 0, not a self coupling -- with the
        diagonal density they imply, and its mismatch against the diagonal."""
        nx, ny, nz = self.grid.grid_nodes
        diag = self.pressure_interface_matrix_diagonal.tensor
        rhs = self.pressure_interface_matrix_rhs.tensor
        vol32 = self._cell_volume_f32()
        obs = self.obstacle.tensor.reshape(-1)
        density = torch.zeros(nx * ny * nz, dtype=diag.dtype, device=diag.device)
        row_count = int(self.pressure_interface_row_count[None])
        capacity = int(self.pressure_interface_row_capacity)
        active_rows, invalid_rows, row_integral, max_t = 0, 0, 0.0, 0.0
        dims = torch.tensor([nx, ny, nz], device=diag.device)
        pairs = None
        if row_count > 0:
            limit = min(row_count, capacity)
            own = self.pressure_interface_row_owner.tensor[:limit].to(torch.int64)
            nbr = self.pressure_interface_row_neighbor.tensor[:limit].to(torch.int64)
            trans = self.pressure_interface_row_transmissibility.tensor[:limit]
            pairs = (own, nbr, trans, torch.ones(limit, dtype=torch.bool, device=diag.device))
        else:
            act = self.pressure_interface_coupling_active.tensor.reshape(-1)
            cells = torch.nonzero((act > 0) & (obs == 0)).reshape(-1)
            if cells.numel() > 0:
                have_extra = "pressure_interface_coupling_extra_neighbor" in self.__dict__
                n_slots = PRESSURE_INTERFACE_COUPLING_SLOT_COUNT if have_extra else 1
                slots = torch.clamp(act[cells], max=PRESSURE_INTERFACE_COUPLING_SLOT_COUNT).to(torch.int64)
                nb0 = self.pressure_interface_coupling_neighbor.tensor.reshape(-1, 3)[cells].to(torch.int64)
                tr0 = self.pressure_interface_coupling_coefficient.tensor.reshape(-1)[cells]
                if have_extra:
                    xnb = self.pressure_interface_coupling_extra_neighbor.tensor.reshape(-1, n_slots - 1, 3)[cells]
                    xtr = self.pressure_interface_coupling_extra_coefficient.tensor.reshape(-1, n_slots - 1)[cells]
                    nbr = torch.cat([nb0[:, None, :], xnb.to(torch.int64)], dim=1).reshape(-1, 3)
                    trans = torch.cat([tr0[:, None], xtr], dim=1).reshape(-1)
                else:
                    nbr, trans = nb0, tr0
                in_use = (torch.arange(n_slots, device=cells.device)[None, :] < slots[:, None]).reshape(-1)
                own_lin = cells.repeat_interleave(n_slots)
                own = torch.stack([own_lin // (ny * nz), (own_lin // nz) % ny, own_lin % nz], dim=1)
                pairs = (own, nbr, trans, in_use)
                if not have_extra:
                    # never-written extra slots hold T = 0: invalid couplings
                    invalid_rows += int((slots - 1).sum())
        if pairs is not None:
            own, nbr, trans, in_use = pairs
            inside = ((own >= 0) & (own < dims)).all(dim=1) & ((nbr >= 0) & (nbr < dims)).all(dim=1)
            oc = torch.where(inside[:, None], own, torch.zeros_like(own))
            nc = torch.where(inside[:, None], nbr, torch.zeros_like(nbr))
            o_lin = (oc[:, 0] * ny + oc[:, 1]) * nz + oc[:, 2]
            n_lin = (nc[:, 0] * ny + nc[:, 1]) * nz + nc[:, 2]
            valid = inside & (obs[o_lin] == 0) & (obs[n_lin] == 0) & (trans > 0.0) & (o_lin != n_lin)
            v_flat = vol32.reshape(-1)
            t_ok = trans[valid & in_use]
            density.index_add_(0, o_lin[valid & in_use],
                               (t_ok / torch.clamp(v_flat[o_lin[valid & in_use]], min=1.0e-30)).to(density.dtype))
            density.index_add_(0, n_lin[valid & in_use],
                               (t_ok / torch.clamp(v_flat[n_lin[valid & in_use]], min=1.0e-30)).to(density.dtype))
            active_rows = int((valid & in_use).sum())
            invalid_rows += int((~valid & in_use).sum())
            row_integral = float((2.0 * t_ok.to(torch.float64)).sum()) if t_ok.numel() else 0.0
            max_t = float(t_ok.max()) if t_ok.numel() else 0.0
        vol64 = vol32.to(torch.float64)
        mismatch = (diag - density.reshape(diag.shape)).to(torch.float64)
        vals = torch.stack(
            [
                (diag.to(torch.float64) * vol64).sum(),
                (rhs.to(torch.float64) * vol64).sum(),
                diag.abs().max().to(torch.float64),
                ((diag.abs() > 0) | (rhs.abs() > 0)).sum().to(torch.float64),
                (mismatch.abs() * vol64).sum(),
                mismatch.abs().max(),
            ]
        ).cpu().tolist()
        return {
            "diagonal_integral": vals[0],
            "rhs_integral": vals[1],
            "max_abs_diagonal": vals[2],
            "active_cells": int(vals[3]),
            "row_count": row_count,
            "row_active_count": active_rows,
            "row_invalid_count": invalid_rows,
            "row_overflow_count": max(row_count - capacity, 0),
            "row_diagonal_integral": row_integral,
            "row_diagonal_integral_abs_mismatch": vals[4],
            "row_diagonal_max_abs_density_mismatch": vals[5],
            "row_max_transmissibility": max_t,
        }

    def project(
        self,
        iterations: int = 40,
        pressure_outlet_zmin: bool = False,
        dt_s: float | None = None,
        preserve_velocity_constraints: bool = False,
        velocity_constraint_blend: float = 1.0,
        velocity_constraint_solid_mobility_ratio: float = 0.0,
        divergence_cleanup_iterations: int = 0,
        divergence_cleanup_relaxation: float = 0.7,
        reset_pressure: bool = False,
        pressure_solver: str = "jacobi",
        multigrid_cycles: int | None = None,
        cg_tolerance: float = 1.0e-6,
        cg_preconditioner: str = "auto",
        pressure_solve_failure_policy: str = "report",
        read_report: bool = True,
    ) -> dict[str, float]:
        if iterations <= 0:
            raise ValueError("iterations must be positive")
        step_dt_s = self.dt if dt_s is None else float(dt_s)
        if step_dt_s <= 0.0:
            raise ValueError("dt_s must be positive")
        if not 0.0 <= float(velocity_constraint_blend) <= 1.0:
            raise ValueError("velocity_constraint_blend must be in [0, 1]")
        ratio = float(velocity_constraint_solid_mobility_ratio)
        if not math.isfinite(ratio) or ratio < 0.0:
            raise ValueError("velocity_constraint_solid_mobility_ratio must be a finite non-negative number")
        if not 0.0 <= float(divergence_cleanup_relaxation) <= 1.0:
            raise ValueError("divergence_cleanup_relaxation must be in [0, 1]")
        tol = float(cg_tolerance)
        if not math.isfinite(tol) or tol < 0.0:
            raise ValueError("cg_tolerance must be a finite non-negative number")
        precond = str(cg_preconditioner)
        if precond not in CG_PRECONDITIONER_CHOICES:
            raise ValueError(f"unsupported cg_preconditioner: {cg_preconditioner!r}")
        policy = str(pressure_solve_failure_policy)
        if policy not in {"report", "raise"}:
            raise ValueError("pressure_solve_failure_policy must be 'report' or 'raise'")
        requested = str(pressure_solver)
        solver = requested
        if solver not in {"jacobi", "compact_jacobi", "fv_jacobi", "fv_multigrid", "fv_cg"}:
            raise ValueError(f"unsupported pressure_solver: {pressure_solver!r}")
        if not self.grid.is_uniform:
            if solver not in {"fv_jacobi", "fv_multigrid", "fv_cg"}:
                raise ValueError("non-uniform CartesianGrid projection requires an FV pressure solver")
            if divergence_cleanup_iterations > 0:
                raise ValueError("non-uniform CartesianGrid divergence cleanup requires non-uniform cleanup operators")
        if multigrid_cycles is not None and int(multigrid_cycles) <= 0:
            raise ValueError("multigrid_cycles must be positive")
        if preserve_velocity_constraints or int(divergence_cleanup_iterations) > 0:
            raise NotImplementedError(
                "velocity-constraint blending and local divergence cleanup are outside the B200 hot path"
            )
        report = bool(read_report)
        outlet = bool(pressure_outlet_zmin)
        self.last_divergence_report_host_reads = 0
        self._refresh_structure()
        iface_active = self._iface_active
        forced = False
        force_reason = ""
        if iface_active and solver == "fv_multigrid":
            solver, forced, force_reason = "fv_cg", True, "pressure_interface_matrix_requires_rowlist_fv_cg"
        anchored = (not outlet) and iface_active
        remove_mean = (not outlet) and solver == "fv_cg" and not anchored
        if outlet:
            nullspace_policy, compat = "pressure_outlet_dirichlet", True
        elif anchored:
            nullspace_policy, compat = "interface_matrix_anchored", solver == "fv_cg"
        elif solver == "fv_cg":
            nullspace_policy, compat = "closed_neumann_fv_cg_zero_mean", True
        else:
            nullspace_policy, compat = "closed_neumann_non_cg_unmeasured", False
        self._reset_project_cg_stats()
        self.last_project_cg_restart_count_measured = solver == "fv_cg"
        self.last_project_cg_restart_policy = "periodic_exact_residual" if solver == "fv_cg" else "not_applicable_non_cg"
        state = {"failed": False, "action": "none"}

        def record_cg_stats() -> None:
            if solver != "fv_cg" or getattr(self, "_device_stats_pending", False):
                return
            self.last_project_cg_project_calls += 1
            self.last_project_cg_iterations_total += int(self.last_cg_iterations)
            self.last_project_cg_iterations_max = max(self.last_project_cg_iterations_max, int(self.last_cg_iterations))
            self.last_project_cg_host_residual_checks += int(self.last_cg_host_residual_checks)
            self.last_project_cg_mean_projection_count += int(self.last_cg_mean_projection_count)
            self.last_project_cg_unreached_set_mean_projection_count += int(
                self.last_cg_unreached_set_mean_projection_count)
            self.last_project_cg_restart_count += int(self.last_cg_restart_count)
            self.last_project_cg_restart_policy = str(self.last_cg_restart_policy)
            if math.isfinite(self.last_cg_initial_relative_residual):
                self.last_project_cg_initial_relative_residual_max = max(
                    self.last_project_cg_initial_relative_residual_max, self.last_cg_initial_relative_residual
                )
            if math.isfinite(self.last_cg_relative_residual):
                self.last_project_cg_relative_residual_max = max(
                    self.last_project_cg_relative_residual_max, self.last_cg_relative_residual
                )
            if not self.last_cg_converged:
                state["failed"] = True
                self.last_project_cg_converged_all = False
                self.last_project_cg_breakdown_count += 1
                self.last_project_cg_breakdown_code = max(self.last_project_cg_breakdown_code, self._last_cg_breakdown_code)
                if math.isfinite(self.last_cg_breakdown_dAd):
                    self.last_project_cg_breakdown_dAd = self.last_cg_breakdown_dAd
                if self.last_cg_breakdown:
                    self.last_project_cg_breakdown = self.last_cg_breakdown

        physical = {"failed": False, "reason": "", "action": "none", "incompatible": 0, "mean": 0.0, "integral": 0.0}

        def record_physical_stats() -> None:
            # fluid.py:7069-7112: an anchored component whose rhs has a
            # non-zero mean cannot be made divergence free
            physical["incompatible"] = max(physical["incompatible"],
                                           int(self.last_hibm_unreached_incompatible_component_count))
            physical["mean"] = max(physical["mean"], float(self.last_hibm_unreached_component_rhs_mean_max_abs))
            physical["integral"] = max(physical["integral"],
                                       float(self.last_hibm_unreached_component_rhs_integral_max_abs))
            if int(self.last_hibm_unreached_incompatible_component_count) > 0:
                physical["failed"] = True
                physical["reason"] = "unreached_component_rhs_incompatible"

        def handle_physical_failure() -> None:
            # fluid.py:7114-7131
            if not physical["failed"]:
                return
            if policy != "raise":
                physical["action"] = "reported"
                return
            physical["action"] = "raised"
            raise RuntimeError(
                "FV-CG pressure projection physical gate failed: unreached component RHS is incompatible with a "
                f"sealed incompressible component (components={physical['incompatible']}, "
                f"max_abs_rhs_mean={physical['mean']:.6g})"
            )

        def handle_failure() -> None:
            if solver != "fv_cg" or self.last_cg_converged or getattr(self, "_device_stats_pending", False):
                return
            if policy != "raise":
                state["action"] = "reported_cleared_pressure_correction"
                self._clear_pressure_kernel()
                return
            raise RuntimeError(
                "FV-CG pressure solve did not converge before pressure-gradient velocity correction "
                f"(iterations={self.last_cg_iterations}, relative_residual={self.last_cg_relative_residual:.6g}, "
                f"breakdown={self.last_cg_breakdown!r})"
            )

        vdir_calls = {"n": 0, "cells": 0, "cells_max": 0, "dsum": 0.0, "dmax": 0.0, "mom": [0.0, 0.0, 0.0]}

        def apply_bc() -> None:
            if self._vdir_active:
                rep = self.apply_velocity_dirichlet_boundary_rows(read_report=report)
                if report and rep is not None:
                    vdir_calls["n"] += 1
                    vdir_calls["cells"] += rep.active_cells
                    vdir_calls["cells_max"] = max(vdir_calls["cells_max"], rep.active_cells)
                    vdir_calls["dsum"] += rep.mean_delta_mps * rep.active_cells
                    vdir_calls["dmax"] = max(vdir_calls["dmax"], rep.max_delta_mps)
                    for a in range(3):
                        vdir_calls["mom"][a] += rep.momentum_delta_n_s[a]
            elif report:
                vdir_calls["n"] += 1
            if outlet:
                self._apply_zmin_no_backflow_kernel()
                self._apply_closed_boundary_no_normal_flow_kernel(1)

        nan_stats = {"max_abs": math.nan, "l2": math.nan}
        f = self.pressure_interface_projection_divergence_s
        _native.call("efsi_zero_buffers", 1, (c_void_p * 1)(f.ptr()),
                     (ctypes.c_int64 * 1)(f.tensor.numel() * f.tensor.element_size()), _stream())
        apply_bc()
        self._compute_divergence_kernel(1 if outlet else 0)
        pre_raw = self.divergence_stats() if report else nan_stats
        pre = self.divergence_residual_stats() if report else nan_stats
        if reset_pressure:
            self._clear_pressure_kernel()
        rhs_scale = self.rho / step_dt_s
        solve_kwargs = dict(
            iterations=int(iterations),
            rhs_scale=float(rhs_scale),
            inv_dx2=1.0 / (self.dx * self.dx),
            inv_dy2=1.0 / (self.dy * self.dy),
            inv_dz2=1.0 / (self.dz * self.dz),
            pressure_outlet_zmin=outlet,
            pressure_solver=solver,
            multigrid_cycles=multigrid_cycles,
            cg_tolerance=tol,
            cg_preconditioner=precond,
            remove_nullspace_mean=remove_mean,
            pressure_interface_matrix_active=iface_active,
        )
        self._solve_pressure_poisson_with_solver(**solve_kwargs)
        record_cg_stats()
        record_physical_stats()
        handle_failure()
        handle_physical_failure()
        self._subtract_pressure_gradient_kernel(step_dt_s / self.rho, 1 if outlet else 0)
        apply_bc()
        self._compute_divergence_kernel(1 if outlet else 0)
        proj_raw = self.divergence_stats() if report else nan_stats
        proj = self.divergence_residual_stats() if report else nan_stats
        post_raw, post = proj_raw, proj
        if outlet:
            # fluid.py:7259-7318: up to three cleanup re-solves while the
            # residual divergence grew more than 5 % over the projection's.
            self.pressure_accum.tensor.copy_(self.pressure.tensor)
            target_stats = self.divergence_residual_stats()
            target_l2 = max(float(target_stats["l2"]) * 1.05, 1.0e-8)
            apply_bc()
            self._compute_divergence_kernel(1)
            current = self.divergence_residual_stats()
            post_raw = self.divergence_stats() if report else nan_stats
            post = current if report else nan_stats
            cleanup_iterations = max(1, min(int(iterations), 256))
            for _ in range(3):
                if current["l2"] <= target_l2:
                    break
                self.pressure.tensor.zero_()
                self.pressure_interface_matrix_rhs.tensor.zero_()
                self._solve_pressure_poisson_with_solver(**{**solve_kwargs, "iterations": cleanup_iterations})
                record_cg_stats()
                record_physical_stats()
                handle_failure()
                handle_physical_failure()
                self._subtract_pressure_gradient_kernel(step_dt_s / self.rho, 1)
                corrected = self.pressure_accum.tensor + self.pressure.tensor
                self.pressure_accum.tensor.copy_(corrected)
                self.pressure.tensor.copy_(corrected)
                self.pressure_tmp.tensor.copy_(corrected)
                apply_bc()
                self._compute_divergence_kernel(1)
                current = self.divergence_residual_stats()
                post_raw = self.divergence_stats() if report else nan_stats
                post = current if report else nan_stats
        else:
            self._apply_closed_boundary_no_normal_flow_kernel(0)
        if not report:
            return {}
        self._compute_divergence_kernel(1 if outlet else 0)
        (final_raw, final, final_int_raw, final_int, near_raw, near, far_raw, far, corr_raw, corr, fixed_raw, fixed,
         int_corr_raw, int_corr, int_fixed_raw, int_fixed) = self.final_and_dirichlet_partition_report_stats(
            pressure_outlet_zmin=outlet)
        iface = self.pressure_interface_matrix_terms_report()
        n_vdir = vdir_calls["cells"]
        return {
            "pressure_solver_requested": requested,
            "pressure_solver": solver,
            "pressure_solver_forced_to_fv_cg": forced,
            "pressure_solver_force_reason": force_reason,
            "l2": final["l2"],
            "max_abs": final["max_abs"],
            "raw_l2": final_raw["l2"],
            "raw_max_abs": final_raw["max_abs"],
            "interior_l2": final_int["l2"],
            "interior_max_abs": final_int["max_abs"],
            "interior_raw_l2": final_int_raw["l2"],
            "interior_raw_max_abs": final_int_raw["max_abs"],
            "pre_projection_l2": pre["l2"],
            "pre_projection_max_abs": pre["max_abs"],
            "pre_projection_raw_l2": pre_raw["l2"],
            "pre_projection_raw_max_abs": pre_raw["max_abs"],
            "projection_l2": proj["l2"],
            "projection_max_abs": proj["max_abs"],
            "projection_raw_l2": proj_raw["l2"],
            "projection_raw_max_abs": proj_raw["max_abs"],
            "post_boundary_l2": post["l2"],
            "post_boundary_max_abs": post["max_abs"],
            "post_boundary_raw_l2": post_raw["l2"],
            "post_boundary_raw_max_abs": post_raw["max_abs"],
            "post_constraint_l2": final["l2"],
            "post_constraint_max_abs": final["max_abs"],
            "post_constraint_raw_l2": final_raw["l2"],
            "post_constraint_raw_max_abs": final_raw["max_abs"],
            "velocity_dirichlet_near_l2": near["l2"],
            "velocity_dirichlet_near_max_abs": near["max_abs"],
            "velocity_dirichlet_near_raw_l2": near_raw["l2"],
            "velocity_dirichlet_near_raw_max_abs": near_raw["max_abs"],
            "velocity_dirichlet_far_l2": far["l2"],
            "velocity_dirichlet_far_max_abs": far["max_abs"],
            "velocity_dirichlet_far_raw_l2": far_raw["l2"],
            "velocity_dirichlet_far_raw_max_abs": far_raw["max_abs"],
            "velocity_dirichlet_boundary_apply_calls": vdir_calls["n"],
            "velocity_dirichlet_boundary_active_cells_total": n_vdir,
            "velocity_dirichlet_boundary_active_cells_max": vdir_calls["cells_max"],
            "velocity_dirichlet_boundary_max_delta_mps": vdir_calls["dmax"],
            "velocity_dirichlet_boundary_mean_delta_mps": vdir_calls["dsum"] / n_vdir if n_vdir > 0 else 0.0,
            "velocity_dirichlet_boundary_momentum_delta_n_s": tuple(vdir_calls["mom"]),
            "pressure_correctable_l2": corr["l2"],
            "pressure_correctable_max_abs": corr["max_abs"],
            "pressure_correctable_cell_count": corr["count"],
            "pressure_correctable_raw_l2": corr_raw["l2"],
            "pressure_correctable_raw_max_abs": corr_raw["max_abs"],
            "pressure_fixed_l2": fixed["l2"],
            "pressure_fixed_max_abs": fixed["max_abs"],
            "pressure_fixed_cell_count": fixed["count"],
            "pressure_fixed_raw_l2": fixed_raw["l2"],
            "pressure_fixed_raw_max_abs": fixed_raw["max_abs"],
            "interior_pressure_correctable_l2": int_corr["l2"],
            "interior_pressure_correctable_max_abs": int_corr["max_abs"],
            "interior_pressure_correctable_cell_count": int_corr["count"],
            "interior_pressure_correctable_raw_l2": int_corr_raw["l2"],
            "interior_pressure_correctable_raw_max_abs": int_corr_raw["max_abs"],
            "interior_pressure_fixed_l2": int_fixed["l2"],
            "interior_pressure_fixed_max_abs": int_fixed["max_abs"],
            "interior_pressure_fixed_cell_count": int_fixed["count"],
            "interior_pressure_fixed_raw_l2": int_fixed_raw["l2"],
            "interior_pressure_fixed_raw_max_abs": int_fixed_raw["max_abs"],
            "pressure_interface_matrix_diagonal_integral": iface["diagonal_integral"],
            "pressure_interface_matrix_rhs_integral": iface["rhs_integral"],
            "pressure_interface_matrix_max_abs_diagonal": iface["max_abs_diagonal"],
            "pressure_interface_matrix_active_cells": iface["active_cells"],
            "pressure_interface_matrix_active": iface_active,
            "pressure_interface_matrix_row_count": iface["row_count"],
            "pressure_interface_matrix_row_active_count": iface["row_active_count"],
            "pressure_interface_matrix_row_invalid_count": iface["row_invalid_count"],
            "pressure_interface_matrix_row_overflow_count": iface["row_overflow_count"],
            "pressure_interface_matrix_row_diagonal_integral": iface["row_diagonal_integral"],
            "pressure_interface_matrix_row_diagonal_integral_abs_mismatch": iface["row_diagonal_integral_abs_mismatch"],
            "pressure_interface_matrix_row_diagonal_max_abs_density_mismatch": iface[
                "row_diagonal_max_abs_density_mismatch"],
            "pressure_interface_matrix_row_max_transmissibility": iface["row_max_transmissibility"],
            "pressure_nullspace_policy": nullspace_policy,
            "pressure_nullspace_compatibility_measured": compat,
            "pressure_nullspace_zero_mean_projection_applied": remove_mean,
            "pressure_system_anchored_by_interface_matrix": anchored,
            "pressure_solve_failure_policy": policy,
            "pressure_solve_failed": state["failed"],
            "pressure_solve_failure_action": state["action"],
            "pressure_projection_physical_failure": physical["failed"],
            "pressure_projection_physical_failure_reason": physical["reason"],
            "pressure_projection_physical_failure_action": physical["action"],
            "hibm_unreached_incompatible_component_count": physical["incompatible"],
            "hibm_unreached_component_rhs_mean_max_abs": physical["mean"],
            "hibm_unreached_component_rhs_integral_max_abs": physical["integral"],
            "cg_project_calls": self.last_project_cg_project_calls,
            "cg_iterations_total": self.last_project_cg_iterations_total,
            "cg_iterations_max": self.last_project_cg_iterations_max,
            "cg_host_residual_checks": self.last_project_cg_host_residual_checks,
            "cg_mean_host_reads": 0,
            "cg_mean_projection_count": self.last_project_cg_mean_projection_count,
            "cg_unreached_set_mean_projection_count": self.last_project_cg_unreached_set_mean_projection_count,
            "hibm_pressure_unreached_cell_count": int(getattr(self, "last_hibm_pressure_unreached_cell_count", 0)),
            "hibm_pressure_reachability_converged": bool(
                getattr(self, "last_hibm_pressure_reachability_converged", True)),
            "cg_unreached_component_count": int(getattr(self, "last_hibm_pressure_unreached_component_count", 0)),
            "cg_unreached_component_overflow": bool(
                getattr(self, "last_hibm_pressure_unreached_component_overflow", False)),
            "unreached_cells_with_interface_diagonal": int(self.last_hibm_unreached_cells_with_interface_diagonal),
            "unreached_cells_with_interface_coupling": int(self.last_hibm_unreached_cells_with_interface_coupling),
            "unreached_components_with_interface_hits": int(self.last_hibm_unreached_components_with_interface_hits),
            "hibm_pressure_component_labels_converged": bool(
                getattr(self, "last_hibm_pressure_component_labels_converged", True)),
            # the solid-band and pressure-fill sweeps (fluid.py:1300-1610,
            # 2100-2170) are not part of this path: their counters keep the
            # reference's "not run" value
            "hibm_solid_band_last_marked_increment": int(getattr(self, "last_hibm_solid_band_marked_increment", 0)),
            "hibm_solid_band_interior_cells": int(getattr(self, "last_hibm_solid_band_interior_cells", -1)),
            "hibm_solid_band_enclosed_water_cells": int(getattr(self, "last_hibm_solid_band_enclosed_water_cells", -1)),
            "hibm_pressure_filled_cell_count": int(getattr(self, "last_hibm_pressure_filled_cell_count", -1)),
            "cg_restart_count": self.last_project_cg_restart_count,
            "cg_restart_count_measured": self.last_project_cg_restart_count_measured,
            "cg_restart_policy": self.last_project_cg_restart_policy,
            "cg_initial_relative_residual_max": self.last_project_cg_initial_relative_residual_max,
            "cg_relative_residual_max": self.last_project_cg_relative_residual_max,
            "cg_converged_all": self.last_project_cg_converged_all,
            "cg_breakdown_count": self.last_project_cg_breakdown_count,
            "cg_breakdown_code": self.last_project_cg_breakdown_code,
            "cg_breakdown_dAd": float(self.last_project_cg_breakdown_dAd),
            "cg_breakdown": self.last_project_cg_breakdown,
        }

    # ------------------------------------------------------------------
    # body-force spreading (fluid.py:3196-3345)
    # ------------------------------------------------------------------
    def spread_surface_forces(
        self, surface_position_m, surface_force_n, vertex_count: int, center_m, force_sign: float = -1.0
    ) -> ForceSpreadingReport:
        if vertex_count <= 0:
            raise ValueError("vertex_count must be positive")
        self._refresh_structure()
        pos = surface_position_m.tensor if isinstance(surface_position_m, Field) else surface_position_m
        frc = surface_force_n.tensor if isinstance(surface_force_n, Field) else surface_force_n
        pos = pos.to(self.device, torch.float32).contiguous()
        frc = frc.to(self.device, torch.float32).contiguous()
        rep = self._report
        _native.call(
            "efsi_spread_surface_forces",
            self._plan,
            byref(self._axes),
            _ptr(pos),
            _ptr(frc),
            int(vertex_count),
            float(center_m[0]),
            float(center_m[1]),
            float(center_m[2]),
            float(force_sign),
            self.force.ptr(),
            _ptr(rep),
            _stream(),
        )
        r = rep[:6].cpu().numpy().astype(np.float32)
        surface = tuple(float(v) for v in r[:3])
        grid_force = tuple(float(v) for v in r[3:6])
        expected = np.float32(force_sign) * r[:3]
        denom = max(float(np.linalg.norm(expected)), 1.0e-12)
        err = float(np.linalg.norm(r[3:6] - expected)) / denom
        active = int((self.force.tensor.norm(dim=-1) > 0).sum().item())
        return ForceSpreadingReport(surface, grid_force, err, active)

    def apply_body_force(self, dt_s: float | None = None, *, read_report: bool = True) -> FluidImpulseReport | None:
        step_dt_s = self.dt if dt_s is None else float(dt_s)
        if step_dt_s <= 0.0:
            raise ValueError("dt_s must be positive")
        self._refresh_structure()
        rep = self._report
        _native.call(
            "efsi_apply_body_force",
            self._plan,
            self.force.ptr(),
            float(step_dt_s),
            float(self.rho),
            self.velocity.ptr(),
            _ptr(rep),
            _stream(),
        )
        if not read_report:
            return None
        r = rep[:7].cpu().tolist()
        impulse = np.asarray(r[:3])
        momentum = np.asarray(r[3:6])
        denom = max(float(np.linalg.norm(impulse)), 1.0e-12)
        return FluidImpulseReport(
            grid_impulse_n_s=tuple(float(v) for v in impulse),
            momentum_delta_n_s=tuple(float(v) for v in momentum),
            impulse_relative_error=float(np.linalg.norm(momentum - impulse)) / denom,
            active_velocity_cells=int(r[6]),
        )
