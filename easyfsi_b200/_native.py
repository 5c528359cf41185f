"""ctypes binding of the easyfsi_b200 C ABI (include/easyfsi_b200.h).

This is the Python side of the drop-in boundary: the solver classes call the
CUDA library only through the functions bound here.  There is no fallback: if
the library cannot be loaded the import of a solver fails loudly.
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, Structure, c_char_p, c_double, c_float, c_int32, c_void_p
from pathlib import Path

_LIB_NAME = "libeasyfsi_b200.so"
_PACKAGE_DIR = Path(__file__).resolve().parent


class LevelDesc(Structure):
    _fields_ = [
        ("nx", c_int32),
        ("ny", c_int32),
        ("nz", c_int32),
        ("wx", c_void_p),
        ("wy", c_void_p),
        ("wz", c_void_p),
        ("cdx", c_void_p),
        ("cdy", c_void_p),
        ("cdz", c_void_p),
    ]


class PcgParams(Structure):
    _fields_ = [
        ("max_iters", c_int32),
        ("precond", c_int32),
        ("remove_mean", c_int32),
        ("outlet", c_int32),
        ("iface_active", c_int32),
        ("use_graphs", c_int32),
        ("tolerance", c_double),
        ("device_loop", c_int32),
    ]


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
        ("used_graphs", c_int32),
        ("learned_iterations", c_int32),
        ("initial_relative_residual", c_double),
        ("relative_residual", c_double),
        ("breakdown_dAd", c_double),
        ("b_norm", c_double),
        ("learned_relative_residual", c_double),
        ("unreached_set_mean_projection_count", c_int32),
    ]


class GridAxes(Structure):
    _fields_ = [("fx", c_void_p), ("fy", c_void_p), ("fz", c_void_p), ("cx", c_void_p), ("cy", c_void_p), ("cz", c_void_p)]


class IbSearchParams(Structure):  # efsi_ib_search_params
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32),
        ("marker_count", c_int32), ("triangle_count", c_int32), ("classify_far_internal_nodes", c_int32),
        ("search_radius_m", c_float), ("interior_probe_distance_m", c_float), ("sign_tolerance_m", c_float),
        ("cell_center_x_m", c_void_p), ("cell_center_y_m", c_void_p), ("cell_center_z_m", c_void_p),
        ("bounds_min_m", c_float * 3), ("spacing_m", c_float * 3),
        ("box_min_m", c_float * 3), ("box_max_m", c_float * 3),
        ("marker_x", c_void_p), ("marker_n", c_void_p), ("triangles", c_void_p),
    ]


class IbSearchFields(Structure):  # efsi_ib_search_fields
    _fields_ = [
        ("node_kind", c_void_p), ("nearest_marker", c_void_p), ("signed_distance_m", c_void_p),
        ("boundary_point_m", c_void_p), ("interior_fluid_point_m", c_void_p),
        ("projection_marker_indices", c_void_p), ("projection_marker_weights", c_void_p), ("report", c_void_p),
    ]


class IbBcReport(Structure):  # efsi_ib_bc_report
    _fields_ = [("no_slip_dirichlet_count", c_int32), ("pressure_neumann_count", c_int32),
                ("inactive_internal_node_count", c_int32), ("max_abs_velocity_mps", c_float)]


class IbVdParams(Structure):  # efsi_ib_vd_params
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32),
        ("face_x_m", c_void_p), ("face_y_m", c_void_p), ("face_z_m", c_void_p),
        ("center_x_m", c_void_p), ("center_y_m", c_void_p), ("center_z_m", c_void_p),
        ("active_ib_node", c_void_p), ("target_velocity", c_void_p), ("target_normal", c_void_p),
        ("boundary_point_m", c_void_p), ("interior_fluid_point_m", c_void_p), ("nearest_marker", c_void_p),
        ("obstacle", c_void_p), ("velocity", c_void_p), ("marker_region_id", c_void_p), ("marker_count", c_int32),
    ]


class IbVdReport(Structure):  # efsi_ib_vd_report
    _fields_ = [(name, c_int32) for name in (
        "active_rows", "blocked_rows", "invalid_rows", "invalid_no_fluid_sample_rows", "invalid_nonpositive_gap_rows",
        "invalid_node_behind_boundary_rows", "invalid_node_beyond_interior_rows", "narrow_gap_rows",
        "relocated_rows", "merged_rows")] + [
        ("max_abs_velocity_mps", c_float), ("min_projection_weight", c_float), ("max_projection_weight", c_float)]


class IbVdFields(Structure):  # efsi_ib_vd_fields
    _fields_ = [("active", c_void_p), ("value_mps", c_void_p), ("projection_weight", c_void_p),
                ("anchor_cell", c_void_p), ("marker_region_id", c_void_p), ("report", c_void_p)]


class CgScalarValues(Structure):  # efsi_cg_scalar_values
    _fields_ = [(name, c_double) for name in (
        "rz", "rz_new", "dAd", "beta_numerator", "alpha", "beta", "breakdown_dAd")] + [("breakdown_code", c_int32)]


class ReachReport(Structure):  # efsi_reach_report
    _fields_ = [("unreached_cells", ctypes.c_int64), ("components", c_int32), ("overflow", c_int32)]


class MpmState(Structure):
    _fields_ = [
        ("particle_count", c_int32),
        ("nx", c_int32),
        ("ny", c_int32),
        ("nz", c_int32),
        ("bmin", c_float * 3),
        ("dx", c_float * 3),
        ("x", c_void_p),
        ("v", c_void_p),
        ("C", c_void_p),
        ("F", c_void_p),
        ("mass", c_void_p),
        ("volume", c_void_p),
        ("fext", c_void_p),
        ("fixed", c_void_p),
        ("region", c_void_p),
        ("rest_x", c_void_p),
        ("normal", c_void_p),
        ("area", c_void_p),
        ("rest_normal", c_void_p),
        ("rest_area", c_void_p),
        ("grid_mass", c_void_p),
        ("grid_velocity", c_void_p),
        ("grid_force", c_void_p),
    ]


class ShellState(Structure):  # efsi_shell_state
    _fields_ = [
        ("particle_count", c_int32), ("face_count", c_int32), ("edge_count", c_int32),
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32),
        ("bmin", c_float * 3), ("dx", c_float * 3),
        ("x", c_void_p), ("u", c_void_p), ("v", c_void_p), ("rest_x", c_void_p), ("mass", c_void_p),
        ("area", c_void_p), ("normal", c_void_p), ("internal_force", c_void_p), ("external_force", c_void_p),
        ("vertex_region", c_void_p), ("fixed", c_void_p), ("faces", c_void_p), ("face_region", c_void_p),
        ("edges", c_void_p), ("grid_mass", c_void_p), ("grid_velocity", c_void_p),
        ("grid_velocity_before", c_void_p), ("grid_force", c_void_p),
    ]


class ShellParams(Structure):  # efsi_shell_params
    _fields_ = [
        ("dt", c_float), ("pressure", c_float), ("velocity_damping", c_float), ("flip_blend", c_float),
        ("body_acceleration", c_float * 3),
        ("c1", c_float), ("c2", c_float), ("membrane_force_scale", c_float),
        ("thickness", c_float), ("primary_thickness", c_float), ("secondary_thickness", c_float),
        ("region_loads", c_int32), ("preserve_external_force", c_int32),
        ("primary_region", c_int32), ("secondary_region", c_int32), ("area_load_region", c_int32),
        ("primary_area_load", c_float * 3), ("primary_reaction", c_float * 3), ("secondary_reaction", c_float * 3),
        ("primary_area", c_float), ("secondary_area", c_float),
    ]


SHELL_SCRATCH_DOUBLES = 48

P = c_void_p
I = c_int32
F = c_float
D = c_double

# name -> argtypes (all return int status except the two string getters)
_PROTOTYPES: dict[str, list] = {
    "efsi_kernel_timing_enable": [I, I],
    "efsi_kernel_timing_read": [I, POINTER(ctypes.c_int64), POINTER(c_double), POINTER(c_double)],
    "efsi_fv_kernel_replay": [P, I, I, POINTER(c_double), POINTER(c_double), P],
    "efsi_fv_autotune": [P, I, POINTER(I), POINTER(c_double), I, P],
    "efsi_fv_plan_create": [POINTER(LevelDesc), I, I, POINTER(c_void_p)],
    "efsi_fv_plan_destroy": [P],
    "efsi_fv_set_masks": [P, P, P, P, P, P],
    "efsi_compute_divergence": [P, P, I, P, P],
    "efsi_mg_prepare_level0": [P, P, P, P, F, P, P],
    "efsi_fv_apply": [P, P, P, I, P],
    "efsi_fv_diagonal": [P, P, I, P],
    "efsi_apply_jacobi_preconditioner": [P, P, P, P, P],
    "efsi_weighted_dot": [P, P, P, POINTER(c_double), P],
    "efsi_weighted_dot_noalloc": [I, I, I, P, P, P, P, P, P, P, P],
    "efsi_fv_jacobi_sweep": [P, I, P, P, P, I, D, P],
    "efsi_fv_residual": [P, I, P, P, P, I, P],
    "efsi_mg_restrict": [P, I, P, P, P, P, P, P, P],
    "efsi_legacy_jacobi_solve": [P, P, P, F, F, F, F, I, I, P, P, P],
    "efsi_mg_prolong": [P, I, P, P, D, P],
    "efsi_mg_vcycle": [P, P, P, I, I, I, I, P],
    "efsi_fv_pcg_solve": [P, P, P, POINTER(PcgParams), POINTER(CgStats), P],
    "efsi_cg_scalars_write": [P, POINTER(CgScalarValues), P],
    "efsi_cg_scalars_read": [P, POINTER(CgScalarValues), P],
    "efsi_cg_compute_alpha": [P, P],
    "efsi_cg_compute_beta": [P, I, P],
    "efsi_fv_multigrid_solve": [P, P, P, I, I, I, P],
    "efsi_fv_jacobi_solve": [P, P, P, I, I, P],
    "efsi_subtract_pressure_gradient": [P, P, P, P, P, F, I, P, P],
    "efsi_apply_closed_boundary": [P, I, P, P],
    "efsi_apply_zmin_no_backflow": [P, P, P],
    "efsi_apply_velocity_dirichlet_rows": [P, P, P, F, P, P, P],
    "efsi_predict": [P, POINTER(GridAxes), P, F, F, I, P, P],
    "efsi_divergence_stats": [P, P, P, P, I, I, POINTER(c_double), P],
    "efsi_spread_surface_forces": [P, POINTER(GridAxes), P, P, I, F, F, F, F, P, P, P],
    "efsi_apply_body_force": [P, P, F, F, P, P, P],
    "efsi_mpm_plan_create": [I, I, I, I, POINTER(c_void_p)],
    "efsi_mpm_plan_destroy": [P],
    "efsi_mpm_step": [P, POINTER(MpmState), F, F, F, F, I, I, P, P],
    "efsi_shell_init": [POINTER(ShellState), P, P, P, F, F, F, F, I, I, I, P, P],
    "efsi_shell_update_normals": [POINTER(ShellState), P],
    "efsi_shell_add_region_area_load": [POINTER(ShellState), I, POINTER(c_float), P],
    "efsi_shell_step": [POINTER(ShellState), POINTER(ShellParams), P, P, P],
    "efsi_sample_pressure_tractions": [I, I, I, POINTER(GridAxes), P, P, P, P, P, I, P, P, P, I, I, F, P, P, P, P],
    "efsi_compute_marker_forces": [I, P, P, P, P],
    "efsi_clear_external_forces": [I, P, P, P],
    "efsi_bin_plan_create": [I, POINTER(c_float), POINTER(c_float), F, POINTER(c_void_p)],
    "efsi_bin_plan_destroy": [P],
    "efsi_bin_particles": [P, P, I, P],
    "efsi_scatter_marker_forces": [P, I, P, P, P, P, P, P],
    "efsi_surface_feedback": [P, I, P, P, P, P, P, P, P, P, F, P, P],
    "efsi_ib_search_plan_create": [POINTER(c_void_p)],
    "efsi_ib_search_plan_destroy": [P],
    "efsi_ib_node_search": [P, POINTER(IbSearchParams), POINTER(IbSearchFields), P],
    "efsi_ib_reset_anchor_cells": [P, ctypes.c_int64, P],
    "efsi_ib_build_boundary_conditions": [ctypes.c_int64, P, P, P, P, P, P, P, I, P, P, P, P, P, P],
    "efsi_ib_velocity_dirichlet_rows": [P, POINTER(IbVdParams), POINTER(IbVdFields), I, P],
    "efsi_fv_bicgstab": [P, P, P, I, I, D, D, I, POINTER(ctypes.c_int64), POINTER(c_double), P],
    "efsi_conv3d_bf16": [I, I, I, I, I, P, P, P, I, P, P, P, P],
    "efsi_conv3d_wgrad": [I, I, I, I, I, P, P, P, P],
    "efsi_unet_create": [I, POINTER(c_void_p)],
    "efsi_unet_destroy": [P],
    "efsi_unet_param_count": [P, POINTER(ctypes.c_int64)],
    "efsi_unet_layer_offsets": [P, P, P, P],
    "efsi_unet_get_params": [P, P, P],
    "efsi_unet_set_params": [P, P],
    "efsi_unet_forward": [P, I, I, I, P, P, P],
    "efsi_unet_accumulate_gradient": [P, I, I, I, P, P, P, POINTER(c_double), P],
    "efsi_unet_backward_from": [P, I, I, I, P, P, P],
    "efsi_unet_zero_grad": [P, P],
    "efsi_unet_adam_step": [P, F, F, F, F, P],
    "efsi_fv_set_learned_preconditioner": [P, P, P],
    "efsi_fv_set_interface_coupling": [P, I, P, P, P, P, P],
    "efsi_fv_copy_rhs": [P, P, P],
    "efsi_zero_buffers": [I, P, P, P],
    "efsi_fv_learned_input": [P, P, P, P],
    "efsi_fv_learned_presmooth": [P, P, P, I, P],
    "efsi_fv_coarse_kernel_blocks": [P, POINTER(c_int32)],
    "efsi_fv_pcg_device_stats": [P, POINTER(CgStats), P],
    "efsi_step_graph_begin": [P],
    "efsi_step_graph_end": [P, POINTER(c_void_p)],
    "efsi_step_graph_launch": [P, P],
    "efsi_step_graph_destroy": [P],
    "efsi_fv_set_unreached_components": [P, P, I, P],
    "efsi_divergence_final_report": [P, P, P, P, P, P, I, P, P],
    "efsi_fv_subtract_unreached_means": [P, P, P, P, P],
    "efsi_reach_plan_create": [POINTER(c_void_p)],
    "efsi_reach_plan_destroy": [P],
    "efsi_outlet_reachability": [P, I, I, I, P, P, P, P, I, I, P, P, POINTER(ReachReport), P],
}

_lib = None


def library_path() -> Path:
    override = os.environ.get("EASYFSI_B200_LIB")
    return Path(override) if override else _PACKAGE_DIR / _LIB_NAME


def load():
    """Load (once) and return the CUDA library with typed prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not path.exists():
        raise RuntimeError(
            f"easyfsi_b200 CUDA library not found at {path}; build it with `python -m easyfsi_b200.build`"
        )
    lib = ctypes.CDLL(str(path))
    lib.efsi_last_error.restype = c_char_p
    lib.efsi_last_error.argtypes = []
    lib.efsi_version.restype = c_char_p
    lib.efsi_version.argtypes = []
    lib.efsi_kernel_launch_count.restype = ctypes.c_uint64
    lib.efsi_kernel_launch_count.argtypes = []
    lib.efsi_fv_graph_error.restype = c_char_p
    lib.efsi_fv_graph_error.argtypes = [c_void_p]
    for name, args in _PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = c_int32
        fn.argtypes = args
    _lib = lib
    return lib


def exported_names() -> list[str]:
    return ["efsi_last_error", "efsi_version", "efsi_kernel_launch_count", "efsi_fv_graph_error", *_PROTOTYPES.keys()]


class NativeError(RuntimeError):
    pass


def check(status: int, what: str = "") -> None:
    if status != 0:
        msg = load().efsi_last_error().decode(errors="replace")
        raise NativeError(f"{what or 'easyfsi_b200'} failed (status {status}): {msg}")


def kernel_launches() -> int:
    return int(load().efsi_kernel_launch_count())


KERNEL_FAMILIES = {
    "spmv_dir": 0,
    "sweep_l0": 1,
    "cg_update": 2,
    "restrict_l0": 3,
    "cg_dots": 4,
    "p2g": 5,
    "predict": 6,
    "grid_update": 7,
    "g2p": 8,
    "scatter": 9,
    "feedback": 10,
    "mpm_step": 11,
    # replay only
    "sweep0_l0": 16,
    "sweep_prolong_l0": 17,
    "sweep_dots_l0": 18,
    "vcycle": 19,
}


def kernel_replay(plan, family: str, reps: int = 50) -> tuple[float, float]:
    """Mean ms per launch and algorithmic bytes per launch of a level-0 family."""
    ms, nbytes = c_double(0.0), c_double(0.0)
    stream = c_void_p(__import__("torch").cuda.current_stream().cuda_stream)
    call("efsi_fv_kernel_replay", plan, KERNEL_FAMILIES[family], int(reps), ctypes.byref(ms), ctypes.byref(nbytes), stream)
    return float(ms.value), float(nbytes.value)


def kernel_timing_enable(family: str, enable: bool = True) -> None:
    call("efsi_kernel_timing_enable", KERNEL_FAMILIES[family], 1 if enable else 0)


def kernel_timing_read(family: str) -> tuple[int, float, float]:
    """(launches, total ms, total algorithmic bytes) of a timed kernel family."""
    n, ms, by = ctypes.c_int64(0), c_double(0.0), c_double(0.0)
    call("efsi_kernel_timing_read", KERNEL_FAMILIES[family], ctypes.byref(n), ctypes.byref(ms), ctypes.byref(by))
    return int(n.value), float(ms.value), float(by.value)


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args), name)
