"""Generate the golden grid / geometry / material fixtures from the reference.

Run in a container where the reference tree is available:

    python tests/golden/make_golden.py /path/to/EasyFsi

The reference's pure-Python host code (CartesianGrid, build_graded_grid, the
multigrid shape / width helpers, NeoHookeanMaterial, make_uv_sphere) is
imported directly from its source under a stand-in ``taichi`` module (Taichi is
not installable here; only class and decorator definitions touch it at import
time) and its outputs are written to ``tests/golden/reference_host.json``.
The tests compare easyfsi_b200's own restatement against this file; nothing at
test time reads the reference tree.
"""

from __future__ import annotations

import importlib
import json
import sys
import types
from pathlib import Path


class _Anything:
    """Permissive stand-in: every attribute / call / subscript yields another
    stand-in; used as a decorator it returns the decorated object unchanged."""

    def __getattr__(self, name):
        return _Anything()

    def __call__(self, *args, **kwargs):
        if len(args) == 1 and not kwargs and (callable(args[0]) or isinstance(args[0], type)):
            return args[0]
        return _Anything()

    def __getitem__(self, item):
        return _Anything()

    def __iter__(self):
        return iter(())

    def __mro_entries__(self, bases):
        return (object,)


def _install_stubs() -> None:
    ti = types.ModuleType("taichi")
    ti.__getattr__ = lambda name: _Anything()  # type: ignore[attr-defined]
    for name in ("data_oriented", "kernel", "func", "pyfunc", "real_func"):
        setattr(ti, name, lambda obj=None, *a, **k: obj)
    sys.modules["taichi"] = ti
    for name in ("trimesh", "gmsh", "pyvista", "matplotlib"):
        sys.modules.setdefault(name, types.ModuleType(name))


def _import_reference(root: Path):
    _install_stubs()
    pkg = types.ModuleType("simulation_core")
    pkg.__path__ = [str(root / "simulation_core")]  # type: ignore[attr-defined]
    sys.modules["simulation_core"] = pkg
    fluid = importlib.import_module("simulation_core.fluid")
    hyper = importlib.import_module("simulation_core.hyperelastic")
    geometry = importlib.import_module("simulation_core.geometry")
    return fluid, hyper, geometry


GRADED_SPECS = [
    # (name, bounds_min, bounds_max, farfield, ratio, regions[(min, max, spacing)])
    ("survey_probe", (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 1.0 / 32.0, 1.05, [((0.3, 0.3, 0.2), (0.7, 0.7, 0.8), 1.0 / 128.0)]),
    ("coarse_box", (0.0, 0.0, 0.0), (1.0, 0.5, 2.0), 0.1, 1.2, [((0.4, 0.1, 0.8), (0.6, 0.3, 1.2), 0.02)]),
    ("two_regions", (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0), 0.25, 1.15,
     [((-0.6, -0.2, -0.2), (-0.3, 0.2, 0.2), 0.03), ((0.3, -0.2, -0.2), (0.6, 0.2, 0.2), 0.05)]),
    ("snap_to_wall", (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 0.08, 1.1, [((0.0, 0.2, 0.5), (0.3, 0.8, 1.0), 0.02)]),
    ("aniso_spacing", (0.0, 0.0, 0.0), (2.0, 1.0, 1.0), (0.2, 0.1, 0.1), 1.08, [((0.8, 0.4, 0.4), (1.2, 0.6, 0.6), (0.02, 0.01, 0.03))]),
    ("merge_close", (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 0.1, 1.3, [((0.2, 0.2, 0.2), (0.4, 0.4, 0.4), 0.02), ((0.41, 0.41, 0.41), (0.6, 0.6, 0.6), 0.03)]),
    ("no_regions", (0.0, 0.0, 0.0), (1.0, 0.7, 0.3), 0.07, 1.2, []),
]

MG_SHAPES = [(64, 64, 64), (128, 128, 256), (256, 256, 256), (192, 192, 192), (5, 5, 5), (4, 7, 9), (12, 12, 16), (96, 96, 111)]


def main(root: Path) -> None:
    fluid, hyper, geometry = _import_reference(root)
    out: dict = {"graded": [], "multigrid_shapes": [], "uniform": [], "material": [], "uv_sphere": []}
    for name, lo, hi, far, ratio, regions in GRADED_SPECS:
        spec = fluid.GradedGridSpec(
            bounds_min_m=lo,
            bounds_max_m=hi,
            farfield_spacing_m=far,
            max_growth_ratio=ratio,
            refinement_regions=tuple(fluid.RefinementRegion(a, b, t) for a, b, t in regions),
        )
        grid = fluid.build_graded_grid(spec)
        shapes = fluid.CartesianFluidSolver._build_multigrid_shapes(grid.grid_nodes)
        mg = fluid.CartesianFluidSolver._build_multigrid_axis_widths(grid, shapes)
        out["graded"].append(
            {
                "name": name,
                "bounds_min": lo,
                "bounds_max": hi,
                "farfield": far,
                "ratio": ratio,
                "regions": regions,
                "widths": [list(grid.cell_widths_x_m), list(grid.cell_widths_y_m), list(grid.cell_widths_z_m)],
                "faces": [list(grid.cell_faces_x_m), list(grid.cell_faces_y_m), list(grid.cell_faces_z_m)],
                "centers": [list(grid.cell_centers_x_m), list(grid.cell_centers_y_m), list(grid.cell_centers_z_m)],
                "center_distances": [list(grid.center_distances_x_m), list(grid.center_distances_y_m), list(grid.center_distances_z_m)],
                "grid_coordinates": [
                    [grid.grid_coordinate_x(v), grid.grid_coordinate_y(v), grid.grid_coordinate_z(v)]
                    for v in (-0.05, 0.0, 0.013, 0.31, 0.5, 0.777, 1.0, 1.3)
                ],
                "is_uniform": grid.is_uniform,
                "mg_shapes": [list(s) for s in shapes],
                "mg_widths": [[list(a) for a in level] for level in mg],
            }
        )
    for shape in MG_SHAPES:
        out["multigrid_shapes"].append({"shape": list(shape), "levels": [list(s) for s in fluid.CartesianFluidSolver._build_multigrid_shapes(shape)]})
    uni = fluid.CartesianGrid.uniform(bounds_min_m=(0.0, -0.5, 1.0), bounds_max_m=(1.0, 0.5, 3.0), grid_nodes=(10, 7, 13))
    out["uniform"].append(
        {
            "widths": [list(uni.cell_widths_x_m), list(uni.cell_widths_y_m), list(uni.cell_widths_z_m)],
            "center_distances": [list(uni.center_distances_x_m), list(uni.center_distances_y_m), list(uni.center_distances_z_m)],
            "is_uniform": uni.is_uniform,
            "spacing": list(uni.uniform_spacing_m),
        }
    )
    for e, nu, rho in ((1.0e5, 0.45, 1100.0), (5.0e4, 0.45, 1100.0), (2.0e5, 0.3, 1000.0)):
        m = hyper.NeoHookeanMaterial.from_youngs_modulus(name="probe", density_kgm3=rho, youngs_modulus_pa=e, poissons_ratio=nu)
        out["material"].append(
            {"E": e, "nu": nu, "rho": rho, "mu": m.shear_modulus_pa, "K": m.bulk_modulus_pa, "lambda": m.lame_lambda_pa,
             "sound_speed": m.sound_speed_mps}
        )
    for lat, lon, r in ((4, 6, 0.5), (8, 16, 0.15)):
        mesh = geometry.make_uv_sphere(geometry.UvSphereResolution(latitude_bands=lat, longitude_segments=lon), r)
        out["uv_sphere"].append(
            {"lat": lat, "lon": lon, "radius": r, "vertices": mesh.vertices.tolist(), "faces": mesh.faces.tolist()}
        )
    path = Path(__file__).resolve().parent / "reference_host.json"
    path.write_text(json.dumps(out, indent=1))
    print(f"wrote {path} ({path.stat().st_size} bytes)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the EasyFsi reference tree>")
    main(Path(sys.argv[1]))
