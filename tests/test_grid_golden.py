"""Host grid metrics against fixtures generated from the reference's own grid
builder (tests/golden/make_golden.py)."""

import json
from pathlib import Path

import numpy as np
import pytest

from easyfsi_b200.geometry import UvSphereResolution, make_uv_sphere
from easyfsi_b200.grid import (
    CartesianGrid,
    FluidDomainSpec,
    GradedGridSpec,
    RefinementRegion,
    build_graded_grid,
    multigrid_axis_widths,
    multigrid_shapes,
)
from easyfsi_b200.hyperelastic import NeoHookeanMaterial

GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "reference_host.json").read_text())


def _spec(case):
    return GradedGridSpec(
        bounds_min_m=tuple(case["bounds_min"]),
        bounds_max_m=tuple(case["bounds_max"]),
        farfield_spacing_m=tuple(case["farfield"]) if isinstance(case["farfield"], list) else case["farfield"],
        max_growth_ratio=case["ratio"],
        refinement_regions=tuple(
            RefinementRegion(tuple(a), tuple(b), tuple(t) if isinstance(t, list) else t) for a, b, t in case["regions"]
        ),
    )


@pytest.mark.parametrize("case", GOLD["graded"], ids=[c["name"] for c in GOLD["graded"]])
def test_graded_grid_matches_reference_bitwise(case):
    grid = build_graded_grid(_spec(case))
    for axis in range(3):
        assert list(grid._widths(axis)) == case["widths"][axis]
        assert list(grid.axis_faces(axis)) == case["faces"][axis]
        assert list(grid.axis_centers(axis)) == case["centers"][axis]
        assert list(grid.axis_center_distances(axis)) == case["center_distances"][axis]
    for v, want in zip((-0.05, 0.0, 0.013, 0.31, 0.5, 0.777, 1.0, 1.3), case["grid_coordinates"]):
        got = [grid.grid_coordinate_x(v), grid.grid_coordinate_y(v), grid.grid_coordinate_z(v)]
        assert got == want
    assert grid.is_uniform == case["is_uniform"]
    shapes = multigrid_shapes(grid.grid_nodes)
    assert [list(s) for s in shapes] == case["mg_shapes"]
    mg = multigrid_axis_widths(grid, shapes)
    assert [[list(a) for a in level] for level in mg] == case["mg_widths"]


@pytest.mark.parametrize("case", GOLD["multigrid_shapes"], ids=lambda c: "x".join(map(str, c["shape"])))
def test_multigrid_depths(case):
    assert [list(s) for s in multigrid_shapes(tuple(case["shape"]))] == case["levels"]


def test_survey_level_counts():
    depth = {tuple(c["shape"]): len(c["levels"]) for c in GOLD["multigrid_shapes"]}
    assert depth[(64, 64, 64)] == 6
    assert depth[(128, 128, 256)] == 7
    assert depth[(256, 256, 256)] == 8
    assert depth[(192, 192, 192)] == 7


def test_uniform_grid():
    ref = GOLD["uniform"][0]
    grid = CartesianGrid.uniform(bounds_min_m=(0.0, -0.5, 1.0), bounds_max_m=(1.0, 0.5, 3.0), grid_nodes=(10, 7, 13))
    for axis in range(3):
        assert list(grid._widths(axis)) == ref["widths"][axis]
        assert list(grid.axis_center_distances(axis)) == ref["center_distances"][axis]
    assert grid.is_uniform == ref["is_uniform"]
    assert list(grid.uniform_spacing_m) == ref["spacing"]


def test_material_cards():
    for ref in GOLD["material"]:
        m = NeoHookeanMaterial.from_youngs_modulus(name="p", density_kgm3=ref["rho"], youngs_modulus_pa=ref["E"], poissons_ratio=ref["nu"])
        assert m.shear_modulus_pa == pytest.approx(ref["mu"], rel=1e-15)
        assert m.bulk_modulus_pa == pytest.approx(ref["K"], rel=1e-15)
        assert m.lame_lambda_pa == pytest.approx(ref["lambda"], rel=1e-12)
        assert m.sound_speed_mps == pytest.approx(ref["sound_speed"], rel=1e-12)


def test_uv_sphere():
    for ref in GOLD["uv_sphere"]:
        mesh = make_uv_sphere(UvSphereResolution(ref["lat"], ref["lon"]), ref["radius"])
        np.testing.assert_allclose(mesh.vertices, np.asarray(ref["vertices"]), rtol=0, atol=1e-15)
        assert mesh.faces.tolist() == ref["faces"]


def test_domain_spec_validation():
    with pytest.raises(ValueError):
        FluidDomainSpec.unit_box(grid_nodes=(3, 8, 8))
    with pytest.raises(ValueError):
        FluidDomainSpec((0, 0, 0), (1, 1, 1), (8, 8, 8), -1.0, 1e-3, 1e-3)
    spec = FluidDomainSpec.unit_box(grid_nodes=(8, 8, 8))
    assert spec.cell_volume_m3 == pytest.approx(1.0 / 512)


def test_multigrid_default_cycles_cover_nonuniform_grids():
    """test_core_fluid.py:704 (fluid.py:688-689, 731-734): graded grids get more
    default V-cycles than uniform ones (host logic, through a stand-in)."""
    from types import SimpleNamespace

    from easyfsi_b200.fluid import CartesianFluidSolver
    from easyfsi_b200.grid import CartesianGrid

    uniform = CartesianGrid(bounds_min_m=(0.0, 0.0, 0.0), cell_widths_x_m=(0.125,) * 8, cell_widths_y_m=(0.125,) * 8,
                            cell_widths_z_m=(0.125,) * 8)
    graded_w = (0.08, 0.09, 0.10, 0.13, 0.14, 0.15, 0.16, 0.15)
    graded = CartesianGrid(bounds_min_m=(0.0, 0.0, 0.0), cell_widths_x_m=graded_w, cell_widths_y_m=(0.125,) * 8,
                           cell_widths_z_m=graded_w)
    cycles = {}
    for name, grid in (("uniform", uniform), ("graded", graded)):
        stub = SimpleNamespace(grid=grid, DEFAULT_MULTIGRID_CYCLES=CartesianFluidSolver.DEFAULT_MULTIGRID_CYCLES,
                               DEFAULT_NONUNIFORM_MULTIGRID_CYCLES=CartesianFluidSolver.DEFAULT_NONUNIFORM_MULTIGRID_CYCLES)
        cycles[name] = CartesianFluidSolver.default_multigrid_cycles(stub)
    assert cycles["uniform"] == CartesianFluidSolver.DEFAULT_MULTIGRID_CYCLES == 12
    assert cycles["graded"] == CartesianFluidSolver.DEFAULT_NONUNIFORM_MULTIGRID_CYCLES == 24
    assert cycles["graded"] > cycles["uniform"] >= 1
