"""efsi_weighted_dot_noalloc: the plan-free, allocation-free weighted dot.

Some callers cannot allocate device memory at the point where they need the
dot: the owner of a caching allocator that must not re-enter it, or code that
holds no solver plan.  This entry point serves them with a static scratch
array.  The file is collected last, so that a run stopping at the first
failure has already run every other test; the test also passes alone.  It
compares the entry point with the plan-based efsi_weighted_dot on calls in a
row, with a smaller grid in between: every call clears the scratch's ticket
itself, so the partials and ticket left by an earlier call do not matter.
"""

import numpy as np
import pytest
import torch

from easyfsi_b200 import _native


def test_noalloc_dot_rejects_grids_beyond_the_static_scratch():
    # argument checks run before any device work, so no GPU is needed
    lib = _native.load()
    status = lib.efsi_weighted_dot_noalloc(1024, 1024, 1024, None, None, None, None, None, None, None, None)
    assert status == 1  # EFSI_ERR_ARG
    assert b"static scratch limit" in lib.efsi_last_error()
    status = lib.efsi_weighted_dot_noalloc(0, 4, 4, None, None, None, None, None, None, None, None)
    assert status == 1


@pytest.mark.gpu
def test_noalloc_dot_matches_plan_dot_on_consecutive_calls():
    from easyfsi_b200.fluid import CartesianFluidSolver, FluidDomainSpec
    from easyfsi_b200.grid import CartesianGrid
    from easyfsi_b200.scenarios import graded_axis_widths

    nx, ny, nz = 40, 24, 48
    grid = CartesianGrid(
        bounds_min_m=(0.0, 0.0, 0.0),
        cell_widths_x_m=graded_axis_widths(nx, 0.0, 1.0, 0.3, 0.7),
        cell_widths_y_m=graded_axis_widths(ny, 0.0, 1.0, 0.3, 0.7),
        cell_widths_z_m=graded_axis_widths(nz, 0.0, 1.0, 0.2, 0.8),
    )
    spec = FluidDomainSpec((0, 0, 0), grid.bounds_max_m, None, 1000.0, 1.0e-3, 1.0e-3, cartesian_grid=grid)
    fl = CartesianFluidSolver(spec)
    rng = np.random.default_rng(41)
    obs = (rng.random((nx, ny, nz)) < 0.1).astype(np.int32)
    fl.obstacle.from_numpy(obs)
    a = rng.normal(size=(nx, ny, nz))
    b = rng.normal(size=(nx, ny, nz))
    fl.pressure_tmp.from_numpy(a)
    fl.cg_d.from_numpy(b)
    expected = fl._weighted_dot_kernel(fl.pressure_tmp, fl.cg_d)

    out = torch.full((1,), float("nan"), dtype=torch.float64, device=fl.device)
    stream = torch.cuda.current_stream(fl.device).cuda_stream
    # a smaller grid first (fewer blocks): the next calls must not depend on
    # the partial sums or the ticket it leaves in the shared scratch
    small = torch.full((1,), float("nan"), dtype=torch.float64, device=fl.device)
    _native.call("efsi_weighted_dot_noalloc", 1, ny, nz, fl.obstacle.ptr(), fl.cell_width_x_m.ptr(),
                 fl.cell_width_y_m.ptr(), fl.cell_width_z_m.ptr(), fl.pressure_tmp.ptr(), fl.cg_d.ptr(),
                 small.data_ptr(), stream)
    for _ in range(2):
        out.fill_(float("nan"))
        _native.call(
            "efsi_weighted_dot_noalloc",
            nx,
            ny,
            nz,
            fl.obstacle.ptr(),
            fl.cell_width_x_m.ptr(),
            fl.cell_width_y_m.ptr(),
            fl.cell_width_z_m.ptr(),
            fl.pressure_tmp.ptr(),
            fl.cg_d.ptr(),
            out.data_ptr(),
            stream,
        )
        torch.cuda.synchronize(fl.device)
        got = float(out.item())
        assert got == pytest.approx(expected, rel=1e-12, abs=1e-300)
    # the same sum in numpy (fluid = obstacle == 0, V from the f32 widths)
    w = [np.asarray(x, np.float32).astype(np.float64) for x in (grid.cell_widths_x_m, grid.cell_widths_y_m, grid.cell_widths_z_m)]
    vol = np.einsum("i,j,k->ijk", *w)
    ref = float(((a * b) * vol)[obs == 0].sum())
    assert got == pytest.approx(ref, rel=1e-10)
