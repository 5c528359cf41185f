"""The membrane oracle against the reference's own known answers (CPU).

Runs every case of ``shell_cases`` (restated from the reference's
tests/test_mooney_shell_mpm.py) on the FP64 oracle, which pins it before the
GPU parity tests use it as the checker."""

import numpy as np
import pytest

import shell_cases as sc
from oracle.oracle_shell import OracleTriShell, unique_undirected_edges


@pytest.mark.parametrize("case", sc.ALL_CASES, ids=sc.CASE_IDS)
def test_oracle_shell_known_answers(case):
    case(sc.OracleShellAdapter)


def test_oracle_unique_edges_of_two_triangles():
    # mooney_shell_mpm.py:53-61: a shared edge is listed once, pairs sorted
    edges = unique_undirected_edges(np.array([[0, 1, 2], [2, 1, 3]]))
    assert edges.tolist() == [[0, 1], [0, 2], [1, 2], [1, 3], [2, 3]]


def test_oracle_region_load_moves_region_and_conserves_momentum():
    # reference tests/test_mooney_shell_mpm.py:1398-1442 (load on the primary region only)
    mesh, region = sc.plate_mesh(8, 6)
    o = OracleTriShell(mesh.vertices, mesh.faces, thickness_m=2e-3, density_kgm3=1000.0, c1_pa=1e5, c2_pa=0.0,
                       face_region_id=region, primary_region_id=1, secondary_region_id=2)
    rep = o.advance_region_loads(dt_s=1e-4, primary_region_id=1, secondary_region_id=2,
                                 primary_area_load_npm2=(0.0, 0.0, 100.0),
                                 primary_interface_reaction_n=(0.0, 0.0, 0.0),
                                 secondary_interface_reaction_n=(0.0, 0.0, 0.0))
    assert rep["primary_mean_velocity_mps"][2] > 0.0
    assert abs(rep["secondary_mean_velocity_mps"][2]) < 0.5 * rep["primary_mean_velocity_mps"][2]
    v32 = mesh.vertices.astype(np.float32).astype(np.float64)  # the membrane stores f32 positions
    area = sum(0.5 * np.linalg.norm(np.cross(v32[f[1]] - v32[f[0]], v32[f[2]] - v32[f[0]]))
               for f, r in zip(mesh.faces, region) if r == 1)
    # vertex forces are stored in f32 as the reference stores them
    assert rep["total_force_n"][2] == pytest.approx(100.0 * area, rel=1e-7)
    assert rep["transfer_relative_error"] < 1e-9
