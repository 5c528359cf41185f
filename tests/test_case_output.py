"""History CSV and snapshot NPZ formats of the case runners
(cases/squid_soft_robot.py:4907-4939, 5714-5757)."""

from types import SimpleNamespace

import numpy as np
import pytest

from easyfsi_b200.case_output import read_csv_rows, write_csv, write_fluid_snapshot_npz


class _HostField:
    def __init__(self, a):
        self.a = np.asarray(a)

    def to_numpy(self):
        return self.a.copy()


def test_history_csv_header_is_the_ordered_union_and_replace_is_atomic(tmp_path):
    path = tmp_path / "history.csv"
    write_csv(path, [{"step": 1, "t": 0.1}, {"step": 2, "extra": "x", "t": 0.2}])
    assert not (tmp_path / "history.csv.tmp").exists()
    assert path.read_text(encoding="utf-8").splitlines()[0] == "step,t,extra"
    rows = read_csv_rows(path)
    assert rows == [{"step": "1", "t": "0.1", "extra": ""}, {"step": "2", "t": "0.2", "extra": "x"}]
    write_csv(path, [])  # no rows: the file is left as it is
    assert len(read_csv_rows(path)) == 2
    assert read_csv_rows(tmp_path / "missing.csv") == []


def _expected_snapshot(vel, obstacle, xg, count):
    # the reference computes the speed over the whole field on the host, then slices
    speed = np.linalg.norm(vel.astype(np.float32), axis=-1).astype(np.float32)
    nx, ny, _ = speed.shape
    return speed[:, ny // 2, :], speed[nx // 2, :, :], obstacle.astype(np.int8)[:, ny // 2, :], xg[:count]


def test_snapshot_npz_keys_dtypes_and_slices_on_host_fields(tmp_path):
    rng = np.random.default_rng(7)
    vel = rng.standard_normal((5, 4, 6, 3)).astype(np.float32)
    obstacle = rng.integers(0, 2, (5, 4, 6)).astype(np.int32)
    xg = rng.standard_normal((9, 3)).astype(np.float32)
    fluid = SimpleNamespace(velocity=_HostField(vel), obstacle=_HostField(obstacle),
                            cell_center_x_m=_HostField(np.arange(5.0)), cell_center_y_m=_HostField(np.arange(4.0)),
                            cell_center_z_m=_HostField(np.arange(6.0)))
    path = write_fluid_snapshot_npz(snapshot_dir=tmp_path / "snaps", step=12, fluid=fluid,
                                    markers=SimpleNamespace(x_gamma_m=_HostField(xg)), marker_count=7,
                                    time_s=0.25, pressure_pa=-3.0)
    assert path.name == "snapshot_000012.npz"
    with np.load(path) as z:
        assert sorted(z.files) == sorted(["step", "time_s", "pressure_pa", "speed_xz", "speed_yz", "obstacle_xz",
                                          "marker_positions_m", "cell_center_x_m", "cell_center_y_m",
                                          "cell_center_z_m"])
        assert z["step"].dtype == np.int64 and int(z["step"]) == 12
        assert z["time_s"].dtype == np.float64 and float(z["pressure_pa"]) == -3.0
        xz, yz, oxz, pos = _expected_snapshot(vel, obstacle, xg, 7)
        np.testing.assert_allclose(z["speed_xz"], xz, rtol=1e-6)
        np.testing.assert_allclose(z["speed_yz"], yz, rtol=1e-6)
        assert z["speed_xz"].dtype == np.float32 and z["obstacle_xz"].dtype == np.int8
        assert np.array_equal(z["obstacle_xz"], oxz) and np.array_equal(z["marker_positions_m"], pos)
        assert z["cell_center_z_m"].dtype == np.float32 and z["cell_center_z_m"].shape == (6,)


def test_snapshot_failure_is_reported_not_raised(tmp_path, capsys):
    assert write_fluid_snapshot_npz(snapshot_dir=tmp_path, step=1, fluid=None, markers=None, marker_count=0,
                                    time_s=0.0, pressure_pa=0.0) is None
    assert "[snapshot] step 1 failed" in capsys.readouterr().out


@pytest.mark.gpu
def test_snapshot_of_a_coupled_scene_matches_its_fields(tmp_path):
    from easyfsi_b200.scenarios import CoupledScene, tiny_config

    scene = CoupledScene(tiny_config())
    scene.step()
    m = scene.markers
    path = write_fluid_snapshot_npz(snapshot_dir=tmp_path, step=1, fluid=scene.fluid, markers=m,
                                    marker_count=m.marker_count, time_s=1e-3, pressure_pa=0.0)
    xz, yz, oxz, pos = _expected_snapshot(scene.fluid.velocity.to_numpy(), scene.fluid.obstacle.to_numpy(),
                                          m.x_gamma_m.to_numpy(), m.marker_count)
    with np.load(path) as z:
        np.testing.assert_allclose(z["speed_xz"], xz, rtol=1e-6, atol=1e-12)
        np.testing.assert_allclose(z["speed_yz"], yz, rtol=1e-6, atol=1e-12)
        assert np.array_equal(z["obstacle_xz"], oxz) and np.array_equal(z["marker_positions_m"], pos)
