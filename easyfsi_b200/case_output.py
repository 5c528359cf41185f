"""On-disk formats of the case runners: the per-step history CSV and the
per-step fluid snapshot NPZ (cases/squid_soft_robot.py:4907-4940 and
:5714-5757).

The formats are the reference's, so its plotting and comparison scripts read
these files unchanged: the CSV header is the ordered union of the rows' keys
(first appearance order) and the file is replaced atomically through a
``.tmp`` sibling, retried while another process holds the destination; the
NPZ holds step, time, pressure, the speed on the y and x mid-planes, the
obstacle on the y mid-plane, the marker positions and the cell centres, with
the reference's key names and dtypes.  On the B200 the snapshot computes the
two speed planes on the device and copies only them (two planes of floats
instead of the whole velocity field).
"""

from __future__ import annotations

import csv
import os
import time
from pathlib import Path

import numpy as np
import torch

WRITE_CSV_REPLACE_ATTEMPTS = 20
WRITE_CSV_REPLACE_BACKOFF_S = 0.25


def write_csv(path: Path, rows: list[dict[str, object]]) -> None:
    """History CSV (squid_soft_robot.py:4907-4932): ordered union header, atomic replace."""
    if not rows:
        return
    path = Path(path)
    fields: dict[str, None] = {}
    for row in rows:
        for key in row:
            fields.setdefault(key, None)
    temp = path.with_name(path.name + ".tmp")
    with temp.open("w", newline="", encoding="utf-8") as handle:
        writer = csv.DictWriter(handle, fieldnames=list(fields))
        writer.writeheader()
        writer.writerows(rows)
    error: PermissionError | None = None
    for _ in range(WRITE_CSV_REPLACE_ATTEMPTS):
        try:
            os.replace(temp, path)
            return
        except PermissionError as exc:  # a reader holds the destination open; retry within the budget
            error = exc
            time.sleep(WRITE_CSV_REPLACE_BACKOFF_S)
    raise error


def read_csv_rows(path: Path) -> list[dict[str, object]]:
    """squid_soft_robot.py:4935-4939."""
    path = Path(path)
    if not path.exists():
        return []
    with path.open("r", newline="", encoding="utf-8") as handle:
        return list(csv.DictReader(handle))


def _device_tensor(field) -> torch.Tensor:
    return field.tensor if hasattr(field, "tensor") else torch.as_tensor(np.asarray(field.to_numpy()))


def write_fluid_snapshot_npz(*, snapshot_dir: Path, step: int, fluid, markers, marker_count: int, time_s: float,
                             pressure_pa: float) -> Path | None:
    """Per-step visualisation snapshot (squid_soft_robot.py:5714-5757).  A
    failure is reported and returns None, so a snapshot never ends a run."""
    try:
        snapshot_dir = Path(snapshot_dir)
        snapshot_dir.mkdir(parents=True, exist_ok=True)
        vel = _device_tensor(fluid.velocity)
        obstacle = _device_tensor(fluid.obstacle)
        nx, ny, nz = (int(v) for v in vel.shape[:3])
        speed_xz = torch.linalg.vector_norm(vel[:, ny // 2, :, :].float(), dim=-1)
        speed_yz = torch.linalg.vector_norm(vel[nx // 2, :, :, :].float(), dim=-1)
        obstacle_xz = obstacle[:, ny // 2, :]
        positions = _device_tensor(markers.x_gamma_m)[: int(marker_count)]

        def host(t, dtype):
            return np.asarray(t.detach().cpu().numpy(), dtype=dtype)

        path = snapshot_dir / f"snapshot_{int(step):06d}.npz"
        np.savez_compressed(
            path,
            step=np.int64(step),
            time_s=np.float64(time_s),
            pressure_pa=np.float64(pressure_pa),
            speed_xz=host(speed_xz, np.float32),
            speed_yz=host(speed_yz, np.float32),
            obstacle_xz=host(obstacle_xz, np.int8),
            marker_positions_m=host(positions, np.float32),
            cell_center_x_m=np.asarray(fluid.cell_center_x_m.to_numpy(), dtype=np.float32),
            cell_center_y_m=np.asarray(fluid.cell_center_y_m.to_numpy(), dtype=np.float32),
            cell_center_z_m=np.asarray(fluid.cell_center_z_m.to_numpy(), dtype=np.float32),
        )
        return path
    except Exception as exc:  # noqa: BLE001 - a snapshot must not end a long run
        print(f"[snapshot] step {step} failed: {exc}", flush=True)
        return None
