"""Rank plumbing of bench.py (replicas only) on CPU with the gloo backend.

Every rank runs an independent replica; the only collective is the max of the
per-rank times, taken by all ranks in the same order.  The reference arm runs
on rank 0 alone.
"""

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    import torch.distributed as dist

    sys.path.insert(0, str(REPO))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        per_rank_ms = [120.0, 150.0][rank]
        max_ms = bench.max_over_ranks(per_rank_ms, world, "cpu")
        out.put((rank, max_ms, bench.replica_steps_per_s(world, 10, max_ms)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank_and_the_summed_throughput():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, max_ms, value in results:
        assert max_ms == pytest.approx(150.0)
        assert value == pytest.approx(2 * 10 / 0.150)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, str(REPO))
    import bench

    monkeypatch.setenv("RANK", "1")
    bench.run_reference_arm(None, None)  # returns before touching its arguments
    assert capsys.readouterr().out == ""
