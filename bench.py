"""Coupled-step throughput of the B200 path (and the CPU reference arm).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c2] [--impl b200|reference]

One step is one coupled FSI step of the graded 128 x 128 x 256 workload
(predict -> MG-PCG projection to relative residual 1e-8 -> marker tractions ->
force spreading -> neo-Hookean MPM substep -> surface feedback) on synthetic
seeded inputs already resident in HBM.  The JSON line carries:

* value: coupled steps/s over all ranks (independent replicas per GPU);
* e2e: the same through the public API with the fluid and particle state
  uploaded from pinned host memory before and downloaded after every step;
* roofline: the dominant kernel family's algorithmic bytes / CUDA-event time
  against the measured HBM copy bandwidth;
* cpu_baseline: the CPU oracle (restatement of the reference path) on the
  host cores, one coupled step of the same workload;
* clocks: SM clocks and throttle reasons sampled during the timed region.

``--impl reference`` times only the CPU oracle (the reference algorithm on the
host cores): the reference itself is Taichi-only and GPU-only.
"""

from __future__ import annotations

import argparse
import json
import os
import signal
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "steps/s; pressure solve ms to rel-res 1e-8, learned+mixed vs plain CG, 1×B200"
WORKING_SET_NOTE = "working set per step > L2 (fluid vectors 13 x 34 MB + MPM grid), no extra flush"


def _measured_peaks() -> dict:
    path = REPO / "MEASURED_PEAKS.json"
    if path.exists():
        try:
            return json.loads(path.read_text())
        except Exception:
            pass
    return {}


def _hbm_peak() -> tuple[float, str]:
    peaks = _measured_peaks()
    if "hbm_gbs" in peaks:
        return float(peaks["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.path = None

    def start(self) -> None:
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"),
                stderr=subprocess.DEVNULL,
            )
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.send_signal(signal.SIGTERM)
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {
            "sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": float(max(smax)) if smax else None,
            "samples": len(sm),
            "reasons": sorted(reasons),
        }


def ib_node_search_stats(scene, reps: int) -> dict:
    """The IB node search (HibmMpmIbNodeSearch.search_and_classify_grid_fields)
    over the scene's fluid cell centres against its markers (the scene has no
    projection triangles, so the markers are the candidates), radius two of
    the finest cells, far nodes classified.  CUDA events around `reps` calls;
    each call includes its two small host reads (bin entry total, report).
    `pairs_per_s` counts the node-marker pairs the reference's all-pairs loop
    would evaluate for the same result."""
    import torch

    from easyfsi_b200.hibm_mpm import HibmMpmIbNodeSearch

    fl, mk = scene.fluid, scene.markers
    g = fl.grid
    search = HibmMpmIbNodeSearch(grid_nodes=g.grid_nodes, bounds_min_m=g.bounds_min_m, bounds_max_m=g.bounds_max_m,
                                 marker_capacity=mk.marker_capacity)
    radius = 2.0 * min(min(g._widths(a)) for a in range(3))
    kwargs = dict(cell_center_x_m=fl.cell_center_x_m, cell_center_y_m=fl.cell_center_y_m,
                  cell_center_z_m=fl.cell_center_z_m, search_radius_m=radius, interior_probe_distance_m=radius,
                  classify_far_internal_nodes=True)
    rep = search.search_and_classify_grid_fields(mk, **kwargs)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        rep = search.search_and_classify_grid_fields(mk, **kwargs)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    nodes = int(np.prod(g.grid_nodes))
    return {
        "ms_per_call": ms,
        "nodes": nodes,
        "markers": int(mk.marker_count),
        "search_radius_m": radius,
        "report": dict(rep.__dict__),
        "pairs_per_s": nodes * int(mk.marker_count) / (ms * 1e-3),
    }


def shell_step_stats(steps: int = 50, warmup: int = 3) -> dict:
    """The triangle Mooney membrane step (TriMooneyShellMpmState.step) on the
    c4 membrane: the 0.4 m x 0.3 m plate of 20,000 triangles (10,201
    vertices), t = 2 mm, C10 = 1e5 Pa, clamped root, its own 36^3 node grid,
    50 Pa pressure and gravity.  CUDA events around `steps` steps without the
    report read (the reference's read_report=False path); one more step reads
    the report."""
    import torch

    from easyfsi_b200 import _native
    from easyfsi_b200.geometry import make_plate_mesh
    from easyfsi_b200.mooney_shell_mpm import TriMooneyShellMpmState

    mesh, region = make_plate_mesh(100, 100)
    st = TriMooneyShellMpmState(mesh, thickness_m=2.0e-3, density_kgm3=1000.0, c1_pa=1.0e5, c2_pa=0.0,
                                face_region_id=region, primary_region_id=1, secondary_region_id=2,
                                fixed_region_id=3)
    kw = dict(dt_s=5.0e-5, pressure_pa=50.0, body_acceleration_mps2=(0.0, 0.0, -9.81), read_report=False)
    for _ in range(warmup):
        st.step(**kw)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    n0 = _native.kernel_launches()
    e0.record(stream)
    for _ in range(steps):
        st.step(**kw)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    launches = (_native.kernel_launches() - n0) / steps
    rep = st.step(**dict(kw, read_report=True))
    return {
        "workload": "c4_membrane_plate_20000_triangles",
        "faces": st.face_count,
        "vertices": st.particle_count,
        "grid_nodes": list(st.grid_nodes),
        "ms_per_step": ms,
        "steps_per_s": 1e3 / ms,
        "launches_per_step": launches,
        "mean_radial_stretch": rep.mean_radial_stretch,
        "transfer_relative_error": rep.transfer_relative_error,
    }


def pressure_solve_stats(scene, reps: int, jacobi_max_iterations: int = 20000) -> dict:
    """One c2 pressure solve to the scene's relative-residual tolerance (the
    Poisson system of a predicted, not yet projected velocity), timed with
    CUDA events per preconditioner: the reference's MG V-cycle, the FP32
    level-0 V-cycle, and Jacobi (plain diagonally preconditioned CG, with a
    larger iteration budget).  The first solve of each captures its graphs
    and is not timed.  The scene's velocity and pressure are restored."""
    import torch

    fl, cfg = scene.fluid, scene.cfg
    saved = (fl.velocity.tensor.clone(), fl.pressure.tensor.clone())
    stream = torch.cuda.current_stream()
    out = {}
    try:
        fl.predict(cfg.dt_s)
        fl.compute_divergence()
        for name, iters in (("fv_multigrid", cfg.cg_max_iterations), ("fv_multigrid_mixed", cfg.cg_max_iterations),
                            ("jacobi", jacobi_max_iterations)):
            times = []
            for r in range(reps + 1):
                fl.pressure.tensor.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fl._solve_pressure_poisson_fv_cg(iterations=iters, rhs_scale=cfg.density_kgm3 / cfg.dt_s,
                                                 pressure_outlet_zmin=False, tolerance=cfg.cg_tolerance,
                                                 preconditioner=name)
                e1.record(stream)
                torch.cuda.synchronize()
                if r > 0:
                    times.append(e0.elapsed_time(e1))
            out[name] = {
                "ms": float(np.median(times)),
                "iterations": int(fl.last_cg_iterations),
                "converged": bool(fl.last_cg_converged),
                "relative_residual": float(fl.last_cg_relative_residual),
            }
        base = out["jacobi"]["ms"]
        for name in ("fv_multigrid", "fv_multigrid_mixed"):
            out[name]["speedup_vs_jacobi"] = base / out[name]["ms"]
        out["tolerance"] = cfg.cg_tolerance
    finally:
        fl.velocity.tensor.copy_(saved[0])
        fl.pressure.tensor.copy_(saved[1])
    return out


PARTICLE_FAMILIES = ("p2g", "grid_update", "g2p", "scatter", "feedback", "mpm_step")


def family_timing(scene, steps: int, peak_gbs: float, world: int) -> dict:
    """Per-launch CUDA-event times of the MPM and HIBM kernel families over
    `steps` coupled steps (timing on, outside the headline's timed region),
    with each family's algorithmic bytes per launch and its fraction of the
    HBM peak."""
    import torch
    import torch.distributed as dist

    from easyfsi_b200 import _native

    for fam in PARTICLE_FAMILIES:
        _native.kernel_timing_enable(fam, True)
    try:
        for _ in range(max(1, steps)):
            scene.step()
        torch.cuda.synchronize()
        out = {}
        for fam in PARTICLE_FAMILIES:
            n, ms, nbytes = _native.kernel_timing_read(fam)
            if n == 0:
                continue
            gbs = nbytes / (ms * 1e-3) / 1e9 if ms > 0 else None
            out[fam] = {"launches": n, "avg_launch_us": 1000.0 * ms / n, "bytes_per_launch": nbytes / n,
                        "achieved_gbs": gbs, "frac": gbs / peak_gbs if gbs else None}
    finally:
        for fam in PARTICLE_FAMILIES:
            _native.kernel_timing_enable(fam, False)
    if world > 1:
        dist.barrier()
    return out


def learned_arm(scene, steps: int, warmup: int, world: int, plain_value: float, train_steps: int) -> dict:
    """The learned preconditioner on the same scene: a U-Net trained on
    (residual, error) pairs harvested from the scene's own MG-PCG solves
    (systems of two predicted velocities; truncated solves of 1..32
    iterations, minus the pre-smoothing), on 32^3 crops; then one pressure
    solve per preconditioner and `steps` coupled steps with
    cg_preconditioner="learned" (flexible PCG; two-level preconditioner: two
    damped-Jacobi sweeps, the network's correction at its energy-minimising
    scale, two sweeps; the 2/24/2 V-cycle taking over a 16-iteration block
    that does not halve the residual), next to the plain FP64 MG-PCG step.
    "learned_no_fallback" runs the two-level preconditioner alone for at most
    256 iterations.  The training is timed apart and is not part of a step."""
    import torch
    import torch.distributed as dist

    from easyfsi_b200.learned import UNetPreconditioner, harvest_pairs

    fl, cfg = scene.fluid, scene.cfg
    stream = torch.cuda.current_stream()
    net = UNetPreconditioner(seed=7)
    fl.set_learned_preconditioner(net)
    saved = (fl.velocity.tensor.clone(), fl.pressure.tensor.clone())
    t0 = time.perf_counter()
    pairs = []
    for _ in range(2):
        fl.predict(cfg.dt_s)
        fl.compute_divergence()
        pairs += harvest_pairs(fl, rhs_scale=cfg.density_kgm3 / cfg.dt_s)
    torch.cuda.synchronize()
    harvest_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    hist = net.train(pairs, steps=train_steps, batch=4, crop=32, lr=1e-3, seed=3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    del pairs
    # one pressure solve of the last predicted velocity's system
    solve = {}
    for name, iters in (("fv_multigrid", cfg.cg_max_iterations), ("learned", cfg.cg_max_iterations),
                        ("learned_no_fallback", 256)):
        times = []
        for r in range(3):
            fl.pressure.tensor.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fl._solve_pressure_poisson_fv_cg(iterations=iters, rhs_scale=cfg.density_kgm3 / cfg.dt_s,
                                             pressure_outlet_zmin=False, tolerance=cfg.cg_tolerance,
                                             preconditioner=name)
            e1.record(stream)
            torch.cuda.synchronize()
            if r > 0:
                times.append(e0.elapsed_time(e1))
        solve[name] = {"ms": float(np.median(times)), "iterations": int(fl.last_cg_iterations),
                       "converged": bool(fl.last_cg_converged),
                       "relative_residual": float(fl.last_cg_relative_residual),
                       "learned_iterations": int(fl.last_cg_learned_iterations),
                       "learned_relative_residual": float(fl.last_cg_learned_relative_residual)}
    fl.velocity.tensor.copy_(saved[0])
    fl.pressure.tensor.copy_(saved[1])
    # coupled steps with the learned preconditioner
    scene.preconditioner = "learned"
    for _ in range(max(1, warmup)):
        scene.step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    its, lits, res = [], [], []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        scene.step()
        its.append(scene.last_cg_iterations)
        lits.append(fl.last_cg_learned_iterations)
        res.append(fl.last_cg_relative_residual)
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    scene.preconditioner = "fv_multigrid"
    value = replica_steps_per_s(world, steps, max_over_ranks(e0.elapsed_time(e1), world, "cuda"))
    fl.set_learned_preconditioner(None)
    return {
        "value": value,
        "unit": "steps/s",
        "ratio_to_fv_multigrid": value / plain_value,
        "preconditioner": "two-level: 2 damped-Jacobi sweeps, U-Net correction (4 levels, 16/32/48/64 ch, BF16, "
                          "FP32 accumulation on tcgen05) at its energy-minimising scale, 2 sweeps; in the FP64 "
                          "flexible PCG; 2/24/2 V-cycle fallback",
        "cg_iterations_mean": float(np.mean(its)),
        "learned_iterations_mean": float(np.mean(lits)),
        "max_relative_residual": float(max(res)),
        "solve": solve,
        "parameters": net.param_count,
        "training": {"steps": train_steps, "batch": 4, "crop": 32, "harvest_s": harvest_s, "train_s": train_s,
                     "loss_first": float(np.mean(hist[:10])), "loss_last": float(np.mean(hist[-10:]))},
    }


def graph_step_arm(scene, steps: int, warmup: int, world: int, plain_value: float) -> dict:
    """The coupled step captured as one CUDA graph (efsi_step_graph_*): the
    pressure solve runs its device-side loop (a WHILE node of 16-iteration
    bodies that stops on the residual test), so the step makes no host reads;
    each timed step is one graph launch.  The statistics of the last step's
    solve are read after the timed region."""
    import torch
    import torch.distributed as dist

    from easyfsi_b200.runtime import StepGraph

    stream = torch.cuda.current_stream()
    fl = scene.fluid
    fl.device_loop_solves = True
    graph = StepGraph()
    try:
        scene.step()  # eager, with the device-side loop
        torch.cuda.synchronize()
        graph.capture(scene.step)
        torch.cuda.synchronize()
        for _ in range(max(1, warmup)):
            graph.launch()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            graph.launch()
        e1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        fl.read_device_pcg_stats()
        value = replica_steps_per_s(world, steps, max_over_ranks(e0.elapsed_time(e1), world, "cuda"))
        return {
            "value": value,
            "unit": "steps/s",
            "ratio_to_fv_multigrid": value / plain_value,
            "graph": "whole coupled step as one CUDA graph; PCG as a device-side WHILE loop of 16-iteration bodies",
            "last_cg_iterations": int(fl.last_cg_iterations),
            "last_cg_converged": bool(fl.last_cg_converged),
            "last_relative_residual": float(fl.last_cg_relative_residual),
        }
    finally:
        graph.close()
        fl.device_loop_solves = False


def batched_arm(steps: int, warmup: int, world: int, count: int, autotune: bool = True) -> dict:
    """The c5 batch: `count` independent coupled instances of uneven size
    (uniform 48^3 .. 128^3 grids, 2k-340k particles each).  Eager: every
    instance's step in turn on one stream (host reads at the PCG's 16-iteration
    checks).  Graph: all instances' steps captured as ONE CUDA graph with one
    branch per instance (runtime.BatchStepGraph; device-side PCG loops), one
    launch per batch step.  The unit is instance-steps/s (each instance
    advanced by one coupled step counts once)."""
    import torch
    import torch.distributed as dist

    from easyfsi_b200.runtime import BatchStepGraph
    from easyfsi_b200.scenarios import CoupledScene, batched_configs

    stream = torch.cuda.current_stream()
    t0 = time.perf_counter()
    cfgs = batched_configs(count)
    scenes = [CoupledScene(c) for c in cfgs]
    picks = [sc.fluid.autotune() for sc in scenes] if autotune else None
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    cells = int(sum(int(np.prod(c.grid_nodes)) for c in cfgs))
    parts = int(sum(sc.solid.particle_count for sc in scenes))

    def timed(run, k):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            run()
        e1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        return max_over_ranks(e0.elapsed_time(e1), world, "cuda")

    def eager():
        for sc in scenes:
            sc.step()

    for _ in range(max(1, warmup)):
        eager()
    eager_ms = timed(eager, steps)
    eager_iters = [int(sc.last_cg_iterations) for sc in scenes]
    graph = BatchStepGraph()
    try:
        for sc in scenes:
            sc.fluid.device_loop_solves = True
        eager()  # every instance once with its device-side loop
        torch.cuda.synchronize()
        graph.capture([sc.step for sc in scenes])
        for _ in range(max(1, warmup)):
            graph.launch()
        graph_ms = timed(graph.launch, steps)
        conv, g_iters = [], []
        for sc in scenes:
            sc.fluid.read_device_pcg_stats()
            conv.append(bool(sc.fluid.last_cg_converged))
            g_iters.append(int(sc.fluid.last_cg_iterations))
    finally:
        graph.close()
        for sc in scenes:
            sc.fluid.device_loop_solves = False
    n_inst = world * count
    eager_v = n_inst * steps / (eager_ms / 1000.0)
    graph_v = n_inst * steps / (graph_ms / 1000.0)
    out = {
        "workload": f"c5: {count} uniform instances of 48^3..128^3 cells (seed 5000+i), one sphere each",
        "instances": count,
        "cells": cells,
        "particles": parts,
        "unit": "instance-steps/s",
        "eager": {"value": eager_v, "ms_per_batch_step": eager_ms / steps},
        "graph": {"value": graph_v, "ms_per_batch_step": graph_ms / steps,
                  "launch": "one CUDA graph launch per batch step, one branch per instance"},
        "ratio_graph_to_eager": graph_v / eager_v,
        "all_converged": all(conv),
        "cg_iterations_eager": eager_iters,
        "cg_iterations_graph": g_iters,
        "setup_s": setup_s,
        "autotune_blocks_per_sm": [[p["blocks_per_sm"] for p in pk] for pk in picks] if picks else None,
    }
    del scenes
    torch.cuda.empty_cache()
    return out


def e2e_serial(state, results, host_in, scene, steps: int, world: int, barrier) -> tuple[float, list]:
    """Every step: the input state copied host -> device, the step, the
    results copied device -> host, all on the compute stream in order."""
    import torch

    stream = torch.cuda.current_stream()
    host_out = {key: torch.empty_like(get(), device="cpu").pin_memory() for key, get in results.items()}
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    iters = []
    for _ in range(steps):
        for key, get in state.items():
            get().copy_(host_in[key], non_blocking=True)
        scene.step()
        iters.append(scene.last_cg_iterations)
        for key, get in results.items():
            host_out[key].copy_(get(), non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    return max_over_ranks(e0.elapsed_time(e1), world, "cuda"), iters


def e2e_pipelined(state, results, host_in, scene, steps: int, world: int, barrier) -> tuple[float, list]:
    """Every step's inputs are copied host -> device and its results device
    -> host, as in e2e_serial, but on two copy streams: step k + 1's inputs
    travel into a device staging buffer while step k computes, and step k's
    results leave from a device snapshot while step k + 1 computes (two
    staging buffers each way, ordered by events).  On the compute stream each
    step starts with a device-to-device copy from its staging buffer into the
    solver state and ends with one into its result snapshot.  The timed region
    opens before the first upload and closes after the last download."""
    import torch

    stream = torch.cuda.current_stream()
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    stage_in = [{key: torch.empty_like(get()) for key, get in state.items()} for _ in range(2)]
    stage_out = [{key: torch.empty_like(get()) for key, get in results.items()} for _ in range(2)]
    host_out = [{key: torch.empty_like(get(), device="cpu").pin_memory() for key, get in results.items()}
                for _ in range(2)]
    in_ready = [torch.cuda.Event() for _ in range(2)]
    in_free = [torch.cuda.Event() for _ in range(2)]
    out_ready = [torch.cuda.Event() for _ in range(2)]
    out_free = [torch.cuda.Event() for _ in range(2)]

    def upload(b):
        with torch.cuda.stream(up):
            for key in state:
                stage_in[b][key].copy_(host_in[key], non_blocking=True)
            in_ready[b].record(up)

    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    up.wait_event(e0)
    down.wait_event(e0)
    upload(0)
    iters = []
    for k in range(steps):
        b = k & 1
        if k + 1 < steps:
            if k >= 1:
                up.wait_event(in_free[1 - b])  # step k - 1 has taken its inputs
            upload(1 - b)
        stream.wait_event(in_ready[b])
        for key, get in state.items():
            get().copy_(stage_in[b][key])
        in_free[b].record(stream)
        scene.step()
        iters.append(scene.last_cg_iterations)
        if k >= 2:
            stream.wait_event(out_free[b])  # step k - 2's results have left
        for key, get in results.items():
            stage_out[b][key].copy_(get())
        out_ready[b].record(stream)
        down.wait_event(out_ready[b])
        with torch.cuda.stream(down):
            for key in results:
                host_out[b][key].copy_(stage_out[b][key], non_blocking=True)
            out_free[b].record(down)
    stream.wait_stream(down)
    stream.wait_stream(up)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    return max_over_ranks(e0.elapsed_time(e1), world, "cuda"), iters


def max_over_ranks(ms: float, world: int, device) -> float:
    """Largest per-rank time over all ranks (every rank calls this in the same
    order; a no-op for one rank)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_steps_per_s(world: int, steps: int, max_ms: float) -> float:
    """Whole-job throughput of `world` independent replicas that each ran
    `steps` steps, timed by the slowest rank."""
    return world * steps / (max_ms / 1000.0)


def cpu_reference(cfg, steps: int, warmup: int, initial_velocity=None) -> dict:
    """Time the CPU oracle's coupled step (all host threads)."""
    from oracle import oracle as orc

    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    scene = orc.OracleScene(cfg, variant="mirror", initial_velocity=initial_velocity, project_initial=initial_velocity is None)
    for _ in range(warmup):
        scene.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        scene.step()
    dt = time.perf_counter() - t0
    return {
        "value": steps / dt,
        "unit": "steps/s",
        "cores": int(os.environ.get("OMP_NUM_THREADS", cores)),
        "kind": "port",
        "sample": f"{steps} coupled step(s) of {cfg.name} after {warmup} warm-up, CPU oracle (C++/OpenMP restatement of the reference)",
        "seconds": dt,
        "cg_iterations": int(scene.last_stats.iterations) if scene.last_stats is not None else None,
    }


def run_reference_arm(args, cfg) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    res = cpu_reference(cfg, args.steps, args.warmup)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": res["value"],
        "unit": "steps/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1000.0 / res["value"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": cfg.name, "grid": list(cfg.grid_nodes), "mpm_nodes": list(cfg.mpm_nodes)},
        "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": res["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference is Taichi-only (GPU-only); this arm times its CPU restatement",
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="c2")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the fv_multigrid_mixed measurement")
    ap.add_argument("--no-ib-search", action="store_true", help="skip the IB node search measurement")
    ap.add_argument("--no-shell", action="store_true", help="skip the Mooney membrane step measurement")
    ap.add_argument("--no-pressure-solve", action="store_true", help="skip the per-preconditioner solve timing")
    ap.add_argument("--cpu-steps", type=int, default=3, help="timed CPU-oracle steps of the GPU arm's cpu_baseline")
    ap.add_argument("--cpu-warmup", type=int, default=1)
    ap.add_argument("--no-family-timing", action="store_true", help="skip the MPM / HIBM kernel-family timing pass")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-preconditioner arm")
    ap.add_argument("--no-graph-step", action="store_true", help="skip the whole-step CUDA graph arm")
    ap.add_argument("--no-batched", action="store_true", help="skip the c5 batched-instances arm")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default V-cycle launch shapes")
    ap.add_argument("--no-overlap-solid", action="store_true",
                    help="run each step's solid part in order instead of beside the next step's fluid work")
    ap.add_argument("--batch-count", type=int, default=32, help="instances of the c5 batched arm")
    ap.add_argument("--learned-train-steps", type=int, default=200)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--replay-reps", type=int, default=50)
    args = ap.parse_args()
    from easyfsi_b200 import scenarios

    cfg = scenarios.CONFIGS[args.config]
    if args.impl == "reference":
        run_reference_arm(args, cfg)
        return

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from easyfsi_b200 import _native
    from easyfsi_b200.scenarios import CoupledScene

    scene = CoupledScene(cfg)
    stream = torch.cuda.current_stream()
    # the V-cycle's launch shapes come from the project's autotuner
    autotune = None if args.no_autotune else scene.fluid.autotune()

    def barrier():
        if world > 1:
            dist.barrier()

    # The clock sampler starts before the warm-up so that nvidia-smi's own
    # start-up does not fall inside the timed region.
    sampler = ClockSampler(local)
    sampler.start()
    # each step's solid part (marker forces, scatter, MPM substep, feedback)
    # runs beside the next step's fluid work (CoupledScene.overlap_solid)
    scene.overlap_solid = not args.no_overlap_solid
    for _ in range(max(args.warmup, 3)):
        scene.step()
    scene.finish()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches0 = _native.kernel_launches()
    iters = []
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        # an NVTX range per timed step lets a profiler select exactly these launches
        with torch.cuda.nvtx.range("coupled_step"):
            scene.step()
        iters.append(scene.last_cg_iterations)
    scene.finish()
    stop.record(stream)
    torch.cuda.synchronize()
    barrier()
    launches = _native.kernel_launches() - launches0
    clocks = sampler.stop()
    elapsed_ms = start.elapsed_time(stop)
    # Per-kernel roofline: every level-0 kernel family replayed back to back on
    # the scene's own buffers (CUDA events on the launching stream).
    iters_mean = float(np.mean(iters)) if iters else 0.0
    # (the CG dots are finished inside the V-cycle's last level-0 sweep, so
    # their stand-alone kernel is not on the path; the zero-guess sweep and
    # the whole update run on one iteration in 16, the other 15 form the
    # sweep in the update's r half and split the update across two streams)
    per_iteration = {"sweep0_l0": 1.0 / 16.0, "sweep_l0": 1, "sweep_prolong_l0": 1, "sweep_dots_l0": 1,
                     "spmv_dir": 1, "cg_update": 1.0 / 16.0, "restrict_l0": 1}
    fam_stats = {}
    for fam, per_it in per_iteration.items():
        avg_ms, nbytes = _native.kernel_replay(scene.fluid._plan, fam, reps=args.replay_reps)
        fam_stats[fam] = {
            "avg_launch_us": 1000.0 * avg_ms,
            "algorithmic_bytes_per_launch": nbytes,
            "achieved_gbs": nbytes / (avg_ms * 1e-3) / 1e9,
            "launches_per_step": per_it * iters_mean,
            "ms_per_step": avg_ms * per_it * iters_mean,
        }
    # the whole preconditioner (levels 0-6 of the V-cycle, dots included), time only
    vc_ms, _ = _native.kernel_replay(scene.fluid._plan, "vcycle", reps=max(1, args.replay_reps // 5))
    level0_us = sum(fam_stats[f]["avg_launch_us"] for f in ("sweep0_l0", "sweep_l0", "sweep_prolong_l0",
                                                            "sweep_dots_l0", "restrict_l0"))
    vcycle_stats = {"avg_us": 1000.0 * vc_ms, "level0_kernels_us": level0_us,
                    "coarse_levels_us": 1000.0 * vc_ms - level0_us, "per_step_ms": vc_ms * iters_mean}
    max_ms = max_over_ranks(elapsed_ms, world, "cuda")
    value = replica_steps_per_s(world, args.steps, max_ms)

    # --- the same coupled step with the mixed-precision preconditioner (FP32
    # level-0 V-cycle inside the FP64 flexible CG), continuing the scene ---
    mixed = None
    if not args.no_mixed:
        scene.preconditioner = "fv_multigrid_mixed"
        for _ in range(args.warmup):  # the first step captures its PCG graphs
            scene.step()
        torch.cuda.synchronize()
        barrier()
        m_iters, m_res = [], []
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        for _ in range(args.steps):
            scene.step()
            m_iters.append(scene.last_cg_iterations)
            m_res.append(scene.fluid.last_cg_relative_residual)
        scene.finish()
        m1.record(stream)
        torch.cuda.synchronize()
        barrier()
        m_value = replica_steps_per_s(world, args.steps, max_over_ranks(m0.elapsed_time(m1), world, "cuda"))
        mixed = {
            "value": m_value,
            "unit": "steps/s",
            "preconditioner": "fv_multigrid_mixed: FP32 level-0 V-cycle; CG, residual, dots and scalars FP64",
            "cg_iterations_mean": float(np.mean(m_iters)),
            "max_relative_residual": float(max(m_res)),
            "ratio_to_fv_multigrid": m_value / value,
        }
        scene.preconditioner = "fv_multigrid"
    scene.finish()
    scene.overlap_solid = False  # the remaining arms run each step in order on one stream

    # --- the same coupled step captured whole as one CUDA graph (device-side
    # PCG loop, no host reads), replayed once per step ---
    graph_step = None
    if not args.no_graph_step:
        try:
            graph_step = graph_step_arm(scene, args.steps, args.warmup, world, value)
        except Exception as exc:  # reported, never fatal to the step's line
            graph_step = {"error": f"{type(exc).__name__}: {exc}"}

    # --- the IB node search on the same grid and markers (not part of the step) ---
    ib_search = None
    if not args.no_ib_search:
        try:
            ib_search = ib_node_search_stats(scene, reps=5)
        except Exception as exc:  # reported, never fatal to the step's line
            ib_search = {"error": f"{type(exc).__name__}: {exc}"}

    # --- the Mooney membrane step on the c4 plate (its own solid; not part of the step) ---
    shell = None
    if not args.no_shell:
        try:
            shell = shell_step_stats()
        except Exception as exc:  # reported, never fatal to the step's line
            shell = {"error": f"{type(exc).__name__}: {exc}"}

    # --- one pressure solve per preconditioner (not part of the step) ---
    psolve = None
    if not args.no_pressure_solve:
        try:
            psolve = pressure_solve_stats(scene, reps=2)
        except Exception as exc:  # reported, never fatal to the step's line
            psolve = {"error": f"{type(exc).__name__}: {exc}"}

    # --- the learned preconditioner (trained here, then timed like the step) ---
    learned = None
    if not args.no_learned:
        try:
            learned = learned_arm(scene, args.steps, args.warmup, world, value, args.learned_train_steps)
        except Exception as exc:  # reported, never fatal to the step's line
            learned = {"error": f"{type(exc).__name__}: {exc}"}

    # --- e2e through the public API with host-resident state ---
    e2e = None
    if not args.no_e2e:
        fl, so, mk = scene.fluid, scene.solid, scene.markers
        n = so.particle_count
        # The full pre-step state (fluid, particles, markers) is uploaded every
        # step, so each e2e step repeats the same complete coupled step.
        state = {  # accessors: predict() exchanges the velocity buffers every step
            "velocity": lambda: fl.velocity.tensor,
            "pressure": lambda: fl.pressure.tensor,
            "x": lambda: so.x.tensor[:n],
            "v": lambda: so.v.tensor[:n],
            "C": lambda: so.C.tensor[:n],
            "F": lambda: so.F.tensor[:n],
            "normal": lambda: so.surface_normal.tensor[:n],
            "area": lambda: so.area_weight_m2.tensor[:n],
            "mx": lambda: mk.x_gamma_m.tensor,
            "mv": lambda: mk.v_gamma_mps.tensor,
            "mn": lambda: mk.n_gamma.tensor,
            "mA": lambda: mk.A_gamma_m2.tensor,
        }
        host_in = {key: get().cpu().pin_memory() for key, get in state.items()}
        results = {  # the step's results read back to the host every step
            "velocity": lambda: fl.velocity.tensor,
            "pressure": lambda: fl.pressure.tensor,
            "x": lambda: so.x.tensor[:n],
        }
        h2d = sum(t_.numel() * t_.element_size() for t_ in host_in.values())
        d2h = sum(get().numel() * get().element_size() for get in results.values())
        serial_ms, e2e_iters = e2e_serial(state, results, host_in, scene, args.steps, world, barrier)
        piped_ms, piped_iters = e2e_pipelined(state, results, host_in, scene, args.steps, world, barrier)
        e2e = {
            "value": replica_steps_per_s(world, args.steps, piped_ms),
            "unit": "steps/s",
            "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h),
            "cg_iterations_mean": float(np.mean(piped_iters)) if piped_iters else None,
            "copies": "every step: H2D of the step's full input state from pinned host memory and D2H of its "
                      "velocity, pressure and particle positions, on two copy streams overlapped with the "
                      "neighbouring steps' compute (double-buffered device staging, device-to-device copies "
                      "into and out of the solver state on the compute stream)",
            "serial": {"value": replica_steps_per_s(world, args.steps, serial_ms),
                       "copies": "the same copies on the compute stream, not overlapped"},
        }

    peak, peak_kind = _hbm_peak()
    # --- MPM and HIBM kernel families: CUDA events around each launch (on its
    # own stream) over `steps` further coupled steps ---
    particle_families = None
    if not args.no_family_timing:
        particle_families = family_timing(scene, args.steps, peak, world)
    # --- the c5 batch of uneven independent instances, eager and as one graph ---
    batched = None
    if not args.no_batched:
        try:
            batched = batched_arm(args.steps, args.warmup, world, args.batch_count, not args.no_autotune)
        except Exception as exc:  # reported, never fatal to the step's line
            batched = {"error": f"{type(exc).__name__}: {exc}"}
    dom = max(fam_stats, key=lambda f: fam_stats[f]["ms_per_step"])
    st = fam_stats[dom]
    traffic = None
    traffic_path = REPO / "profiles" / "dram_traffic.json"
    if traffic_path.exists():
        try:
            per_cell = json.loads(traffic_path.read_text()).get(dom, {}).get("dram_bytes_per_cell")
            if per_cell is not None:
                traffic = per_cell * scene.fluid.nx * scene.fluid.ny * scene.fluid.nz
        except Exception:
            traffic = None
    roofline = {
        "bound": "hbm",
        "kernel": dom,
        "achieved": st["achieved_gbs"],
        "peak": peak,
        "unit": "GB/s",
        "frac": st["achieved_gbs"] / peak,
        "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6.65 TB/s",
        "traffic": traffic,
        "avg_launch_us": st["avg_launch_us"],
        "algorithmic_bytes_per_launch": st["algorithmic_bytes_per_launch"],
        "timing": f"CUDA events around {args.replay_reps} back-to-back launches on the scene's level-0 buffers",
    }
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_reference(cfg, args.cpu_steps, args.cpu_warmup, initial_velocity=scene.fluid.velocity.to_numpy())
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "steps/s", "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {exc}"}
    if rank == 0:
        solve_ms, solve_iters = None, None
        if isinstance(psolve, dict) and "error" not in psolve:
            names = [k for k, v in psolve.items() if isinstance(v, dict) and "ms" in v]
            solve_ms = {k: round(psolve[k]["ms"], 4) for k in names}
            solve_iters = {k: psolve[k]["iterations"] for k in names}
        # the whole MG-PCG iteration against HBM: 267 algorithmic bytes per
        # cell (89 for the SpMV, update and direction, 178 for the V-cycle),
        # over the c2 solve's time per iteration (its once-per-solve setup
        # included)
        pcg_iteration = None
        if solve_ms and solve_iters and solve_iters.get("fv_multigrid"):
            cells = scene.fluid.nx * scene.fluid.ny * scene.fluid.nz
            us = 1000.0 * solve_ms["fv_multigrid"] / solve_iters["fv_multigrid"]
            gbs = 267.0 * cells / (us * 1e-6) / 1e9
            pcg_iteration = {"bytes_per_cell": 267, "cells": int(cells), "us": us, "achieved_gbs": gbs,
                             "frac": gbs / peak, "timing": "fv_multigrid solve ms / iterations"}
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": max(args.warmup, 3),
            "ms_per_step": max_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": {
                "workload": cfg.name,
                "grid": list(cfg.grid_nodes),
                "mpm_nodes": list(cfg.mpm_nodes),
                "particles": int(scene.solid.particle_count),
                "markers": int(scene.markers.marker_count),
                "dt_s": cfg.dt_s,
                "cg": "flexible MG-PCG (fv_multigrid 2/24/2), rel-res 1e-8",
                "parallelism": f"replicas x{world}",
                "solid_part": "in order" if args.no_overlap_solid else
                              "beside the next step's fluid work on a side stream (joined before its tractions)",
                "l2": WORKING_SET_NOTE,
            },
            "e2e": e2e,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "solve_ms": solve_ms,
            "pcg_iteration_roofline": pcg_iteration,
            "solve_iterations": solve_iters,
            "cg_iterations_mean": float(np.mean(iters)) if iters else None,
            "mixed_precision": mixed,
            "graph_step": graph_step,
            "batched": batched,
            "learned": learned,
            "particle_families": particle_families,
            "kernel_families": fam_stats,
            "autotune": autotune,
            "preconditioner": vcycle_stats,
            "pressure_solve": psolve,
            "ib_node_search": ib_search,
            "shell_step": shell,
            "cg_iterations": iters,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
