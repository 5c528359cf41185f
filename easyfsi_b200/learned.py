"""The learned preconditioner of the flexible PCG (no counterpart in the reference).

``UNetPreconditioner`` owns one device U-Net (``efsi_unet_*`` in
``csrc/efsi_unet.cu``: 4 levels, 16/32/48/64 channels, about 0.69 M
parameters, BF16 activations and weights with FP32 accumulation on the tensor
cores, FP32 master weights and Adam).  It is trained on (residual, error)
pairs that the solver's own multigrid-preconditioned CG produces, and is then
attached to a ``CartesianFluidSolver`` as ``cg_preconditioner="learned"``.

Inside the flexible PCG of the reference (fluid.py:6535-6811) the network is
the coarse correction of a two-level preconditioner: two damped-Jacobi sweeps
of the V-cycle's level-0 smoother from zero (z_pre), the network's estimate n
of the error that remains, added at the scale that minimises the energy norm
of the error (s = <r', n>_V / <n, A n>_V with r' = r - A z_pre), and two more
sweeps.  The sweeps remove the rough error the network leaves; the network
removes the smooth error the sweeps cannot.  The 2/24/2 V-cycle takes over
whenever a 16-iteration block does not halve the residual, and every solve
ends on the same true-residual test as the plain method.

Pairs (``harvest_pairs``): for a prepared right-hand side b, the multigrid
PCG is run to convergence (x*) and, from zero, truncated after k iterations
(x_k; k = 0 gives r = b, e = x*); r_k = b - A x_k and e_k = x* - x_k (both
with the closed-domain mean removed) satisfy A e_k = r_k.  The pre-smoothing
z_pre of r_k is subtracted as inside the PCG: the pair is (r_k - A z_pre,
e_k - z_pre).  The network input is the solver's own encoding of that
residual (``efsi_fv_learned_input``: r over its volume-weighted RMS, the
fluid mask, log2 cell widths); the target is the error over its RMS (the
energy-minimising scale makes the correction independent of the output's
scale).  Training takes random crops of the pairs.
"""

from __future__ import annotations

import ctypes
from ctypes import byref, c_double, c_void_p
from dataclasses import dataclass

import numpy as np
import torch

from . import _native

IN_CHANNELS = 16
OUT_CHANNELS = 16


def _stream() -> c_void_p:
    return c_void_p(torch.cuda.current_stream().cuda_stream)


@dataclass
class TrainingPair:
    """One (residual, error) pair on a solver's full grid."""

    input: torch.Tensor  # BF16 [nx, ny, nz, 16] (the PCG's input encoding of r)
    target: torch.Tensor  # FP32 [nx, ny, nz] (e over its RMS)
    mask: torch.Tensor  # FP32 [nx, ny, nz] (fluid cells)
    iterations: int  # k of the truncated solve


class UNetPreconditioner:
    """A device U-Net with its parameters, Adam state and workspace."""

    def __init__(self, seed: int = 0):
        handle = c_void_p()
        _native.call("efsi_unet_create", int(seed), byref(handle))
        self.handle = handle
        count = ctypes.c_int64(0)
        _native.call("efsi_unet_param_count", self.handle, byref(count))
        self.param_count = int(count.value)
        self.losses: list[float] = []

    def __del__(self):
        handle = getattr(self, "handle", None)
        if handle is not None and handle.value:
            try:
                _native.load().efsi_unet_destroy(handle)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self.handle = c_void_p()

    # -- parameters ---------------------------------------------------------
    def layer_layout(self) -> list[dict]:
        w = (ctypes.c_int64 * 15)()
        b = (ctypes.c_int64 * 15)()
        shp = (ctypes.c_int32 * 60)()
        _native.call("efsi_unet_layer_offsets", self.handle, w, b, shp)
        return [{"weight_offset": int(w[l]), "bias_offset": int(b[l]), "level": int(shp[4 * l]),
                 "cin": int(shp[4 * l + 1]), "cout": int(shp[4 * l + 2]), "relu": bool(shp[4 * l + 3])}
                for l in range(15)]

    def parameters(self) -> np.ndarray:
        out = np.zeros(self.param_count, np.float32)
        _native.call("efsi_unet_get_params", self.handle, out.ctypes.data_as(c_void_p), None)
        return out

    def gradients(self) -> np.ndarray:
        out = np.zeros(self.param_count, np.float32)
        _native.call("efsi_unet_get_params", self.handle, None, out.ctypes.data_as(c_void_p))
        return out

    def set_parameters(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, np.float32)
        if p.size != self.param_count:
            raise ValueError(f"expected {self.param_count} parameters, got {p.size}")
        _native.call("efsi_unet_set_params", self.handle, p.ctypes.data_as(c_void_p))

    # -- passes -------------------------------------------------------------
    @staticmethod
    def _check_input(x: torch.Tensor) -> tuple[int, int, int]:
        if x.dtype != torch.bfloat16 or x.dim() != 4 or x.shape[3] != IN_CHANNELS or not x.is_contiguous():
            raise ValueError("input must be a contiguous BF16 tensor of shape (nx, ny, nz, 16)")
        return int(x.shape[0]), int(x.shape[1]), int(x.shape[2])

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """FP32 output (nx, ny, nz, 16) of a BF16 input (nx, ny, nz, 16)."""
        nx, ny, nz = self._check_input(x)
        out = torch.empty((nx, ny, nz, OUT_CHANNELS), dtype=torch.float32, device=x.device)
        _native.call("efsi_unet_forward", self.handle, nx, ny, nz, c_void_p(x.data_ptr()),
                     c_void_p(out.data_ptr()), _stream())
        return out

    def accumulate_gradient(self, x: torch.Tensor, target: torch.Tensor, mask: torch.Tensor) -> float:
        """Forward, masked mean-square loss on output channel 0, backward;
        gradients are added to the accumulated ones.  Returns the loss."""
        nx, ny, nz = self._check_input(x)
        t = target.to(torch.float32).contiguous()
        m = mask.to(torch.float32).contiguous()
        loss = c_double(0.0)
        _native.call("efsi_unet_accumulate_gradient", self.handle, nx, ny, nz, c_void_p(x.data_ptr()),
                     c_void_p(t.data_ptr()), c_void_p(m.data_ptr()), byref(loss), _stream())
        return float(loss.value)

    def zero_grad(self) -> None:
        _native.call("efsi_unet_zero_grad", self.handle, _stream())

    def adam_step(self, lr: float = 1.0e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1.0e-8) -> None:
        _native.call("efsi_unet_adam_step", self.handle, float(lr), float(beta1), float(beta2), float(eps),
                     _stream())

    # -- training -----------------------------------------------------------
    def train(self, pairs: list[TrainingPair], *, steps: int, batch: int = 4, crop: int = 32, lr: float = 1.0e-3,
              seed: int = 0) -> list[float]:
        """Adam on random crops (edge ``crop``, clipped to the grid) of the
        pairs; returns the mean loss of every step."""
        if not pairs:
            raise ValueError("no training pairs")
        rng = np.random.default_rng(seed)
        history = []
        for _ in range(int(steps)):
            total = 0.0
            for _ in range(int(batch)):
                p = pairs[int(rng.integers(len(pairs)))]
                nx, ny, nz = p.target.shape
                cx, cy, cz = min(crop, nx), min(crop, ny), min(crop, nz)
                i0 = int(rng.integers(0, nx - cx + 1))
                j0 = int(rng.integers(0, ny - cy + 1))
                k0 = int(rng.integers(0, nz - cz + 1))
                sl = (slice(i0, i0 + cx), slice(j0, j0 + cy), slice(k0, k0 + cz))
                total += self.accumulate_gradient(p.input[sl].contiguous(), p.target[sl], p.mask[sl])
            self.adam_step(lr=lr)
            history.append(total / batch)
        self.losses.extend(history)
        return history


def harvest_pairs(solver, *, rhs_scale: float, truncations=(0, 1, 2, 4, 8, 16, 32), tolerance: float = 1.0e-10,
                  max_iterations: int = 400) -> list[TrainingPair]:
    """(residual, error) pairs from the solver's own MG-PCG on the system of
    its current divergence (closed domain, zero-mean pressure): for every
    truncated iterate x_k, the residual r_k = b - A x_k and error x* - x_k
    minus the learned preconditioner's pre-smoothing z_pre of r_k, i.e. the
    residual r_k - A z_pre and error x* - x_k - z_pre that its network
    corrects.  The network must already be attached (its input encoding uses
    the finest widths)."""
    fl = solver
    saved = fl.pressure.tensor.clone()
    try:
        fl.pressure.tensor.zero_()
        fl._solve_pressure_poisson_fv_cg(iterations=max_iterations, rhs_scale=rhs_scale, pressure_outlet_zmin=False,
                                         tolerance=tolerance, preconditioner="fv_multigrid")
        x_star = fl.pressure.tensor.clone()
        fluid = (fl.obstacle.tensor == 0)
        vol = fl._cell_volume_f32().to(torch.float64)
        fvol = float((vol * fluid).sum())

        def zero_mean(f: torch.Tensor) -> torch.Tensor:
            m = float((f * vol * fluid).sum()) / max(fvol, 1e-300)
            return torch.where(fluid, f - m, torch.zeros_like(f))

        # b: the positive rhs of the solve (fluid.py:6589-6601)
        b = zero_mean(torch.where(fluid, -fl._mg_rhs[0].tensor, torch.zeros_like(fl._mg_rhs[0].tensor)))
        pairs = []
        for k in truncations:
            fl.pressure.tensor.zero_()
            if int(k) > 0:  # k = 0: x_0 = 0, r = b, e = x*
                fl._solve_pressure_poisson_fv_cg(iterations=int(k), rhs_scale=rhs_scale, pressure_outlet_zmin=False,
                                                 tolerance=0.0, preconditioner="fv_multigrid")
            x_k = fl.pressure.tensor.clone()
            fl._fv_laplacian_apply_kernel(fl.pressure, fl.cg_Ad, 0)
            r_k = zero_mean(b - fl.cg_Ad.tensor).contiguous()
            # what the network sees inside the PCG: the residual and error left
            # after the pre-smoothing sweeps
            z_pre = torch.zeros_like(r_k)
            _native.call("efsi_fv_learned_presmooth", fl._plan, c_void_p(r_k.data_ptr()), c_void_p(z_pre.data_ptr()),
                         0, _stream())
            az = torch.zeros_like(r_k)
            _native.call("efsi_fv_apply", fl._plan, c_void_p(z_pre.data_ptr()), c_void_p(az.data_ptr()), 0, _stream())
            r = zero_mean(r_k - az)
            e = zero_mean(x_star - x_k - z_pre)
            rms_e = float(torch.sqrt((e * e * vol * fluid).sum() / max(fvol, 1e-300)))
            if not np.isfinite(rms_e) or rms_e <= 0.0:
                continue
            shape = tuple(fl.grid.grid_nodes)
            x_in = torch.empty(shape + (IN_CHANNELS,), dtype=torch.bfloat16, device=fl.device)
            _native.call("efsi_fv_learned_input", fl._plan, c_void_p(r.contiguous().data_ptr()),
                         c_void_p(x_in.data_ptr()), _stream())
            pairs.append(TrainingPair(input=x_in, target=(e / rms_e).to(torch.float32).contiguous(),
                                      mask=fluid.to(torch.float32).contiguous(), iterations=int(k)))
        return pairs
    finally:
        fl.pressure.tensor.copy_(saved)


def _demo(argv=None) -> None:
    """Train a network on one graded grid and compare solves:

        python -m easyfsi_b200.learned [--nodes 96 96 96] [--steps 200]

    prints one JSON line with the training loss, and ms / iterations to the
    relative residual 1e-8 of the MG-PCG, the Jacobi-PCG, the learned PCG
    with the V-cycle fallback and without it."""
    import argparse
    import json
    import time

    from .fluid import CartesianFluidSolver, FluidDomainSpec
    from .grid import CartesianGrid
    from .scenarios import graded_axis_widths

    ap = argparse.ArgumentParser()
    ap.add_argument("--nodes", type=int, nargs=3, default=(96, 96, 96))
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args(argv)
    nodes = tuple(args.nodes)
    grid = CartesianGrid(bounds_min_m=(0.0, 0.0, 0.0),
                         cell_widths_x_m=graded_axis_widths(nodes[0], 0.0, 1.0, 0.3, 0.7),
                         cell_widths_y_m=graded_axis_widths(nodes[1], 0.0, 1.0, 0.3, 0.7),
                         cell_widths_z_m=graded_axis_widths(nodes[2], 0.0, 1.0, 0.2, 0.8))
    fl = CartesianFluidSolver(FluidDomainSpec((0, 0, 0), grid.bounds_max_m, None, 1000.0, 1.0e-3, 1.0e-3,
                                              cartesian_grid=grid))
    rng = np.random.default_rng(args.seed)
    net = UNetPreconditioner(seed=args.seed)
    fl.set_learned_preconditioner(net)
    pairs = []
    for _ in range(2):
        fl.divergence.from_numpy(rng.normal(size=nodes).astype(np.float32))
        pairs += harvest_pairs(fl, rhs_scale=1.0e6)
    t0 = time.perf_counter()
    hist = net.train(pairs, steps=args.steps, batch=4, crop=32, lr=1.0e-3, seed=args.seed)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    fl.divergence.from_numpy(rng.normal(size=nodes).astype(np.float32))
    out = {"nodes": list(nodes), "parameters": net.param_count, "train_s": train_s,
           "loss_first": float(np.mean(hist[:10])), "loss_last": float(np.mean(hist[-10:]))}
    for name, iters in (("fv_multigrid", 400), ("jacobi", 4000), ("learned", 400), ("learned_no_fallback", 4000)):
        for rep in range(2):
            fl.pressure.tensor.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fl._solve_pressure_poisson_fv_cg(iterations=iters, rhs_scale=1.0e6, pressure_outlet_zmin=False,
                                             tolerance=1.0e-8, preconditioner=name)
            torch.cuda.synchronize()
            ms = 1e3 * (time.perf_counter() - t0)
        out[name] = {"ms": ms, "iterations": fl.last_cg_iterations, "converged": fl.last_cg_converged,
                     "relative_residual": fl.last_cg_relative_residual,
                     "learned_iterations": fl.last_cg_learned_iterations}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    _demo()
