"""The learned preconditioner on the GPU: the tensor-core convolution and the
weight gradient against numpy, the U-Net's loss and parameter gradients
against the CPU oracle (oracle/oracle_unet.py, which rounds to BF16 where the
device does), and the trained network inside the flexible PCG against the
same PCG without it."""

import math
import time

import numpy as np
import pytest
import torch

from oracle import oracle_unet as ou

pytestmark = pytest.mark.gpu


def _bf16_tensor(a: np.ndarray) -> torch.Tensor:
    return torch.as_tensor(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16).cuda().contiguous()


def _rel(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("cin,cout,shape,relu", [(16, 16, (6, 5, 7), 0), (48, 32, (9, 4, 11), 1),
                                                 (112, 48, (5, 6, 9), 1), (32, 112, (7, 7, 7), 0)])
def test_tensor_core_conv3d_matches_numpy(cin, cout, shape, relu):
    """tcgen05 implicit-GEMM convolution (BF16 operands, FP32 accumulation)
    against float64 numpy on the same BF16 values; partial last tiles."""
    from easyfsi_b200 import _native

    rng = np.random.default_rng(cin + cout)
    x = ou.bf16(rng.normal(size=shape + (cin,)))
    w = ou.bf16(rng.normal(0.0, 1.0 / math.sqrt(27 * cin), size=(cout, 27, cin)))
    b = rng.normal(size=cout).astype(np.float32)
    xt, wt = _bf16_tensor(x), _bf16_tensor(w)
    bt = torch.as_tensor(b).cuda()
    yf = torch.zeros(shape + (cout,), dtype=torch.float32, device="cuda")
    yb = torch.zeros(shape + (cout,), dtype=torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _native.call("efsi_conv3d_bf16", *shape, cin, cout, xt.data_ptr(), wt.data_ptr(), bt.data_ptr(), relu,
                 yb.data_ptr(), yf.data_ptr(), err.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = ou.conv(x, w, b.astype(np.float64))
    if relu:
        ref = np.maximum(ref, 0.0)
    got = yf.cpu().numpy()
    assert _rel(got, ref) <= 1e-5
    np.testing.assert_array_equal(yb.cpu().to(torch.float32).numpy(), ou.bf16(got).astype(np.float32))


def test_weight_gradient_matches_numpy():
    from easyfsi_b200 import _native

    rng = np.random.default_rng(9)
    shape, cin, cout = (7, 6, 9), 48, 32
    x = ou.bf16(rng.normal(size=shape + (cin,)))
    g = ou.bf16(rng.normal(size=shape + (cout,)))
    dw = torch.zeros((cout, 27, cin), dtype=torch.float32, device="cuda")
    xt, gt = _bf16_tensor(x), _bf16_tensor(g)  # kept alive until the kernel has run
    _native.call("efsi_conv3d_wgrad", *shape, cin, cout, xt.data_ptr(), gt.data_ptr(), dw.data_ptr(),
                 torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert _rel(dw.cpu().numpy(), ou.conv_weight_grad(x, g)) <= 1e-5


def test_unet_loss_and_gradients_match_oracle():
    """Forward, masked mean-square loss and every layer's weight and bias
    gradient of the device U-Net against the oracle on an odd-sized volume
    (ceil pooling at every level).  Both round to BF16 at the same points;
    what remains is FP32 against float64 accumulation, which moves some BF16
    roundings by one unit."""
    from easyfsi_b200.learned import UNetPreconditioner

    net = UNetPreconditioner(seed=5)
    rng = np.random.default_rng(12)
    layout = net.layer_layout()
    params = np.zeros(net.param_count, np.float32)
    for L in layout:
        nw = L["cout"] * 27 * L["cin"]
        params[L["weight_offset"] : L["weight_offset"] + nw] = rng.normal(0.0, math.sqrt(2.0 / (27 * L["cin"])), nw)
        params[L["bias_offset"] : L["bias_offset"] + L["cout"]] = 0.05 * rng.normal(size=L["cout"])
    net.set_parameters(params)
    shape = (10, 7, 13)
    x = ou.bf16(rng.normal(size=shape + (16,)))
    target = rng.normal(size=shape)
    mask = (rng.random(shape) < 0.85).astype(np.float64)
    out_ref, _ = ou.forward(params.astype(np.float64), x)
    out = net.forward(_bf16_tensor(x)).cpu().numpy()
    assert _rel(out[..., 0], out_ref[..., 0]) <= 2e-2
    net.zero_grad()
    loss = net.accumulate_gradient(_bf16_tensor(x), torch.as_tensor(target, dtype=torch.float32).cuda(),
                                   torch.as_tensor(mask, dtype=torch.float32).cuda())
    grads = net.gradients()
    loss_ref, grad_ref = ou.loss_and_grad(params.astype(np.float64), x, target, mask)
    assert loss == pytest.approx(loss_ref, rel=1e-2)
    worst = 0.0
    for l, L in enumerate(layout):
        w0, b0 = L["weight_offset"], L["bias_offset"]
        nw = L["cout"] * 27 * L["cin"]
        ew = _rel(grads[w0 : w0 + nw], grad_ref[w0 : w0 + nw])
        eb = _rel(grads[b0 : b0 + L["cout"]], grad_ref[b0 : b0 + L["cout"]])
        worst = max(worst, ew, eb)
        assert ew <= 5e-2 and eb <= 5e-2, (l, ew, eb)
    print(f"unet: loss {loss:.6e} oracle {loss_ref:.6e}; worst layer gradient rel-L2 {worst:.3e}")


def _graded_solver(nodes, seed):
    from easyfsi_b200.fluid import CartesianFluidSolver, FluidDomainSpec
    from easyfsi_b200.grid import CartesianGrid
    from easyfsi_b200.scenarios import graded_axis_widths

    grid = CartesianGrid(bounds_min_m=(0.0, 0.0, 0.0),
                         cell_widths_x_m=graded_axis_widths(nodes[0], 0.0, 1.0, 0.3, 0.7),
                         cell_widths_y_m=graded_axis_widths(nodes[1], 0.0, 1.0, 0.3, 0.7),
                         cell_widths_z_m=graded_axis_widths(nodes[2], 0.0, 1.0, 0.2, 0.8))
    spec = FluidDomainSpec((0, 0, 0), grid.bounds_max_m, None, 1000.0, 1.0e-3, 1.0e-3, cartesian_grid=grid)
    fl = CartesianFluidSolver(spec)
    rng = np.random.default_rng(seed)
    obs = np.zeros(nodes, np.int32)
    nx, ny, nz = nodes
    obs[nx // 3 : nx // 3 + 4, ny // 2 - 2 : ny // 2 + 2, nz // 2 : nz // 2 + 5] = 1
    fl.obstacle.from_numpy(obs)
    return fl, rng


def _solve(fl, div, precond, iterations=2000):
    fl.divergence.from_numpy(div)
    fl.pressure.tensor.zero_()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fl._solve_pressure_poisson_fv_cg(iterations=iterations, rhs_scale=1.0e6, pressure_outlet_zmin=False,
                                     tolerance=1e-8, preconditioner=precond)
    torch.cuda.synchronize()
    return {"iterations": fl.last_cg_iterations, "converged": fl.last_cg_converged,
            "learned_iterations": getattr(fl, "last_cg_learned_iterations", 0),
            "residual": fl.last_cg_relative_residual, "ms": 1e3 * (time.perf_counter() - t0)}


def test_learned_preconditioner_trains_and_reduces_iterations():
    """Pairs harvested from the solver's own MG-PCG, training on crops, then a
    new right-hand side, solved to the relative residual 1e-8.  The trained
    two-level preconditioner alone (no fallback) takes fewer iterations than
    the same preconditioner with an untrained network (the sweeps alone, in
    effect) and than Jacobi-PCG, the method without it; with the V-cycle
    fallback it also converges.  The training loss falls."""
    from easyfsi_b200.learned import UNetPreconditioner, harvest_pairs

    nodes = (32, 32, 40)
    fl, rng = _graded_solver(nodes, seed=31)
    untrained = UNetPreconditioner(seed=2)
    net = UNetPreconditioner(seed=2)
    fl.set_learned_preconditioner(net)
    pairs = []
    for _ in range(3):
        fl.divergence.from_numpy(rng.normal(size=nodes).astype(np.float32))
        pairs += harvest_pairs(fl, rhs_scale=1.0e6)
    assert len(pairs) >= 12
    hist = net.train(pairs, steps=200, batch=4, crop=32, lr=1e-3, seed=4)
    first, last = float(np.mean(hist[:20])), float(np.mean(hist[-20:]))
    print(f"training loss {first:.4f} -> {last:.4f}")
    assert last < 0.7 * first

    div = rng.normal(size=nodes).astype(np.float32)
    res = {"jacobi": _solve(fl, div, "jacobi"), "fv_multigrid": _solve(fl, div, "fv_multigrid"),
           "trained": _solve(fl, div, "learned_no_fallback"), "learned": _solve(fl, div, "learned")}
    fl.set_learned_preconditioner(untrained)
    res["untrained"] = _solve(fl, div, "learned_no_fallback")
    fl.set_learned_preconditioner(net)
    print("solves to 1e-8:", res)
    for name, r in res.items():
        assert r["converged"] and r["residual"] <= 1e-8, name
    assert res["trained"]["iterations"] < res["untrained"]["iterations"]
    assert res["trained"]["iterations"] < res["jacobi"]["iterations"]
    assert res["trained"]["learned_iterations"] == res["trained"]["iterations"]
    assert res["learned"]["learned_iterations"] > 0
