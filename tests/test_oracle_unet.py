"""Pins the CPU restatement of the learned preconditioner's U-Net
(oracle/oracle_unet.py) by central finite differences in float64: the
analytic parameter gradient of the masked mean-square loss against
(L(p + h e_i) - L(p - h e_i)) / 2h for parameters of every layer, on a small
odd-sized volume that exercises the ceil pooling at every level."""

import numpy as np

from oracle import oracle_unet as ou


def test_unet_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    shape = (5, 4, 6)
    offs, total = ou.param_layout()
    params = np.zeros(total)
    for (w, b), (_, cin, cout, _) in zip(offs, ou.LAYERS):
        params[w : w + cout * 27 * cin] = rng.normal(0.0, np.sqrt(2.0 / (27 * cin)), cout * 27 * cin)
        params[b : b + cout] = 0.05 * rng.normal(size=cout)
    x = rng.normal(size=shape + (16,))
    target = rng.normal(size=shape)
    mask = (rng.random(shape) < 0.8).astype(np.float64)
    loss, grad = ou.loss_and_grad(params, x, target, mask, rounding=False)
    assert np.isfinite(loss) and loss > 0.0
    h = 1e-6
    for (w, b), _ in zip(offs, ou.LAYERS):
        for idx in (w + int(rng.integers(0, b - w)), b):
            p1, p2 = params.copy(), params.copy()
            p1[idx] += h
            p2[idx] -= h
            l1, _ = ou.loss_and_grad(p1, x, target, mask, rounding=False)
            l2, _ = ou.loss_and_grad(p2, x, target, mask, rounding=False)
            fd = (l1 - l2) / (2 * h)
            assert abs(fd - grad[idx]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (idx, fd, grad[idx])


def test_bf16_rounding_is_round_to_nearest_even():
    vals = np.array([1.0, 1.0 + 2.0**-8, 1.0 + 3 * 2.0**-9, -2.5, 3.14159265], np.float64)
    got = ou.bf16(vals)
    assert got[0] == 1.0
    assert got[1] == 1.0  # halfway to the next BF16 value: ties to even
    assert got[2] == 1.0 + 2.0**-7
    assert got[3] == -2.5
    assert abs(got[4] - 3.140625) < 1e-12
