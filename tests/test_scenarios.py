"""Seeded synthetic workloads (host side, no GPU)."""

import numpy as np

from easyfsi_b200.scenarios import BATCH_GRID_SIZES, batched_configs, particles


def test_batched_configs_are_seeded_and_uneven():
    """The c5 batch: 32 instances whose grid size, sphere radius and Young's
    modulus come from seed + i (the same list every call), spanning every
    grid size, radii in [0.08, 0.18] and moduli in [1e4, 1e6] Pa."""
    a, b = batched_configs(), batched_configs()
    assert a == b
    assert len(a) == 32
    sizes = {c.grid_nodes for c in a}
    assert sizes == {(n, n, n) for n in BATCH_GRID_SIZES}
    for c in a:
        assert not c.graded and c.mpm_nodes == c.grid_nodes
        (body,) = c.bodies
        r = body.semi_axes[0]
        assert body.semi_axes == (r, r, r) and 0.08 <= r <= 0.18
        assert 1.0e4 <= body.youngs_modulus_pa <= 1.0e6
        assert c.dt_s == 1.0e-4
    assert len({c.velocity_seed for c in a}) == 32 and len({c.particle_seed for c in a}) == 32
    # instance 0 alone, with a different size list, keeps its seeded draws
    (one,) = batched_configs(1, sizes=(32,))
    assert one.grid_nodes == (32, 32, 32)


def test_batched_instances_hold_uneven_particle_counts():
    """8 particles per MPM cell inside each sphere: the smallest and largest
    instances differ by two orders of magnitude."""
    counts = [particles(c)["x"].shape[0] for c in batched_configs(8)]
    assert min(counts) > 1000
    assert max(counts) / min(counts) > 10.0
    for c, n in zip(batched_configs(8), counts):
        r, nn = c.bodies[0].semi_axes[0], c.grid_nodes[0]
        expected = 8.0 * (4.0 / 3.0) * np.pi * r**3 * nn**3
        assert abs(n - expected) / expected < 0.15
