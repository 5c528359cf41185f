"""Host-side logic of the IB node search (no GPU): the default sign tolerance
(hibm_mpm.py:5477-5492) and the argument checks (hibm_mpm.py:6069-6094) of
HibmMpmIbNodeSearch, called on a stand-in object with the fields they read."""

import math
from types import SimpleNamespace

import pytest

from easyfsi_b200.hibm_mpm import HibmMpmIbNodeSearch


def _box(nodes=(4, 4, 4), bmin=(0.0, 0.0, 0.0), bmax=(1.0, 1.0, 1.0), capacity=8):
    spacing = tuple((hi - lo) / n for lo, hi, n in zip(bmin, bmax, nodes))
    return SimpleNamespace(grid_nodes=nodes, bounds_min_m=bmin, bounds_max_m=bmax, spacing_m=spacing,
                           marker_capacity=capacity, _F32_EPSILON=HibmMpmIbNodeSearch._F32_EPSILON)


def _tolerance(box):
    return HibmMpmIbNodeSearch._default_sign_tolerance_m(box)


def _validate(box, markers, **kw):
    stub = SimpleNamespace(**vars(box), _default_sign_tolerance_m=lambda: _tolerance(box))
    return HibmMpmIbNodeSearch._validate_search_inputs(stub, markers, **kw)


def test_default_sign_tolerance_follows_the_spacing_and_the_f32_coordinate_scale():
    # unit box, 4 cells: 1e-6 * 0.25 wins over 2 eps * 1
    assert _tolerance(_box()) == pytest.approx(max(0.25e-6, 2.0 * 1.1920928955078125e-7))
    # far from the origin the f32 coordinate scale wins
    far = _box(bmin=(1000.0, 0.0, 0.0), bmax=(1001.0, 1.0, 1.0))
    assert _tolerance(far) == pytest.approx(2.0 * 1.1920928955078125e-7 * 1001.0)
    # fine grids keep the 1e-12 floor or the spacing term
    fine = _box(nodes=(10**6, 4, 4))
    assert _tolerance(fine) >= 1.0e-12


def test_validation_returns_the_three_scalars_and_the_default_tolerance():
    box = _box()
    mk = SimpleNamespace(marker_count=3)
    r, p, t = _validate(box, mk, search_radius_m=0.1, interior_probe_distance_m=0.05, sign_tolerance_m=None)
    assert (r, p) == (0.1, 0.05) and t == pytest.approx(_tolerance(box))
    assert _validate(box, mk, search_radius_m=0.1, interior_probe_distance_m=0.05, sign_tolerance_m=0.0)[2] == 0.0


@pytest.mark.parametrize("kw,msg", [
    ({"search_radius_m": 0.0}, "search_radius_m"),
    ({"search_radius_m": math.nan}, "search_radius_m"),
    ({"interior_probe_distance_m": math.inf}, "interior_probe_distance_m"),
    ({"interior_probe_distance_m": -0.1}, "interior_probe_distance_m"),
    ({"sign_tolerance_m": -1e-9}, "sign_tolerance_m"),
])
def test_validation_rejects_bad_scalars(kw, msg):
    args = {"search_radius_m": 0.1, "interior_probe_distance_m": 0.05, "sign_tolerance_m": None, **kw}
    with pytest.raises(ValueError, match=msg):
        _validate(_box(), SimpleNamespace(marker_count=1), **args)


def test_validation_rejects_more_markers_than_capacity():
    with pytest.raises(ValueError, match="marker_capacity"):
        _validate(_box(capacity=2), SimpleNamespace(marker_count=3), search_radius_m=0.1,
                  interior_probe_distance_m=0.05, sign_tolerance_m=None)
