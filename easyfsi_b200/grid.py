"""Graded Cartesian grid metrics and the fluid domain spec (host side, f64).

Same dataclasses and results as the reference's grid layer
(simulation_core/fluid.py:20-647 of lizhuoh9/EasyFsi): ``CartesianGrid``
(per-axis cell widths; faces, centres and centre distances derived by running
sums), ``RefinementRegion`` / ``GradedGridSpec`` / ``build_graded_grid``
(geometric grading between refined boxes and the far field), and
``FluidDomainSpec``.  The metric arrays built here are what the CUDA path and
the oracle both consume, so they follow the reference's arithmetic order
(accumulated faces, centre = face + w/2, distance[0] = w[0]).  Fixtures
generated from the reference's own builder pin them (tests/golden).
"""

from __future__ import annotations

from dataclasses import dataclass

_GROWTH_SLACK = 1.0 + 1.0e-10


def _as_float3(values, name: str) -> tuple[float, float, float]:
    out = tuple(float(v) for v in values)
    if len(out) != 3:
        raise ValueError(f"{name} must have three coordinates")
    return out  # type: ignore[return-value]


@dataclass(frozen=True)
class CartesianGrid:
    """Non-uniform tensor-product grid given by its per-axis cell widths (fluid.py:20-182)."""

    bounds_min_m: tuple[float, float, float]
    cell_widths_x_m: tuple[float, ...]
    cell_widths_y_m: tuple[float, ...]
    cell_widths_z_m: tuple[float, ...]

    def __post_init__(self) -> None:
        lo = tuple(float(v) for v in self.bounds_min_m)
        if len(lo) != 3:
            raise ValueError("bounds_min_m must have three coordinates")
        axes = [tuple(float(v) for v in w) for w in (self.cell_widths_x_m, self.cell_widths_y_m, self.cell_widths_z_m)]
        if any(len(a) == 0 for a in axes):
            raise ValueError("CartesianGrid axes must contain at least one cell")
        if any(w <= 0.0 for a in axes for w in a):
            raise ValueError("CartesianGrid cell widths must be positive")
        object.__setattr__(self, "bounds_min_m", lo)
        object.__setattr__(self, "cell_widths_x_m", axes[0])
        object.__setattr__(self, "cell_widths_y_m", axes[1])
        object.__setattr__(self, "cell_widths_z_m", axes[2])

    @classmethod
    def uniform(cls, *, bounds_min_m, bounds_max_m, grid_nodes) -> "CartesianGrid":
        if any(int(n) <= 0 for n in grid_nodes):
            raise ValueError("grid_nodes must be positive in every dimension")
        per_axis = []
        for lo, hi, n in zip(bounds_min_m, bounds_max_m, grid_nodes, strict=True):
            per_axis.append((float((hi - lo) / n),) * int(n))
        return cls(
            bounds_min_m=tuple(float(v) for v in bounds_min_m),
            cell_widths_x_m=per_axis[0],
            cell_widths_y_m=per_axis[1],
            cell_widths_z_m=per_axis[2],
        )

    # -- per-axis derived metrics (running sums in f64, reference order) --
    @staticmethod
    def _axis_faces(origin: float, widths) -> tuple[float, ...]:
        faces = [float(origin)]
        for w in widths:
            faces.append(faces[-1] + w)
        return tuple(faces)

    @staticmethod
    def _axis_centers(origin: float, widths) -> tuple[float, ...]:
        out = []
        face = float(origin)
        for w in widths:
            out.append(face + 0.5 * w)
            face += w
        return tuple(out)

    @staticmethod
    def _axis_center_distances(centers, widths) -> tuple[float, ...]:
        dist = [float(widths[0])]
        dist.extend(float(centers[n] - centers[n - 1]) for n in range(1, len(centers)))
        return tuple(dist)

    @staticmethod
    def _axis_is_uniform(widths) -> bool:
        first = widths[0]
        tol = max(abs(first), 1.0) * 1.0e-12
        return all(abs(w - first) <= tol for w in widths)

    @staticmethod
    def _axis_grid_coordinate(value: float, faces, centers) -> float:
        if value <= centers[0]:
            half = max(centers[0] - faces[0], 1.0e-18)
            return -0.5 * (centers[0] - value) / half
        if value >= centers[-1]:
            half = max(faces[-1] - centers[-1], 1.0e-18)
            return float(len(centers) - 1) + 0.5 * (value - centers[-1]) / half
        for n in range(len(centers) - 1):
            a, b = centers[n], centers[n + 1]
            if a <= value <= b:
                return float(n) + (value - a) / max(b - a, 1.0e-18)
        return 0.0

    @property
    def grid_nodes(self) -> tuple[int, int, int]:
        return (len(self.cell_widths_x_m), len(self.cell_widths_y_m), len(self.cell_widths_z_m))

    @property
    def bounds_max_m(self) -> tuple[float, float, float]:
        lo = self.bounds_min_m
        return (lo[0] + sum(self.cell_widths_x_m), lo[1] + sum(self.cell_widths_y_m), lo[2] + sum(self.cell_widths_z_m))

    def _widths(self, axis: int):
        return (self.cell_widths_x_m, self.cell_widths_y_m, self.cell_widths_z_m)[axis]

    def axis_faces(self, axis: int) -> tuple[float, ...]:
        return self._axis_faces(self.bounds_min_m[axis], self._widths(axis))

    def axis_centers(self, axis: int) -> tuple[float, ...]:
        return self._axis_centers(self.bounds_min_m[axis], self._widths(axis))

    def axis_center_distances(self, axis: int) -> tuple[float, ...]:
        return self._axis_center_distances(self.axis_centers(axis), self._widths(axis))

    cell_centers_x_m = property(lambda self: self.axis_centers(0))
    cell_centers_y_m = property(lambda self: self.axis_centers(1))
    cell_centers_z_m = property(lambda self: self.axis_centers(2))
    cell_faces_x_m = property(lambda self: self.axis_faces(0))
    cell_faces_y_m = property(lambda self: self.axis_faces(1))
    cell_faces_z_m = property(lambda self: self.axis_faces(2))
    center_distances_x_m = property(lambda self: self.axis_center_distances(0))
    center_distances_y_m = property(lambda self: self.axis_center_distances(1))
    center_distances_z_m = property(lambda self: self.axis_center_distances(2))

    @property
    def is_uniform(self) -> bool:
        return all(self._axis_is_uniform(self._widths(a)) for a in range(3))

    @property
    def uniform_spacing_m(self) -> tuple[float, float, float]:
        if not self.is_uniform:
            raise ValueError("uniform_spacing_m is only available for a uniform CartesianGrid")
        return (self.cell_widths_x_m[0], self.cell_widths_y_m[0], self.cell_widths_z_m[0])

    def grid_coordinate_x(self, x_m: float) -> float:
        return self._axis_grid_coordinate(float(x_m), self.axis_faces(0), self.axis_centers(0))

    def grid_coordinate_y(self, y_m: float) -> float:
        return self._axis_grid_coordinate(float(y_m), self.axis_faces(1), self.axis_centers(1))

    def grid_coordinate_z(self, z_m: float) -> float:
        return self._axis_grid_coordinate(float(z_m), self.axis_faces(2), self.axis_centers(2))


@dataclass(frozen=True)
class RefinementRegion:
    """Box refined to ``target_spacing_m`` (fluid.py:185-209)."""

    bounds_min_m: tuple[float, float, float]
    bounds_max_m: tuple[float, float, float]
    target_spacing_m: float | tuple[float, float, float]

    def __post_init__(self) -> None:
        lo = tuple(float(v) for v in self.bounds_min_m)
        hi = tuple(float(v) for v in self.bounds_max_m)
        if len(lo) != 3 or len(hi) != 3:
            raise ValueError("RefinementRegion bounds must have three coordinates")
        if any(b <= a for a, b in zip(lo, hi, strict=True)):
            raise ValueError("RefinementRegion bounds_max_m must be greater than bounds_min_m")
        sp = self.target_spacing_m
        if isinstance(sp, tuple):
            target = tuple(float(v) for v in sp)
            if len(target) != 3:
                raise ValueError("target_spacing_m tuple must have three values")
        else:
            target = (float(sp),) * 3
        if any(v <= 0.0 for v in target):
            raise ValueError("target_spacing_m must be positive")
        object.__setattr__(self, "bounds_min_m", lo)
        object.__setattr__(self, "bounds_max_m", hi)
        object.__setattr__(self, "target_spacing_m", target)


@dataclass(frozen=True)
class GradedGridSpec:
    """Far-field spacing, growth limit and refinement boxes (fluid.py:212-246)."""

    bounds_min_m: tuple[float, float, float]
    bounds_max_m: tuple[float, float, float]
    farfield_spacing_m: float | tuple[float, float, float]
    max_growth_ratio: float
    refinement_regions: tuple[RefinementRegion, ...] = ()
    max_cells: int | None = None

    def __post_init__(self) -> None:
        lo = tuple(float(v) for v in self.bounds_min_m)
        hi = tuple(float(v) for v in self.bounds_max_m)
        if len(lo) != 3 or len(hi) != 3:
            raise ValueError("GradedGridSpec bounds must have three coordinates")
        if any(b <= a for a, b in zip(lo, hi, strict=True)):
            raise ValueError("bounds_max_m must be greater than bounds_min_m")
        sp = self.farfield_spacing_m
        if isinstance(sp, tuple):
            far = tuple(float(v) for v in sp)
            if len(far) != 3:
                raise ValueError("farfield_spacing_m tuple must have three values")
        else:
            far = (float(sp),) * 3
        if any(v <= 0.0 for v in far):
            raise ValueError("farfield_spacing_m must be positive")
        if self.max_growth_ratio <= 1.0:
            raise ValueError("max_growth_ratio must be greater than 1")
        cap = None if self.max_cells is None else int(self.max_cells)
        if cap is not None and cap <= 0:
            raise ValueError("max_cells must be positive when provided")
        object.__setattr__(self, "bounds_min_m", lo)
        object.__setattr__(self, "bounds_max_m", hi)
        object.__setattr__(self, "farfield_spacing_m", far)
        object.__setattr__(self, "refinement_regions", tuple(self.refinement_regions))
        object.__setattr__(self, "max_cells", cap)


# ---------------------------------------------------------------------------
# One-axis grading (fluid.py:249-536).  Widths between two anchors are the
# smallest number of cells whose per-cell bounds (geometric decay from / growth
# to the anchors, capped by the far-field spacing) can cover the distance; the
# cells are then interpolated between those bounds.
# ---------------------------------------------------------------------------


def _uniform_interior_faces(left: float, right: float, spacing: float) -> list[float]:
    length = right - left
    if length <= 0.0:
        return []
    n = max(1, int(round(length / spacing)))
    while length / n > spacing * _GROWTH_SLACK:
        n += 1
    step = length / n
    return [left + step * m for m in range(1, n)]


def _growth_ok(widths, ratio: float, left=None, right=None) -> bool:
    seq = ([] if left is None else [float(left)]) + [float(w) for w in widths] + ([] if right is None else [float(right)])
    for a, b in zip(seq, seq[1:]):
        if a <= 0.0 or b <= 0.0:
            return False
        if max(a / b, b / a) > float(ratio) * _GROWTH_SLACK:
            return False
    return True


def _interpolate_between(distance: float, lower: list[float], upper: list[float]) -> tuple[float, ...]:
    lo_sum, hi_sum = sum(lower), sum(upper)
    if hi_sum <= lo_sum:
        return tuple(lower)
    t = (float(distance) - lo_sum) / (hi_sum - lo_sum)
    return tuple(a + t * (b - a) for a, b in zip(lower, upper, strict=True))


def _cell_budget(distance: float, *anchors: float) -> int:
    smallest = max(min(anchors), 1.0e-12)
    return max(64, int(distance / smallest) * 8 + 64)


def _fits(distance: float, lower: list[float], upper: list[float]) -> bool:
    return not (distance < sum(lower) * (1.0 - 1.0e-10) or distance > sum(upper) * _GROWTH_SLACK)


def _side_widths(distance: float, inner: float, farfield: float, ratio: float) -> tuple[float, ...]:
    """Cells from a refined edge (width ``inner``) out to a domain wall (fluid.py:260-303)."""
    if distance <= 0.0:
        return ()
    g = float(ratio)
    for n in range(1, _cell_budget(distance, inner, farfield) + 1):
        lower, upper = [], []
        for m in range(1, n + 1):
            lo = float(inner) / (g**m)
            hi = min(float(farfield), float(inner) * (g**m))
            if lo > hi * _GROWTH_SLACK:
                break
            lower.append(lo)
            upper.append(hi)
        if len(lower) != n or not _fits(distance, lower, upper):
            continue
        widths = _interpolate_between(distance, lower, upper)
        if _growth_ok(widths, ratio, left=inner):
            return widths
    raise ValueError("could not build graded side satisfying max_growth_ratio")


def _bridge_widths(distance: float, left: float, right: float, farfield: float, ratio: float) -> tuple[float, ...]:
    """Cells between two refined segments (fluid.py:337-402)."""
    if distance <= 0.0:
        return ()
    g = float(ratio)
    far = float(farfield)
    for n in range(1, _cell_budget(distance, left, right, farfield) + 1):

        def grown(start: float) -> list[float]:
            out, v = [], float(start)
            for _ in range(n):
                v = min(far, v * g)
                out.append(v)
            return out

        from_left, from_right = grown(left), grown(right)
        lower, upper = [], []
        ok = True
        for m in range(n):
            lo = max(float(left) / (g ** (m + 1)), float(right) / (g ** (n - m)))
            hi = min(far, from_left[m], from_right[n - m - 1])
            if lo > hi * _GROWTH_SLACK:
                ok = False
                break
            lower.append(lo)
            upper.append(hi)
        if not ok or not _fits(distance, lower, upper):
            continue
        widths = _interpolate_between(distance, lower, upper)
        if _growth_ok(widths, ratio, left=left, right=right):
            return widths
    raise ValueError("could not build graded bridge satisfying max_growth_ratio")


@dataclass(frozen=True)
class _Segment:
    left: float
    right: float
    width: float
    cells: int


def _refined_segments(lo: float, hi: float, farfield: float, ratio: float, intervals, tol: float) -> list[_Segment]:
    """Clip, snap, sort and merge the refinement intervals of one axis (fluid.py:405-478)."""
    spans = []
    for a, b, target in intervals:
        left, right, t = max(lo, float(a)), min(hi, float(b)), float(target)
        if right <= lo or left >= hi or right <= left:
            continue
        snap = t / float(ratio)
        if left - lo < snap:
            left = lo
        if hi - right < snap:
            right = hi
        spans.append([left, right, t])
    if not spans:
        return []
    spans.sort(key=lambda s: (s[0], s[1]))
    merged: list[list[float]] = []
    for left, right, t in spans:
        if not merged:
            merged.append([left, right, t])
            continue
        prev = merged[-1]
        gap = left - prev[1]
        join = left <= prev[1] + max(tol, min(prev[2], t) / float(ratio))
        if not join and gap > 0.0:
            try:
                _bridge_widths(gap, prev[2], t, farfield, ratio)
            except ValueError:
                join = True
        if join:
            prev[1] = max(prev[1], right)
            prev[2] = min(prev[2], t)
        else:
            merged.append([left, right, t])
    out = []
    for left, right, t in merged:
        n = max(1, int(round((right - left) / t)))
        while (right - left) / n > t:
            n += 1
        out.append(_Segment(left, right, (right - left) / n, n))
    return out


def _graded_axis(lo: float, hi: float, farfield: float, ratio: float, intervals) -> tuple[float, ...]:
    """Cell widths of one axis (fluid.py:481-536)."""

    def uniform() -> tuple[float, ...]:
        faces = [lo, *_uniform_interior_faces(lo, hi, farfield), hi]
        return tuple(faces[n + 1] - faces[n] for n in range(len(faces) - 1))

    if not intervals:
        return uniform()
    tol = max(abs(hi - lo), 1.0) * 1.0e-12
    segs = _refined_segments(lo, hi, farfield, ratio, intervals, tol)
    if not segs:
        return uniform()
    widths: list[float] = list(reversed(_side_widths(segs[0].left - lo, segs[0].width, farfield, ratio)))
    widths.extend([segs[0].width] * segs[0].cells)
    for prev, seg in zip(segs, segs[1:]):
        widths.extend(_bridge_widths(seg.left - prev.right, prev.width, seg.width, farfield, ratio))
        widths.extend([seg.width] * seg.cells)
    widths.extend(_side_widths(hi - segs[-1].right, segs[-1].width, farfield, ratio))
    return tuple(widths)


def build_graded_grid(spec: GradedGridSpec) -> CartesianGrid:
    """Graded grid of a spec (fluid.py:539-570)."""
    per_axis = [[], [], []]
    for region in spec.refinement_regions:
        for a in range(3):
            per_axis[a].append((region.bounds_min_m[a], region.bounds_max_m[a], region.target_spacing_m[a]))
    widths = [
        _graded_axis(spec.bounds_min_m[a], spec.bounds_max_m[a], spec.farfield_spacing_m[a], float(spec.max_growth_ratio), tuple(per_axis[a]))
        for a in range(3)
    ]
    count = len(widths[0]) * len(widths[1]) * len(widths[2])
    if spec.max_cells is not None and count > int(spec.max_cells):
        raise ValueError(f"graded grid cell count {count} exceeds max_cells {int(spec.max_cells)}")
    return CartesianGrid(
        bounds_min_m=spec.bounds_min_m, cell_widths_x_m=widths[0], cell_widths_y_m=widths[1], cell_widths_z_m=widths[2]
    )


@dataclass(frozen=True)
class FluidDomainSpec:
    """Fluid box, material and grid (fluid.py:573-647)."""

    bounds_min_m: tuple[float, float, float]
    bounds_max_m: tuple[float, float, float]
    grid_nodes: tuple[int, int, int] | None
    density_kgm3: float
    viscosity_pa_s: float
    dt_s: float
    cartesian_grid: CartesianGrid | None = None
    graded_grid: GradedGridSpec | None = None

    @classmethod
    def unit_box(cls, grid_nodes=(32, 32, 32), density_kgm3=1000.0, viscosity_pa_s=1.0e-3, dt_s=1.0e-3):
        return cls(
            bounds_min_m=(0.0, 0.0, 0.0),
            bounds_max_m=(1.0, 1.0, 1.0),
            grid_nodes=grid_nodes,
            density_kgm3=density_kgm3,
            viscosity_pa_s=viscosity_pa_s,
            dt_s=dt_s,
        )

    def __post_init__(self) -> None:
        if any(b <= a for a, b in zip(self.bounds_min_m, self.bounds_max_m, strict=True)):
            raise ValueError("bounds_max_m must be greater than bounds_min_m")
        if self.density_kgm3 <= 0.0:
            raise ValueError("density_kgm3 must be positive")
        if self.viscosity_pa_s < 0.0:
            raise ValueError("viscosity_pa_s must be non-negative")
        if self.dt_s <= 0.0:
            raise ValueError("dt_s must be positive")
        if self.cartesian_grid is not None and self.graded_grid is not None:
            raise ValueError("cartesian_grid and graded_grid are mutually exclusive")
        if self.graded_grid is not None:
            grid = build_graded_grid(self.graded_grid)
        elif self.cartesian_grid is not None:
            grid = self.cartesian_grid
        else:
            if self.grid_nodes is None:
                raise ValueError("grid_nodes is required when no cartesian_grid or graded_grid is provided")
            grid = CartesianGrid.uniform(
                bounds_min_m=self.bounds_min_m, bounds_max_m=self.bounds_max_m, grid_nodes=self.grid_nodes
            )
        nodes = grid.grid_nodes if self.grid_nodes is None else tuple(int(n) for n in self.grid_nodes)
        if any(n < 4 for n in nodes):
            raise ValueError("grid_nodes must be at least 4 in every dimension")
        if grid.grid_nodes != nodes:
            raise ValueError("cartesian_grid grid_nodes must match FluidDomainSpec.grid_nodes")
        for got, want in zip(grid.bounds_min_m, self.bounds_min_m, strict=True):
            if abs(got - want) > max(abs(want), 1.0) * 1.0e-12:
                raise ValueError("cartesian_grid bounds_min_m must match FluidDomainSpec.bounds_min_m")
        for got, want in zip(grid.bounds_max_m, self.bounds_max_m, strict=True):
            if abs(got - want) > max(abs(want), 1.0) * 1.0e-12:
                raise ValueError("cartesian_grid bounds_max_m must match FluidDomainSpec.bounds_max_m")
        object.__setattr__(self, "grid_nodes", nodes)
        object.__setattr__(self, "cartesian_grid", grid)

    @property
    def spacing_m(self) -> tuple[float, float, float]:
        return self.cartesian_grid.uniform_spacing_m

    @property
    def cell_volume_m3(self) -> float:
        dx, dy, dz = self.spacing_m
        return dx * dy * dz


# ---------------------------------------------------------------------------
# Multigrid hierarchy (fluid.py:692-729): halve each axis (ceil) while every
# axis has more than 3 cells; coarse widths are pairwise sums.
# ---------------------------------------------------------------------------


def multigrid_shapes(shape) -> tuple[tuple[int, int, int], ...]:
    shapes = [tuple(int(n) for n in shape)]
    cur = shapes[0]
    while min(cur) > 3:
        nxt = tuple(max(2, (n + 1) // 2) for n in cur)
        if nxt == cur:
            break
        shapes.append(nxt)
        cur = nxt
    return tuple(shapes)


def coarsen_axis_widths(widths) -> tuple[float, ...]:
    return tuple(sum(widths[n : min(n + 2, len(widths))]) for n in range(0, len(widths), 2))


def multigrid_axis_widths(grid: CartesianGrid, shapes) -> tuple[tuple[tuple[float, ...], ...], ...]:
    levels = []
    cur = (grid.cell_widths_x_m, grid.cell_widths_y_m, grid.cell_widths_z_m)
    for shape in shapes:
        if tuple(len(a) for a in cur) != tuple(shape):
            raise ValueError("multigrid axis widths do not match multigrid shapes")
        levels.append(cur)
        cur = tuple(coarsen_axis_widths(a) for a in cur)
    return tuple(levels)
