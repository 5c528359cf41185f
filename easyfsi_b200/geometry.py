"""Latitude / longitude sphere tessellation used to place surface markers
(same vertex and face layout as simulation_core/geometry.py:76-122)."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class UvSphereResolution:
    latitude_bands: int
    longitude_segments: int


@dataclass(frozen=True)
class SurfaceMesh:
    vertices: np.ndarray
    faces: np.ndarray

    @property
    def vertex_count(self) -> int:
        return int(np.asarray(self.vertices).shape[0])

    @property
    def face_count(self) -> int:
        return int(self.faces.shape[0])


def make_uv_sphere(resolution: UvSphereResolution, radius_m: float) -> SurfaceMesh:
    if radius_m <= 0.0:
        raise ValueError("radius_m must be positive")
    lat, lon = int(resolution.latitude_bands), int(resolution.longitude_segments)
    verts = [(0.0, 0.0, radius_m)]
    for band in range(1, lat):
        theta = np.pi * band / lat
        for seg in range(lon):
            phi = 2.0 * np.pi * seg / lon
            verts.append((radius_m * np.sin(theta) * np.cos(phi), radius_m * np.sin(theta) * np.sin(phi), radius_m * np.cos(theta)))
    south = len(verts)
    verts.append((0.0, 0.0, -radius_m))

    def ring(r: int, s: int) -> int:
        return 1 + (r - 1) * lon + (s % lon)

    faces = [(0, ring(1, s), ring(1, s + 1)) for s in range(lon)]
    for r in range(1, lat - 1):
        for s in range(lon):
            a, b, c, d = ring(r, s), ring(r, s + 1), ring(r + 1, s + 1), ring(r + 1, s)
            faces.append((a, d, c))
            faces.append((a, c, b))
    faces.extend((south, ring(lat - 1, s + 1), ring(lat - 1, s)) for s in range(lon))
    v = np.asarray(verts, dtype=np.float64)
    f = np.asarray(faces, dtype=np.int64)
    # orient every face so that its normal points away from the centroid
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    normals = np.cross(b - a, c - a)
    centroid = v.mean(axis=0)
    flip = np.einsum("ij,ij->i", normals, (a + b + c) / 3.0 - centroid) < 0.0
    f[flip] = f[flip][:, [0, 2, 1]]
    return SurfaceMesh(v, f)


def make_plate_mesh(nu: int, nv: int, size_m: tuple[float, float] = (0.4, 0.3), seed: int = 4001):
    """Flat rectangular membrane of 2 nu nv triangles in the xy plane with a
    seeded 1 mm out-of-plane jitter, and its face regions: 1 for the half at
    x > size/2, 2 for the other half, 3 for the first column of quads (the
    root, to be clamped).  The c4 membrane is the 0.4 m x 0.3 m plate with
    nu = nv = 100 (20,000 triangles)."""
    xs = np.linspace(0.0, size_m[0], nu + 1)
    ys = np.linspace(0.0, size_m[1], nv + 1)
    gx, gy = np.meshgrid(xs, ys, indexing="ij")
    gz = 1.0e-3 * np.random.default_rng(seed).standard_normal(gx.shape)
    verts = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)
    idx = np.arange((nu + 1) * (nv + 1)).reshape(nu + 1, nv + 1)
    a, b, c, d = idx[:-1, :-1].ravel(), idx[1:, :-1].ravel(), idx[1:, 1:].ravel(), idx[:-1, 1:].ravel()
    faces = np.concatenate([np.stack([a, b, c], 1), np.stack([a, c, d], 1)]).astype(np.int32)
    cx = verts[faces, 0].mean(axis=1)
    region = np.where(cx > 0.5 * size_m[0], 1, 2).astype(np.int32)
    region[cx < size_m[0] / nu] = 3
    return SurfaceMesh(vertices=verts, faces=faces), region
