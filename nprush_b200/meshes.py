"""Procedural triangle meshes in the reference's vertex layout.

The reference loads its scenes from GLB files (src/lib/gpu/loadGlb.ts) into
MeshData: `vertices` of 12 floats per vertex [px py pz, nx ny nz, r g b a,
u v] and u32 `indices`, three per triangle.  Colour alpha is the path
tracer's material switch: below 0.5 a perfect mirror, else diffuse
(path_trace.wgsl:46, 248).  These builders make meshes in that layout for
synthetic scenes; `concat` joins meshes as
GpuPathTracePipelineManager.setMeshes does (GpuPathTracePipelineManager.ts:103-122).
Faces wind counter-clockwise seen from outside.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

VSTRIDE = 12


@dataclass
class MeshData:
    vertices: np.ndarray  # (V, 12) float32
    indices: np.ndarray   # (3T,) uint32

    @property
    def n_vertices(self) -> int:
        return self.vertices.shape[0]

    @property
    def n_tris(self) -> int:
        return self.indices.shape[0] // 3


def _vert(p, n, c, uv=(0.0, 0.0)):
    return [p[0], p[1], p[2], n[0], n[1], n[2], c[0], c[1], c[2], c[3], uv[0], uv[1]]


def _rgba(color):
    c = list(color)
    return c + [1.0] * (4 - len(c))


def quad(center, size, color=(0.8, 0.8, 0.8, 1.0), axis: int = 2) -> MeshData:
    """Square of side `size` facing +axis (default +z, the ground of a z-up scene)."""
    c = np.asarray(center, np.float64)
    u_ax, v_ax = [(1, 2), (2, 0), (0, 1)][axis]
    n = [0.0, 0.0, 0.0]
    n[axis] = 1.0
    col = _rgba(color)
    vs = []
    for su, sv, uv in ((-1, -1, (0, 0)), (1, -1, (1, 0)), (1, 1, (1, 1)), (-1, 1, (0, 1))):
        p = c.copy()
        p[u_ax] += su * size * 0.5
        p[v_ax] += sv * size * 0.5
        vs.append(_vert(p, n, col, uv))
    return MeshData(np.array(vs, np.float32), np.array([0, 1, 2, 0, 2, 3], np.uint32))


def box(center, half, color=(0.8, 0.8, 0.8, 1.0)) -> MeshData:
    """Axis-aligned box with flat-shaded faces (24 vertices, 12 triangles)."""
    c = np.asarray(center, np.float64)
    h = np.broadcast_to(np.asarray(half, np.float64), (3,))
    col = _rgba(color)
    vs, idx = [], []
    for axis in range(3):
        for sign in (-1.0, 1.0):
            n = [0.0, 0.0, 0.0]
            n[axis] = sign
            u_ax, v_ax = [(1, 2), (2, 0), (0, 1)][axis]
            base = len(vs)
            for su, sv in ((-1, -1), (1, -1), (1, 1), (-1, 1)):
                p = c.copy()
                p[axis] += sign * h[axis]
                p[u_ax] += su * h[u_ax]
                p[v_ax] += sv * h[v_ax]
                vs.append(_vert(p, n, col))
            quad_idx = [0, 1, 2, 0, 2, 3] if sign > 0 else [0, 2, 1, 0, 3, 2]
            idx += [base + k for k in quad_idx]
    return MeshData(np.array(vs, np.float32), np.array(idx, np.uint32))


def uv_sphere(center, radius, color=(0.8, 0.8, 0.8, 1.0), n_lat: int = 12, n_lon: int = 24) -> MeshData:
    """Latitude-longitude sphere with smooth normals (z is the pole axis)."""
    c = np.asarray(center, np.float64)
    col = _rgba(color)
    vs = []
    for i in range(n_lat + 1):
        th = math.pi * i / n_lat
        for j in range(n_lon + 1):
            ph = 2.0 * math.pi * j / n_lon
            n = (math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th))
            vs.append(_vert(c + radius * np.asarray(n), n, col, (j / n_lon, i / n_lat)))
    idx = []
    row = n_lon + 1
    for i in range(n_lat):
        for j in range(n_lon):
            a, b = i * row + j, i * row + j + 1
            cc, d = a + row, b + row
            if i > 0:
                idx += [a, cc, b]
            if i < n_lat - 1:
                idx += [b, cc, d]
    return MeshData(np.array(vs, np.float32), np.array(idx, np.uint32))


def concat(meshes) -> MeshData:
    """One vertex / index buffer for several meshes, indices offset by the
    vertices before them (GpuPathTracePipelineManager.ts:103-122)."""
    vs, ids, off = [], [], 0
    for m in meshes:
        vs.append(np.asarray(m.vertices, np.float32).reshape(-1, VSTRIDE))
        ids.append(np.asarray(m.indices, np.uint32).reshape(-1) + np.uint32(off))
        off += vs[-1].shape[0]
    if not vs:
        return MeshData(np.zeros((0, VSTRIDE), np.float32), np.zeros(0, np.uint32))
    return MeshData(np.concatenate(vs), np.concatenate(ids))


def demo_scene(n_objects: int = 6, seed: int = 0, mirror_fraction: float = 0.25, sphere_detail: int = 12):
    """A ground quad (z = 0) with `n_objects` random spheres and boxes on it,
    diffuse with random albedo or (a `mirror_fraction` of them) mirrors."""
    rng = np.random.default_rng(seed)
    parts = [quad((0.0, 0.0, 0.0), 8.0, (0.7, 0.7, 0.7, 1.0))]
    for k in range(n_objects):
        pos = rng.uniform(-2.0, 2.0, 2)
        size = float(rng.uniform(0.25, 0.6))
        alpha = 0.0 if rng.random() < mirror_fraction else 1.0
        col = tuple(rng.uniform(0.2, 0.9, 3)) + (alpha,)
        if k % 2 == 0:
            parts.append(uv_sphere((pos[0], pos[1], size), size, col, sphere_detail, 2 * sphere_detail))
        else:
            parts.append(box((pos[0], pos[1], size), size * rng.uniform(0.6, 1.0, 3), col))
    return concat(parts)


def sky_env(w: int = 64, h: int = 32) -> np.ndarray:
    """A smooth equirectangular sky (h, w, 4): bright towards +z, a band at the
    horizon, a small sun, darker below; v = 0 is the zenith
    (path_trace.wgsl:200-205)."""
    v = (np.arange(h) + 0.5) / h
    u = (np.arange(w) + 0.5) / w
    elev = (0.5 - v)[:, None] * math.pi + 0.0 * u[None, :]
    az = (u[None, :] - 0.5) * 2.0 * math.pi + 0.0 * v[:, None]
    up = np.clip(np.sin(elev), 0.0, 1.0)
    band = np.exp(-(elev / 0.2) ** 2)
    sun = np.exp(-((az - 0.8) ** 2 + (elev - 0.6) ** 2) / 0.02) * 6.0
    img = np.zeros((h, w, 4), np.float32)
    img[..., 0] = 0.3 + 0.5 * up + 0.6 * band + sun
    img[..., 1] = 0.35 + 0.6 * up + 0.4 * band + sun
    img[..., 2] = 0.45 + 0.9 * up + 0.2 * band + 0.9 * sun
    img[..., 3] = 1.0
    img[v > 0.5, :, :3] *= 0.3
    return img
