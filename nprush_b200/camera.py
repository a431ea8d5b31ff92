"""Camera matrices, column-major, WebGPU clip conventions.

Mirrors the reference's camera (src/lib/viewer/Camera.svelte.ts:18-33):
proj = perspective(fov, aspect, zNear=0.01, zFar=100) with clip z in [0, 1],
viewProj = proj * view, viewProjInv = inverse(viewProj); matrices are uploaded
as 16 column-major floats (WGSL mat4x4f, m[c][r] = column c, row r).  The
reference takes these from wgpu-matrix 3.4.2 (npm, not vendored); they are
derived here from the standard formulas (right-handed view space, camera
looking down -z, clip.w = view depth).
"""
from __future__ import annotations

import math

import numpy as np

Z_NEAR = 0.01
Z_FAR = 100.0


def perspective(fovy: float, aspect: float, z_near: float = Z_NEAR, z_far: float = Z_FAR) -> np.ndarray:
    """4x4 (row-major numpy, M @ v) perspective with clip z in [0, 1]."""
    f = math.tan(math.pi * 0.5 - 0.5 * fovy)
    m = np.zeros((4, 4), np.float64)
    m[0, 0] = f / aspect
    m[1, 1] = f
    range_inv = 1.0 / (z_near - z_far)
    m[2, 2] = z_far * range_inv
    m[2, 3] = z_far * z_near * range_inv
    m[3, 2] = -1.0
    return m


def look_at(eye, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """World -> view matrix (row-major numpy)."""
    eye = np.asarray(eye, np.float64)
    target = np.asarray(target, np.float64)
    up = np.asarray(up, np.float64)
    z = eye - target
    z /= np.linalg.norm(z)
    x = np.cross(up, z)
    if np.linalg.norm(x) < 1e-12:  # looking along up: pick another up
        x = np.cross(np.array([0.0, 0.0, 1.0]), z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    m = np.eye(4)
    m[0, :3], m[1, :3], m[2, :3] = x, y, z
    m[:3, 3] = -m[:3, :3] @ eye
    return m


def col_major(m: np.ndarray) -> np.ndarray:
    """Row-major numpy 4x4 -> 16 float32 in WGSL column-major order."""
    return np.ascontiguousarray(np.asarray(m, np.float64).T.reshape(16), dtype=np.float32)


def view_proj(eye, target, fovy: float, aspect: float, up=(0.0, 1.0, 0.0)):
    """Returns (vp, vp_inv) as 16-float column-major float32 arrays."""
    vp = perspective(fovy, aspect) @ look_at(eye, target, up)
    return col_major(vp), col_major(np.linalg.inv(vp))


def fibonacci_sphere(n: int, radius: float) -> np.ndarray:
    """n camera positions spread on a sphere (golden-angle spiral)."""
    i = np.arange(n, dtype=np.float64) + 0.5
    phi = np.arccos(1.0 - 2.0 * i / n)
    theta = math.pi * (1.0 + 5.0 ** 0.5) * i
    return radius * np.stack([np.cos(theta) * np.sin(phi), np.cos(phi), np.sin(theta) * np.sin(phi)], axis=1)


def sphere_cameras(n: int, radius: float, fovy: float, aspect: float):
    """(vp[n,16], vp_inv[n,16]) for n cameras on a sphere looking at the origin."""
    vps, invs = [], []
    for eye in fibonacci_sphere(n, radius):
        up = (0.0, 1.0, 0.0) if abs(eye[1]) < 0.99 * radius else (0.0, 0.0, 1.0)
        a, b = view_proj(eye, (0.0, 0.0, 0.0), fovy, aspect, up)
        vps.append(a)
        invs.append(b)
    return np.stack(vps), np.stack(invs)
