"""Seeded synthetic scenes shared by the tests.

Splat records follow the reference layout (GpuSplatOptimizerManager.ts:58-86:
16 floats: pos.xyz, sx, rgb, opacity, quat wxyz, sy, shape_a, shape_b, sz) and
its init distribution, but seeded.  Bezier records follow
GpuBezierOptimizerManager.ts:60-95 (20 floats).
"""
from __future__ import annotations

import math

import numpy as np

from nprush_b200.camera import view_proj


def splat_scene(n, seed, alive=None, spread=0.3, scale=(0.05, 0.12), random_quat=True, random_shape=False):
    rng = np.random.default_rng(seed)
    s = np.zeros((n, 16), np.float32)
    s[:, 0:3] = (rng.random((n, 3)) * 2 - 1) * spread
    s[:, 3] = scale[0] + rng.random(n) * (scale[1] - scale[0])
    s[:, 4:7] = rng.random((n, 3))
    s[:, 7] = 0.3 + rng.random(n) * 0.6
    if alive is not None:
        s[alive:, 7] = 0.0
    if random_quat:
        q = rng.normal(size=(n, 4))
        q /= np.linalg.norm(q, axis=1, keepdims=True)
        s[:, 8:12] = q
    else:
        s[:, 8] = 1.0
    s[:, 12] = scale[0] + rng.random(n) * (scale[1] - scale[0])
    s[:, 13] = 2.0
    s[:, 14] = 0.5
    if random_shape:
        s[:, 13] = 1.5 + rng.random(n) * 3.0
        s[:, 14] = 0.3 + rng.random(n) * 0.6
    s[:, 15] = scale[0] + rng.random(n) * (scale[1] - scale[0])
    return s


def camera(w, h, dist=1.6, fov=math.pi / 3, eye=None):
    eye = (0.3, 0.4, dist) if eye is None else eye
    return view_proj(eye, (0.0, 0.0, 0.0), fov, w / h)


def targets(w, h, seed, fg_frac=0.6):
    rng = np.random.default_rng(seed)
    rgba = np.zeros((h, w, 4), np.float32)
    rgba[..., :3] = np.clip(rng.normal(0.5, 0.2, (h, w, 3)), 0, 1)
    rgba[..., 3] = 1.0
    depth = np.where(rng.random((h, w)) < fg_frac, 0.9 + 0.06 * rng.random((h, w)), 1.0).astype(np.float32)
    return rgba, depth


def bezier_scene(n, seed, alive=None, width=(0.01, 0.04)):
    rng = np.random.default_rng(seed)
    b = np.zeros((n, 20), np.float32)
    c = (rng.random((n, 2)) * 2 - 1) * 0.5
    ln = 0.2 + rng.random(n) * 0.2
    ang = rng.random(n) * 2 * math.pi
    dx, dy = np.cos(ang) * ln, np.sin(ang) * ln
    jit = lambda: (rng.random(n) - 0.5) * 0.08  # noqa: E731
    b[:, 0] = c[:, 0] - dx * 0.5
    b[:, 1] = c[:, 1] - dy * 0.5
    b[:, 2] = (rng.random(n) * 2 - 1) * 0.3
    b[:, 3] = width[0] + rng.random(n) * (width[1] - width[0])
    b[:, 4] = c[:, 0] - dx * 0.15 + jit()
    b[:, 5] = c[:, 1] - dy * 0.15 + jit()
    b[:, 6] = (rng.random(n) * 2 - 1) * 0.3
    b[:, 7] = 0.005 + rng.random(n) * 0.01
    b[:, 8] = c[:, 0] + dx * 0.15 + jit()
    b[:, 9] = c[:, 1] + dy * 0.15 + jit()
    b[:, 10] = (rng.random(n) * 2 - 1) * 0.3
    b[:, 12] = c[:, 0] + dx * 0.5
    b[:, 13] = c[:, 1] + dy * 0.5
    b[:, 14] = (rng.random(n) * 2 - 1) * 0.3
    b[:, 16:19] = rng.random((n, 3))
    b[:, 19] = 0.3 + 0.6 * rng.random(n)
    if alive is not None:
        b[alive:, 19] = 0.0
    return b


def bezier_textures(w, h, seed):
    rng = np.random.default_rng(seed)
    tgt, depth = targets(w, h, seed)
    bg = np.zeros((h, w, 4), np.float32)
    bg[..., :3] = rng.random((h, w, 3))
    bg_depth = (0.9 + 0.1 * rng.random((h, w))).astype(np.float32)
    normal = np.zeros((h, w, 4), np.float32)
    normal[..., :3] = rng.random((h, w, 3))
    return tgt, depth, bg, bg_depth, normal
