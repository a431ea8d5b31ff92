"""Seeded Gaussian scenes for the tests (the small-case distribution: means
U[-1,1]^3, log-scales N(-4, 0.5), random unit quaternions, opacity logits
N(0,1), RGB U[0,1]; camera fov 60 deg at (0, 0, 4) looking at the origin)."""
import math

import numpy as np

from nprush_b200.camera import view_proj
from nprush_b200.gaussians import random_gaussians, view_records


def gs_scene(n, seed, deg=0, log_scale_mean=-4.0, spread=1.0):
    p = random_gaussians(n, seed, sh_degree=deg)
    if log_scale_mean != -4.0:
        p[:, 3:6] += log_scale_mean + 4.0
    p[:, 0:3] *= spread
    return p


def gs_views(w, h, eyes=((0.0, 0.0, 4.0),), fov_deg=60.0):
    vps, vpis = [], []
    for e in eyes:
        up = (0.0, 1.0, 0.0) if abs(e[1]) < 0.99 * np.linalg.norm(e) else (0.0, 0.0, 1.0)
        a, b = view_proj(e, (0.0, 0.0, 0.0), math.radians(fov_deg), w / h, up)
        vps.append(a)
        vpis.append(b)
    vp, vpi = np.stack(vps), np.stack(vpis)
    return vp, vpi, view_records(vp, vpi)


def gs_targets(nt, w, h, seed):
    rng = np.random.default_rng(seed)
    t = np.zeros((nt, h, w, 4), np.float32)
    t[..., :3] = np.clip(rng.normal(0.5, 0.2, (nt, h, w, 3)), 0, 1)
    t[..., 3] = 1.0
    return t
