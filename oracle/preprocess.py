"""CPU restatement (numpy, float64 accumulation) of the reference's target
preprocessing shaders — test infrastructure, checked against the reference's
own shaders run on the host (tests/golden/preprocess.npz).

  blur            src/lib/gpu/blur.wgsl:23-48
  depth_aware     src/lib/gpu/depth_aware_blur.wgsl:12-53
  splat_edge      src/lib/gpu/splat_edge.wgsl:13-44
"""
import numpy as np


def _srgb_to_linear(c):
    return np.where(c > 0.04045, ((c + 0.055) / 1.055) ** 2.4, c / 12.92)


def _linear_to_srgb(c):
    s = np.maximum(c, 0.0)
    return np.where(s > 0.0031308, 1.055 * s ** (1.0 / 2.4) - 0.055, s * 12.92)


def unorm8(x):
    return np.rint(np.clip(x, 0.0, 1.0) * 255.0) / 255.0


def blur(color, direction, radius, flags, sigma):
    h, w = color.shape[:2]
    yy, xx = np.mgrid[0:h, 0:w]
    acc = np.zeros((h, w, 3))
    ws = 0.0
    for i in range(-radius, radius + 1):
        cx = np.clip(xx + direction[0] * i, 0, w - 1)
        cy = np.clip(yy + direction[1] * i, 0, h - 1)
        c = color[cy, cx, :3].astype(np.float64)
        if flags & 1:
            c = _srgb_to_linear(c)
        wt = np.exp(-float(i * i) / (2.0 * sigma * sigma))
        acc += c * wt
        ws += wt
    r = acc / ws
    if flags & 2:
        r = _linear_to_srgb(r)
    out = np.ones((h, w, 4))
    out[..., :3] = r
    return out


def depth_aware_blur(color, depth, radius):
    h, w = color.shape[:2]
    yy, xx = np.mgrid[0:h, 0:w]
    cc = color[..., :3].astype(np.float64)
    cd = depth[..., 0].astype(np.float64)
    acc = np.zeros((h, w, 3))
    sw = np.zeros((h, w))
    for dy in range(-radius, radius + 1):
        for dx in range(-radius, radius + 1):
            nx, ny = xx + dx, yy + dy
            inb = (nx >= 0) & (nx < w) & (ny >= 0) & (ny < h)
            sx, sy = np.clip(nx, 0, w - 1), np.clip(ny, 0, h - 1)
            nc = cc[sy, sx]
            nd = cd[sy, sx]
            wr = (np.exp(-(dx * dx + dy * dy) / (2.0 * 100.0)) * np.exp(-((nc - cc) ** 2).sum(-1) / (2.0 * 0.25))
                  * np.exp(-((nd - cd) ** 2) / (2.0 * 0.25)))
            wt = np.where(inb, wr, 0.0)
            acc += nc * wt[..., None]
            sw += wt
    out = np.ones((h, w, 4))
    out[..., :3] = acc / np.maximum(sw, 1e-5)[..., None]
    return out


def splat_edge(depth, thr_min, thr_max):
    h, w = depth.shape[:2]
    d = depth[..., 0].astype(np.float64)
    p = np.pad(d, 1, mode="edge")
    tl, tc, tr = p[:-2, :-2], p[:-2, 1:-1], p[:-2, 2:]
    ml, mr = p[1:-1, :-2], p[1:-1, 2:]
    bl, bc, br = p[2:, :-2], p[2:, 1:-1], p[2:, 2:]
    gx = -tl - 2 * ml - bl + tr + 2 * mr + br
    gy = -tl - 2 * tc - tr + bl + 2 * bc + br
    e = np.sqrt(gx * gx + gy * gy)
    t = np.clip((e - thr_min) / (thr_max - thr_min), 0.0, 1.0)
    v = t * t * (3 - 2 * t)
    out = np.ones((h, w, 4))
    out[..., 0] = out[..., 1] = out[..., 2] = v
    return out
