"""Scalar CPU restatement of the reference's path tracer — test
infrastructure.

Follows src/lib/gpu/path_trace.wgsl operation by operation in float32
(numpy float32 scalars, each operation rounded): pcg / rand2 (:34-43), the
watertight triangle test (:60-131), the slab test (:133-144), the explicit
stack traversal with its 64-entry limit (:148-192), the equirectangular
environment lookup through a linear sampler with u repeating and v clamped
(:200-205, GpuPathTracePipelineManager.ts:204-208), the cosine hemisphere
(:208-219) and the 8-bounce loop (:222-268); and path_trace_resolve.wgsl
(:20-30).  Slow (milliseconds per path): meant for a grid of pixels,
checked against the reference's shader run on the host
(tests/golden/path_trace.npz).

    radiance = trace_pixel(scene, inv_view_proj, x, y, w, h, frame)
"""
from __future__ import annotations

import numpy as np

F = np.float32
M32 = 0xFFFFFFFF
LEAF_FLAG = 0x80000000
MAX_STACK = 64
PI = F(3.14159265358979)


class Scene:
    def __init__(self, vertices, nodes, tri_indices, env):
        self.v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 12)
        self.nodes = np.ascontiguousarray(nodes, np.float32).reshape(-1, 8)
        self.bits = self.nodes.view(np.uint32)
        self.tris = np.ascontiguousarray(tri_indices, np.uint32).reshape(-1, 3)
        self.env = np.ascontiguousarray(env, np.float32)


def pcg(v: int) -> int:
    s = (v * 747796405 + 2891336453) & M32
    w = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & M32
    return ((w >> 22) ^ w) & M32


def rand2(seed: int):
    seed = pcg(seed)
    a = seed
    seed = pcg(seed)
    b = seed
    return seed, F(a) / F(4294967296.0), F(b) / F(4294967296.0)


def add(a, b):
    return tuple(x + y for x, y in zip(a, b))


def sub(a, b):
    return tuple(x - y for x, y in zip(a, b))


def scale(a, s):
    return tuple(x * s for x in a)


def dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def normalize(a):
    return scale(a, F(1.0) / np.sqrt(dot(a, a)))


def cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def intersect_tri(sc, ro, rd, i0, i1, i2, t_max):
    """path_trace.wgsl:60-131; returns (t, norm, color) or None."""
    p0, p1, p2 = (tuple(F(x) for x in sc.v[i, :3]) for i in (i0, i1, i2))
    ad = tuple(abs(x) for x in rd)
    kz = 0
    if ad[1] > ad[0]:
        kz = 1
    if ad[2] > max(ad[0], ad[1]):
        kz = 2
    kx = (kz + 1) % 3
    ky = (kx + 1) % 3
    if rd[kz] < 0:
        kx, ky = ky, kx
    sz = F(1.0) / rd[kz]
    sx = rd[kx] * sz
    sy = rd[ky] * sz
    A, B, C = sub(p0, ro), sub(p1, ro), sub(p2, ro)
    ax, ay = A[kx] - sx * A[kz], A[ky] - sy * A[kz]
    bx, by = B[kx] - sx * B[kz], B[ky] - sy * B[kz]
    cx, cy = C[kx] - sx * C[kz], C[ky] - sy * C[kz]
    U = cx * by - cy * bx
    V = ax * cy - ay * cx
    W = bx * ay - by * ax
    if (U < 0 or V < 0 or W < 0) and (U > 0 or V > 0 or W > 0):
        return None
    det = U + V + W
    if det == 0:
        return None
    az, bz, cz = sz * A[kz], sz * B[kz], sz * C[kz]
    T = U * az + V * bz + W * cz
    inv_det = F(1.0) / det
    t = T * inv_det
    if t < F(1e-4) or t >= t_max:
        return None
    u, v, w = U * inv_det, V * inv_det, W * inv_det
    n0, n1, n2 = (tuple(F(x) for x in sc.v[i, 3:6]) for i in (i0, i1, i2))
    c0, c1, c2 = (tuple(F(x) for x in sc.v[i, 6:10]) for i in (i0, i1, i2))
    norm = normalize(add(add(scale(n0, u), scale(n1, v)), scale(n2, w)))
    color = tuple(u * a + v * b + w * c for a, b, c in zip(c0, c1, c2))
    return t, norm, color


def aabb_hit(sc, ro, inv_rd, node, t_max):
    n = sc.nodes[node]
    mn, mx = (F(n[0]), F(n[1]), F(n[2])), (F(n[4]), F(n[5]), F(n[6]))
    t0 = tuple((a - o) * i for a, o, i in zip(mn, ro, inv_rd))
    t1 = tuple((a - o) * i for a, o, i in zip(mx, ro, inv_rd))
    tmin = np.fmax(np.fmax(np.fmin(t0[0], t1[0]), np.fmin(t0[1], t1[1])), np.fmin(t0[2], t1[2]))
    tmax = np.fmin(np.fmin(np.fmax(t0[0], t1[0]), np.fmax(t0[1], t1[1])), np.fmax(t0[2], t1[2]))
    return tmax >= 0 and tmax >= tmin and tmin < t_max


def scene_hit(sc, ro, rd):
    best = None
    best_t = F(1e30)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        inv_rd = (F(1.0) / rd[0], F(1.0) / rd[1], F(1.0) / rd[2])
        stack = [0]
        while stack:
            node = stack.pop()
            if not aabb_hit(sc, ro, inv_rd, node, best_t):
                continue
            d1 = int(sc.bits[node, 7])
            if d1 & LEAF_FLAG:
                first = int(sc.bits[node, 3])
                for k in range(d1 & ~LEAF_FLAG & M32):
                    i0, i1, i2 = (int(x) for x in sc.tris[first + k])
                    h = intersect_tri(sc, ro, rd, i0, i1, i2, best_t)
                    if h is not None:
                        best, best_t = h, h[0]
            else:
                left, right = int(sc.bits[node, 3]), d1
                if len(stack) + 1 < MAX_STACK:
                    stack.append(right)
                if len(stack) < MAX_STACK:
                    stack.append(left)
    return best


def _texel(env, x, y):
    return tuple(F(c) for c in env[y, x, :3])


def sample_env(sc, d):
    u = np.arctan2(d[1], d[0]) / (F(2.0) * PI) + F(0.5)
    v = F(0.5) - np.arcsin(np.fmin(np.fmax(d[2], F(-1.0)), F(1.0))) / PI
    h, w = sc.env.shape[:2]
    fx = (u - np.floor(u)) * F(w) - F(0.5)
    fy = v * F(h) - F(0.5)
    x0f, y0f = np.floor(fx), np.floor(fy)
    ax, ay = fx - x0f, fy - y0f
    x0, y0 = int(x0f), int(y0f)
    xs = (x0 % w, (x0 + 1) % w)
    ys = (min(max(y0, 0), h - 1), min(max(y0 + 1, 0), h - 1))
    a, b = _texel(sc.env, xs[0], ys[0]), _texel(sc.env, xs[1], ys[0])
    c, e = _texel(sc.env, xs[0], ys[1]), _texel(sc.env, xs[1], ys[1])
    out = []
    for i in range(3):
        top = a[i] + (b[i] - a[i]) * ax
        bot = c[i] + (e[i] - c[i]) * ax
        out.append(top + (bot - top) * ay)
    return tuple(out)


def cosine_hemisphere(n, seed):
    seed, rx, ry = rand2(seed)
    phi = F(2.0) * PI * rx
    sr = np.sqrt(ry)
    x, y, z = np.cos(phi) * sr, np.sin(phi) * sr, np.sqrt(max(F(0.0), F(1.0) - ry))
    up = (F(0.0), F(1.0), F(0.0))
    if abs(n[1]) > F(0.99):
        up = (F(1.0), F(0.0), F(0.0))
    t = normalize(cross(up, n))
    b = cross(n, t)
    return seed, normalize(add(add(scale(t, x), scale(b, y)), scale(n, z)))


def trace_pixel(sc, inv_view_proj, x, y, w, h, frame):
    """One sample of pixel (x, y): the radiance path_trace.wgsl adds (:222-262)."""
    m = np.asarray(inv_view_proj, np.float32).reshape(4, 4)  # m[c] = column c
    pixel = (y * w + x) & M32
    seed = pcg(pixel ^ ((frame * 2654435761) & M32))
    seed, jx, jy = rand2(seed)
    jx, jy = jx - F(0.5), jy - F(0.5)
    ux = (F(x) + F(0.5) + jx) / F(w)
    uy = (F(y) + F(0.5) + jy) / F(h)
    nx, ny = ux * F(2.0) - F(1.0), F(1.0) - uy * F(2.0)

    def mul(vz):
        return tuple(m[0][r] * nx + m[1][r] * ny + m[2][r] * vz + m[3][r] * F(1.0) for r in range(4))

    nh, fh = mul(F(0.0)), mul(F(1.0))
    ro = (nh[0] / nh[3], nh[1] / nh[3], nh[2] / nh[3])
    rd = normalize(sub((fh[0] / fh[3], fh[1] / fh[3], fh[2] / fh[3]), ro))
    rad = (F(0.0), F(0.0), F(0.0))
    thr = (F(1.0), F(1.0), F(1.0))
    o, d = ro, rd
    for _ in range(8):
        hit = scene_hit(sc, o, d)
        if hit is None:
            rad = add(rad, tuple(a * b for a, b in zip(thr, sample_env(sc, d))))
            break
        t, norm, color = hit
        n = scale(norm, F(-1.0)) if dot(norm, d) > 0 else norm
        o2 = add(add(o, scale(d, t)), scale(n, F(5e-4)))
        if color[3] < F(0.5):
            k = F(2.0) * dot(n, d)
            d = sub(d, scale(n, k))
        else:
            thr = tuple(a * b for a, b in zip(thr, color[:3]))
            seed, d = cosine_hemisphere(n, seed)
        o = o2
    return np.array(rad, np.float32)


def resolve(accum):
    """path_trace_resolve.wgsl:20-30 (the stored floats), numpy float32."""
    a = np.asarray(accum, np.float32)
    n = np.maximum(a[..., 3:4], F(1.0))
    c = (a[..., :3] / n) * F(4.0)
    out = np.ones(a.shape, np.float32)
    out[..., :3] = c / (c + F(1.0))
    return out
