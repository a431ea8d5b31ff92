"""CPU restatement of the reference's mesh render pass — test infrastructure.

What it draws is the optimisation-resolution pass of the reference's viewer
(src/lib/viewer/GpuRunner.svelte.ts:611-634): the environment background
(envmap.wgsl, depth test "always", no depth write), then the mesh with
mesh.wgsl's standard pipeline (GpuMeshRenderPipelineManager.ts:84-112:
triangle list, back faces culled, counter-clockwise front, depth "less" into a
z-buffer cleared to 1.0) writing two colour targets: the shaded colour and
the reciprocal-encoded depth (mesh.wgsl:37-47, cleared to 1.0).

The vertex and fragment stages are functions: `vert`, `frag`, `env_frag`
below restate mesh.wgsl / envmap.wgsl in float32, and the generator of the
fixtures runs the reference's own functions instead (translated to C++).
The fixed-function part is WebGPU's, restated here; where WebGPU leaves a
choice to the implementation this file makes one (the CUDA kernels make the
same one):
  * clipping against 0 <= z <= w and a guard band |x|, |y| <= 64 w
    (Sutherland-Hodgman, then a fan from the first vertex)
  * vertices snapped to 1/256 pixel and edge functions evaluated exactly in
    integers (watertight: a pixel centre on an edge shared by two triangles
    belongs to exactly one of them); pixel centres sampled; a centre exactly
    on an edge is kept when the edge is a top or left edge
  * depth z/w interpolated linearly in screen space, clamped to [0, 1],
    compared as float32 (a depth24plus buffer may round it)
  * varyings interpolated perspective-correctly from the clipped triangle,
    clipped vertices carrying clip-space weights of the original three
  * textures sampled bilinearly at level 0 with exact float32 weights
  * the background's ndc is the pixel centre's
Every float operation is float32 in the order the CUDA kernels use.

    color, depth = render(vertices, indices, uniforms52, w, h, stages)
"""
from __future__ import annotations

import numpy as np

F = np.float32
DEPTH_NEAR = F(0.1)   # mesh.wgsl:37
PI = F(3.14159265358979)
SUBPIX = 256          # sub-pixel steps per pixel
GUARD = F(64.0)       # guard band, in units of w
N_PLANES = 6
MAX_SUBS = 7          # a triangle clipped by 6 planes has <= 9 vertices: <= 7 fan triangles


# ------------------------------------------------------------ float32 helpers
def mat_vec(m16, v):
    """WGSL M * v (m16 column-major): ((c0 v0 + c1 v1) + c2 v2) + c3 v3."""
    m = np.asarray(m16, np.float32).reshape(4, 4)
    return np.array([m[0][r] * F(v[0]) + m[1][r] * F(v[1]) + m[2][r] * F(v[2]) + m[3][r] * F(v[3])
                     for r in range(4)], np.float32)


def normalize(v):
    v = np.asarray(v, np.float32)
    d = v[0] * v[0] + v[1] * v[1] + v[2] * v[2]
    return (v * (F(1.0) / np.sqrt(d))).astype(np.float32)


def reinhard(c):
    return (c / (c + F(1.0))).astype(np.float32)


def sample(tex, u, v, repeat_u, repeat_v):
    """Bilinear level-0 sample (WebGPU filtering, exact float32 weights)."""
    h, w = tex.shape[:2]
    u, v = F(u), F(v)
    if repeat_u:
        u = u - np.floor(u)
    if repeat_v:
        v = v - np.floor(v)
    fx, fy = u * F(w) - F(0.5), v * F(h) - F(0.5)
    # bounded texel coordinates: the same taps for every finite input (beyond
    # the edges both taps clamp to the edge texel), defined for NaN
    fx = np.fmin(np.fmax(fx, F(-2.0)), F(w + 1))
    fy = np.fmin(np.fmax(fy, F(-2.0)), F(h + 1))
    x0f, y0f = np.floor(fx), np.floor(fy)
    ax, ay = fx - x0f, fy - y0f
    x0, y0 = int(x0f), int(y0f)

    def wrap(i, n, rep):
        return i % n if rep else min(max(i, 0), n - 1)

    xa, xb = wrap(x0, w, repeat_u), wrap(x0 + 1, w, repeat_u)
    ya, yb = wrap(y0, h, repeat_v), wrap(y0 + 1, h, repeat_v)
    a, b, c, d = tex[ya, xa], tex[ya, xb], tex[yb, xa], tex[yb, xb]
    top = a + (b - a) * ax
    bot = c + (d - c) * ax
    return (top + (bot - top) * ay).astype(np.float32)


# --------------------------------------------- restated vertex / fragment stages
# VertexOutput as 17 floats: position(4) normal(3) viewDepth(1) viewNormal(3) color(4) uv(2)
def vert(vin, uni):
    """mesh.wgsl:39-50."""
    vin = np.asarray(vin, np.float32)
    pos = mat_vec(uni[0:16], (vin[0], vin[1], vin[2], 1.0))
    vn = mat_vec(uni[16:32], (vin[3], vin[4], vin[5], 0.0))[:3]
    lin = np.fmax(pos[3], DEPTH_NEAR)
    vd = np.fmin(np.fmax(F(1.0) - DEPTH_NEAR / lin, F(0.0)), F(1.0))
    return np.concatenate([pos, vin[3:6], [vd], vn, vin[6:10], vin[10:12]]).astype(np.float32)


def frag(vo, uni, matcap):
    """mesh.wgsl:52-70: (colour, depth) outputs."""
    nc = ((normalize(vo[4:7]) + F(1.0)) * F(0.5)).astype(np.float32)
    vn = normalize(vo[8:11])
    uvx, uvy = vn[0] * F(0.5) + F(0.5), vn[1] * F(0.5) + F(0.5)
    mc = sample(matcap, uvx, F(1.0) - uvy, False, False)[:3]
    tinted = (mc * vo[11:14]).astype(np.float32)
    final = nc if uni[32] < F(0.5) else tinted
    col = np.concatenate([reinhard(final * F(4.0)), [1.0]]).astype(np.float32)
    d = vo[7]
    return col, np.array([d, d, d, 1.0], np.float32)


def cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]], np.float32)


def frag_pbr(vo, uni, matcap, albedo_tex, normal_tex):
    """mesh.wgsl:87-121 (the ground's PBR stage): albedo and tangent-space
    normal map (linear, repeating), TBN from the interpolated normal, matcap
    lit by the perturbed view-space normal."""
    uv = vo[15:17]
    albedo = sample(albedo_tex, uv[0], uv[1], True, True)[:3]
    ts = (sample(normal_tex, uv[0], uv[1], True, True)[:3] * F(2.0) - F(1.0)).astype(np.float32)
    N = normalize(vo[4:7])
    up = np.array([0.0, 0.0, 1.0], np.float32)
    if abs(N[0] * up[0] + N[1] * up[1] + N[2] * up[2]) > F(0.99):
        up = np.array([1.0, 0.0, 0.0], np.float32)
    T = normalize(cross(up, N))
    B = cross(N, T)
    wn = normalize((T * ts[0] + B * ts[1] + N * ts[2]).astype(np.float32))
    vn = normalize(mat_vec(uni[16:32], (wn[0], wn[1], wn[2], 0.0))[:3])
    mx, my = vn[0] * F(0.5) + F(0.5), vn[1] * F(0.5) + F(0.5)
    mc = sample(matcap, mx, F(1.0) - my, False, False)[:3]
    lit = (mc * albedo).astype(np.float32)
    nc = ((wn + F(1.0)) * F(0.5)).astype(np.float32)
    final = nc if uni[32] < F(0.5) else lit
    col = np.concatenate([reinhard(final * F(4.0)), [1.0]]).astype(np.float32)
    d = vo[7]
    return col, np.array([d, d, d, 1.0], np.float32)


def env_frag(ndc, uni, env):
    """envmap.wgsl:36-52."""
    inv = uni[36:52]
    nh = mat_vec(inv, (ndc[0], ndc[1], 0.0, 1.0))
    fh = mat_vec(inv, (ndc[0], ndc[1], 1.0, 1.0))
    nw = nh[:3] / nh[3]
    fw = fh[:3] / fh[3]
    d = normalize(fw - nw)
    lon = np.arctan2(d[1], d[0])
    lat = np.arcsin(np.fmin(np.fmax(d[2], F(-1.0)), F(1.0)))
    u = lon / (F(2.0) * PI) + F(0.5)
    v = F(0.5) - lat / PI
    c = sample(env, u, v, True, False)[:3]
    return np.concatenate([reinhard(c * F(4.0)), [1.0]]).astype(np.float32)


class RestatedStages:
    """The stage functions above, with the textures they sample (albedo and
    normal map for the PBR stage)."""

    def __init__(self, matcap, env, albedo=None, normal_map=None):
        self.matcap = np.ascontiguousarray(matcap, np.float32)
        self.env = np.ascontiguousarray(env, np.float32)
        self.albedo = None if albedo is None else np.ascontiguousarray(albedo, np.float32)
        self.normal_map = None if normal_map is None else np.ascontiguousarray(normal_map, np.float32)

    def vert(self, vin, uni):
        return vert(vin, uni)  # vert_pbr is the same function

    def frag(self, vo, uni, pbr=False):
        if pbr:
            return frag_pbr(vo, uni, self.matcap, self.albedo, self.normal_map)
        return frag(vo, uni, self.matcap)

    def env_frag(self, ndc, uni):
        return env_frag(ndc, uni, self.env)


# --------------------------------------------------------- fixed function
def plane_dist(p, plane):
    x, y, z, w = p[0], p[1], p[2], p[3]
    if plane == 0:
        return z
    if plane == 1:
        return w - z
    g = GUARD * w
    return (g - x, g + x, g - y, g + y)[plane - 2]


def clip_polygon(clip, c):
    """Sutherland-Hodgman against z >= 0, w - z >= 0 and the guard band.
    clip: 3 x 4 clip positions, c: 3 x 3 weights of the original vertices."""
    poly = [(np.asarray(clip[i], np.float32), np.asarray(c[i], np.float32)) for i in range(3)]
    if all(plane_dist(p[0], k) >= 0 for p in poly for k in range(N_PLANES)):
        return poly
    for plane in range(N_PLANES):
        out = []
        n = len(poly)
        for i in range(n):
            a, b = poly[i], poly[(i + 1) % n]
            da, db = plane_dist(a[0], plane), plane_dist(b[0], plane)
            if da >= 0:
                out.append(a)
            if (da >= 0) != (db >= 0):
                t = da / (da - db)
                out.append(((a[0] + t * (b[0] - a[0])).astype(np.float32),
                            (a[1] + t * (b[1] - a[1])).astype(np.float32)))
        poly = out
        if len(poly) < 3:
            return []
    return poly


def screen(p, w, h):
    """Clip position -> (fx, fy, z_ndc, 1/w) in framebuffer coordinates."""
    X, Y, Z, W = (F(x) for x in p)
    nx, ny, nz = X / W, Y / W, Z / W
    fx = (nx + F(1.0)) * F(0.5) * F(w)
    fy = (F(1.0) - ny) * F(0.5) * F(h)
    return fx, fy, nz, F(1.0) / W


def setup(poly, k, w, h):
    """Sub-triangle k of the clipped polygon, or None when culled: screen
    vertices, snapped vertices, area (in 1/256-pixel units squared), pixel
    box, clip weights."""
    if len(poly) < k + 3:
        return None
    vs = [poly[0], poly[k + 1], poly[k + 2]]
    if any(not (v[0][3] > 0) for v in vs):
        return None
    s = [screen(v[0], w, h) for v in vs]
    if not all(np.isfinite(x) for sv in s for x in sv):
        return None
    X = [int(np.rint(sv[0] * F(SUBPIX))) for sv in s]
    Y = [int(np.rint(sv[1] * F(SUBPIX))) for sv in s]
    A = (X[1] - X[0]) * (Y[2] - Y[0]) - (X[2] - X[0]) * (Y[1] - Y[0])
    if A >= 0:  # back-facing (or degenerate): counter-clockwise on screen is the front
        return None
    half = SUBPIX // 2
    bx0 = max(0, -((-(min(X) - half)) // SUBPIX))
    bx1 = min(w - 1, (max(X) - half) // SUBPIX)
    by0 = max(0, -((-(min(Y) - half)) // SUBPIX))
    by1 = min(h - 1, (max(Y) - half) // SUBPIX)
    if bx0 > bx1 or by0 > by1:
        return None
    return dict(s=s, X=X, Y=Y, area=-A, box=(bx0, bx1, by0, by1), c=[v[1] for v in vs])


def _top_left(ax, ay, bx, by):
    return (by > ay) or (by == ay and bx < ax)


def coverage(st, px, py):
    """Exact edge functions at pixel centres (arrays of pixel indices):
    inside mask, screen barycentrics, depth."""
    X, Y = st["X"], st["Y"]
    cx = px.astype(np.int64) * SUBPIX + SUBPIX // 2
    cy = py.astype(np.int64) * SUBPIX + SUBPIX // 2

    def edge(a, b):
        return (Y[b] - Y[a]) * (cx - X[a]) - (X[b] - X[a]) * (cy - Y[a])

    e0, e1, e2 = edge(1, 2), edge(2, 0), edge(0, 1)
    ins = ((e0 > 0) | ((e0 == 0) & _top_left(X[1], Y[1], X[2], Y[2]))) & \
          ((e1 > 0) | ((e1 == 0) & _top_left(X[2], Y[2], X[0], Y[0]))) & \
          ((e2 > 0) | ((e2 == 0) & _top_left(X[0], Y[0], X[1], Y[1])))
    area = np.int64(st["area"]).astype(np.float32)
    l0, l1, l2 = e0.astype(np.float32) / area, e1.astype(np.float32) / area, e2.astype(np.float32) / area
    z0, z1, z2 = st["s"][0][2], st["s"][1][2], st["s"][2][2]
    z = np.fmin(np.fmax(l0 * z0 + l1 * z1 + l2 * z2, F(0.0)), F(1.0))
    return ins, (l0, l1, l2), z


def render(vertices, indices, uni, w, h, stages, draw_env=True, first_pbr=None):
    """The pass: (colour, depth) float32 (h, w, 4) images (the stored floats,
    before an 8-bit target rounds them).  Triangles from first_pbr on are
    drawn with the PBR stage (the reference draws its PBR mesh last)."""
    uni = np.asarray(uni, np.float32)
    v = np.asarray(vertices, np.float32).reshape(-1, 12)
    idx = np.asarray(indices, np.uint32).reshape(-1, 3)
    vout = np.array([stages.vert(v[i], uni) for i in range(v.shape[0])], np.float32).reshape(-1, 17)
    zbuf = np.ones((h, w), np.float32)
    owner = np.full((h, w), -1, np.int64)
    one_hot = np.eye(3, dtype=np.float32)
    for t in range(idx.shape[0]):
        poly = clip_polygon([vout[i, 0:4] for i in idx[t]], one_hot)
        for k in range(MAX_SUBS):
            st = setup(poly, k, w, h)
            if st is None:
                continue
            bx0, bx1, by0, by1 = st["box"]
            py, px = np.mgrid[by0:by1 + 1, bx0:bx1 + 1]
            ins, _, z = coverage(st, px, py)
            upd = ins & (z < zbuf[by0:by1 + 1, bx0:bx1 + 1])  # depth "less", in draw order
            zbuf[by0:by1 + 1, bx0:bx1 + 1][upd] = z[upd]
            owner[by0:by1 + 1, bx0:bx1 + 1][upd] = MAX_SUBS * t + k
    color = np.zeros((h, w, 4), np.float32)
    depth = np.ones((h, w, 4), np.float32)
    for y in range(h):
        for x in range(w):
            sid = owner[y, x]
            if sid < 0:
                if draw_env:
                    color[y, x] = stages.env_frag(ndc_center(x, y, w, h), uni)
                else:
                    color[y, x] = (0.05, 0.05, 0.05, 1.0)
                continue
            t, k = divmod(int(sid), MAX_SUBS)
            poly = clip_polygon([vout[i, 0:4] for i in idx[t]], one_hot)
            st = setup(poly, k, w, h)
            _, (l0, l1, l2), z = coverage(st, np.array([x]), np.array([y]))
            iw = [sv[3] for sv in st["s"]]
            q0, q1, q2 = l0[0] * iw[0], l1[0] * iw[1], l2[0] * iw[2]
            qs = q0 + q1 + q2
            b = (q0 / qs, q1 / qs, q2 / qs)
            c = st["c"]
            wts = [b[0] * c[0][j] + b[1] * c[1][j] + b[2] * c[2][j] for j in range(3)]
            vo = vout[idx[t]]
            interp = (wts[0] * vo[0] + wts[1] * vo[1] + wts[2] * vo[2]).astype(np.float32)
            interp[0:4] = (F(x) + F(0.5), F(y) + F(0.5), z[0], F(0.0))  # builtin position (unused)
            pbr = first_pbr is not None and t >= first_pbr
            col, dep = stages.frag(interp, uni, pbr) if pbr else stages.frag(interp, uni)
            color[y, x], depth[y, x] = col, dep
    return color, depth


def ndc_center(x, y, w, h):
    """The background's ndc at pixel (x, y), float32."""
    return ((F(x) + F(0.5)) / F(w) * F(2.0) - F(1.0), F(1.0) - (F(y) + F(0.5)) / F(h) * F(2.0))


