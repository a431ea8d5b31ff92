"""Fixed-function steps of the display forwards' render pipelines, restated.

TEST INFRASTRUCTURE ONLY (the fixture generator tests/golden/make_forward_golden.py
and the tests).  The pipelines are those of

* GpuSplatForwardPipelineManager (src/lib/gpu/GpuSplatForwardPipelineManager.ts:56-92,
  :114-137): triangle list, 6 vertices per instance, no face culling, two
  attachments (colour, encoded depth) blended with
  rgb = src.rgb * src.a + dst.rgb * (1 - src.a), a = src.a + dst.a * (1 - src.a);
* GpuBezierForwardPipelineManager (src/lib/gpu/GpuBezierForwardPipelineManager.ts:62-99,
  :131-148): triangle strip, 4 vertices per instance, one attachment blended
  premultiplied, rgb = src.rgb + dst.rgb * (1 - src.a), a = src.a + dst.a * (1 - src.a).

The vertex and fragment stages are callables (in the fixture generator the
reference's own functions, translated by oracle/build_ref.py).  The steps
between them, with the implementation choices this restatement makes:

* clipping: both vertex stages give every vertex of an instance one common
  clip z and w, and cull an instance by moving it outside the clip volume.
  A primitive is drawn when w > 0 and 0 <= z <= w (inclusive) and dropped
  otherwise; x and y are not clipped, only pixel centres inside the viewport
  are sampled (a guard band);
* coverage: screen positions snapped to 1/256 pixel, exact integer edge
  functions at pixel centres with the top-left rule, both windings;
* interpolation: barycentric weights from the unsnapped screen positions in
  float64, cast to float32; the vertices of a primitive share w, so the
  perspective-correct weights are these; flat attributes from the first
  vertex of the primitive;
* blending: in draw order (instance, then primitive) in float32; the
  reference's rgba8unorm attachments are not emulated.
"""
from __future__ import annotations

import numpy as np

SUBPIX = 256


def _screen(clip, w, h):
    """Framebuffer position (y down) of a clip-space vertex, float64."""
    x = (float(clip[0]) / float(clip[3]) + 1.0) * 0.5 * w
    y = (1.0 - float(clip[1]) / float(clip[3])) * 0.5 * h
    return x, y


def _top_left(ax, ay, bx, by):
    return (by > ay) or (by == ay and bx < ax)


def raster_triangle(clips, w, h):
    """Pixel centres a triangle covers: (px, py, lam) with lam the float64
    barycentric weights (n x 3) of the three vertices, or None when nothing
    is drawn."""
    zs = {(float(c[2]), float(c[3])) for c in clips}
    if len(zs) != 1:
        raise ValueError("these pipelines emit one clip z and w per primitive")
    z, cw = zs.pop()
    if not (cw > 0 and 0.0 <= z <= cw):
        return None
    s = [_screen(c, w, h) for c in clips]
    X = [int(np.rint(p[0] * SUBPIX)) for p in s]
    Y = [int(np.rint(p[1] * SUBPIX)) for p in s]
    A = (X[1] - X[0]) * (Y[2] - Y[0]) - (X[2] - X[0]) * (Y[1] - Y[0])
    if A == 0:
        return None
    order = [0, 1, 2] if A < 0 else [0, 2, 1]  # one orientation for the edge tests
    X = [X[k] for k in order]
    Y = [Y[k] for k in order]
    half = SUBPIX // 2
    bx0 = max(0, -((-(min(X) - half)) // SUBPIX))
    bx1 = min(w - 1, (max(X) - half) // SUBPIX)
    by0 = max(0, -((-(min(Y) - half)) // SUBPIX))
    by1 = min(h - 1, (max(Y) - half) // SUBPIX)
    if bx0 > bx1 or by0 > by1:
        return None
    py, px = np.mgrid[by0:by1 + 1, bx0:bx1 + 1]
    px, py = px.ravel(), py.ravel()
    cx = px.astype(np.int64) * SUBPIX + half
    cy = py.astype(np.int64) * SUBPIX + half

    def edge(a, b):
        return (Y[b] - Y[a]) * (cx - X[a]) - (X[b] - X[a]) * (cy - Y[a])

    e0, e1, e2 = edge(1, 2), edge(2, 0), edge(0, 1)
    ins = (((e0 > 0) | ((e0 == 0) & _top_left(X[1], Y[1], X[2], Y[2])))
           & ((e1 > 0) | ((e1 == 0) & _top_left(X[2], Y[2], X[0], Y[0])))
           & ((e2 > 0) | ((e2 == 0) & _top_left(X[0], Y[0], X[1], Y[1]))))
    px, py = px[ins], py[ins]
    if px.size == 0:
        return None
    # barycentrics of the unsnapped triangle at the pixel centres
    (x0, y0), (x1, y1), (x2, y2) = s
    fx, fy = px + 0.5, py + 0.5
    area = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0)
    l0 = ((x1 - fx) * (y2 - fy) - (x2 - fx) * (y1 - fy)) / area
    l1 = ((x2 - fx) * (y0 - fy) - (x0 - fx) * (y2 - fy)) / area
    lam = np.stack([l0, l1, 1.0 - l0 - l1], 1)
    return px, py, lam


def triangles(topology, n_vertices):
    """Vertex indices of the primitives of one instance."""
    if topology == "triangle-list":
        return [(k, k + 1, k + 2) for k in range(0, n_vertices - 2, 3)]
    if topology == "triangle-strip":  # odd triangles keep the strip's winding
        return [(k, k + 1, k + 2) if k % 2 == 0 else (k + 1, k, k + 2) for k in range(n_vertices - 2)]
    raise ValueError(topology)


def blend_src_alpha(src, dst):
    """src-alpha / one-minus-src-alpha colour, one / one-minus-src-alpha alpha."""
    a = np.float32(src[3])
    one = np.float32(1.0)
    out = np.empty(4, np.float32)
    out[:3] = src[:3] * a + dst[:3] * (one - a)
    out[3] = a + dst[3] * (one - a)
    return out


def blend_premultiplied(src, dst):
    """one / one-minus-src-alpha on every channel."""
    a = np.float32(src[3])
    return (src + dst * (np.float32(1.0) - a)).astype(np.float32)


def draw(n_instances, n_vertices, topology, vert, frag, w, h, attachments, blends, interp, flat):
    """Runs one draw: vert(vi, ii) -> vertex output floats (clip position in
    0-3), frag(fragment input floats) -> list of per-attachment colours or
    None (discarded).  `interp` / `flat` are the output float indices that are
    interpolated / copied from the first vertex; attachments are float32
    H x W x 4 images blended in place with blends[k]."""
    for ii in range(n_instances):
        outs = [np.asarray(vert(vi, ii), np.float32) for vi in range(n_vertices)]
        for tri in triangles(topology, n_vertices):
            vs = [outs[k] for k in tri]
            r = raster_triangle([v[:4] for v in vs], w, h)
            if r is None:
                continue
            px, py, lam = r
            for j in range(px.size):
                fin = np.zeros_like(vs[0])
                fin[flat] = vs[0][flat]
                for k in interp:
                    fin[k] = np.float32(lam[j, 0] * vs[0][k] + lam[j, 1] * vs[1][k] + lam[j, 2] * vs[2][k])
                cw = float(vs[0][3])
                fin[0:4] = (px[j] + 0.5, py[j] + 0.5, float(vs[0][2]) / cw, 1.0 / cw)
                res = frag(fin)
                if res is None:
                    continue
                for att, blend, col in zip(attachments, blends, res):
                    att[py[j], px[j]] = blend(np.asarray(col, np.float32), att[py[j], px[j]])
