"""CPU restatement of the reference's SAH BVH builder (src/lib/gpu/bvh.ts) —
test infrastructure.

JavaScript numbers are IEEE doubles and Python floats are too, so every
quantity is computed here as bvh.ts computes it; node bounds are rounded to
float32 when written (DataView.setFloat32, bvh.ts:90-97) and the data words
hold u32 bits (setUint32, :99-103).  There is no JavaScript runtime on this
machine; bvh.ts itself runs here through oracle/ts2py.py (refrun.build_bvh),
and this restatement equals it bit for bit (tests/test_golden_path_trace.py).

    nodes, tris = build_bvh(vertices, indices)
        vertices: (V, 12) float32 [pos, normal, rgba, uv]; indices: (T*3,) u32
        nodes: (N, 8) float32 (columns 3 and 7 hold u32 bits); tris: (T, 3) u32
"""
from __future__ import annotations

import math
import sys

import numpy as np

LEAF_FLAG = 0x80000000  # bvh.ts:15
MAX_LEAF_TRIS = 4       # bvh.ts:16
SAH_BINS = 8            # bvh.ts:17
INF = math.inf


def _union(a, b):  # bvh.ts:38-43
    return ([min(a[0][i], b[0][i]) for i in range(3)], [max(a[1][i], b[1][i]) for i in range(3)])


def _area(a):  # bvh.ts:45-50
    dx, dy, dz = (a[1][i] - a[0][i] for i in range(3))
    return 2 * (dx * dy + dy * dz + dz * dx)


def _empty():
    return ([INF, INF, INF], [-INF, -INF, -INF])


def _bin(c, cmin, cmax):  # bvh.ts:147-148
    return min(math.floor(((c - cmin) / (cmax - cmin)) * SAH_BINS), SAH_BINS - 1)


def build_bvh(vertices, indices):
    v = np.asarray(vertices, np.float32).reshape(-1, 12)
    idx = np.asarray(indices, np.uint32).reshape(-1)
    pos = [[float(x) for x in row[:3]] for row in v]
    eps = 1e-4  # bvh.ts:66
    tris = []
    for t in range(len(idx) // 3):  # bvh.ts:208-216
        i0, i1, i2 = int(idx[3 * t]), int(idx[3 * t + 1]), int(idx[3 * t + 2])
        a, b, c = pos[i0], pos[i1], pos[i2]
        box = ([min(a[k], b[k], c[k]) - eps for k in range(3)], [max(a[k], b[k], c[k]) + eps for k in range(3)])
        cen = [(box[0][k] + box[1][k]) * 0.5 for k in range(3)]
        tris.append((i0, i1, i2, box, cen))

    nodes: list = []   # [minx, miny, minz, data0, maxx, maxy, maxz, data1]
    out_tris: list = []

    def build_node(ts):  # bvh.ts:106-200
        bounds, cent = _empty(), _empty()
        for t in ts:
            bounds = _union(bounds, t[3])
            cent = _union(cent, (t[4], t[4]))
        node = len(nodes)
        nodes.append([bounds[0][0], bounds[0][1], bounds[0][2], 0, bounds[1][0], bounds[1][1], bounds[1][2], 0])
        if len(ts) <= MAX_LEAF_TRIS:
            start = len(out_tris)
            out_tris.extend((t[0], t[1], t[2]) for t in ts)
            nodes[node][3], nodes[node][7] = start, (len(ts) | LEAF_FLAG)
            return node
        best_cost, best_axis, best_split = INF, 0, 0
        parent_sa = _area(bounds)
        for axis in range(3):
            cmin, cmax = cent[0][axis], cent[1][axis]
            if cmax - cmin < 1e-8:
                continue
            bin_box = [_empty() for _ in range(SAH_BINS)]
            bin_count = [0] * SAH_BINS
            for t in ts:
                b = _bin(t[4][axis], cmin, cmax)
                bin_box[b] = _union(bin_box[b], t[3])
                bin_count[b] += 1
            left_box, left_count = [], []
            lb, lc = _empty(), 0
            for i in range(SAH_BINS - 1):
                lb = _union(lb, bin_box[i])
                lc += bin_count[i]
                left_box.append(lb)
                left_count.append(lc)
            rb, rc = _empty(), 0
            for i in range(SAH_BINS - 2, -1, -1):
                rb = _union(rb, bin_box[i + 1])
                rc += bin_count[i + 1]
                # an empty side has infinite area: Infinity * 0 is NaN and
                # NaN < x is false, in JavaScript as in Python
                cost = (_area(left_box[i]) * left_count[i] + _area(rb) * rc) / parent_sa
                if cost < best_cost:
                    best_cost, best_axis, best_split = cost, axis, i
        cmin, cmax = cent[0][best_axis], cent[1][best_axis]
        if cmax - cmin < 1e-8 or best_cost >= len(ts):
            mid = len(ts) // 2
            left, right = ts[:mid], ts[mid:]
        else:
            left, right = [], []
            for t in ts:
                (left if _bin(t[4][best_axis], cmin, cmax) <= best_split else right).append(t)
            if not left or not right:
                mid = len(ts) // 2
                left, right = ts[:mid], ts[mid:]
        li = build_node(left)
        ri = build_node(right)
        nodes[node][3], nodes[node][7] = li, ri
        return node

    old = sys.getrecursionlimit()
    sys.setrecursionlimit(max(old, 10000))
    try:
        build_node(tris)
    finally:
        sys.setrecursionlimit(old)
    out = np.zeros((len(nodes), 8), np.float32)
    bits = out.view(np.uint32)
    for k, nd in enumerate(nodes):
        out[k, [0, 1, 2, 4, 5, 6]] = np.array([nd[0], nd[1], nd[2], nd[4], nd[5], nd[6]], np.float64).astype(np.float32)
        bits[k, 3], bits[k, 7] = nd[3], nd[7]
    return out, np.array(out_tris, np.uint32).reshape(-1, 3)
