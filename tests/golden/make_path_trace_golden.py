"""Generates tests/golden/path_trace.npz: scenes, their BVHs and the outputs of
the reference's own path tracer (src/lib/gpu/path_trace.wgsl and
path_trace_resolve.wgsl, translated to C++ and run on the host by
oracle/build_ref.py).  The BVHs come from the reference's own builder
(src/lib/gpu/bvh.ts, translated to Python by oracle/ts2py.py).  Needs the
reference checkout (NPRUSH_REFERENCE, else oracle/reference_path.txt); the GPU tests
read only the .npz.

Cases (image 45 x 37, not a multiple of the 8 x 8 workgroup):
  diffuse  ground + spheres and boxes (one box a mirror), sky environment;
           accumulation after frame 0 and after frames 0-2, resolved output
  mirror   the same geometry with every surface a mirror (no random bounce
           directions: the paths depend only on exact arithmetic until the
           environment lookup)
  empty    no triangles: every pixel is the environment seen by its ray

    python tests/golden/make_path_trace_golden.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT))

import refrun  # noqa: E402
from nprush_b200 import camera, meshes  # noqa: E402

W, H = 45, 37


def scene():
    sc = meshes.demo_scene(6, seed=3, mirror_fraction=0.0, sphere_detail=8)
    v = sc.vertices.copy()
    first_box = 4 + 9 * 17  # after the ground quad and the first 8 x 16 sphere
    v[first_box:first_box + 24, 9] = 0.0
    return meshes.MeshData(v, sc.indices)


def trace(mesh, env, inv, frames):
    nodes, tris = refrun.build_bvh(mesh.vertices, mesh.indices)
    acc = np.zeros((H, W, 4), np.float32)
    snaps = []
    for f in frames:
        refrun.path_trace(mesh.vertices, nodes, tris, env, inv, f, acc)
        snaps.append(acc.copy())
    return nodes, tris, snaps


def main():
    env = meshes.sky_env(64, 32)
    vp, inv = camera.view_proj((3.2, -2.6, 1.9), (0.0, 0.0, 0.4), 0.9, W / H, up=(0.0, 0.0, 1.0))
    diffuse = scene()
    nodes, tris, snaps = trace(diffuse, env, inv, [0, 1, 2])
    mirror = meshes.MeshData(diffuse.vertices.copy(), diffuse.indices)
    mirror.vertices[:, 9] = 0.0
    _, _, msnaps = trace(mirror, env, inv, [5])
    empty = meshes.MeshData(np.zeros((0, 12), np.float32), np.zeros(0, np.uint32))
    enodes, _, esnaps = trace(empty, env, inv, [0])
    data = dict(
        env=env, inv_view_proj=inv, vertices=diffuse.vertices, indices=diffuse.indices,
        mirror_vertices=mirror.vertices, nodes=nodes, tris=tris, empty_nodes=enodes,
        accum_f0=snaps[0], accum_f012=snaps[2], resolved_f012=refrun.path_trace_resolve(snaps[2]),
        mirror_accum_f5=msnaps[0], empty_accum_f0=esnaps[0],
    )
    np.savez_compressed(HERE / "path_trace.npz", **data)


if __name__ == "__main__":
    main()
