"""Generates tests/golden/mesh_raster.npz: the reference viewer's mesh render
pass (environment background, then the mesh with mesh.wgsl's standard
pipeline) on synthetic scenes.  The vertex and fragment stages are the
reference's own functions (src/lib/gpu/mesh.wgsl vert / frag,
src/lib/gpu/envmap.wgsl frag, translated to C++ by oracle/build_ref.py); the
fixed-function rasterisation between them is the restatement in
oracle/mesh_raster.py.  Needs the reference checkout (NPRUSH_REFERENCE,
else oracle/reference_path.txt); the GPU tests read only the .npz.

Scene: ground + spheres and boxes, a long thin wall that runs from behind the
camera into the view (near-plane clipping) and a 400-unit ground slab that
reaches past the far plane (far clipping); 61 x 45 pixels.  Cases: normals
shading (the viewer's default) and matcap shading.

    python tests/golden/make_mesh_raster_golden.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT))

import mesh_raster as mr  # noqa: E402
import refrun  # noqa: E402
from nprush_b200 import camera, meshes  # noqa: E402

W, H = 61, 45
EYE, TARGET = (3.2, -2.6, 1.9), (0.0, 0.0, 0.4)


# mesh.wgsl vert / frag and envmap.wgsl frag, the reference's own code
ReferenceStages = refrun.MeshStages


def wall():
    """A quad in the plane of the view direction and the up vector, 0.5 to the
    right of the eye, from 2 behind the eye to 6 in front; both windings (the
    one facing away is culled)."""
    eye, tgt = np.array(EYE), np.array(TARGET)
    f = (tgt - eye) / np.linalg.norm(tgt - eye)
    r = np.cross(f, (0.0, 0.0, 1.0))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    pts = [eye + f * s + r * 0.5 + u * v for s, v in ((-2.0, -0.8), (6.0, -0.8), (6.0, 0.8), (-2.0, 0.8))]
    vs = []
    for n in (-r, r):
        for p in pts:
            vs.append(list(p) + list(n) + [0.6, 0.5, 0.4, 1.0, 0.0, 0.0])
    idx = [0, 1, 2, 0, 2, 3, 4, 6, 5, 4, 7, 6]
    return meshes.MeshData(np.array(vs, np.float32), np.array(idx, np.uint32))


def scene():
    sc = meshes.demo_scene(6, seed=3, mirror_fraction=0.0, sphere_detail=8)
    slab = meshes.quad((0.0, 0.0, -0.01), 400.0, (0.3, 0.35, 0.3, 1.0))
    return meshes.concat([sc, wall(), slab])


def pbr_ground():
    """A ground quad drawn with the PBR stage, its uv repeating the maps 3 x 3."""
    q = meshes.quad((0.0, 0.0, -0.005), 12.0, (1.0, 1.0, 1.0, 1.0))
    q.vertices[:, 10:12] *= 3.0
    return q


def pbr_textures(n=24):
    """Linear albedo (checker + tint) and a tangent-space normal map of bumps."""
    yy, xx = np.mgrid[0:n, 0:n]
    u, v = (xx + 0.5) / n, (yy + 0.5) / n
    alb = np.zeros((n, n, 4), np.float32)
    chk = ((xx // 6 + yy // 6) % 2).astype(np.float32)
    alb[..., 0], alb[..., 1], alb[..., 2], alb[..., 3] = 0.3 + 0.4 * chk, 0.35 + 0.2 * u, 0.25 + 0.3 * v, 1.0
    nx, ny = 0.4 * np.sin(2 * np.pi * 2 * u), 0.4 * np.cos(2 * np.pi * 3 * v)
    nz = np.sqrt(1 - nx * nx - ny * ny)
    nm = np.zeros((n, n, 4), np.float32)
    nm[..., 0], nm[..., 1], nm[..., 2], nm[..., 3] = nx * 0.5 + 0.5, ny * 0.5 + 0.5, nz * 0.5 + 0.5, 1.0
    return alb, nm


def matcap_image(n=32):
    yy, xx = np.mgrid[0:n, 0:n]
    u, v = (xx + 0.5) / n * 2 - 1, (yy + 0.5) / n * 2 - 1
    r2 = np.clip(u * u + v * v, 0, 1)
    img = np.zeros((n, n, 4), np.float32)
    img[..., 0] = 0.2 + 0.8 * (1 - r2) + 0.3 * np.clip(-v, 0, 1)
    img[..., 1] = 0.2 + 0.7 * (1 - r2)
    img[..., 2] = 0.3 + 0.5 * (1 - r2) + 0.3 * np.clip(u, 0, 1)
    img[..., 3] = 1.0
    return img


def uniforms(shading_mode):
    vp, inv = camera.view_proj(EYE, TARGET, 0.9, W / H, up=(0.0, 0.0, 1.0))
    view = camera.col_major(camera.look_at(EYE, TARGET, (0.0, 0.0, 1.0)))
    u = np.zeros(52, np.float32)  # GpuUniformsBufferManager.ts: 208 bytes
    u[0:16], u[16:32], u[32], u[36:52] = vp, view, shading_mode, inv
    return u


def main():
    sc = scene()
    matcap, env = matcap_image(), meshes.sky_env(64, 32)
    out = dict(vertices=sc.vertices, indices=sc.indices, matcap=matcap, env=env)
    for name, mode in (("normals", 0.0), ("shaded", 1.0)):
        uni = uniforms(mode)
        col, dep = mr.render(sc.vertices, sc.indices, uni, W, H, ReferenceStages(uni, matcap, env))
        out[f"uniforms_{name}"] = uni
        out[f"color_{name}"] = col
        out[f"depth_{name}"] = dep
    # the same scene with a PBR-shaded ground drawn last (setPbrMesh)
    pbr = meshes.concat([sc, pbr_ground()])
    alb, nm = pbr_textures()
    out.update(pbr_vertices=pbr.vertices, pbr_indices=pbr.indices, pbr_first=np.uint32(sc.n_tris), albedo=alb,
               normal_map=nm)
    for name, mode in (("normals", 0.0), ("shaded", 1.0)):
        uni = uniforms(mode)
        col, dep = mr.render(pbr.vertices, pbr.indices, uni, W, H, ReferenceStages(uni, matcap, env, alb, nm),
                             first_pbr=sc.n_tris)
        out[f"pbr_color_{name}"] = col
        out[f"pbr_depth_{name}"] = dep
    np.savez_compressed(HERE / "mesh_raster.npz", **out)


if __name__ == "__main__":
    main()
