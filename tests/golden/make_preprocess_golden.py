"""Generates tests/golden/preprocess.npz: inputs and outputs of the reference's
own target-preprocessing shaders (src/lib/gpu/blur.wgsl,
depth_aware_blur.wgsl, splat_edge.wgsl), translated to C++ and run on the
host by oracle/build_ref.py.  Needs the reference checkout (NPRUSH_REFERENCE,
else oracle/reference_path.txt); the GPU tests read only the .npz.

    python tests/golden/make_preprocess_golden.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))

from build_ref import RefModule, gpu_constants  # noqa: E402

W, H = 61, 45  # not multiples of the 16 x 16 workgroup


def images(seed):
    rng = np.random.default_rng(seed)
    color = np.zeros((H, W, 4), np.float32)
    color[..., :3] = rng.random((H, W, 3))
    color[..., 3] = 1.0
    yy, xx = np.mgrid[0:H, 0:W]
    disk = (xx - 27.3) ** 2 + (yy - 20.1) ** 2 < 13.0 ** 2
    depth = np.zeros((H, W, 4), np.float32)
    depth[..., 0] = np.where(disk, 0.3 + 0.002 * xx, 1.0) + rng.normal(0, 0.002, (H, W))
    depth[..., 3] = 1.0
    return color, depth


def run_blur(color, direction, radius, flags, sigma):
    m = RefModule("blur", 0)
    params = np.zeros(8, np.float32)
    pi = params.view(np.int32)
    pi[0], pi[1], pi[2] = direction[0], direction[1], radius
    params.view(np.uint32)[3] = flags
    params[4] = sigma
    out = np.zeros_like(color)
    m.bind_tex(0, color)
    m.bind_storage_tex(1, out)
    m.bind(2, params)
    m.dispatch(-(-W // 16), -(-H // 16))
    return out


def run_depth_blur(color, depth, radius):
    m = RefModule("depth_aware_blur", 0)
    params = np.zeros(4, np.int32)
    params[0] = radius
    out = np.zeros_like(color)
    m.bind_tex(0, color)
    m.bind_tex(1, depth)
    m.bind_storage_tex(2, out)
    m.bind(3, params)
    m.dispatch(-(-W // 16), -(-H // 16))
    return out


def run_edge(depth):
    m = RefModule("splat_edge", 0)
    out = np.zeros_like(depth)
    m.bind_tex(0, depth)
    m.bind_storage_tex(1, out)
    m.dispatch(-(-W // 16), -(-H // 16))
    return out


def main():
    color, depth = images(5)
    c = gpu_constants()
    blur_cases = [((1, 0), 6, 0, 3.0), ((0, 1), 4, 3, 2.0), ((1, 0), 0, 2, 1.0)]
    data = dict(color=color, depth=depth, blur_cases=np.array([[d[0], d[1], r, f] for d, r, f, _ in blur_cases],
                                                               np.int32),
                blur_sigmas=np.array([s for *_, s in blur_cases], np.float32),
                edge_thresholds=np.array([c["SPLAT_EDGE_THRESHOLD_MIN"], c["SPLAT_EDGE_THRESHOLD_MAX"]], np.float32),
                depth_blur_radii=np.array([0, 3], np.int32))
    for k, (d, r, f, s) in enumerate(blur_cases):
        data[f"blur{k}"] = run_blur(color, d, r, f, s)
    for k, r in enumerate(data["depth_blur_radii"]):
        data[f"depth_blur{k}"] = run_depth_blur(color, depth, int(r))
    data["edge"] = run_edge(depth)
    np.savez_compressed(HERE / "preprocess.npz", **data)
    print("wrote", HERE / "preprocess.npz", {k: v.shape for k, v in data.items()})


if __name__ == "__main__":
    main()
