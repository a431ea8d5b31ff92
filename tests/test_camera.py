"""Camera convention pins (CPU).  The reference builds its matrices with
wgpu-matrix (Camera.svelte.ts:18-33: proj = mat4.perspective(fov, aspect,
zNear = 0.01, zFar = 100), viewProj = proj * view, viewProjInv =
inverse(viewProj)) and uploads them column-major as WGSL mat4x4f.  These
tests pin nprush_b200.camera to the closed forms of that convention: WebGPU
clip z in [0, 1], clip w equal to the view depth, the look-at target at NDC
(0, 0), camera up on screen up, and column-major storage (element 4c + r is
column c, row r)."""
import math

import numpy as np
import pytest

from nprush_b200 import camera
from nprush_b200.gaussians import view_records

CASES = [
    ((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), math.pi / 2, 16 / 9),
    ((3.0, -2.0, 1.5), (0.2, 0.1, -0.3), (0.0, 0.0, 1.0), math.radians(50.0), 1.0),
    ((-1.0, 5.0, 2.0), (0.5, 0.0, 0.0), (0.0, 1.0, 0.0), math.radians(60.0), 0.75),
]


def _clip(vp16, p):
    m = np.asarray(vp16, np.float64).reshape(4, 4).T  # column-major -> row-major
    return m @ np.array([p[0], p[1], p[2], 1.0])


def test_perspective_closed_form():
    """wgpu-matrix perspective: f = tan(pi/2 - fov/2); column-major elements
    [0] = f / aspect, [5] = f, [10] = zFar / (zNear - zFar), [11] = -1,
    [14] = zFar zNear / (zNear - zFar), every other element 0."""
    for fov, aspect in ((math.pi / 2, 16 / 9), (math.radians(50.0), 1.0), (0.3, 2.5)):
        m = camera.col_major(camera.perspective(fov, aspect))
        f = math.tan(math.pi / 2 - fov / 2)
        want = np.zeros(16)
        want[0], want[5] = f / aspect, f
        want[10] = camera.Z_FAR / (camera.Z_NEAR - camera.Z_FAR)
        want[11] = -1.0
        want[14] = camera.Z_FAR * camera.Z_NEAR / (camera.Z_NEAR - camera.Z_FAR)
        np.testing.assert_allclose(m, want.astype(np.float32), rtol=1e-6, atol=0)


@pytest.mark.parametrize("eye,target,up,fov,aspect", CASES)
def test_view_projection_convention(eye, target, up, fov, aspect):
    vp, vpi = camera.view_proj(eye, target, fov, aspect, up)
    eye, target, up = (np.asarray(x, np.float64) for x in (eye, target, up))
    fwd = (target - eye) / np.linalg.norm(target - eye)
    # the look-at target lands at NDC (0, 0), in front of the camera
    c = _clip(vp, target)
    assert abs(c[0] / c[3]) < 1e-6 and abs(c[1] / c[3]) < 1e-6
    # clip w is the view depth (distance along the viewing direction)
    rng = np.random.default_rng(0)
    for p in rng.normal(0, 2, (20, 3)):
        c = _clip(vp, p)
        assert abs(c[3] - np.dot(p - eye, fwd)) < 1e-5 * max(1.0, abs(c[3]))
    # clip z / w: 0 on the near plane, 1 on the far plane (WebGPU depth range)
    for d, want in ((camera.Z_NEAR, 0.0), (camera.Z_FAR, 1.0)):
        c = _clip(vp, eye + d * fwd)
        assert abs(c[2] / c[3] - want) < 2e-4
    # the vertical field of view spans NDC y in [-1, 1]; x is scaled by the aspect
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    cam_up = np.cross(right, fwd)
    d = 3.0
    top = eye + d * fwd + d * math.tan(fov / 2) * cam_up
    c = _clip(vp, top)
    assert abs(c[1] / c[3] - 1.0) < 1e-5 and abs(c[0] / c[3]) < 1e-5
    side = eye + d * fwd + d * math.tan(fov / 2) * aspect * right
    c = _clip(vp, side)
    assert abs(c[0] / c[3] - 1.0) < 1e-5 and abs(c[1] / c[3]) < 1e-5
    # vp_inv is the inverse, and the camera centre the kernels use is the eye
    m = np.asarray(vp, np.float64).reshape(4, 4).T
    mi = np.asarray(vpi, np.float64).reshape(4, 4).T
    np.testing.assert_allclose(m @ mi, np.eye(4), atol=2e-4)
    np.testing.assert_allclose(view_records(vp[None], vpi[None])[0, 32:35], eye, atol=2e-4)


def test_sphere_cameras_look_at_origin():
    vp, vpi = camera.sphere_cameras(32, 4.0, math.radians(50.0), 1.0)
    eyes = camera.fibonacci_sphere(32, 4.0)
    np.testing.assert_allclose(np.linalg.norm(eyes, axis=1), 4.0, rtol=1e-12)
    for k in range(32):
        c = _clip(vp[k], (0.0, 0.0, 0.0))
        assert abs(c[0] / c[3]) < 1e-6 and abs(c[1] / c[3]) < 1e-6
        assert abs(c[3] - 4.0) < 1e-5
