"""CPU checks of the Python mirrors' surface: every public method of the
reference's manager classes has a counterpart under its own (camelCase) name,
and the host-side logic of the split VP writes and the shading-mode check
(methods called on stand-in objects; no library calls)."""
import types

import numpy as np
import pytest

from nprush_b200 import bezier, mesh_render, path_trace, splat, targets

# reference class -> (mirror class, public methods of the reference class)
REFERENCE_METHODS = {
    # GpuSplatOptimizerManager.ts:281-402 (addDraw is the viewer's screen draw: render())
    "GpuSplatOptimizerManager": (splat.GpuSplatOptimizerManager,
                                 ["writeSplatVPMatrix", "setBackwardTarget", "setEdgeTarget", "dispatch",
                                  "dispatchEdge"]),
    # GpuBezierOptimizerManager.ts:269-406
    "GpuBezierOptimizerManager": (bezier.GpuBezierOptimizerManager,
                                  ["writeVPMatrix", "writeVPInvMatrix", "writeMode", "writeBgPenalty", "writeMaxWidth",
                                   "writeKillThresholds", "setAdcPeriod", "writeNoKill", "setBackwardTarget",
                                   "dispatch"]),
    # GpuPathTracePipelineManager.ts:101-247
    "GpuPathTracePipelineManager": (path_trace.GpuPathTracePipelineManager,
                                    ["setMeshes", "setOutputSize", "reset", "writeInvViewProjMat", "dispatch"]),
    # GpuSplatForwardPipelineManager.ts:94-137, GpuBezierForwardPipelineManager.ts:102-148
    "GpuSplatForwardPipelineManager": (splat.GpuSplatForwardPipelineManager, ["writeVPMatrix", "setTarget", "dispatch"]),
    "GpuBezierForwardPipelineManager": (bezier.GpuBezierForwardPipelineManager,
                                        ["writeVPMatrix", "setTarget", "dispatch"]),
    # GpuBlurPipelineManager.ts:46-99, GpuDepthAwareBlurPipelineManager.ts:41-70
    "GpuBlurPipelineManager": (targets.GpuBlurPipelineManager, ["blur"]),
    "GpuDepthAwareBlurPipelineManager": (targets.GpuDepthAwareBlurPipelineManager, ["blur"]),
    # GpuMeshRenderPipelineManager.ts:127-247 and GpuUniformsBufferManager.ts:59-93
    # (addDraw of the mesh and envmap managers: render())
    "GpuMeshRenderPipelineManager": (mesh_render.GpuMeshRenderPipelineManager,
                                     ["setGroundMesh", "setPbrMesh", "writeViewProjMat", "writeViewMat",
                                      "writeShadingMode", "writeInvViewProjMat", "render"]),
}


@pytest.mark.parametrize("name", sorted(REFERENCE_METHODS))
def test_reference_methods_exist(name):
    cls, methods = REFERENCE_METHODS[name]
    missing = [m for m in methods if not callable(getattr(cls, m, None))]
    assert not missing, f"{name} mirror lacks {missing}"


def _bezier_stub():
    calls = []
    stub = types.SimpleNamespace(_vp=None, _vp_inv=None)

    def write_vp(vp, vpi):
        calls.append((np.array(vp), np.array(vpi)))
        stub._vp, stub._vp_inv = np.array(vp), np.array(vpi)

    stub.write_vp = write_vp
    return stub, calls


def test_split_vp_writes_keep_the_other_matrix():
    cls = bezier.GpuBezierOptimizerManager
    a = np.arange(16, dtype=np.float32)
    b = -np.arange(16, dtype=np.float32)
    stub, calls = _bezier_stub()
    cls.write_vp_matrix(stub, a)  # the inverse was never written: zeros
    np.testing.assert_array_equal(calls[-1][0], a.reshape(1, 16))
    np.testing.assert_array_equal(calls[-1][1], np.zeros((1, 16), np.float32))
    cls.write_vp_inv_matrix(stub, b)  # keeps the view-projection
    np.testing.assert_array_equal(calls[-1][0], a.reshape(1, 16))
    np.testing.assert_array_equal(calls[-1][1], b.reshape(1, 16))
    # a new number of views: the other matrix reads as zeros until it is written
    cls.write_vp_matrix(stub, np.stack([a, a]))
    assert calls[-1][0].shape == (2, 16) and not calls[-1][1].any()


def test_shading_mode_values():
    stub = types.SimpleNamespace(uniforms=np.full(52, 7.0, np.float32))
    mesh_render.MeshRenderer.write_shading_mode(stub, "normals")
    assert stub.uniforms[32] == 0.0
    mesh_render.MeshRenderer.write_shading_mode(stub, "shaded")
    assert stub.uniforms[32] == 1.0
    with pytest.raises(ValueError):
        mesh_render.MeshRenderer.write_shading_mode(stub, "phong")
