"""The on-disk scene container (nprush_b200/scene.py): round trips, the
layout a TypeScript reader relies on (magic, version, JSON header, 16-byte
aligned little-endian blobs), and rejection of foreign or damaged files."""
import json
import struct

import numpy as np
import pytest

from nprush_b200 import scene


def sample_arrays(rng):
    return {
        "splats": rng.random((37, 16)).astype(np.float32),
        "splats.adam_m": rng.random((37, 16)).astype(np.float32),
        "beziers": rng.random((5, 20)).astype(np.float32),
        "gaussians": rng.random((11, 64)).astype(np.float32),
        "cameras.view_proj": rng.random((3, 16)).astype(np.float32),
        "mesh.indices": rng.integers(0, 1000, 3 * 7).astype(np.uint32),
        "grads": rng.integers(-5, 5, (4, 18)).astype(np.int32),
        "empty": np.zeros((0, 16), np.float32),
    }


def test_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    arrays = sample_arrays(rng)
    meta = {"splats.adam_t": 12.0, "splats.step_count": 50, "note": "x" * 300}
    scene.save(tmp_path / "a.npsc", arrays, meta)
    sc = scene.load(tmp_path / "a.npsc")
    assert sc.meta == meta
    assert set(sc.arrays) == set(arrays)
    for k, v in arrays.items():
        assert sc[k].dtype == v.dtype and sc[k].shape == v.shape
        np.testing.assert_array_equal(sc[k], v)


def test_layout_for_a_typescript_reader(tmp_path):
    """What `new Float32Array(buf.buffer, off, n)` needs: the fields at the
    documented offsets, every blob 16-byte aligned, little-endian."""
    rng = np.random.default_rng(1)
    arrays = sample_arrays(rng)
    scene.save(tmp_path / "b.npsc", arrays, {"w": 64})
    raw = (tmp_path / "b.npsc").read_bytes()
    assert raw[:4] == b"NPSC"
    version, hlen, zero = struct.unpack("<III", raw[4:16])
    assert version == 1 and zero == 0 and hlen % 16 == 0
    hdr = json.loads(raw[16:16 + hlen].decode())
    assert hdr["format"] == "nprush-scene" and hdr["meta"] == {"w": 64}
    for k, d in hdr["arrays"].items():
        assert d["offset"] % 16 == 0 and d["offset"] >= 16 + hlen
        v = np.frombuffer(raw, dtype={"f32": "<f4", "i32": "<i4", "u32": "<u4"}[d["dtype"]],
                          count=d["bytes"] // 4, offset=d["offset"]).reshape(d["shape"])
        np.testing.assert_array_equal(v, arrays[k])


def test_rejects_foreign_and_damaged_files(tmp_path):
    p = tmp_path / "c.npsc"
    p.write_bytes(b"PLY\n" + b"\0" * 64)
    with pytest.raises(ValueError):
        scene.load(p)
    scene.save(p, {"x": np.ones(4, np.float32)})
    raw = bytearray(p.read_bytes())
    raw[4:8] = struct.pack("<I", 99)
    p.write_bytes(bytes(raw))
    with pytest.raises(ValueError):
        scene.load(p)
    scene.save(p, {"x": np.ones(4096, np.float32)})
    p.write_bytes(p.read_bytes()[:-100])  # truncated
    with pytest.raises(ValueError):
        scene.load(p)
    with pytest.raises(TypeError):
        scene.save(p, {"x": np.ones(4, np.float64)})


class _FakeSplatOpt:
    """The calls write_scene / restore_splats make, on host arrays."""

    def __init__(self, n, rng=None):
        self.num_splats = n
        z = np.zeros((n, 16), np.float32)
        self.state = dict(splats=z.copy(), grads=np.zeros((n, 16), np.int32), adam_m=z.copy(), adam_v=z.copy(),
                          adam_t=0.0, grad_accum=np.zeros(n, np.float32))
        if rng is not None:
            for k in ("splats", "adam_m", "adam_v"):
                self.state[k] = rng.random((n, 16)).astype(np.float32)
            self.state["grad_accum"] = rng.random(n).astype(np.float32)
            self.state["adam_t"] = 7.0
        self.steps = 0 if rng is None else 33

    def read_state(self):
        return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.state.items()}

    def stats(self):
        return {"step_count": self.steps}

    def write_params(self, s):
        self.state["splats"] = np.array(s)

    def write_state(self, adam_m=None, adam_v=None, adam_t=0.0, grad_accum=None, grads=None):
        self.state.update(adam_m=np.array(adam_m), adam_v=np.array(adam_v), adam_t=adam_t,
                          grad_accum=np.array(grad_accum), grads=np.array(grads))

    def set_step_count(self, n):
        self.steps = n


def test_write_and_restore_through_the_manager_calls(tmp_path):
    from nprush_b200 import camera, meshes
    rng = np.random.default_rng(2)
    a, b = _FakeSplatOpt(19, rng), _FakeSplatOpt(19)
    vp, vpi = camera.sphere_cameras(4, 3.0, 0.9, 1.0)
    mesh = meshes.box((0, 0, 0), 1.0)
    scene.write_scene(tmp_path / "d.npsc", splat_opt=a, cameras=(vp, vpi), mesh=mesh, meta={"width": 256})
    sc = scene.read_scene(tmp_path / "d.npsc")
    sc.restore_splats(b)
    for k in ("splats", "adam_m", "adam_v", "grad_accum", "grads"):
        np.testing.assert_array_equal(b.state[k], a.state[k])
    assert b.state["adam_t"] == 7.0 and b.steps == 33
    np.testing.assert_array_equal(sc["cameras.inv_view_proj"], vpi.astype(np.float32))
    np.testing.assert_array_equal(sc["mesh.indices"], mesh.indices)
    assert sc.meta["width"] == 256
    with pytest.raises(ValueError):
        sc.restore_splats(_FakeSplatOpt(20))
