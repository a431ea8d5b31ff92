"""On-disk scene: trained primitives, their optimiser state, cameras and
meshes in one file that the reference's TypeScript viewer can read with
`fetch` / `Deno.readFile`, a `JSON.parse` and typed-array views — no parser
of its own.

Layout (little-endian):

    bytes 0-3    "NPSC"
    bytes 4-7    u32 format version (1)
    bytes 8-11   u32 header length H (bytes)
    bytes 12-15  0
    bytes 16..   UTF-8 JSON header, space-padded to a multiple of 16
    then one blob per array, each at a 16-byte aligned file offset

    header = {"format": "nprush-scene", "version": 1, "meta": {...},
              "arrays": {name: {"dtype": "f32" | "i32" | "u32",
                                "shape": [...], "offset": o, "bytes": b}}}

Arrays hold exactly the reference's GPU buffer layouts, so the viewer can
hand them to `device.queue.writeBuffer` as they are:

    splats              N x 16 f32   splatBuffer (splat_forward.wgsl:1-6)
    splats.adam_m/_v    N x 16 f32   adamBuffer's m and v halves
    splats.grad_accum   N f32        adcBuffer
    splats.grads        N x 16 i32   gradBuffer (fixed point)
    beziers             N x 20 f32   bezierBuffer (bezier_forward.wgsl:1-7)
    beziers.adam_m/_v   N x 18 f32
    beziers.grad_accum / .loss_accum   N f32
    beziers.grads       N x 18 i32, beziers.pixel_loss   i32 (the pixel-loss map)
    gaussians           N x 64 f32   3D Gaussian records (mean, log-scale,
                                     quaternion, opacity logit, SH)
    gaussians.adam_m/_v N x 64 f32
    cameras.view_proj / cameras.inv_view_proj   V x 16 f32 (column-major)
    mesh.vertices       V x 12 f32   MeshData.vertices (pos, normal, rgba, uv)
    mesh.indices        3T u32

and "meta" the scalars: Adam step counters (`splats.adam_t`,
`beziers.adam_t`, `gaussians.step`), dispatch counters (`splats.step_count`,
`beziers.step_count`), image size, SH degree.

    write_scene(path, splat_opt=..., bezier_opt=..., trainer=..., cameras=(vp, vp_inv), mesh=..., meta={...})
    sc = read_scene(path)          # arrays are read-only views of the file
    sc.restore_splats(opt); sc.restore_beziers(opt); sc.restore_gaussians(trainer)
"""
from __future__ import annotations

import json
import struct
from pathlib import Path

import numpy as np

MAGIC = b"NPSC"
VERSION = 1
_DT = {"f32": np.dtype("<f4"), "i32": np.dtype("<i4"), "u32": np.dtype("<u4")}
_NAME = {np.dtype(np.float32): "f32", np.dtype(np.int32): "i32", np.dtype(np.uint32): "u32"}


def _align(n: int, a: int = 16) -> int:
    return (n + a - 1) // a * a


def save(path, arrays: dict, meta: dict | None = None):
    """Writes `arrays` (name -> numpy array of f32 / i32 / u32) and `meta`."""
    arrays = {k: np.ascontiguousarray(v) for k, v in arrays.items() if v is not None}
    for k, v in arrays.items():
        if v.dtype not in _NAME:
            raise TypeError(f"{k}: dtype {v.dtype} (f32, i32 or u32 only)")
    desc = {}
    # offsets depend on the header length, which depends on the offsets'
    # digits: lay out twice with a generous header bound
    header_len = 0
    for _ in range(3):
        off = _align(16 + header_len)
        desc = {}
        for k, v in arrays.items():
            desc[k] = {"dtype": _NAME[v.dtype], "shape": list(v.shape), "offset": off, "bytes": int(v.nbytes)}
            off = _align(off + v.nbytes)
        hdr = json.dumps({"format": "nprush-scene", "version": VERSION, "meta": meta or {}, "arrays": desc},
                         sort_keys=True).encode()
        need = _align(len(hdr))
        if need <= header_len:
            break
        header_len = need + 64
    hdr = hdr.ljust(header_len, b" ")
    path = Path(path)
    tmp = path.with_suffix(path.suffix + ".tmp")
    with open(tmp, "wb") as f:
        f.write(MAGIC + struct.pack("<III", VERSION, header_len, 0))
        f.write(hdr)
        for k, v in arrays.items():
            f.seek(desc[k]["offset"])
            f.write(v.astype(v.dtype.newbyteorder("<"), copy=False).tobytes())
    tmp.replace(path)


class Scene:
    def __init__(self, arrays: dict, meta: dict):
        self.arrays, self.meta = arrays, meta

    def __getitem__(self, k):
        return self.arrays[k]

    def __contains__(self, k):
        return k in self.arrays

    # ---- restoring optimiser state
    def restore_splats(self, opt):
        """Into a GpuSplatOptimizerManager of the same size."""
        s = self.arrays["splats"]
        if s.shape[0] != opt.num_splats:
            raise ValueError(f"scene has {s.shape[0]} splats, the manager {opt.num_splats}")
        opt.write_params(np.array(s))
        opt.write_state(adam_m=np.array(self.arrays["splats.adam_m"]), adam_v=np.array(self.arrays["splats.adam_v"]),
                        adam_t=float(self.meta.get("splats.adam_t", 0.0)),
                        grad_accum=np.array(self.arrays["splats.grad_accum"]),
                        grads=np.array(self.arrays["splats.grads"]) if "splats.grads" in self.arrays else None)
        opt.set_step_count(int(self.meta.get("splats.step_count", 0)))

    def restore_beziers(self, opt):
        """Into a GpuBezierOptimizerManager of the same size."""
        b = self.arrays["beziers"]
        if b.shape[0] != opt.num_beziers:
            raise ValueError(f"scene has {b.shape[0]} curves, the manager {opt.num_beziers}")
        opt.write_params(np.array(b))
        opt.write_state(adam_m=np.array(self.arrays["beziers.adam_m"]), adam_v=np.array(self.arrays["beziers.adam_v"]),
                        adam_t=float(self.meta.get("beziers.adam_t", 0.0)),
                        grad_accum=np.array(self.arrays["beziers.grad_accum"]),
                        loss_accum=np.array(self.arrays["beziers.loss_accum"]),
                        grads=np.array(self.arrays["beziers.grads"]) if "beziers.grads" in self.arrays else None,
                        pixel_loss=(np.array(self.arrays["beziers.pixel_loss"])
                                    if "beziers.pixel_loss" in self.arrays else None))
        opt.set_step_count(int(self.meta.get("beziers.step_count", 0)))

    def restore_gaussians(self, trainer):
        """Into a GaussianTrainer with room for them."""
        g = self.arrays["gaussians"]
        if g.shape[0] > trainer.capacity:
            raise ValueError(f"scene has {g.shape[0]} Gaussians, the trainer room for {trainer.capacity}")
        trainer.write_params(np.array(g))
        if "gaussians.adam_m" in self.arrays:
            trainer.write_state(np.array(self.arrays["gaussians.adam_m"]), np.array(self.arrays["gaussians.adam_v"]),
                                int(self.meta.get("gaussians.step", 0)))


def load(path) -> Scene:
    data = np.memmap(path, dtype=np.uint8, mode="r")
    if bytes(data[:4]) != MAGIC:
        raise ValueError(f"{path}: not an nprush scene (magic {bytes(data[:4])!r})")
    version, header_len, _ = struct.unpack("<III", bytes(data[4:16]))
    if version != VERSION:
        raise ValueError(f"{path}: scene format version {version}, this reader knows {VERSION}")
    hdr = json.loads(bytes(data[16:16 + header_len]).decode())
    arrays = {}
    for k, d in hdr["arrays"].items():
        off, nbytes = int(d["offset"]), int(d["bytes"])
        if off % 16 or off + nbytes > data.size:
            raise ValueError(f"{path}: array {k} outside the file or misaligned")
        a = data[off:off + nbytes].view(_DT[d["dtype"]])
        arrays[k] = a.reshape(d["shape"])
    return Scene(arrays, hdr.get("meta", {}))


def write_scene(path, splat_opt=None, bezier_opt=None, trainer=None, cameras=None, mesh=None, meta=None):
    """Gathers the managers' state (and cameras / a mesh) into one file."""
    arrays, m = {}, dict(meta or {})
    if splat_opt is not None:
        st = splat_opt.read_state()
        arrays.update({"splats": st["splats"], "splats.adam_m": st["adam_m"], "splats.adam_v": st["adam_v"],
                       "splats.grad_accum": st["grad_accum"], "splats.grads": st["grads"]})
        m["splats.adam_t"] = float(st["adam_t"])
        m["splats.step_count"] = int(splat_opt.stats()["step_count"])
    if bezier_opt is not None:
        st = bezier_opt.read_state()
        arrays.update({"beziers": st["beziers"], "beziers.adam_m": st["adam_m"], "beziers.adam_v": st["adam_v"],
                       "beziers.grad_accum": st["grad_accum"], "beziers.loss_accum": st["loss_accum"],
                       "beziers.grads": st["grads"], "beziers.pixel_loss": st["pixel_loss"]})
        m["beziers.adam_t"] = float(st["adam_t"])
        m["beziers.step_count"] = int(bezier_opt.stats()["step_count"])
    if trainer is not None:
        st = trainer.read_state()
        arrays.update({"gaussians": st["params"], "gaussians.adam_m": st["adam_m"], "gaussians.adam_v": st["adam_v"]})
        m["gaussians.sh_degree"] = int(trainer.sh_degree)
        m["gaussians.step"] = int(trainer.stats()["step_count"])  # Adam steps taken
    if cameras is not None:
        vp, vpi = cameras
        arrays["cameras.view_proj"] = np.asarray(vp, np.float32).reshape(-1, 16)
        arrays["cameras.inv_view_proj"] = np.asarray(vpi, np.float32).reshape(-1, 16)
    if mesh is not None:
        arrays["mesh.vertices"] = np.asarray(mesh.vertices, np.float32).reshape(-1, 12)
        arrays["mesh.indices"] = np.asarray(mesh.indices, np.uint32).reshape(-1)
    save(path, arrays, m)


def read_scene(path) -> Scene:
    return load(path)
