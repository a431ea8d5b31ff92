"""Build recipe for oracle/_ref: the reference's own WGSL compute shaders,
translated to C++ (oracle/wgsl2cpp.py) and compiled with g++ for the host.

TEST INFRASTRUCTURE ONLY.  Reads the reference checkout (the directory named
by NPRUSH_REFERENCE, else the one in oracle/reference_path.txt) at build time;
outputs go only
to oracle/_ref/ (git-ignored).  Sizes are baked into the shaders exactly as the
reference bakes them at pipeline creation (`{@NUM_SPLATS}` etc.), so one shared
object is built per (shader, size) and cached by content hash.

Each shared object exports:
  wg_bind(group, binding, void*)          storage / uniform buffer binding
  wg_bind_tex(group, binding, rgba*, w, h) texture_2d<f32> binding (fp32 RGBA)
  wg_bind_storage_tex(group, binding, rgba*, w, h) texture_storage_2d output (the stored floats)
  wg_bind_sampler(group, binding, linear, address_u, address_v)  sampler state (address 0 clamp, 1 repeat)
  wg_size(unsigned[3])                    @workgroup_size
  wg_run_one(x, y, z, gx, gy, gz)         run one workgroup to completion
  wg_dispatch(gx, gy, gz)                 run all workgroups in x-fastest order
  call_<fn>(in*, out*), size_<fn>(o[2])   a @vertex / @fragment function of one input
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import re
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_OUT = HERE / "_ref"
SHADERS = ("splat_backward", "splat_step", "splat_adc", "bezier_backward", "bezier_step", "bezier_adc")
# target preprocessing (GpuBlurPipelineManager, GpuDepthAwareBlurPipelineManager, the splat edge pass):
# no size baked in (built with n = 0)
IMAGE_SHADERS = ("blur", "depth_aware_blur", "splat_edge", "path_trace", "path_trace_resolve")
# render pipelines: their @vertex / @fragment functions, callable one invocation at a time
# (the display forwards with their instance count baked in, as their managers inject it)
STAGE_SHADERS = ("mesh", "envmap", "splat_forward", "bezier_forward")


REF_PATH_FILE = HERE / "reference_path.txt"


def reference_root() -> Path:
    """The reference checkout: $NPRUSH_REFERENCE, else the first line of
    oracle/reference_path.txt (where this build's checkout lies)."""
    env = os.environ.get("NPRUSH_REFERENCE")
    if env:
        return Path(env)
    if REF_PATH_FILE.is_file():
        line = REF_PATH_FILE.read_text().strip().splitlines()
        if line:
            return Path(line[0].strip())
    return HERE / "_no_reference_configured"



def reference_available() -> bool:
    return (reference_root() / "src/lib/gpu/splat_backward.wgsl").is_file()


def gpu_constants() -> dict:
    """GPU_CONSTANTS parsed from the reference's src/lib/gpu/constants.ts:5-42."""
    text = (reference_root() / "src/lib/gpu/constants.ts").read_text()
    body = text[text.index("GPU_CONSTANTS = {"):]
    body = body[: body.index("};")]
    out = {}
    for m in re.finditer(r"^\s*([A-Z0-9_]+)\s*:\s*([^,/\n]+),", body, re.M):
        expr = m.group(2).strip()
        if not re.fullmatch(r"[0-9eE.+\-*/ ()]+", expr):
            raise ValueError(f"unexpected constant expression {expr!r}")
        out[m.group(1)] = eval(expr, {"__builtins__": {}})  # numeric literal arithmetic only
    return out


def splat_consts(n: int) -> dict:
    # GpuSplatOptimizerManager.ts:127-136
    c = dict(gpu_constants())
    c.update(NUM_SPLATS=n, NUM_SPLATS_PLUS_ONE=n + 1, NUM_SPLATS_MINUS_ONE=n - 1,
             NUM_SPLATS_DIV_32=-(-n // 32), NUM_PARAMS=n * 16)
    return c


def bezier_consts(n: int) -> dict:
    # GpuBezierOptimizerManager.ts:146-158 (OPTIM_WIDTH/HEIGHT are baked as 256)
    c = dict(gpu_constants())
    c.update(NUM_BEZIERS=n, NUM_BEZIERS_PLUS_ONE=n + 1, NUM_BEZIERS_MINUS_ONE=n - 1,
             NUM_BEZIERS_DIV_32=-(-n // 32), NUM_BEZIER_PARAMS=n * 18,
             PIXEL_LOSS_SIZE=c["PIXEL_LOSS_MAX"], OPTIM_WIDTH=256, OPTIM_HEIGHT=256)
    return c


def build(shader: str, n: int) -> Path:
    """Translate + compile `shader` with N baked in; returns the .so path."""
    from wgsl2cpp import TRANSLATOR_VERSION, translate  # noqa: local import (sys.path set by caller)

    if shader not in SHADERS + IMAGE_SHADERS + STAGE_SHADERS:
        raise ValueError(shader)
    src_path = reference_root() / "src/lib/gpu" / f"{shader}.wgsl"
    src = src_path.read_text()
    if shader in IMAGE_SHADERS + STAGE_SHADERS:
        consts = dict(gpu_constants())
        if shader == "splat_forward":  # GpuSplatForwardPipelineManager.ts:45-48
            consts["NUM_SPLATS"] = n
        elif shader == "bezier_forward":  # GpuBezierForwardPipelineManager.ts:58-61
            consts["NUM_BEZIERS"] = n
    else:
        consts = splat_consts(n) if shader.startswith("splat") else bezier_consts(n)
    rt = (HERE / "wgsl_rt.h").read_text()
    key = hashlib.sha256(
        (src + repr(sorted(consts.items())) + TRANSLATOR_VERSION + rt + (HERE / "wgsl2cpp.py").read_text()).encode()
    ).hexdigest()[:16]
    REF_OUT.mkdir(exist_ok=True)
    so = REF_OUT / f"{shader}_n{n}_{key}.so"
    if so.exists():
        return so
    cpp = REF_OUT / f"{shader}_n{n}_{key}.cpp"
    cpp.write_text(translate(src, consts, f"src/lib/gpu/{shader}.wgsl"))
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
           "-w", f"-I{HERE}", "-o", str(so) + ".tmp", str(cpp)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed for {shader}:\n{r.stderr[-4000:]}")
    os.replace(str(so) + ".tmp", so)
    # one build per (shader, n): readers without the reference checkout (bench.py on
    # another machine) find it by name
    for old in REF_OUT.glob(f"{shader}_n{n}_*"):
        if not old.name.startswith(f"{shader}_n{n}_{key}"):
            old.unlink(missing_ok=True)
    return so


def load_ts(name: str):
    """The reference's host-side TypeScript module src/lib/gpu/<name>.ts,
    translated to Python by oracle/ts2py.py (cached under oracle/_ref, one
    translation per source) and imported."""
    import importlib.util
    import sys

    from ts2py import TS2PY_VERSION, translate  # noqa: local import (sys.path set by caller)

    if str(HERE) not in sys.path:
        sys.path.insert(0, str(HERE))  # js_rt
    REF_OUT.mkdir(exist_ok=True)
    src_path = reference_root() / "src/lib/gpu" / f"{name}.ts"
    if src_path.exists():
        src = src_path.read_text()
        key = hashlib.sha256((src + TS2PY_VERSION + (HERE / "ts2py.py").read_text()
                              + (HERE / "js_rt.py").read_text()).encode()).hexdigest()[:16]
        py = REF_OUT / f"{name}_ts_{key}.py"
        if not py.exists():
            tmp = py.with_suffix(f".{os.getpid()}.tmp")
            tmp.write_text(translate(src, f"src/lib/gpu/{name}.ts"))
            os.replace(tmp, py)
            for old in REF_OUT.glob(f"{name}_ts_*.py"):
                if old != py:
                    old.unlink(missing_ok=True)
    else:
        found = sorted(REF_OUT.glob(f"{name}_ts_*.py"))
        if not found:
            raise FileNotFoundError(f"{src_path} absent and no translation in {REF_OUT}")
        py = found[-1]
    spec = importlib.util.spec_from_file_location(py.stem, py)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class RefModule:
    """ctypes handle on one compiled reference shader."""

    def __init__(self, shader: str, n: int, path=None):
        import sys
        if str(HERE) not in sys.path:
            sys.path.insert(0, str(HERE))
        self.path = Path(path) if path is not None else build(shader, n)
        self.lib = ctypes.CDLL(str(self.path))
        self.lib.wg_bind.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        self.lib.wg_bind_tex.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint]
        self.lib.wg_bind_storage_tex.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint,
                                                 ctypes.c_uint]
        self.lib.wg_bind_sampler.argtypes = [ctypes.c_int] * 5
        self.lib.wg_run_one.argtypes = [ctypes.c_uint] * 6
        self.lib.wg_dispatch.argtypes = [ctypes.c_uint] * 3
        ws = (ctypes.c_uint * 3)()
        self.lib.wg_size(ws)
        self.wgsize = tuple(ws)
        self._keep = []

    @classmethod
    def from_path(cls, path):
        """Loads an already built module (no reference checkout needed)."""
        return cls("", 0, path=path)

    def bind(self, binding: int, arr, group: int = 0):
        self._keep.append(arr)
        self.lib.wg_bind(group, binding, arr.ctypes.data)

    def bind_tex(self, binding: int, rgba, group: int = 0):
        assert rgba.dtype.name == "float32" and rgba.ndim == 3 and rgba.shape[2] == 4 and rgba.flags.c_contiguous
        self._keep.append(rgba)
        self.lib.wg_bind_tex(group, binding, rgba.ctypes.data, rgba.shape[1], rgba.shape[0])

    def bind_storage_tex(self, binding: int, rgba, group: int = 0):
        """Output texture: receives the float values the shader stores (before
        the texture format's conversion)."""
        assert rgba.dtype.name == "float32" and rgba.ndim == 3 and rgba.shape[2] == 4 and rgba.flags.c_contiguous
        self._keep.append(rgba)
        self.lib.wg_bind_storage_tex(group, binding, rgba.ctypes.data, rgba.shape[1], rgba.shape[0])

    def bind_sampler(self, binding: int, linear: bool = True, address_u: str = "clamp-to-edge",
                     address_v: str = "clamp-to-edge", group: int = 0):
        mode = {"clamp-to-edge": 0, "repeat": 1}
        self.lib.wg_bind_sampler(group, binding, int(bool(linear)), mode[address_u], mode[address_v])

    def call(self, fn: str, arg):
        """Runs the @vertex / @fragment function `fn` on one input (its bytes
        in `arg`); returns the result as float32."""
        sizes = (ctypes.c_uint * 2)()
        getattr(self.lib, f"size_{fn}")(sizes)
        a = np.ascontiguousarray(arg)
        assert a.nbytes == sizes[0], (fn, a.nbytes, sizes[0])
        out = np.zeros(sizes[1] // 4, np.float32)
        f = getattr(self.lib, f"call_{fn}")
        f.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        f(a.ctypes.data, out.ctypes.data)
        return out

    def discarded(self) -> bool:
        """Whether the last call() ended in `discard`."""
        return bool(self.lib.wg_discarded())

    def dispatch(self, gx: int, gy: int = 1, gz: int = 1):
        self.lib.wg_dispatch(gx, gy, gz)

    def run_one(self, x, y, z, gx, gy, gz):
        self.lib.wg_run_one(x, y, z, gx, gy, gz)


if __name__ == "__main__":
    import sys
    sys.path.insert(0, str(HERE))
    for sh in SHADERS:
        print(build(sh, 64))
