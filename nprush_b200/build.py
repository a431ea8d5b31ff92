"""Builds libnprush_cuda.so in-tree with nvcc for sm_100a.

    python -m nprush_b200.build [--force]

Sources in nprush_b200/csrc are compiled separately (files whose kernels
reproduce the reference's fp32 operation order get --fmad=false) and linked
into nprush_b200/libnprush_cuda.so with the CUDA runtime linked statically.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "libnprush_cuda.so"
BUILD_DIR = HERE / "_build"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=default",
          f"-I{HERE.parent / 'include'}"]
# reference-semantics kernels: keep every fp32 operation separately rounded
NO_FMAD = {"compat_splat.cu", "compat_bezier.cu", "binning.cu", "path_trace.cu", "mesh_raster.cu"}


def sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _needs(obj: Path, deps) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD_DIR.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "nprush.h"]
    objs = []
    for src in sources():
        obj = BUILD_DIR / (src.name + ".o")
        objs.append(obj)
        if not force and not _needs(obj, [src] + headers):
            continue
        flags = list(COMMON) + ARCH
        if src.name in NO_FMAD:
            flags += ["--fmad=false", "-Xcompiler", "-ffp-contract=off"]
        cmd = [NVCC] + flags + ["-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    if force or _needs(OUT, objs):
        tmp = str(OUT) + ".tmp"
        cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + [str(o) for o in objs] + ["-lcudart_static", "-lrt", "-ldl",
                                                                                "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(p)
