"""Build recipe of libnebula_b200.so: every CUDA source compiled for sm_100a with nvcc.

FP64 sources are compiled without fused multiply-add so the double-precision path rounds like
the reference; the FP32 pair passes keep fused multiply-add.  The library is written in place
(next to this file) so it travels with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libnebula_b200.so")
OBJ = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "--expt-relaxed-constexpr", "-Xptxas", "-O3"]  # fmt: skip
# source -> fused multiply-add allowed
SOURCES = {
    "neighbours.cu": False,
    "sph64.cu": False,
    "sph32.cu": True,
    "gravity.cu": False,
    "engine.cu": False,
    "steps.cu": False,
    "capi.cu": False,
    "noalloc.cu": False,
    "mlp.cu": True,
    "deposit.cu": False,
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "nebula_b200.h"))
    objs = []
    for src, fma in SOURCES.items():
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(obj)
        if not _stale(obj, [path, *headers, __file__]):
            continue
        cmd = [nvcc(), *ARCH, *COMMON, "-fmad=true" if fma else "-fmad=false", "-c", path, "-o",
               obj, *(extra or [])]  # fmt: skip
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-cudart=static", *objs, "-o", LIB]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
