"""Build libpantometry_b200.so in-tree for sm_100a with nvcc.

The plain f64 kernels (plain_f64.cu) are compiled with --fmad=false so that no multiply-add is
contracted; every other unit keeps nvcc's default. The CUDA runtime is linked statically, so the
library needs only the driver at run time.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libpantometry_b200.so")
BUILD = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]
UNITS = {
    "plain_f64.cu": ["--fmad=false"],
    "fields_f32.cu": [],
    "runtime.cu": [],
    "heat.cu": [],
    "hall.cu": [],
    "room.cu": [],
    "tube.cu": [],
    "bar.cu": [],
    "cavity.cu": [],
    "ensemble.cu": [],
    "noalloc.cu": [],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build pantometry_b200")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "pantometry_gpu.h"))
    objs = []
    cc = nvcc()
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [cc, *ARCH, *COMMON, *flags, "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    if force or _stale(OUT, objs):
        cmd = [cc, *ARCH, "-shared", "-o", OUT, *objs, "-cudart", "static"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
