"""Builds the CUDA library libblacktracer_b200.so in-tree for sm_100a.

Each translation unit has its own flags: the plain FP64 integrator and the
grid builder are compiled with --fmad=false so their double arithmetic rounds
like the reference's host build; the mixed integrator and the per-pixel map
keep FMA contraction.

    python -m blacktracer_b200.build [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libblacktracer_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
          "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]

# translation unit -> extra flags
UNITS = {
    "integrate.cu": ["--fmad=false"],
    "grid.cu": ["--fmad=false"],
    "mixed.cu": [],
    "map.cu": ["--fmad=false"],
    "stars.cu": ["--fmad=false"],
    "map_api.cu": [],
    "noalloc.cu": [],
    "server.cu": [],
    "cache.cu": [],
    "trails.cu": ["--fmad=false"],
}
HEADERS = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
           if f.endswith((".h", ".cuh"))] + [os.path.join(ROOT, "include", "blacktracer.h")]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OBJ, exist_ok=True)
    objs, cmds = [], []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(OBJ, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [src] + HEADERS + [__file__]):
            cmd = [NVCC] + ARCH + COMMON + flags + ["-c", src, "-o", obj]
            if verbose:
                cmd += ["-Xptxas", "-v"]
                print(" ".join(cmd), file=sys.stderr)
            cmds.append(cmd)
    # translation units compile independently
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        list(ex.map(lambda c: subprocess.run(c, check=True), cmds))
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
