"""In-tree build of the native libraries.

* ``libmaspcg.so``  -- the CUDA solver behind ``include/maspcg.h`` (sm_100a).
* ``libmassynth.so`` -- host C generator of the synthetic Newton systems.

Both land next to this file so that they travel with the source tree.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_synth(force: bool = False) -> str:
    out = os.path.join(HERE, "libmassynth.so")
    src = [os.path.join(CSRC, "synth.c")]
    if force or _newer(out, src):
        subprocess.run(["gcc", "-O2", "-fPIC", "-fopenmp", "-std=c11", "-Wall", "-shared", "-o", out, *src, "-lm"],
                       check=True)
    return out


def build_cuda(force: bool = False, verbose_ptxas: bool = False, extra=()) -> str:
    out = os.path.join(HERE, "libmaspcg.so")
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    deps = srcs + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + sorted(glob.glob(os.path.join(INCLUDE, "*.h")))
    if not (force or _newer(out, deps)):
        return out
    cmd = [_nvcc(), *NVCC_ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC,
           "-o", out, *srcs, "-lcudart"]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    cmd.extend(extra)
    subprocess.run(cmd, check=True)
    return out


def build_all(force: bool = False) -> None:
    build_synth(force)
    build_cuda(force)


if __name__ == "__main__":
    import sys
    build_all(force="--force" in sys.argv)
