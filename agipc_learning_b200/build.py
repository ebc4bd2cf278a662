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
    """Compile every ``csrc/*.cu`` to an object under ``_build/`` (in parallel;
    a source is recompiled when it or any shared header changed), then link
    ``libmaspcg.so``.  No file shares device symbols with another, so the
    objects are whole-program device code and need no device link step."""
    from concurrent.futures import ThreadPoolExecutor

    out = os.path.join(HERE, "libmaspcg.so")
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + sorted(glob.glob(os.path.join(INCLUDE, "*.h")))
    objdir = os.path.join(ROOT, "_build", "maspcg")
    os.makedirs(objdir, exist_ok=True)
    flags = [*NVCC_ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler",
             "-fvisibility=hidden", "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC, *extra]
    if verbose_ptxas:
        flags.insert(0, "-Xptxas=-v")
    objs = [os.path.join(objdir, os.path.basename(s)[:-3] + ".o") for s in srcs]
    todo = [(s, o) for s, o in zip(srcs, objs) if force or verbose_ptxas or extra or _newer(o, [s, *headers])]
    if not todo and not _newer(out, objs):
        return out

    def compile_one(so):
        src, obj = so
        return subprocess.run([_nvcc(), *flags, "-c", "-o", obj, src], capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, todo))
    for (src, _), r in zip(todo, results):
        if verbose_ptxas or r.returncode:
            print(r.stdout + r.stderr)
        if r.returncode:
            raise subprocess.CalledProcessError(r.returncode, f"nvcc {src}")
    subprocess.run([_nvcc(), *NVCC_ARCH, "-shared", "-o", out, *objs, "-lcudart"], check=True)
    return out


def build_all(force: bool = False) -> None:
    build_synth(force)
    build_cuda(force)


if __name__ == "__main__":
    import sys
    build_all(force="--force" in sys.argv)
