"""Build the engine's shared library in-tree: radtranbook_b200/libimcb200.so (sm_100a).

Each CUDA source is compiled separately (the FP64 bookkeeping file without FMA
contraction, so its per-cell numbers match the CPU oracle exactly) and linked into one
shared object whose exported symbols are the C ABI of include/imcb200.h.

build(checked=True) makes the bounds-checked variant libimcb200_checked.so (every source
compiled with IMC_CHECKED: the tracking and comb kernels verify cell, group and bin indices
and particle weights, skip an access that fails and report IMC_FLAG_BOUNDS).  The library
loader picks it when the environment sets IMCB200_CHECKED=1.
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libimcb200.so"
LIB_CHECKED = HERE / "libimcb200_checked.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]
PER_FILE = {"imc_bookkeeping.cu": ["-fmad=false"], "imc_batch_plan.cu": ["-fmad=false"]}
SOURCES = ["imc_capi.cu", "imc_bookkeeping.cu", "imc_source.cu", "imc_transport.cu", "imc_comb.cu",
           "imc_batch.cu", "imc_batch_plan.cu", "imc_adjoint.cu"]
HEADERS = ["imc_device.cuh", "imc_internal.h", "imc_block.cuh", "imc_sample.cuh", "imc_batch.h"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libimcb200.so")
    return path


def _stale(target: pathlib.Path, deps: list[pathlib.Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None,
          checked: bool = False) -> pathlib.Path:
    bdir = BUILD / "checked" if checked else BUILD
    lib = LIB_CHECKED if checked else LIB
    extra = (extra or []) + (["-DIMC_CHECKED"] if checked else [])
    bdir.mkdir(parents=True, exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [HERE.parent / "include" / "imcb200.h"]
    objs = []
    for src in SOURCES:
        s = CSRC / src
        o = bdir / (s.stem + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc(), *ARCH, *COMMON, *PER_FILE.get(src, []), *(extra or []), "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(lib, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(lib), *map(str, objs)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    import sys

    print(build(force="--force" in sys.argv, verbose=True))
    print(build(force="--force" in sys.argv, verbose=True, checked=True))
