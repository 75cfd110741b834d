"""Build the CPU oracle (test infrastructure only): oracle/liboracle.so from imc_oracle.cpp.

Plain g++ with OpenMP; no FMA (x86-64 baseline ISA), so its FP64 bookkeeping matches the
CUDA path's FMA-free bookkeeping kernels operation for operation.
"""
from __future__ import annotations

import pathlib
import shutil
import subprocess

HERE = pathlib.Path(__file__).resolve().parent
SRC = HERE / "imc_oracle.cpp"
LIB = HERE / "liboracle.so"


def build(force: bool = False) -> pathlib.Path:
    deps = [SRC, HERE / "philox_ref.h"]
    if force or not LIB.exists() or any(d.stat().st_mtime > LIB.stat().st_mtime for d in deps):
        gxx = shutil.which("g++") or "g++"
        subprocess.run([gxx, "-O2", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off", "-std=c++17",
                        "-o", str(LIB), str(SRC)], check=True)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
