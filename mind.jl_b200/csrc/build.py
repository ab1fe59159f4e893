"""Build libmindgpu.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

    python mind.jl_b200/csrc/build.py [--verbose]

-fmad=false keeps every FP64 rounding step the one the source writes, which is
what makes the FP64 mode reproduce the CPU oracle bit for bit; fused
multiply-adds are written out with fma() where wanted.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PACKAGE = os.path.dirname(HERE)
OUT_DIR = os.path.join(PACKAGE, "lib")
OUTPUT = os.path.join(OUT_DIR, "libmindgpu.so")
SOURCES = [os.path.join(HERE, "mindgpu.cu"), os.path.join(HERE, "surrogate.cu"), os.path.join(HERE, "planner.cpp")]
DEPENDS = SOURCES + [os.path.join(HERE, f) for f in ("device.cuh", "kernels.cuh", "macro.cuh", "mind_math.h",
                                                     "gen_runtime.cuh", "generated_mechanisms.cuh", "mlp_umma.cuh")] + [
    os.path.join(os.path.dirname(PACKAGE), "include", "mindgpu.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-shared", "-cudart", "shared",
]


def nvcc() -> str:
    for candidate in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if candidate and (os.path.sep not in candidate or os.path.exists(candidate)):
            return candidate
    return "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(OUTPUT):
        return False
    built = os.path.getmtime(OUTPUT)
    return all(os.path.getmtime(p) <= built for p in DEPENDS if os.path.exists(p))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUTPUT
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [nvcc(), *NVCC_FLAGS, *(["-Xptxas", "-v"] if verbose else []), "-o", OUTPUT, *SOURCES, "-ldl"]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed ({result.returncode}):\n{result.stderr}\n{result.stdout}")
    if verbose:
        sys.stderr.write(result.stderr)
    return OUTPUT


if __name__ == "__main__":
    print(build(force=True, verbose="--verbose" in sys.argv))
