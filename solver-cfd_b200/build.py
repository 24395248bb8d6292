"""Build recipe of the CUDA library ``libacs_b200.so`` (sm_100a) next to this file.

Every CUDA source is compiled by nvcc for ``-gencode arch=compute_100a,code=sm_100a``;
``kernels_exact.cu`` and the boundary/control kernels are compiled with ``-fmad=false`` so each
product and sum is rounded separately, as in the reference arithmetic.  Objects go to
``_build/`` beside this file; the shared library is written in-tree so it travels with the
source tree.  Usage: ``python build.py [--force] [--verbose]``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libacs_b200.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
               "-I", os.path.join(ROOT, "include")] + ARCH

# source -> extra flags
SOURCES = {
    "kernels_exact.cu": ["-fmad=false"],
    "engine_exact.cu": ["-fmad=false"],
    "control.cu": ["-fmad=false"],
    "output.cu": ["-fmad=false"],
    "mesh_device.cu": [],
    "engine_fast.cu": [],
    "kernels_fast.cu": [],
    "tile_engine.cu": [],
    "fast_tables.cu": [],
    "noalloc.cu": [],
    "warmstart.cu": ["-fmad=false"],
    "solver.cu": [],
    "../unet/csrc/unet_gemm.cu": [],
    "../unet/csrc/unet_ops.cu": [],
}
CXX_SOURCES = {"mesh.cpp": ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off"]}
HEADERS = [os.path.join(ROOT, "include", "unet.h"), "acs_dev.cuh", "kernels.h", "fast.h", "engine.cuh", "engine_api.h", "points_exact.cuh", "points_fast.cuh", "bc_exact.cuh", "warmstart.h", "tile_engine.h",
           "../unet/csrc/gemm_tc.cuh"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "acs.h")]
    objs = []
    for src, extra in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs + [__file__]):
            cmd = [nvcc(), "-c", s, "-o", o] + NVCC_COMMON + extra
            if verbose:
                cmd += ["-Xptxas", "-v"]
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    for src, flags in CXX_SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs + [__file__]):
            cmd = ["g++", "-c", s, "-o", o, "-I", os.path.join(ROOT, "include")] + flags
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _newer(LIB, objs):
        cmd = [nvcc(), "-shared", "-o", LIB] + objs + ARCH + ["-lcuda"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
