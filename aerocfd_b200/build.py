"""Builds libaerocfd_gpu.so in-tree for sm_100a with nvcc.

    python -m aerocfd_b200.build          # incremental
    python -m aerocfd_b200.build --clean  # rebuild everything

FP64 parity needs the reference's operation order, so the kernels are compiled
with -fmad=false (no contraction of separate multiplies and adds).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libaerocfd_gpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["aero_flux.cu", "aero_implicit.cu", "aero_bc.cu", "aero_transfer.cu",
           "aero_runtime.cu", "aero_topology.cpp", "aero_geometry.cu", "aero_sa.cu",
           "aero_noalloc.cu", "aero_forces.cu", "aero_crank.cu", "aero_mlp.cu", "aero_crmath.cu"]
HEADERS = ["aero_device.cuh", "aero_kernels.h", "aero_topology.h", "aero_mlp_gemm.cuh", "aero_crmath.h",
           "aero_crmath_tables.h"]
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
         "-I" + INCLUDE, "-I" + CSRC]


def _newer(src: str, dst: str, deps) -> bool:
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(p) > t for p in [src, *deps])


def build(clean: bool = False, verbose: bool = False) -> str:
    if clean and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "aerocfd_gpu.h")]
    objs = []
    rebuilt = False
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, os.path.splitext(s)[0] + ".o")
        objs.append(obj)
        if _newer(src, obj, deps):
            cmd = [NVCC, "-x", "cu", *ARCH, *FLAGS, "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
            rebuilt = True
    if rebuilt or not os.path.exists(LIB):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.clean, a.verbose))
    sys.exit(0)
