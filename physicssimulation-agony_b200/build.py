"""Builds libag2d.so (the CUDA library behind include/ag2d.h) in-tree for sm_100a.

Every kernel is compiled with --fmad=false: the pipeline reproduces the reference's fp32 operation order, so the
compiler may not contract a*b+c into an FMA (the one FMA the reference issues is written explicitly). Division
and square root stay IEEE-rounded (-prec-div/-prec-sqrt are nvcc's defaults without --use_fast_math, and are
passed explicitly). Host code gets -ffp-contract=off for the same reason (object creation arithmetic).

    python physicssimulation-agony_b200/build.py [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "ag2d", "libag2d.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
              "-Xcompiler", "-fPIC,-ffp-contract=off", f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}"]
CU_SOURCES = ["k_spatial.cu", "k_contact.cu", "k_islands.cu", "k_events.cu", "k_joints.cu", "k_repack.cu", "capi.cu", "solve_noalloc.cu"]
CPP_SOURCES = ["host_objects.cpp", "polygon_decompose.cpp"]
HEADERS = ["ag2d_math.cuh", "ag2d_world.cuh", "ag2d_kernels.cuh", "ag2d_solver.cuh", "ag2d_ccd.cuh", "host_objects.hpp"]


def _newer(src_paths, dst):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(p) > t for p in src_paths)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "ag2d.h")]
    objs = []
    for src in CU_SOURCES + CPP_SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(OUT_DIR, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        if force or _newer([path] + headers, obj):
            if src.endswith(".cu"):
                cmd = [NVCC] + ARCH + CUDA_FLAGS + ["-c", path, "-o", obj]
            else:
                cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", f"-I{CSRC}",
                       f"-I{os.path.join(ROOT, 'include')}", "-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    if force or _newer(objs, LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
