#!/usr/bin/env python3
"""Builds libirbc.so (sm_100a CUDA kernels + C ABI) in place with nvcc.

FP64 kernels are compiled with --fmad=false so that every expression rounds
like the reference's x86-64 build (no fused multiply-add contraction)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libirbc.so")
MAIN = os.path.join(HERE, "MAIN")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("IRBC_CXX", "g++")
CUDA_LIB = os.path.join(os.path.dirname(os.path.dirname(NVCC)), "lib64")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-O2",
         "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]
SOURCES = ["kernels.cu", "fast.cu", "binning.cu", "binning_noalloc.cu", "api.cu", "batch.cu"]
# every header and included .cuh: a change to any of them rebuilds every source
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith((".h", ".cuh")))


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False):
    objs = []
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "irbc.h")]
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(CSRC, src.replace(".cu", ".o"))
        if _newer(obj, [path] + hdrs + [__file__]):
            cmd = [NVCC] + ARCH + FLAGS + ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError("nvcc failed on " + src)
        objs.append(obj)
    if _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    # MAIN: the reference's command line over the library
    src = os.path.join(HERE, "main.cpp")
    if _newer(MAIN, [src, LIB, os.path.join(ROOT, "include", "irbc.h")]):
        cmd = [CXX, "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), src, "-o", MAIN, "-L" + HERE,
               "-lirbc", "-L" + CUDA_LIB, "-lcudart", "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + CUDA_LIB]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("MAIN failed to build")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
