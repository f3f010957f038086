"""Builds libshape_b200.so (the engine's C ABI) in-tree for sm_100a.

    python shape-cuda-v1.2_b200/build.py [--force]

Object files go to shape-cuda-v1.2_b200/_build/, the library to
shape-cuda-v1.2_b200/lib/libshape_b200.so. Translation units whose FP64
arithmetic must match the reference CPU code bit for bit are compiled with
-fmad=false (no FMA contraction); the FP32 rasterizer keeps contraction.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libshape_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                 "-Xcompiler", "-ffp-contract=off", "-I", os.path.join(REPO, "include"),
                 "-I", CSRC]

# (source, extra flags)
UNITS = [
    ("core.cu", ["-fmad=false"]),
    ("raster_f64.cu", ["-fmad=false"]),
    ("raster_f32.cu", []),
    ("engine.cu", ["-fmad=false"]),
    ("noalloc.cu", ["-fmad=false"]),
    ("posview.cu", ["-fmad=false"]),
    ("fit.cu", ["-fmad=false"]),
    ("server.cu", ["-fmad=false"]),
    ("spin.cu", ["-fmad=false"]),
    ("penalty.cu", ["-fmad=false"]),
    ("modfile.cu", []),
]

HEADERS = ["engine_internal.h", "engine_impl.h", "kernels.h", "raster_impl.cuh", "posmask_dev.cuh", "viewgeom.cuh",
           "spin_impl.cuh"]


def _newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    deps = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(REPO, "include", "shape_types.h"), os.path.join(REPO, "include", "shape_b200.h"),
        os.path.abspath(__file__)]
    objs = []
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer([s] + deps, o):
            cmd = [NVCC] + COMMON + flags + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _newer(objs, LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread",
                                                                   "-Xlinker", "-soname=libshape_b200.so"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
