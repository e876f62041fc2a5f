"""Build the sm_100a CUDA library in-tree: banshee_b200/libbanshee_gpu.so.

nvcc compiles every .cu for sm_100a only (-gencode arch=compute_100a,code=sm_100a)
with -fmad=false and IEEE division / square root, which the bit-exact
Moller-Trumbore path relies on (cache.cu, the radiance cache, is off that path
and contracts multiply-adds).  Host C++ is compiled by g++ with
-ffp-contract=off.  No GPU is needed to build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbanshee_gpu.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

CU_SOURCES = ["api.cu", "render.cu", "cache.cu", "batch.cu", "gpu_build.cu", "sah_build.cu", "scene_records.cu"]
CXX_SOURCES = ["bvh_build.cpp", "image.cpp"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
              "-Xcompiler", "-fPIC,-ffp-contract=off", "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


# The radiance cache's kernels (encoding, MLP, Adam) are not part of the
# bit-exact path: they may contract multiply-adds.
FMAD_FILES = {"cache.cu"}


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "banshee_gpu.h")]


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    deps = _deps()
    objs = []
    for src in CU_SOURCES + CXX_SOURCES:
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not force and not _newer(obj, deps):
            continue
        path = os.path.join(CSRC, src)
        if src.endswith(".cu"):
            flags = [("-fmad=true" if (f == "-fmad=false" and src in FMAD_FILES) else f) for f in NVCC_FLAGS]
            cmd = [NVCC] + flags + ["-c", path, "-o", obj]
        else:
            cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-pthread",
                   "-I" + os.path.join(CUDA_HOME, "include"), "-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    if force or _newer(LIB, objs):
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB] + objs + ["-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
