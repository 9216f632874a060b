"""Builds the native libraries of the package in-tree:

  fusion_b200/libfusion_b200.so  CUDA kernels + C ABI (nvcc, sm_100a)
  fusion_b200/libfbsynth.so      seeded synthetic RGB-D generator (g++, OpenMP)

    python -m fusion_b200.build
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
CU_SOURCES = ["preprocess.cu", "track.cu", "map.cu", "raycast.cu", "session.cu", "static_scratch.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB = os.path.join(HERE, "libfusion_b200.so")
SYNTH = os.path.join(HERE, "libfbsynth.so")


def _nvcc():
    for cand in [os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")]:
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build_cuda(force=False, verbose=False):
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES]
    deps = srcs + [os.path.join(CSRC, "fb_common.cuh"), os.path.join(CSRC, "fb_internal.h"),
                   os.path.join(ROOT, "include", "fusion_b200.h")]
    if not force and _newer(LIB, deps):
        return LIB
    cmd = [_nvcc(), "-std=c++17", "-O3", "-lineinfo", *ARCH, "-shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-Xptxas", "-warn-spills",
           "-I", os.path.join(ROOT, "include"), "-o", LIB, *srcs]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return LIB


def build_synth(force=False):
    src = os.path.join(CSRC, "synth", "synth.cpp")
    deps = [src, os.path.join(CSRC, "synth", "synth.h")]
    if not force and _newer(SYNTH, deps):
        return SYNTH
    # the environment's CXX may lack OpenMP; the system g++ has it
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
                           "-o", SYNTH, src])
    return SYNTH


def build_all(force=False, verbose=False):
    build_synth(force)
    build_cuda(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
