"""Builds the native libraries of the package in-tree:

  fusion_b200/libfusion_b200.so  CUDA kernels + C ABI (nvcc, sm_100a)

    python -m fusion_b200.build

Each CUDA source is compiled to an object under fusion_b200/_build/ (in
parallel), then linked.  track.cu is compiled without contraction of
multiplies and adds into FMAs (-fmad=false): its kernels exist in two
register budgets that must compute the same bits.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
CU_SOURCES = ["preprocess.cu", "track.cu", "map.cu", "raycast.cu", "session.cu", "keyframe_track.cu", "stage_api.cu",
              "persist.cu", "batch_step.cu", "shade.cu", "static_scratch.cu", "mesh.cu", "keypoints.cu"]
EXTRA_FLAGS = {"track.cu": ["-fmad=false"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB = os.path.join(HERE, "libfusion_b200.so")


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


def _compile(src, verbose):
    obj = os.path.join(OBJ, os.path.splitext(os.path.basename(src))[0] + ".o")
    cmd = [_nvcc(), "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", "-Xcompiler",
           "-fvisibility=hidden", "-Xptxas", "-warn-spills", *EXTRA_FLAGS.get(os.path.basename(src), []),
           "-I", os.path.join(ROOT, "include"), "-c", "-o", obj, src]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return obj


def build_cuda(force=False, verbose=False):
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES]
    deps = srcs + [os.path.join(CSRC, "fb_common.cuh"), os.path.join(CSRC, "fb_internal.h"),
                   os.path.join(CSRC, "fb_fused.cuh"), os.path.join(CSRC, "fb_async.cuh"),
                   os.path.join(CSRC, "session_internal.h"),
                   os.path.join(ROOT, "include", "fusion_b200.h"), os.path.abspath(__file__)]
    if not force and _newer(LIB, deps):
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB, *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return LIB


def build_all(force=False, verbose=False):
    build_cuda(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
