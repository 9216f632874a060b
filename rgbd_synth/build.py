"""Builds the seeded RGB-D generator in-tree: rgbd_synth/libfbsynth.so (g++,
OpenMP).  The generator is input data for the tests and the benchmark (both of
its arms), so it lives apart from the fusion library.

    python -m rgbd_synth.build
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libfbsynth.so")


def build(force=False):
    src = os.path.join(HERE, "synth.cpp")
    deps = [src, os.path.join(HERE, "synth.h"), os.path.abspath(__file__)]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(d) <= os.path.getmtime(LIB) for d in deps):
        return LIB
    # the environment's CXX may lack OpenMP; the system g++ has it
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
                           "-o", LIB, src])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
