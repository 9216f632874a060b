"""The C++ shim (include/fusion_b200_shim.hpp) against the reference's own
boundary headers: a translation unit that includes the reference's
Tracking/Reduction.h (which includes Mapping/RenderScene.h) and then the
shim, takes the address of every free function the two headers declare --
except BuildAdjacencyMatrix and FilterKeyMatching, which stay in the
reference's Tracking/KeyPoints.cu -- and links against libfusion_b200.so
alone.  A shim definition whose signature differed from the reference's
declaration would be a second overload: taking the address would be
ambiguous and the declared function would stay undefined at link time.
CPU only (compiles and links, runs nothing); skipped where the reference's
sources or nvcc are absent.  The OpenCV umbrella header the reference
includes is the oracle's stand-in (declares cv::cuda::GpuMat only)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _reference_dir():
    """FB_REFERENCE_DIR, else the reference tree the last build() compiled
    (recorded in oracle/_ref/REFERENCE_DIR); empty when neither exists."""
    if os.environ.get("FB_REFERENCE_DIR"):
        return os.environ["FB_REFERENCE_DIR"]
    rec = os.path.join(ROOT, "oracle", "_ref", "REFERENCE_DIR")
    if os.path.exists(rec):
        return open(rec).read().strip()
    return ""


REF = _reference_dir()
LIB = os.path.join(ROOT, "fusion_b200", "libfusion_b200.so")

TU = r"""
#include "Reduction.h"
#include "fusion_b200_shim.hpp"

template <class F> static void* addr(F f) { return (void*)f; }

int main(int argc, char**) {
    void* fns[] = {
        addr(&FilterDepth), addr(&ComputeVMap), addr(&ComputeNMap),
        addr(static_cast<void (*)(const DeviceArray2D<float>&, DeviceArray2D<float>&)>(&PyrDownGauss)),
        addr(static_cast<void (*)(const DeviceArray2D<unsigned char>&, DeviceArray2D<unsigned char>&)>(
            &PyrDownGauss)),
        addr(&ImageToIntensity), addr(&ComputeDerivativeImage), addr(&ResizeMap), addr(&RenderImage),
        addr(&DepthToImage), addr(&RgbImageToRgba), addr(&ForwardWarping), addr(&SO3Step), addr(&ICPStep),
        addr(&RGBStep),
        addr(&ResetMap), addr(&ResetKeyPoints), addr(&InsertKeyPoints), addr(&CollectKeyPoints),
        addr(&Raycast), addr(&CreateRenderingBlocks), addr(&MeshScene), addr(&CheckBlockVisibility),
        addr(&FuseMapColor),
    };
    int n = 0;
    for (void* f : fns) n += f != nullptr;
    return argc > 100 ? n : 0;
}
"""


def _nvcc():
    for c in [os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")]:
        if c and os.path.exists(c):
            return c
    return None


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "Tracking")), reason="reference sources absent")
def test_shim_matches_the_reference_declarations_and_links(tmp_path):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc absent")
    if not os.path.exists(LIB):
        pytest.skip("libfusion_b200.so not built")
    src = tmp_path / "shim_tu.cu"
    src.write_text(TU)
    exe = tmp_path / "shim_tu"
    cmd = [nvcc, "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-w",
           "-I", os.path.join(ROOT, "oracle", "ref_harness", "stub"),
           "-I", os.path.join(REF, "Utility"), "-I", os.path.join(REF, "Mapping"),
           "-I", os.path.join(REF, "Tracking"), "-I", os.path.join(ROOT, "include"),
           "-o", str(exe), str(src), "-L", os.path.dirname(LIB), "-lfusion_b200",
           "-Xlinker", "--no-undefined"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert exe.exists()
