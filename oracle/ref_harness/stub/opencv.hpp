// ORACLE / TEST INFRASTRUCTURE ONLY.
// Minimal stand-in for OpenCV's umbrella header.  The reference's
// Tracking/Reduction.h:7 includes <opencv.hpp> only to declare the SURF
// matching helpers (Reduction.h:85-96), which take cv::cuda::GpuMat.  Those
// helpers are not on the dense per-frame path and are never called by the
// harness; declaring the type is enough to compile the hot-path kernels.
#pragma once
namespace cv {
namespace cuda {
struct GpuMat {};
}  // namespace cuda
}  // namespace cv
