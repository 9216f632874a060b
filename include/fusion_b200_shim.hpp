/* fusion_b200_shim.hpp -- the reference's kernel free functions with their
 * exact signatures (Tracking/Reduction.h:18-83, Mapping/RenderScene.h:3-52),
 * defined on top of libfusion_b200's C ABI, so that the reference's host
 * classes (Frame, Tracker, Mapping, System) relink unchanged against the
 * library in place of Tracking/Pyrdown.cu, Tracking/Reduction.cu,
 * Mapping/DeviceMap.cu, Mapping/FuseMap.cu, Mapping/RenderScene.cu and
 * Mapping/MeshScene.cu.  Tracking/KeyPoints.cu (BuildAdjacencyMatrix,
 * FilterKeyMatching: OpenCV CUDA) stays as it is.
 *
 * Include it in exactly one translation unit of the reference's executable,
 * after the reference's Reduction.h (it uses the reference's DeviceArray2D,
 * DeviceArray, Matrix3f, Intrinsics, DeviceMap, KeyMap, HashEntry,
 * RenderingBlock and SURF), compile that unit with nvcc, and link with
 * -lfusion_b200.
 *
 * Semantics:
 * - Image and tracking functions: the library's per-stage entry points on the
 *   reference's buffers (device pointer, pitch `step`, cols, rows), on the
 *   legacy default stream, so they are ordered with the reference's own
 *   default-stream work as its kernels were.  ICPStep and RGBStep return the
 *   normal equations on the host, synchronously, as the reference's do; their
 *   reduction buffers (sum, out, sumRes, outRes) are not used.
 * - The map: the library keeps the hash table and the voxel blocks in its own
 *   layout inside an fb_session.  The first FuseMapColor or
 *   CheckBlockVisibility creates that session with the reference's map
 *   constants (fb_default_config) and the camera of the call; every later
 *   map call -- on the reference's one DeviceMap -- goes to it.  The
 *   reference's DeviceMap buffers stay allocated by Mapping and are not read.
 *   Mapping::RayTrace calls CreateRenderingBlocks and then Raycast;
 *   fb_raycast does both (z ranges, then the rays), so CreateRenderingBlocks
 *   only records the camera and reports whether any block is visible, and
 *   Raycast leaves the maps untouched when no rendering rectangle results,
 *   as the reference does when CreateRenderingBlocks returns false.
 * - Errors print the library's message and exit(0), as the reference's
 *   SafeCall does.
 * - Not provided by the library, defined here as such: SO3Step (its only
 *   caller, Tracker::ComputeSO3, is never called) and ForwardWarping (its only
 *   caller, Mapping::ForwardWarp, is never called) report and exit; the
 *   reference's SURF key map (ResetKeyPoints, InsertKeyPoints,
 *   CollectKeyPoints) is kept empty -- key points, keyframes and
 *   relocalisation are the session's own (fb_session_set_keypoints). */
#ifndef FUSION_B200_SHIM_HPP
#define FUSION_B200_SHIM_HPP

#include <cuda_runtime_api.h>

#include <cstdlib>
#include <iostream>

#include "fusion_b200.h"

namespace fusion_b200_shim {

inline void check(int st, const char* fn) {
    if (st != FB_OK) {
        std::cout << "Error: " << fn << ": " << fb_status_string(st);
        if (st == FB_ECUDA) std::cout << " (" << fb_last_error() << ")";
        std::cout << std::endl;
        std::exit(0);
    }
}

inline void unsupported(const char* fn) {
    std::cout << "Error: " << fn << " is not provided by libfusion_b200" << std::endl;
    std::exit(0);
}

template <class A>
inline fb_image img(const A& a) {
    return fb_image{a.data, a.step, a.cols, a.rows};
}

inline void* legacy() { return (void*)cudaStreamLegacy; }

inline const float* rows(const Matrix3f& m) { return &m.rowx.x; }   // three float3 rows, contiguous

// Scratch of ICPStep / RGBStep (the reference allocates per call,
// Reduction.cu:572), grown on demand and kept.
inline void* step_scratch(int cols, int rows_, size_t* bytes) {
    static void* buf = nullptr;
    static size_t size = 0;
    const size_t need = fb_step_scratch_bytes(cols, rows_);
    if (size < need) {
        if (buf) cudaFree(buf);
        buf = nullptr;
        size = 0;
        if (cudaMalloc(&buf, need) != cudaSuccess) check(FB_ENOMEM, "ICPStep/RGBStep scratch");
        size = need;
    }
    *bytes = size;
    return buf;
}

// The session holding the map, and the camera of the last
// CreateRenderingBlocks call (Raycast receives only 1/fx and 1/fy).
struct MapState {
    fb_session* session = nullptr;
    float K[4] = {0.f, 0.f, 0.f, 0.f};
};

inline MapState& map_state() {
    static MapState m;
    return m;
}

inline fb_session* bind_map(int cols, int rows_, float fx, float fy, float cx, float cy, float depthMin,
                            float depthMax) {
    MapState& m = map_state();
    if (!m.session) {
        fb_config c;
        fb_default_config(&c, cols, rows_);
        c.fx = fx;
        c.fy = fy;
        c.cx = cx;
        c.cy = cy;
        c.depth_min = depthMin;
        c.depth_max = depthMax;
        check(fb_session_create(&c, legacy(), &m.session), "fb_session_create");
    }
    return m.session;
}

}  // namespace fusion_b200_shim

// ------------------------------------------------ Tracking/Reduction.h

void FilterDepth(const DeviceArray2D<unsigned short>& depth, DeviceArray2D<float>& rawDepth,
                 DeviceArray2D<float>& filteredDepth, float depthScale, float depthCutoff) {
    using namespace fusion_b200_shim;
    fb_image d = img(depth), r = img(rawDepth), f = img(filteredDepth);
    check(fb_filter_depth(&d, &r, &f, depthScale, depthCutoff, legacy()), "FilterDepth");
}

void ComputeVMap(const DeviceArray2D<float>& depth, DeviceArray2D<float4>& vmap, float fx, float fy, float cx,
                 float cy, float depthCutoff) {
    using namespace fusion_b200_shim;
    fb_image d = img(depth), v = img(vmap);
    check(fb_compute_vmap(&d, &v, fx, fy, cx, cy, depthCutoff, legacy()), "ComputeVMap");
}

void ComputeNMap(const DeviceArray2D<float4>& vmap, DeviceArray2D<float4>& nmap) {
    using namespace fusion_b200_shim;
    fb_image v = img(vmap), n = img(nmap);
    check(fb_compute_nmap(&v, &n, legacy()), "ComputeNMap");
}

void PyrDownGauss(const DeviceArray2D<float>& src, DeviceArray2D<float>& dst) {
    using namespace fusion_b200_shim;
    fb_image s = img(src), d = img(dst);
    check(fb_pyrdown_gauss_f32(&s, &d, legacy()), "PyrDownGauss");
}

void PyrDownGauss(const DeviceArray2D<unsigned char>& src, DeviceArray2D<unsigned char>& dst) {
    using namespace fusion_b200_shim;
    fb_image s = img(src), d = img(dst);
    check(fb_pyrdown_gauss_u8(&s, &d, legacy()), "PyrDownGauss");
}

void ImageToIntensity(const DeviceArray2D<uchar3>& rgb, DeviceArray2D<unsigned char>& image) {
    using namespace fusion_b200_shim;
    fb_image s = img(rgb), d = img(image);
    check(fb_image_to_intensity(&s, &d, legacy()), "ImageToIntensity");
}

void ComputeDerivativeImage(DeviceArray2D<unsigned char>& image, DeviceArray2D<short>& dx,
                            DeviceArray2D<short>& dy) {
    using namespace fusion_b200_shim;
    fb_image g = img(image), x = img(dx), y = img(dy);
    check(fb_compute_derivative_image(&g, &x, &y, legacy()), "ComputeDerivativeImage");
}

void ResizeMap(const DeviceArray2D<float4>& vsrc, const DeviceArray2D<float4>& nsrc, DeviceArray2D<float4>& vdst,
               DeviceArray2D<float4>& ndst) {
    using namespace fusion_b200_shim;
    fb_image a = img(vsrc), b = img(nsrc), c = img(vdst), d = img(ndst);
    check(fb_resize_map(&a, &b, &c, &d, legacy()), "ResizeMap");
}

void RenderImage(const DeviceArray2D<float4>& points, const DeviceArray2D<float4>& normals, const float3 light_pose,
                 DeviceArray2D<uchar4>& image) {
    using namespace fusion_b200_shim;
    fb_image v = img(points), n = img(normals), o = img(image);
    check(fb_render_image(&v, &n, &light_pose.x, &o, legacy()), "RenderImage");
}

void DepthToImage(const DeviceArray2D<float>& depth, DeviceArray2D<uchar4>& image) {
    using namespace fusion_b200_shim;
    fb_image d = img(depth), o = img(image);
    check(fb_depth_to_image(&d, &o, legacy()), "DepthToImage");
}

void RgbImageToRgba(const DeviceArray2D<uchar3>& image, DeviceArray2D<uchar4>& rgba) {
    using namespace fusion_b200_shim;
    fb_image s = img(image), o = img(rgba);
    check(fb_rgb_to_rgba(&s, &o, legacy()), "RgbImageToRgba");
}

void ForwardWarping(const DeviceArray2D<float4>&, const DeviceArray2D<float4>&, DeviceArray2D<float4>&,
                    DeviceArray2D<float4>&, Matrix3f, Matrix3f, float3, float3, float, float, float, float) {
    fusion_b200_shim::unsupported("ForwardWarping");
}

void SO3Step(const DeviceArray2D<unsigned char>&, const DeviceArray2D<unsigned char>&, const DeviceArray2D<short>&,
             const DeviceArray2D<short>&, Matrix3f, Matrix3f, Intrinsics, DeviceArray2D<float>&,
             DeviceArray<float>&, float*, double*, double*) {
    fusion_b200_shim::unsupported("SO3Step");
}

void ICPStep(DeviceArray2D<float4>& nextVMap, DeviceArray2D<float4>& lastVMap, DeviceArray2D<float4>& nextNMap,
             DeviceArray2D<float4>& lastNMap, Matrix3f Rcurr, float3 tcurr, Matrix3f Rlast, Matrix3f RlastInv,
             float3 tlast, Intrinsics K, DeviceArray2D<float>&, DeviceArray<float>&, float* residual,
             double* matrixA_host, double* vectorB_host) {
    using namespace fusion_b200_shim;
    fb_image vc = img(nextVMap), vl = img(lastVMap), nc = img(nextNMap), nl = img(lastNMap);
    const float k[4] = {K.fx, K.fy, K.cx, K.cy};
    size_t bytes = 0;
    void* scratch = step_scratch(vc.cols, vc.rows, &bytes);
    check(fb_icp_step(&vc, &vl, &nc, &nl, rows(Rcurr), &tcurr.x, rows(Rlast), rows(RlastInv), &tlast.x, k, scratch,
                      bytes, residual, matrixA_host, vectorB_host, legacy()),
          "ICPStep");
}

void RGBStep(const DeviceArray2D<unsigned char>& nextImage, const DeviceArray2D<unsigned char>& lastImage,
             const DeviceArray2D<float4>& nextVMap, const DeviceArray2D<float4>& lastVMap,
             const DeviceArray2D<short>& dIdx, const DeviceArray2D<short>& dIdy, Matrix3f Rcurr, Matrix3f RcurrInv,
             Matrix3f Rlast, Matrix3f RlastInv, float3 tcurr, float3 tlast, Intrinsics K, DeviceArray2D<float>&,
             DeviceArray<float>&, DeviceArray2D<int>&, DeviceArray<int>&, float* residual, double* matrixA_host,
             double* vectorB_host) {
    using namespace fusion_b200_shim;
    fb_image gc = img(nextImage), gl = img(lastImage), vc = img(nextVMap), vl = img(lastVMap), dx = img(dIdx),
             dy = img(dIdy);
    const float k[4] = {K.fx, K.fy, K.cx, K.cy};
    size_t bytes = 0;
    void* scratch = step_scratch(gc.cols, gc.rows, &bytes);
    check(fb_rgb_step(&gc, &gl, &vc, &vl, &dx, &dy, rows(Rcurr), rows(RcurrInv), rows(Rlast), rows(RlastInv),
                      &tcurr.x, &tlast.x, k, scratch, bytes, residual, matrixA_host, vectorB_host, legacy()),
          "RGBStep");
}

// ------------------------------------------------ Mapping/RenderScene.h

void ResetMap(DeviceMap) {
    using namespace fusion_b200_shim;
    // before the first frame there is no session yet: it starts empty
    if (map_state().session) check(fb_reset_map(map_state().session), "ResetMap");
}

void ResetKeyPoints(KeyMap) {}

void InsertKeyPoints(KeyMap, DeviceArray<SURF>&, DeviceArray<int>&, size_t) {}

void CollectKeyPoints(KeyMap, DeviceArray<SURF>&, DeviceArray<uint>& noKeys) {
    const uint zero = 0;
    cudaMemcpy(noKeys.data, &zero, sizeof zero, cudaMemcpyHostToDevice);
}

void CheckBlockVisibility(DeviceMap, DeviceArray<uint>&, Matrix3f Rview, Matrix3f RviewInv, float3 tview, int cols,
                          int rows_, float fx, float fy, float cx, float cy, float depthMax, float depthMin,
                          uint* host_data) {
    using namespace fusion_b200_shim;
    fb_session* s = bind_map(cols, rows_, fx, fy, cx, cy, depthMin, depthMax);
    const float k[4] = {fx, fy, cx, cy};
    uint32_t n = 0;
    check(fb_check_block_visibility(s, rows(Rview), rows(RviewInv), &tview.x, cols, rows_, k, &n, legacy()),
          "CheckBlockVisibility");
    if (host_data) *host_data = n;
}

void FuseMapColor(const DeviceArray2D<float>& depth, const DeviceArray2D<uchar3>& color,
                  const DeviceArray2D<float4>& nmap, DeviceArray<uint>&, Matrix3f Rview, Matrix3f RviewInv,
                  float3 tview, DeviceMap, float fx, float fy, float cx, float cy, float depthMax, float depthMin,
                  uint* host_data) {
    using namespace fusion_b200_shim;
    fb_session* s = bind_map(depth.cols, depth.rows, fx, fy, cx, cy, depthMin, depthMax);
    fb_image d = img(depth), c = img(color), n = img(nmap);
    const float k[4] = {fx, fy, cx, cy};
    uint32_t no = 0;
    check(fb_fuse_map_color(s, &d, &c, &n, rows(Rview), rows(RviewInv), &tview.x, k, &no, legacy()),
          "FuseMapColor");
    if (host_data) *host_data = no;
}

bool CreateRenderingBlocks(const DeviceArray<HashEntry>&, DeviceArray2D<float>&, DeviceArray2D<float>&,
                           const float&, const float&, DeviceArray<RenderingBlock>&, DeviceArray<uint>&, Matrix3f,
                           float3, uint noVisibleBlocks, float fx, float fy, float cx, float cy) {
    fusion_b200_shim::MapState& m = fusion_b200_shim::map_state();
    m.K[0] = fx;
    m.K[1] = fy;
    m.K[2] = cx;
    m.K[3] = cy;
    return m.session != nullptr && noVisibleBlocks > 0;
}

void Raycast(DeviceMap, DeviceArray2D<float4>& vmap, DeviceArray2D<float4>& nmap, DeviceArray2D<float>&,
             DeviceArray2D<float>&, Matrix3f Rview, Matrix3f RviewInv, float3 tview, float, float, float, float) {
    using namespace fusion_b200_shim;
    MapState& m = map_state();
    if (!m.session) return;
    fb_image v = img(vmap), n = img(nmap);
    int rendered = 0;
    check(fb_raycast(m.session, &v, &n, rows(Rview), rows(RviewInv), &tview.x, m.K, &rendered, legacy()),
          "Raycast");
}

uint MeshScene(DeviceArray<uint>&, DeviceArray<uint>&, DeviceMap, const DeviceArray<int>&, const DeviceArray<int>&,
               const DeviceArray2D<int>&, DeviceArray<float3>& normal, DeviceArray<float3>& vertex,
               DeviceArray<uchar3>& color, DeviceArray<int3>&) {
    using namespace fusion_b200_shim;
    MapState& m = map_state();
    if (!m.session) return 0;
    size_t cap = vertex.size < normal.size ? vertex.size : normal.size;
    if (color.size < cap) cap = color.size;
    uint64_t n = 0;
    check(fb_mesh_scene(m.session, (float*)vertex.data, (float*)normal.data, (uint8_t*)color.data, cap / 3, &n,
                        legacy()),
          "MeshScene");
    return (uint)(n < cap / 3 ? n : cap / 3);
}

#endif
