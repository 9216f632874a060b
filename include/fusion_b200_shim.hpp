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
 *   layout inside an fb_session, one per DeviceMap -- keyed by the address of
 *   the DeviceMap's hashEntries buffer, i.e. one per Mapping.  The first
 *   FuseMapColor or CheckBlockVisibility on a DeviceMap creates its session
 *   with the reference's map constants (fb_default_config) and the camera of
 *   the call.  What the reference's callers read back is written into their
 *   own buffers:
 *     - FuseMapColor and CheckBlockVisibility fill the DeviceMap's
 *       visibleEntries (the reference's 32-byte HashEntry layout, in order)
 *       and its noVisibleBlocks counter, and return the count in host_data;
 *     - CreateRenderingBlocks fills the caller's zRangeX / zRangeY images and
 *       the rendering-tile count in noRenderingBlocks (the RenderingBlock list
 *       itself is the reference's intermediate: not written), and returns
 *       false when there is no tile, as the reference does;
 *     - Raycast writes vmap / nmap (it recomputes the z ranges itself);
 *     - ResetMap empties the session's map.
 *   The hash table, heap, counters and voxel blocks of the DeviceMap are not
 *   kept up to date frame by frame (that would copy the whole map every
 *   frame): code that reads them directly, such as System::WriteMapToDisk,
 *   calls fusion_b200_shim::ExportMap(mapping) first, which writes the
 *   session's map into them in the reference's layouts.
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
#include <map>

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

// The session holding one DeviceMap's map, and the camera of its last
// CreateRenderingBlocks call (Raycast receives only 1/fx and 1/fy).
struct MapState {
    fb_session* session = nullptr;
    float K[4] = {0.f, 0.f, 0.f, 0.f};
};

// Sessions by the address of the DeviceMap's hashEntries buffer, and the
// same sessions by the address of its visibleEntries buffer (what
// CreateRenderingBlocks receives).
inline std::map<const void*, MapState>& map_states() {
    static std::map<const void*, MapState> m;
    return m;
}

inline std::map<const void*, MapState*>& by_visible() {
    static std::map<const void*, MapState*> m;
    return m;
}

inline MapState* find_map(const DeviceMap& map) {
    auto it = map_states().find((const void*)map.hashEntries.data);
    return it == map_states().end() ? nullptr : &it->second;
}

inline MapState& bind_map(const DeviceMap& map, int cols, int rows_, float fx, float fy, float cx, float cy,
                          float depthMin, float depthMax) {
    MapState& m = map_states()[(const void*)map.hashEntries.data];
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
        by_visible()[(const void*)map.visibleEntries.data] = &m;
    }
    return m;
}

// After visibility: the DeviceMap's visibleEntries and noVisibleBlocks, as
// the reference's CheckBlockVisibility leaves them.
inline void write_visible(const DeviceMap& map, fb_session* s) {
    if (!map.visibleEntries.data) return;   // a DeviceMap without buffers
    uint32_t n = 0;
    check(fb_map_export_visible(s, map.visibleEntries.data, (uint32_t)map.visibleEntries.size, &n, legacy()),
          "visible entries");
    if (map.noVisibleBlocks.data)
        cudaMemcpyAsync(map.noVisibleBlocks.data, &n, sizeof n, cudaMemcpyHostToDevice, cudaStreamLegacy);
    cudaStreamSynchronize(cudaStreamLegacy);
}

// The session's whole map written into the DeviceMap's own buffers
// (hashEntries, voxelBlocks, heapMem, heapCounter, entryPtr, and the visible
// list), in the reference's layouts.  Call it before code that reads
// Mapping's device buffers directly, such as System::WriteMapToDisk.
inline void ExportMap(const DeviceMap& map) {
    MapState* m = find_map(map);
    if (!m) return;
    check(fb_map_export_reference(m->session, map.hashEntries.data, map.hashEntries.size, map.voxelBlocks.data,
                                  map.voxelBlocks.size, map.heapMem.data, map.heapMem.size, map.heapCounter.data,
                                  map.entryPtr.data, legacy()),
          "ExportMap");
    write_visible(map, m->session);
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

void ResetMap(DeviceMap map) {
    using namespace fusion_b200_shim;
    // a DeviceMap without a session yet (before its first frame) is empty
    if (MapState* m = find_map(map)) check(fb_reset_map(m->session), "ResetMap");
}

void ResetKeyPoints(KeyMap) {}

void InsertKeyPoints(KeyMap, DeviceArray<SURF>&, DeviceArray<int>&, size_t) {}

void CollectKeyPoints(KeyMap, DeviceArray<SURF>&, DeviceArray<uint>& noKeys) {
    const uint zero = 0;
    cudaMemcpy(noKeys.data, &zero, sizeof zero, cudaMemcpyHostToDevice);
}

void CheckBlockVisibility(DeviceMap map, DeviceArray<uint>& noVisibleBlocks, Matrix3f Rview, Matrix3f RviewInv,
                          float3 tview, int cols, int rows_, float fx, float fy, float cx, float cy, float depthMax,
                          float depthMin, uint* host_data) {
    using namespace fusion_b200_shim;
    fb_session* s = bind_map(map, cols, rows_, fx, fy, cx, cy, depthMin, depthMax).session;
    const float k[4] = {fx, fy, cx, cy};
    uint32_t n = 0;
    check(fb_check_block_visibility(s, rows(Rview), rows(RviewInv), &tview.x, cols, rows_, k, &n, legacy()),
          "CheckBlockVisibility");
    write_visible(map, s);
    if (noVisibleBlocks.data && noVisibleBlocks.data != map.noVisibleBlocks.data)
        cudaMemcpy(noVisibleBlocks.data, &n, sizeof n, cudaMemcpyHostToDevice);
    if (host_data) *host_data = n;
}

void FuseMapColor(const DeviceArray2D<float>& depth, const DeviceArray2D<uchar3>& color,
                  const DeviceArray2D<float4>& nmap, DeviceArray<uint>& noVisibleBlocks, Matrix3f Rview,
                  Matrix3f RviewInv, float3 tview, DeviceMap map, float fx, float fy, float cx, float cy,
                  float depthMax, float depthMin, uint* host_data) {
    using namespace fusion_b200_shim;
    fb_session* s = bind_map(map, depth.cols, depth.rows, fx, fy, cx, cy, depthMin, depthMax).session;
    fb_image d = img(depth), c = img(color), n = img(nmap);
    const float k[4] = {fx, fy, cx, cy};
    uint32_t no = 0;
    check(fb_fuse_map_color(s, &d, &c, &n, rows(Rview), rows(RviewInv), &tview.x, k, &no, legacy()),
          "FuseMapColor");
    write_visible(map, s);
    if (noVisibleBlocks.data && noVisibleBlocks.data != map.noVisibleBlocks.data)
        cudaMemcpy(noVisibleBlocks.data, &no, sizeof no, cudaMemcpyHostToDevice);
    if (host_data) *host_data = no;
}

bool CreateRenderingBlocks(const DeviceArray<HashEntry>& visibleBlocks, DeviceArray2D<float>& zRangeX,
                           DeviceArray2D<float>& zRangeY, const float&, const float&, DeviceArray<RenderingBlock>&,
                           DeviceArray<uint>& noRenderingBlocks, Matrix3f RviewInv, float3 tview,
                           uint noVisibleBlocks, float fx, float fy, float cx, float cy) {
    using namespace fusion_b200_shim;
    auto it = by_visible().find((const void*)visibleBlocks.data);
    if (it == by_visible().end() || noVisibleBlocks == 0) return false;
    MapState& m = *it->second;
    m.K[0] = fx;
    m.K[1] = fy;
    m.K[2] = cx;
    m.K[3] = cy;
    fb_image zx = img(zRangeX), zy = img(zRangeY);
    uint32_t tiles = 0;
    check(fb_create_rendering_blocks(m.session, rows(RviewInv), &tview.x, m.K, &zx, &zy, &tiles, legacy()),
          "CreateRenderingBlocks");
    if (noRenderingBlocks.data) cudaMemcpy(noRenderingBlocks.data, &tiles, sizeof tiles, cudaMemcpyHostToDevice);
    return tiles > 0;
}

void Raycast(DeviceMap map, DeviceArray2D<float4>& vmap, DeviceArray2D<float4>& nmap, DeviceArray2D<float>&,
             DeviceArray2D<float>&, Matrix3f Rview, Matrix3f RviewInv, float3 tview, float, float, float, float) {
    using namespace fusion_b200_shim;
    MapState* m = find_map(map);
    if (!m) return;
    fb_image v = img(vmap), n = img(nmap);
    int rendered = 0;
    check(fb_raycast(m->session, &v, &n, rows(Rview), rows(RviewInv), &tview.x, m->K, &rendered, legacy()),
          "Raycast");
}

uint MeshScene(DeviceArray<uint>&, DeviceArray<uint>&, DeviceMap map, const DeviceArray<int>&,
               const DeviceArray<int>&, const DeviceArray2D<int>&, DeviceArray<float3>& normal,
               DeviceArray<float3>& vertex, DeviceArray<uchar3>& color, DeviceArray<int3>&) {
    using namespace fusion_b200_shim;
    MapState* m = find_map(map);
    if (!m) return 0;
    size_t cap = vertex.size < normal.size ? vertex.size : normal.size;
    if (color.size < cap) cap = color.size;
    uint64_t n = 0;
    check(fb_mesh_scene(m->session, (float*)vertex.data, (float*)normal.data, (uint8_t*)color.data, cap / 3, &n,
                        legacy()),
          "MeshScene");
    return (uint)(n < cap / 3 ? n : cap / 3);
}

#endif
