// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference's per-frame dense path, used as the checker
// of the CUDA implementation (tests/, __graft_entry__.smoke) and as the timed
// CPU baseline (bench.py).  Nothing in fusion_b200/ links or loads it.
//
// Every function is templated on the arithmetic type R:
//   R = double : the FP64 oracle.  All arithmetic the reference does in float
//                is done in double.
//   R = float  : reference precision.  Expressions the reference evaluates in
//                float are evaluated in IEEE binary32, one operation at a time,
//                in the order they are written in the reference (the file is
//                built with -ffp-contract=off), and sub-expressions the
//                reference evaluates in double stay in double.  The CUDA
//                implementation evaluates the same expressions with
//                non-contracting intrinsics, so integer, byte and index
//                results (pixels, voxel and block coordinates, hash slots,
//                weights, colours, counts) match it bit for bit.
// Sums over pixels (normal equations) are always accumulated in double.
//
// Parity of this file with the reference is pinned by the golden vectors in
// tests/golden/, produced by running the reference's own CUDA kernels.
#ifndef FB_ORACLE_HPP
#define FB_ORACLE_HPP

#include <cstdint>
#include <vector>

extern "C" {

// Runtime form of the reference's compile-time constants
// (Mapping/DeviceMap.h:135-151, Tracking/Tracking.h:99-104, Core/Frame.cc:13-14).
typedef struct fbo_config {
    int width, height;
    float fx, fy, cx, cy;       // level-0 intrinsics
    float depth_scale;          // Frame::mDepthScale
    float depth_cutoff;         // Frame::mDepthCutoff
    float voxel_size;           // DeviceMap::VoxelSize
    float trunc_dist;           // DeviceMap::TruncateDist
    float depth_min, depth_max; // DeviceMap::DepthMin / DepthMax
    int num_buckets, num_excess, num_blocks;
    int iters[3];               // ICP iterations at pyramid levels 0, 1, 2
    int precision;              // 64 or 32 (see above)
} fbo_config;

// ---- stage functions (row-major contiguous arrays) ----
int fbo_filter_depth(int prec, int W, int H, const uint16_t* depth, float depth_scale,
                     float depth_cutoff, float* raw, float* filtered);
int fbo_intensity(int W, int H, const uint8_t* rgb, uint8_t* gray);
int fbo_pyrdown_f32(int prec, int W, int H, const float* src, float* dst);
int fbo_pyrdown_u8(int prec, int W, int H, const uint8_t* src, uint8_t* dst);
int fbo_vmap(int prec, int W, int H, const float* depth, float fx, float fy, float cx, float cy,
             float depth_cutoff, float* vmap);
int fbo_nmap(int prec, int W, int H, const float* vmap, float* nmap);
int fbo_derivative(int W, int H, const uint8_t* gray, int16_t* dx, int16_t* dy);
int fbo_resize_map(int prec, int W, int H, const float* vsrc, const float* nsrc, float* vdst,
                   float* ndst);
// sums29: 28 upper-triangle products of the 7-wide rows + count (double)
int fbo_icp_step(int prec, int W, int H, const float* vcurr, const float* vlast,
                 const float* ncurr, const float* nlast, const double* pose_curr,
                 const double* pose_last, float fx, float fy, float cx, float cy, double* sums29);
// res2: count and sum of squared intensity differences (64-bit)
int fbo_rgb_step(int prec, int W, int H, const uint8_t* gcurr, const uint8_t* glast,
                 const float* vcurr, const float* vlast, const int16_t* dx, const int16_t* dy,
                 const double* pose_curr, const double* pose_last, float fx, float fy, float cx,
                 float cy, double* sums29, int64_t* res2);

// ---- map (voxel-block hash + TSDF) ----
void* fbo_map_create(const fbo_config* cfg);
void fbo_map_destroy(void* m);
void fbo_map_reset(void* m);
// Block allocation + visibility + integration of one frame (FuseMapColor).
int fbo_map_fuse(void* m, const float* raw_depth, const uint8_t* rgb, const float* nmap,
                 const double* pose, uint32_t* no_visible);
// Allocation only; returns the number of blocks inserted.
int fbo_map_allocate(void* m, const float* raw_depth, const double* pose, uint32_t* n_new);
// Rendering-block z ranges + raycast (Mapping::RayTrace) of the current
// visible list; zmin/zmax are ceil(W/8) x ceil(H/8) (may be NULL).  Returns
// the number of rendering tiles; with none, vmap/nmap are left unchanged.
int fbo_map_raycast(void* m, const double* pose, float* vmap, float* nmap, float* zmin,
                    float* zmax);
int fbo_map_counters(void* m, int32_t* heap_counter, int32_t* entry_ptr, uint32_t* no_visible);
// entries: (num_buckets + num_excess) x {x, y, z, ptr, offset}; ptr is a voxel index
int fbo_map_entries(void* m, int32_t* entries);
int fbo_map_visible(void* m, int32_t* slots);
// voxels of n blocks given by voxel-index ptrs (as in the entries)
int fbo_map_voxels(void* m, const int32_t* ptrs, int n, double* sdf, uint8_t* weight, uint8_t* rgb);
// Start from a given state (teacher forcing): n occupied slots with their
// {x, y, z, ptr, offset} (all other slots emptied) and the two counters; the
// visible list; the voxels of n blocks given by voxel-index ptrs.
int fbo_map_set_entries(void* m, const int32_t* slots, const int32_t* entries, int n,
                        int32_t heap_counter, int32_t entry_ptr);
int fbo_map_set_visible(void* m, const int32_t* slots, int n);
int fbo_map_load_blocks(void* m, const int32_t* ptrs, int n, const double* sdf,
                        const uint8_t* weight, const uint8_t* rgb);
// CheckBlockVisibility (Mapping/FuseMap.cu:206-249) at pose T for the
// configured camera and depth range; *nv = visible blocks.
int fbo_map_visibility(void* m, const double* T, uint32_t* nv);
// MeshScene (Mapping/MeshScene.cu:20-295) with a given case table (tri:
// 256 x 16 edge triples, ntri: triangles per case): *count = triangles; the
// first min(count, cap) written (3 vertices each: V, N float3, C uchar3).
// fused: 1 rounds the normal's multiply-adds fused, 0 as written.
int fbo_map_mesh(void* m, const int8_t* tri, const int32_t* ntri, int fused, float* V, float* N, uint8_t* C,
                 uint64_t cap, uint64_t* count);

// ---- whole per-frame loop (System::GrabImage) ----
void* fbo_system_create(const fbo_config* cfg);
void fbo_system_destroy(void* s);
// info: [0] GrabFrame result, [1] tracker state, [2] visible blocks,
// [3] icp error, [4] icp count, [5] rgb error, [6] rgb count, [7] fused
int fbo_system_grab(void* s, const uint16_t* depth, const uint8_t* rgb, double* info);
int fbo_system_pose(void* s, int which, double* T);
void* fbo_system_map(void* s);
// level maps of frame `which` (0 = last, 1 = next); any output may be NULL
int fbo_system_level(void* s, int which, int level, float* vmap, float* nmap, float* depth,
                     uint8_t* image, int16_t* dx, int16_t* dy);
// Tracker::ComputeSE3 alone on given inputs (teacher forcing): the next
// frame's level maps (vertex, normal, gray, Sobel x/y) and the last frame's
// (vertex, normal, gray), three levels each, and the last pose.  out_pose is
// the next frame's pose (rolled back to last_pose on failure); info: [0] ok,
// [1] icp error, [2] icp count, [3] rgb error, [4] rgb count.
int fbo_track(const fbo_config* cfg, const float* const* next_vmap, const float* const* next_nmap,
              const uint8_t* const* next_gray, const int16_t* const* next_dx,
              const int16_t* const* next_dy, const float* const* last_vmap,
              const float* const* last_nmap, const uint8_t* const* last_gray,
              const double* last_pose, double* out_pose, double* info);
// fbo_track in reference precision, summing the normal equations in the order
// of the library's tracking kernels for their grid size grid[level] (a
// multiple of 4) and solving in its solver's order; -1 on a bad grid.
int fbo_track_gpu_order(const fbo_config* cfg, const int* grid, const float* const* next_vmap,
                        const float* const* next_nmap, const uint8_t* const* next_gray,
                        const int16_t* const* next_dx, const int16_t* const* next_dy,
                        const float* const* last_vmap, const float* const* last_nmap,
                        const uint8_t* const* last_gray, const double* last_pose, double* out_pose,
                        double* info);
int fbo_num_threads(void);
}

#endif
