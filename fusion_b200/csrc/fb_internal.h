// Internal interfaces between the translation units of libfusion_b200.so.
#ifndef FB_INTERNAL_H
#define FB_INTERNAL_H

#include <cuda_runtime.h>
#include <stdint.h>

#include "fb_common.cuh"

namespace fb {

// ------------------------------------------------------------------ tracking

constexpr int kTrackMaxBlocks = 592;   // 4 resident blocks of 256 threads per SM
// The per-iteration kernels run in thread-block clusters of kTrackCluster
// blocks; each cluster reduces its blocks' sums through distributed shared
// memory into one group sum.
constexpr int kTrackCluster = 4;
constexpr int kTrackMaxGroups = kTrackMaxBlocks / kTrackCluster;
constexpr int kTrackWarps = 8;         // warps per block of the per-iteration kernels

// One pyramid level of the current (next) and last frames.  Pitches in
// elements: vp for float4 maps, gp for u8 images, sp for i16 derivatives.
struct TrackLevel {
    int W, H, vp, gp, sp;
    Intr k;
    const float4* vcurr;
    const float4* ncurr;
    const float4* vlast;
    const float4* nlast;
    const uint8_t* gcurr;
    const uint8_t* glast;
    const int16_t* dx;
    const int16_t* dy;
    const uint8_t* rgbok;   // pose-independent photometric eligibility (may be null)
};

// Device-resident tracker state of one session (Tracker's poses, residuals).
struct TrackState {
    double last_pose[16];   // pose of the last (model) frame
    double pose[16];        // current estimate of the next frame's pose
    double init_pose[16];   // the next pose when ComputeSE3 started
    double delta[16];       // accumulated increment (Tracking.cc:314, 392)
    DevPose cur, last;      // float views of pose / last_pose
    int failed;             // tracking of this frame failed (pose rolled back)
    int pad0;
    float icp_error, icp_count, rgb_error, rgb_count;
    float sigma;
    int pad1;
    long long rgb_cnt, rgb_sq;
    double icp_sums[29];
    double rgb_sums[29];
    long long scratch_cnt[kTrackMaxBlocks];
    long long scratch_sq[kTrackMaxBlocks];
    // per-cluster group sums of the per-iteration kernels (FP64, fixed order)
    double grp_icp[kTrackMaxGroups][32];
    double grp_rgb[kTrackMaxGroups][32];
    long long grp_cnt[kTrackMaxGroups];
    long long grp_sq[kTrackMaxGroups];
    // precision form: the group sums as compensated FP32 pairs (hi, lo)
    float2 grp_icp2[kTrackMaxGroups][32];
    float2 grp_rgb2[kTrackMaxGroups][32];
};

int track_grid(int n);
int track_cluster_grid(int n);   // track_grid rounded up to whole clusters
int launch_track_begin(TrackState* st, cudaStream_t s);
// residual: per-warp compact segments of photometric correspondences
// (int2: the pixel's Sobel derivatives dx | dy << 16, packed last pixel + difference), capacity track_list_capacity;
// counts: entries per segment (kTrackMaxBlocks * kTrackWarps ints)
// shared_gpu: the instance with four resident blocks per SM (other sessions'
// kernels run beside it); same results as the two-block instance
int launch_track_iter(const TrackLevel& L, TrackState* st, unsigned int* tickets, int2* residual, int* counts,
                      int min_count, bool is_final, cudaStream_t s, bool shared_gpu = false,
                      bool compensated = false);
size_t track_list_capacity(int n_pixels);
int launch_step_icp(const TrackLevel& L, const DevPose& cur, const DevPose& last, float* partials,
                     unsigned int* ticket, double* out, cudaStream_t s);
int launch_step_rgb(const TrackLevel& L, const DevPose& cur, const DevPose& last, float* partials,
                     unsigned int* tickets, int* residual, double* out, cudaStream_t s);

// ------------------------------------------------------------- preprocessing

int launch_level0(const uint16_t* depth, int dpitch, const uint8_t* rgb, int rgbpitch, int W, int H,
                   float depth_scale, float cutoff, float* raw, int rawpitch, float* filt, int fpitch,
                   uint8_t* gray, int gpitch, cudaStream_t st);
int launch_pyrdown(const float* sd, int sdp, const uint8_t* sg, int sgp, int SW, int SH, float* dd, int ddp,
                    uint8_t* dg, int dgp, cudaStream_t st);
// Where the level-0 map kernel writes the fusion records of its pixels
// (fuse_record): the raw depth and RGB8 image they are made from, the fusion
// depth range, and the destinations (W wide); rec null: none.
struct FuseRecDst {
    const float* raw;
    int rp;
    const uint8_t* rgb;
    int cp;
    float dmin, dmax;
    float4* rec;
    uint32_t* col;
    int packed;   // 1: the precision form's 16-byte records (fuse_record_packed) in rec, col unused
};
int launch_maps(const float* depth, int dp, const uint8_t* gray, int gp, int W, int H, const Intr& k,
                 float cutoff, float4* vmap, int vp, float4* nmap, int np, int16_t* dx, int16_t* dy, int sp,
                 cudaStream_t st, uint8_t* rgbok = nullptr, const FuseRecDst* fr = nullptr);
int launch_nmap(const float4* vmap, int vp, int W, int H, float4* nmap, int np, cudaStream_t st);
int launch_resize(const float4* vs, const float4* ns, int sp, int SW, int SH, float4* vd, float4* nd, int dp,
                   cudaStream_t st);

// One launch of a frame's preprocessing whose blocks take up to four roles,
// each the kernel of the same name above over its own image as a grid of
// 32 x 8 blocks (gx x gy; 0 x 0: role absent); the launch's 1-D grid holds
// the roles' grids one after another in the order level 0, resize, pyrdown,
// maps.  Roles in one launch must not depend on each other.
struct Level0Args {
    const uint16_t* depth;
    int dpitch;
    const uint8_t* rgb;
    int rgbpitch, W, H;
    float inv, cutoff;
    float* raw;
    int rawpitch;
    float* filt;
    int fpitch;
    uint8_t* gray;
    int gpitch;
};
struct ResizeArgs {
    const float4* vs;
    const float4* ns;
    int sp, SW, SH;
    float4* vd;
    float4* nd;
    int dp;
};
struct PyrArgs {
    const float* sd;
    int sdp;
    const uint8_t* sg;
    int sgp, SW, SH;
    float* dd;
    int ddp;
    uint8_t* dg;
    int dgp;
};
struct MapsArgs {
    const float* depth;
    int dp;
    const uint8_t* gray;
    int gp, W, H;
    Intr k;
    float cutoff;
    float4* vmap;
    int vp;
    float4* nmap;
    int np;
    int16_t* dxo;
    int16_t* dyo;
    int sp;
    uint8_t* rgbok;
    FuseRecDst fr;
};
struct PreLaunch {
    Level0Args l0;
    ResizeArgs rs;
    PyrArgs py;
    MapsArgs mp;
    int gx[4], gy[4];
};
// Role setters (same arguments as the launchers above) and the launch.
void pre_level0(PreLaunch& P, const uint16_t* depth, int dpitch, const uint8_t* rgb, int rgbpitch, int W, int H,
                float depth_scale, float cutoff, float* raw, int rawpitch, float* filt, int fpitch, uint8_t* gray,
                int gpitch);
void pre_resize(PreLaunch& P, const float4* vs, const float4* ns, int sp, int SW, int SH, float4* vd, float4* nd,
                int dp);
void pre_pyrdown(PreLaunch& P, const float* sd, int sdp, const uint8_t* sg, int sgp, int SW, int SH, float* dd,
                 int ddp, uint8_t* dg, int dgp);
void pre_maps(PreLaunch& P, const float* depth, int dp, const uint8_t* gray, int gp, int W, int H, const Intr& k,
              float cutoff, float4* vmap, int vp, float4* nmap, int np, int16_t* dx, int16_t* dy, int sp,
              uint8_t* rgbok, const FuseRecDst* fr);
int launch_pre(const PreLaunch& P, cudaStream_t st);

// ----------------------------------------------------------------------- map

struct MapCounters {
    int heap_counter;      // top of the free-block stack (DeviceMap heapCounter)
    int entry_ptr;         // next excess-list slot, 1-based (DeviceMap entryPtr)
    int holes;             // an entry with ptr -1 was linked (pool exhausted once)
    int n_alloc;           // entries in the allocated list
    int n_req;             // new blocks requested this frame
    int n_new;             // blocks inserted by the last allocation
    int n_visible;         // visible blocks of the last fusion / visibility pass
    int n_tiles;           // rendering rectangles of the last z-range pass
    // dense block index of the last z-range pass: the box of the visible
    // blocks (+1 block each side) when it fits the grid's capacity
    int bmin[3], bmax[3];
    int g_o[3], g_n[3], g_on;
    int excess_total;      // new blocks going to the excess list this frame
    unsigned int err;      // ErrFlag bits, sticky
    int seq_path;          // last allocation used the sequential path
    // snapshot taken before insertion (read by the insert kernel only)
    int snap_M, snap_hc, snap_ep, snap_na;
    int fast;              // the parallel insertion path applies
    unsigned int ray_next; // tile counter of the queued raycast (zeroed with the z ranges)
    unsigned int scan_ticket; // chunk-scan blocks done this frame (the last one resets it)
};

struct NewBlock {
    short x, y, z, pad;
    uint32_t bucket;
    int setslot;           // slot in the request set (cleared after insertion)
    int j;                 // arrival index inside the bucket
    int rank;              // canonical rank: order by (bucket, x, y, z)
    int pad2;
};

// Geometry of the map (runtime form of DeviceMap's constants).
struct MapGeom {
    float voxel_size, voxel_size_inv, trunc_dist, step_scale, block_width;
    float depth_min, depth_max;
};

struct MapView {
    HEntry* entries;
    int NB, NE, NS;
    uint32_t nb_mask;           // NB - 1 when NB is a power of two, else 0
    int* heap;
    Voxel* voxels;              // reference form: NS x 512 voxels of 8 B
    uint8_t* cvox;              // precision form: NS blocks of kCBlockBytes (voxels then null)
    MapCounters* ctr;
    int* alloc_list;            // slots of allocated entries, allocation order (NS)
    int* visible;               // slots of visible entries (NS)
    HEntry* vis_blocks;         // the visible entries themselves (NS), same order
    int* grid;                  // dense block index for the raycast (grid_cap cells, -1: none)
    int grid_cap;
    unsigned long long* reqset; // request set, open addressing (reqcap, power of 2)
    int reqcap;
    NewBlock* newblk;           // this frame's new blocks (newcap)
    int newcap;
    int* order;                 // canonical order -> newblk index (newcap)
    int* arrival;               // bucket segment -> newblk index (newcap)
    int* bucket_cnt;            // NB, zero between frames
    int* bucket_start;          // NB
    int* bucket_x;              // NB: excess start << 1 | head-was-empty
    int* chunk_sums;            // 2 * nchunks
    int nchunks;
    float* zmin;                // z-range image, zc x zr
    float* zmax;
    int zc, zr;
    float4* frec;               // fusion records, 8 zc x 8 zr: {depth or NaN, normal xyz} (fuse_record), or
                                // in the precision form one packed 16-byte word each (fuse_record_packed)
    uint32_t* fcol;             // reference form: the records' colours r | g << 8 | b << 16
    // raycast block order (a scheduling hint; no result depends on it): each
    // raycast warp records its duration in rc_cost[tile] (clock cycles, max
    // over the tile's warps); the z-range pass turns the last raycast's costs
    // into rc_order = {tile count n, then the n tiles slowest first} and
    // clears them; a raycast of n tiles runs its blocks in that order
    uint32_t* rc_cost;          // rc_cap
    int* rc_order;              // 1 + rc_cap
    int rc_cap;
    MapGeom g;
};

// Tiles of the raycast's block grid for a W x H image in bx x by blocks, and
// the most any block shape of 32..128 threads (a multiple of 32) can need.
inline int raycast_tiles(int W, int H, int bx, int by) {
    return bx > 0 && by > 0 ? ((W + bx - 1) / bx) * ((H + by - 1) / by) : 0;
}
inline int raycast_tile_cap(int W, int H) { return W * H / 32 + W + H + 1; }

constexpr int kScanChunk = 4096;
constexpr int kMinNewBlocks = 1 << 16;

int launch_map_reset(const MapView& m, cudaStream_t s);
// pose: device pointer; skip: device flag (nonzero: do nothing), may be null
int launch_allocate(const MapView& m, const float* raw, int rp, int W, int H, const Intr& k, const DevPose* pose,
                     const int* skip, cudaStream_t s);
// after_allocate: launched right after launch_allocate, whose last kernel
// already zeroed the visible-block and rendering-rectangle counters.
int launch_visibility(const MapView& m, int W, int H, const Intr& k, const DevPose* pose, const int* skip,
                       cudaStream_t s, bool after_allocate = false);
// The visible entries (at most `capacity`) in the reference's 32-byte
// HashEntry layout at dst; the table, voxels and counters in the reference's
// layouts (the reference form's voxels are the reference's already: the
// caller copies them).
int launch_export_visible(const MapView& m, void* dst, int capacity, cudaStream_t s);
int launch_export_reference(const MapView& m, void* entries, void* voxels, int* heap_counter, int* entry_ptr,
                            cudaStream_t s);
// Fusion records (m.frec / m.fcol, W wide) of a raw depth map, RGB8 image and
// normal map; the frame path makes them in the level-0 map kernel instead.
int launch_fuse_records(const MapView& m, const float* raw, int rp, const uint8_t* rgb, int cp, const float4* nmap,
                        int np, int W, int H, cudaStream_t s);
// Integration of the visible blocks from the fusion records of a W x H frame.
// ctas_per_sm: the grid (CTAs per SM, each taking every grid-th visible
// block); 0: the form's default.  Results do not depend on it.
int launch_integrate(const MapView& m, int W, int H, const Intr& k, const DevPose* pose, const int* skip,
                     cudaStream_t s, int ctas_per_sm = 0);
// rc_tiles: tiles of the raycast that follows (raycast_tiles), whose block
// order this pass prepares from the last raycast's costs; 0: leave it as it is.
int launch_zrange(const MapView& m, const Intr& k, const DevPose* pose, const int* skip, cudaStream_t s,
                  int rc_tiles = 0);
// tile bx x by threads: bx * by <= 128 (the kernel's launch bound), a multiple
// of 32; bx = by = 0: the queued raycast (warps take 8 x 4 pixel tiles from a counter)
int launch_raycast(const MapView& m, float4* vmap, float4* nmap, int p, int W, int H, const Intr& k,
                    const DevPose* pose, const int* skip, cudaStream_t s, int bx = 16, int by = 8);

// ----------------------------------------------------------------- key points

constexpr int kSurfOctaves = 4;      // SURF_CUDA defaults: 4 octaves ...
constexpr int kSurfLayers = 4;       // ... of nOctaveLayers + 2 = 4 filter sizes
constexpr int kSurfMaxCand = 16384;  // candidates ranked per detection
constexpr int kKeyDesc = 64;         // descriptor values

// Device scratch of one detection on a W x H image.
struct KeyScratch {
    int W, H, max_keys;              // max_keys: 1 % of the pixels (SURF_CUDA keypointsRatio)
    uint32_t* integral;              // (W + 1) x (H + 1)
    float* det[kSurfOctaves];        // [layer][H >> o][W >> o]
    int ow[kSurfOctaves], oh[kSurfOctaves];
    float4* cand;                    // kSurfMaxCand: x, y, scale, response
    unsigned long long* keys;        // kSurfMaxCand sort keys
    int* slotmap;                    // sample index -> candidate slot
    int* counter;
    float4* kp;                      // max_keys selected: x, y, scale, angle
    float* desc;                     // max_keys x kKeyDesc
};

// The key points of a frame that have a 3-D point (Frame::ExtractKeyPoints).
struct KeySet {
    float4* kp;     // x, y, scale, angle
    float4* pt;     // camera-space point, w = 1
    float4* nrm;    // normal (level-0 normal map, interpolated)
    float* desc;    // kKeyDesc per key
    int cap;
};

size_t key_scratch_bytes(int W, int H);
int key_scratch_carve(void* base, size_t bytes, int W, int H, KeyScratch& ks);
// detection and description on the level-0 gray image; *n_keys = key points
// described into ks.kp / ks.desc (synchronises st)
int launch_surf(const uint8_t* gray, int gp, float threshold, const KeyScratch& ks, int* n_keys, cudaStream_t st);
// the key points with a depth and a normal -> out (count in *d_n, device)
int launch_backproject(const KeyScratch& ks, int n, const float* depth, int dp, const float4* nmap, int np,
                       const Intr& k, float cutoff, const KeySet& out, int* d_n, cudaStream_t st);
// two nearest train descriptors per query: idx {best, second}, dist {d1, d2}
int launch_match2(const float* q, int nq, const float* t, int nt, int2* idx, float2* dist, cudaStream_t st);
// Solver::PoseEstimate: T (4x4, row-major) maps ref points onto src points;
// outlier[i] = 0 for the final inliers.  Host.
bool pose_estimate(const double* src, const double* ref, int n, int iterations, bool check_angle, uint64_t seed,
                   double T[16], uint8_t* outlier);

// Marching-cubes mesh of the map over its n_blocks allocated blocks: *total =
// triangles found; the first min(total, cap) written to V / N (float3 per
// vertex) and C (uchar3) when all three are given.  Synchronous on st.
int launch_mesh(const MapView& m, int n_blocks, float* V, float* N, uint8_t* C, unsigned long long cap,
                unsigned long long* total, cudaStream_t st);

}  // namespace fb

// Text returned by fb_last_error() in the calling thread.
void fb_set_error_text(const char* msg);

#endif
