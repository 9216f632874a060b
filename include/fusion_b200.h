/*
 * fusion_b200 -- C ABI of the B200 implementation of the per-frame dense
 * RGB-D fusion path of cnxyang/Fusion: depth/intensity pyramid, projective
 * ICP + photometric tracking, voxel-block hash allocation, TSDF/colour
 * integration and hash-table raycasting.
 *
 * Two groups of entry points:
 *   1. A session API: one session owns the frames, the tracker state and the
 *      voxel-block map of one camera, and runs the reference's per-frame
 *      System::GrabImage (Core/System.cc:92-138) on the GPU.
 *   2. Per-stage entry points with the meaning of the reference's kernel
 *      free functions (Tracking/Reduction.h:18-83, Mapping/RenderScene.h:3-52)
 *      over plain device pointers with pitches, so that the reference's host
 *      classes (Frame, Tracker, Mapping) can call them through a thin shim.
 *
 * All functions return a status code (FB_OK = 0) and never terminate the
 * process (the reference's SafeCall exits, Utility/SafeCall.h:13-21).
 * Images are row-major; `pitch` is in bytes.  `stream` is a cudaStream_t or
 * NULL for the session's / the default stream.
 */
#ifndef FUSION_B200_H
#define FUSION_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FB_API __attribute__((visibility("default")))
#else
#define FB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define FB_OK 0
#define FB_EINVAL 1        /* bad argument */
#define FB_ENOMEM 2        /* device or pinned allocation failed */
#define FB_ECUDA 3         /* a CUDA call failed; see fb_last_error() */
#define FB_ETRACK_LOST 4   /* frame not tracked (the tracker rolled back) */

/* device-side error flags reported in fb_frame_result.error_flags (sticky) */
#define FB_ERR_HEAP_EXHAUSTED 0x1u    /* voxel-block pool full: blocks not allocated */
#define FB_ERR_EXCESS_FULL 0x2u       /* excess list full: blocks not allocated */
#define FB_ERR_REQUEST_SET_FULL 0x4u  /* per-frame block-request set overflowed */
#define FB_ERR_COORD_RANGE 0x8u       /* a block beyond +-32767 blocks was skipped */
#define FB_ERR_NEW_LIST_FULL 0x10u    /* more new blocks in one frame than the pool */
#define FB_ERR_VISIBLE_FULL 0x20u     /* visible list full */
#define FB_ERR_SEQUENTIAL_INSERT 0x40u /* pool/excess edge case: exact sequential insert used */
#define FB_ERR_TIMEOUT 0x80u          /* a bounded device-side wait (a staged copy) gave up; integration stopped */
#define FB_ERR_NORMAL_W 0x100u        /* fb_fuse_map_color: a valid normal's w lane was not 1 (ComputeNMap's) */

/* Runtime form of the reference's compile-time constants:
 * Mapping/DeviceMap.h:135-151 (voxel size, truncation, depth range, table
 * sizes), Tracking/Tracking.h:98-100 (iterations per pyramid level),
 * Core/Frame.cc:13-14 and Core/System.h:16-27 (depth scale / cutoff, camera). */
typedef struct fb_config {
    int width, height;          /* level-0 image size */
    float fx, fy, cx, cy;       /* level-0 intrinsics */
    float depth_scale;          /* depth units per metre (Frame::mDepthScale) */
    float depth_cutoff;         /* pyramid depth cutoff, m (Frame::mDepthCutoff) */
    float voxel_size;           /* m (DeviceMap::VoxelSize) */
    float trunc_dist;           /* m (DeviceMap::TruncateDist) */
    float depth_min, depth_max; /* fusion depth range, m (DeviceMap::DepthMin/Max) */
    int num_buckets;            /* hash buckets (DeviceMap::NumBuckets) */
    int num_excess;             /* excess-list entries (DeviceMap::NumExcess) */
    int num_blocks;             /* voxel blocks of 8^3 in the pool (DeviceMap::NumSdfBlocks) */
    int iters[3];               /* Gauss-Newton iterations at levels 0, 1, 2 */
    int form;                   /* FB_FORM_REFERENCE (0) or FB_FORM_PRECISION (1); no reference counterpart */
} fb_config;

/* fb_config.form.  FB_FORM_REFERENCE: the reference's arithmetic, operation
 * by operation, 8-byte voxels {f32 sdf, u8 weight, u8 r, g, b}.
 * FB_FORM_PRECISION: 6-byte voxels (FP16 TSDF, u8 weight, RGB8, stored per
 * block as separate arrays), integration in contracted FP32 with the
 * per-block camera-space basis, tracking rows in FP32 with the normal
 * equations reduced in compensated (two-float) FP32 and only the 6x6
 * solve and pose update in FP64.  Block allocation, visibility and the
 * raycast's stepping rule are the same in both forms. */
#define FB_FORM_REFERENCE 0
#define FB_FORM_PRECISION 1

/* Result of one frame (System::GrabImage). */
typedef struct fb_frame_result {
    int status;              /* FB_OK, or FB_ETRACK_LOST when not tracked */
    int tracked;             /* Tracker::GrabFrame result */
    int tracker_state;       /* Tracker::state: 1 initialising, 0 tracking, -1 lost */
    int fused;               /* the frame was integrated into the map */
    uint32_t no_visible;     /* visible blocks (FuseMapColor's host_data) */
    uint32_t no_allocated;   /* entries in the map */
    uint32_t no_new;         /* blocks allocated by this frame */
    uint32_t error_flags;    /* FB_ERR_* */
    float icp_error, icp_count, rgb_error, rgb_count;  /* last Gauss-Newton iteration */
    double pose[16];         /* camera-to-world pose, row-major (Frame::pose) */
    uint64_t frame_id;
} fb_frame_result;

typedef struct fb_session fb_session;

/* ---------------------------------------------------------------- session */

/* The reference's defaults for a width x height camera: 6 mm voxels,
 * truncation 8 voxels, depth 0.1-3.0 m, 1e6 buckets, 5e5 excess entries,
 * 7e5 blocks, iterations {10, 5, 3}, fx = fy = 525 * width / 640. */
FB_API void fb_default_config(fb_config* cfg, int width, int height);
FB_API const char* fb_status_string(int status);
/* Text of the last CUDA error seen by this library in the calling thread. */
FB_API const char* fb_last_error(void);
/* Device bytes a session with this configuration allocates. */
FB_API size_t fb_session_bytes(const fb_config* cfg);
/* Frame-graph executables: those kept for reuse by later sessions (the
 * executables of closed sessions, rewritten with cudaGraphExecUpdate when a
 * session of the same image size, form and options captures its frame
 * graphs), and the counts of captures served by an update and by a new
 * instantiation since the library was loaded.  Any pointer may be NULL. */
FB_API void fb_graph_exec_stats(long long* pooled, long long* updated, long long* instantiated);

/* Replaces: System::System (Core/System.cc:16-73) -- Mapping::Create,
 * Tracker::Tracker, Frame::Create. stream: cudaStream_t or NULL (a stream is
 * created).  FB_EINVAL for images outside width 16-4096, height 16-2048
 * (the photometric correspondences pack a 12-bit column and an 11-bit row). */
FB_API int fb_session_create(const fb_config* cfg, void* stream, fb_session** out);
FB_API int fb_session_destroy(fb_session* s);
/* Replaces: System::RebootSystem / Mapping::Reset + Tracker::ResetTracking. */
FB_API int fb_session_reset(fb_session* s);

/* Replaces: System::GrabImage (Core/System.cc:92-138), without the viewer's
 * RenderTopDown and the SURF key points.  depth: u16 in 1/depth_scale m;
 * rgb: packed RGB8.  on_device = 0: host pointers (copied in), 1: device
 * pointers.  Synchronous: returns when the frame is done. */
FB_API int fb_grab_frame(fb_session* s, const uint16_t* depth, size_t depth_pitch, const uint8_t* rgb,
                  size_t rgb_pitch, int on_device, fb_frame_result* out);
/* No counterpart in the reference.  Starts the host-to-device copy of a
 * later frame's depth and colour (host memory; pinned for the copy to run
 * asynchronously) on a copy stream of the session and returns.  A
 * fb_grab_frame call with depth = rgb = NULL takes the oldest staged frame
 * instead of copying, so the copy overlaps the frames before it: stage
 * frame k+1, then grab frame k.  At most two frames are staged at a time
 * (FB_EINVAL beyond).  The host memory must stay unchanged until the
 * fb_grab_frame that takes the frame has returned.  The staging buffers
 * (2 x 5 bytes per pixel) are allocated at the first call, outside
 * fb_session_bytes. */
FB_API int fb_stage_frame(fb_session* s, const uint16_t* depth, size_t depth_pitch, const uint8_t* rgb,
                          size_t rgb_pitch);

/* Tracing (the reference has none; Utility/StopWatch.h is never called):
 * with profiling on, every frame records CUDA events around its stages and
 * accumulates device milliseconds per stage: 0 resize of the last frame's
 * maps (its kernels run inside the pyramid's launches, so its own time is
 * only the events'), 1 pyramid and resize, 2 tracking, 3 block allocation,
 * 4 visibility, 5 integration, 6 z ranges, 7 raycast.  Switching it on
 * resets the sums. */
FB_API int fb_session_set_profiling(fb_session* s, int on);
FB_API int fb_session_stage_times(fb_session* s, double* ms, uint64_t* calls, int n);
/* Frames run as captured CUDA graphs (default on; one capture per tracker
 * mode and frame parity, made on first use).  Off: kernels launched one by
 * one.  Profiled frames always launch kernels one by one. */
FB_API int fb_session_set_graphs(fb_session* s, int on);
/* Kernels this session has launched so far. */
FB_API int fb_session_launch_count(fb_session* s, uint64_t* launches);
/* Bytes fb_grab_frame moves per frame with host inputs: h2d = depth + rgb,
 * d2h = the frame result read back. */
FB_API int fb_frame_transfer_bytes(const fb_config* cfg, size_t* h2d, size_t* d2h);

/* Captures now every frame graph the session can use (tracker modes, fusion
 * on and off, both frame parities), for frames run alone and in batch steps
 * of one to three sessions (shared = 0) or in batch steps of more sessions
 * (shared = 1, tracking kernels that leave room for the other sessions'
 * frames; the same results), so that later frames launch without capture
 * work on the host.  No reference counterpart. */
FB_API int fb_session_prepare(fb_session* s, int shared);
/* As fb_session_prepare, capturing at most max_graphs graphs now;
 * *remaining = how many are still missing.  Lets a request loop spread the
 * capture work of a newly admitted session over several steps (graph
 * instantiation takes driver locks that other threads' launches and copies
 * wait for). */
FB_API int fb_session_prepare_some(fb_session* s, int shared, int max_graphs, int* remaining);
/* The model raycast's launch shape for this session: one thread per pixel
 * in CUDA blocks of bx x by threads (bx * by <= 128 and a multiple of 32;
 * default 16 x 8), or with bx = by = 0 the queued raycast, a grid of
 * resident CTAs whose warps take 8 x 4 pixel tiles from a work counter until
 * every tile is taken.  Results do not depend on it
 * (every pixel is traced alone, by the same operations).  Cached frame
 * graphs are rebuilt on the next frame.  No reference counterpart: a tuning
 * knob for the batched form's autotuner. */
FB_API int fb_session_set_raycast_tile(fb_session* s, int bx, int by);
/* The integration kernel's grid: ctas_per_sm CTAs per SM (1..32), each
 * taking every grid-th visible block; 0 (default) is the form's own (8 CTAs
 * of 256 threads, or 7 of 128 in the precision form).  Results do not depend
 * on it.  Cached frame graphs are rebuilt on the next frame.  No reference
 * counterpart: a tuning knob for the batched form's autotuner. */
FB_API int fb_session_set_integration_grid(fb_session* s, int ctas_per_sm);

/* Snapshots (System::WriteMapToDisk / ReadMapFromDisk, Core/System.cc:195-271,
 * in memory and with the tracker included): everything a session needs to
 * continue exactly where it was -- tracker state, both frames, counters, the
 * whole hash table, the free-block stack, the allocated and visible lists
 * and the used prefix of the voxel pool (the reference writes its whole
 * pool).  A session of the same configuration restored from a snapshot gives
 * the same results, bit for bit, as the original would have.  Uses:
 * persistence, and evicting a session from HBM to bring it back later.  The
 * buffer's layout is this library's own. */
FB_API int fb_snapshot_bytes(fb_session* s, size_t* bytes);
FB_API int fb_snapshot(fb_session* s, void* host_buf, size_t capacity, size_t* written);
FB_API int fb_restore(fb_session* s, const void* host_buf, size_t size);

/* ------------------------------------------- batched and served forms
 * No reference counterpart (the reference runs one System per process).
 * A batch steps many independent sessions -- any sizes, cameras and voxel
 * sizes -- by one frame each, with all of their frames in flight on the GPU
 * together.  Every session's result is the one fb_grab_frame gives for the
 * same input on that session alone (the same kernels on the same data). */
typedef struct fb_batch fb_batch;

typedef struct {
    const uint16_t* depth;   /* u16 depth, depth_pitch bytes per row */
    size_t depth_pitch;
    const uint8_t* rgb;      /* packed RGB8, rgb_pitch bytes per row */
    size_t rgb_pitch;
    int on_device;           /* 0: host pointers (copied in), 1: device pointers */
} fb_frame_input;

/* stream: the stream the batch orders its work after (NULL: its own).
 * Session memory is one stream-ordered allocation from the device's default
 * memory pool; creating a batch sets that pool to keep freed memory for reuse
 * (release threshold) so that sessions created and destroyed while others
 * run never wait for the device. */
FB_API int fb_batch_create(void* stream, fb_batch** out);
FB_API int fb_batch_destroy(fb_batch* b);
/* Maps `bytes` of device memory into the default pool now (allocated and
 * freed at once; the pool keeps it), so that sessions created later while
 * others run do not map new memory, which the driver serialises with kernel
 * launches. */
FB_API int fb_batch_reserve(fb_batch* b, size_t bytes);
/* How a step reaches the GPU.  0 (default): each session's own frame graph
 * is launched on one of the batch's streams (no capture when the set of
 * sessions changes).  1: one graph per step holding every session's frame,
 * captured once per composition (sessions, their tracker modes and frame
 * parities) and launched as a single graph; best for a fixed set of sessions
 * stepped together.  2: fused launches -- each stage kernel of the frame runs
 * ONCE for all sessions of the step, its grid the concatenation of the
 * sessions' grids (ragged resolutions, cameras and voxel sizes in one
 * launch), so a step makes about as many launches as one frame instead of
 * one frame's launches per session; a composition seen before runs as one
 * captured graph.  Results are the same in every mode. */
FB_API int fb_batch_set_mode(fb_batch* b, int mode);
/* One frame for each of n distinct sessions; out[i] as fb_grab_frame's.
 * Synchronous.  A session must not be used elsewhere during the call. */
FB_API int fb_batch_step(fb_batch* b, fb_session* const* sessions, int n, const fb_frame_input* in,
                         fb_frame_result* out);
/* fb_batch_step in two halves: submit starts the step and collect waits for
 * it and writes out[i] for the sessions in submission order.  The inputs are
 * read by the device after submit returns: they must stay unchanged until
 * collect.  One step per batch is in flight at a time
 * (FB_EINVAL otherwise); until collect, its sessions must not be used
 * elsewhere, in particular not in another batch.  Two batches over disjoint
 * sessions, stepped alternately, keep two steps in flight: one step's last
 * kernels overlap the other's first. */
FB_API int fb_batch_submit(fb_batch* b, fb_session* const* sessions, int n, const fb_frame_input* in);
FB_API int fb_batch_collect(fb_batch* b, fb_frame_result* out);
/* Graph launches and captures so far (mode 1 captures once per composition). */
FB_API int fb_batch_stats(fb_batch* b, uint64_t* steps, uint64_t* captures);
/* Mode 2: the step's sessions are split into `lanes` groups of about equal
 * pixel counts (1..32, default 4); each group's fused launches run on a
 * stream of their own, so one group's latency-bound tracking overlaps
 * another's throughput-bound raycast and integration.  Results do not depend
 * on it. */
FB_API int fb_batch_set_lanes(fb_batch* b, int lanes);
/* Mode 2: kernel launches of the last step, and the per-session kernel
 * launches they carried (the launches modes 0 and 1 make for that step). */
FB_API int fb_batch_launch_stats(fb_batch* b, int* launches, int* kernels);

/* Pose of the last tracked frame (LastFrame->pose). */
FB_API int fb_get_pose(fb_session* s, double pose[16]);

/* Download one pyramid level of the last (which = 0) or next (1) frame to
 * host memory; any pointer may be NULL.  vmap/nmap: float4 per pixel. */
FB_API int fb_download_level(fb_session* s, int which, int level, float* vmap, float* nmap, float* depth,
                      uint8_t* gray, int16_t* dx, int16_t* dy);
/* Raw (unfiltered) level-0 depth of a frame, metres (Frame::range). */
FB_API int fb_download_raw(fb_session* s, int which, float* raw);

typedef struct fb_map_stats {
    int32_t heap_counter;   /* DeviceMap heapCounter */
    int32_t entry_ptr;      /* DeviceMap entryPtr */
    uint32_t no_allocated, no_visible, no_new, no_tiles, error_flags;
    int32_t sequential;     /* last allocation used the exact sequential path */
} fb_map_stats;
FB_API int fb_map_get_stats(fb_session* s, fb_map_stats* out);
/* All hash slots as {x, y, z, ptr, offset} with ptr a voxel index (block *
 * 512) or -1, in the reference's HashEntry order; entries has room for
 * (num_buckets + num_excess) * 5 ints. */
FB_API int fb_map_download_entries(fb_session* s, int32_t* entries);
/* Voxels of n blocks given by voxel-index ptrs: sdf, weight, rgb (n*512). */
FB_API int fb_map_download_blocks(fb_session* s, const int32_t* ptrs, int n, float* sdf, uint8_t* weight,
                           uint8_t* rgb);
/* Slots of the visible entries of the last fusion / visibility pass. */
FB_API int fb_map_download_visible(fb_session* s, int32_t* slots, uint32_t capacity, uint32_t* n);

/* -------------------------------------------------------- per-stage entries
 * Device images with pitches; the meaning of each argument is that of the
 * reference function named in the comment. */

typedef struct fb_image {
    void* data;     /* device pointer */
    size_t pitch;   /* bytes between rows */
    int cols, rows;
} fb_image;

/* Replaces: FilterDepth (Tracking/Pyrdown.cu:43-54). depth: u16; raw,
 * filtered: float. */
FB_API int fb_filter_depth(const fb_image* depth, fb_image* raw, fb_image* filtered, float depth_scale,
                    float depth_cutoff, void* stream);
/* Replaces: ImageToIntensity (Tracking/Pyrdown.cu:195-205). rgb: uchar3; gray: u8. */
FB_API int fb_image_to_intensity(const fb_image* rgb, fb_image* gray, void* stream);
/* Replaces: PyrDownGauss(float) (Tracking/Pyrdown.cu:160-169). */
FB_API int fb_pyrdown_gauss_f32(const fb_image* src, fb_image* dst, void* stream);
/* Replaces: PyrDownGauss(uchar) (Tracking/Pyrdown.cu:171-181). */
FB_API int fb_pyrdown_gauss_u8(const fb_image* src, fb_image* dst, void* stream);
/* Replaces: ComputeVMap (Tracking/Pyrdown.cu:80-91). vmap: float4. */
FB_API int fb_compute_vmap(const fb_image* depth, fb_image* vmap, float fx, float fy, float cx, float cy,
                    float depth_cutoff, void* stream);
/* Replaces: ComputeNMap (Tracking/Pyrdown.cu:116-125). */
FB_API int fb_compute_nmap(const fb_image* vmap, fb_image* nmap, void* stream);
/* Replaces: ComputeDerivativeImage (Tracking/Pyrdown.cu:239-249). dx, dy: int16. */
FB_API int fb_compute_derivative_image(const fb_image* gray, fb_image* dx, fb_image* dy, void* stream);
/* Replaces: ResizeMap (Tracking/Pyrdown.cu:281-291). */
FB_API int fb_resize_map(const fb_image* vsrc, const fb_image* nsrc, fb_image* vdst, fb_image* ndst,
                  void* stream);

/* Scratch the two step functions need, like the reference's sum / out /
 * sumRes / outRes arrays and the per-call Residual buffer
 * (Tracking/Tracking.cc:29-34, Reduction.cu:572). */
FB_API size_t fb_step_scratch_bytes(int cols, int rows);

/* No counterpart in the reference.  The grid (blocks of 256 threads, a
 * multiple of 4) of a session's per-iteration tracking kernels at a pyramid
 * level of `pixels` pixels on the current device.  The normal equations are
 * summed in a fixed order that depends only on this number, so a checker can
 * sum in the same order and compare the tracker bit for bit.  0 on error. */
FB_API int fb_track_reduction_grid(int pixels);

/* Replaces: ICPStep (Tracking/Reduction.cu:319-375).  R* are row-major 3x3
 * (Matrix3f), t* 3-vectors, K = {fx, fy, cx, cy} of the level.  Outputs on
 * the host as the reference's: residual = {sum of squared point-to-plane
 * residuals, correspondence count}, A (6x6 row-major), b (6).
 * Synchronous. */
FB_API int fb_icp_step(const fb_image* vcurr, const fb_image* vlast, const fb_image* ncurr,
                const fb_image* nlast, const float Rcurr[9], const float tcurr[3], const float Rlast[9],
                const float RlastInv[9], const float tlast[3], const float K[4], void* scratch,
                size_t scratch_bytes, float residual[2], double A[36], double b[6], void* stream);

/* Replaces: RGBStep (Tracking/Reduction.cu:547-627).  gray: u8, dx/dy: int16
 * of the current frame.  Synchronous. */
FB_API int fb_rgb_step(const fb_image* gcurr, const fb_image* glast, const fb_image* vcurr,
                const fb_image* vlast, const fb_image* dx, const fb_image* dy, const float Rcurr[9],
                const float RcurrInv[9], const float Rlast[9], const float RlastInv[9],
                const float tcurr[3], const float tlast[3], const float K[4], void* scratch,
                size_t scratch_bytes, float residual[2], double A[36], double b[6], void* stream);

/* No counterpart in the reference.  fb_rgb_step for callers that cannot
 * allocate device memory when they track a frame -- frame loops that cannot
 * pay for cudaFree's device-wide wait, plug-ins in hosts whose device memory
 * all belongs to the host's own allocator.  Same arguments without the
 * scratch: the library keeps 1.25 MiB of device memory per GPU for it, so
 * images may have at most fb_rgb_step_static_max_pixels() (640 x 480)
 * pixels; larger ones are rejected with FB_EINVAL.  The first call on a
 * device looks up that memory's address and should come before any stream
 * capture.  Every call shares the memory: calls that overlap on the GPU
 * (other streams, unordered threads) corrupt each other's results.
 * Synchronous: returns once the sums are on the host. */
FB_API int fb_rgb_step_static(const fb_image* gcurr, const fb_image* glast, const fb_image* vcurr,
                              const fb_image* vlast, const fb_image* dx, const fb_image* dy,
                              const float Rcurr[9], const float RcurrInv[9], const float Rlast[9],
                              const float RlastInv[9], const float tcurr[3], const float tlast[3],
                              const float K[4], float residual[2], double A[36], double b[6], void* stream);
FB_API size_t fb_rgb_step_static_max_pixels(void);

/* Replaces: ResetMap (Mapping/FuseMap.cu:352-364) on the session's map. */
FB_API int fb_reset_map(fb_session* s);

/* Replaces: FuseMapColor (Mapping/FuseMap.cu:251-319) on the session's map:
 * block allocation, visibility and integration of one frame.  depth: raw
 * float depth; rgb: uchar3; nmap: float4; Rview/RviewInv row-major; K =
 * {fx, fy, cx, cy}; depth range from the session config.  no_visible:
 * visible block count (host). */
FB_API int fb_fuse_map_color(fb_session* s, const fb_image* depth, const fb_image* rgb, const fb_image* nmap,
                      const float Rview[9], const float RviewInv[9], const float tview[3],
                      const float K[4], uint32_t* no_visible, void* stream);

/* Replaces: CheckBlockVisibility (Mapping/FuseMap.cu:206-249) for a cols x
 * rows camera. */
FB_API int fb_check_block_visibility(fb_session* s, const float Rview[9], const float RviewInv[9],
                              const float tview[3], int cols, int rows, const float K[4],
                              uint32_t* no_visible, void* stream);

/* Replaces: CreateRenderingBlocks (Mapping/RenderScene.cu:199-276, declared
 * at Mapping/RenderScene.h:20-27): the z ranges of the session's visible
 * blocks seen from (RviewInv, tview) with intrinsics K, written into the
 * caller's z-range images zmin / zmax (float, at least ceil(W/8) x ceil(H/8)
 * of the session's camera; tiles with no block hold 100 and 0, as the
 * reference initialises them), and the number of rendering tiles.  The
 * reference's RenderingBlock list is an intermediate of its own; the library
 * keeps a dense block index instead and writes no list. */
FB_API int fb_create_rendering_blocks(fb_session* s, const float RviewInv[9], const float tview[3],
                                      const float K[4], fb_image* zmin, fb_image* zmax, uint32_t* no_tiles,
                                      void* stream);

/* Replaces the visibleEntries array that CheckBlockVisibility and
 * FuseMapColor fill in the reference (Mapping/FuseMap.cu:206-249): the
 * session's visible entries, in order, written to device memory `entries`
 * (16-byte aligned) in the reference's 32-byte HashEntry layout
 * (Mapping/DeviceMap.h:17-59: int3 pos, int ptr = voxel index or -1, int
 * offset, padding).  *n = the number of visible entries; FB_EINVAL when more
 * than `capacity`. */
FB_API int fb_map_export_visible(fb_session* s, void* entries, uint32_t capacity, uint32_t* n, void* stream);

/* The session's map written into the reference's own device buffers -- the
 * DeviceMap views Mapping::operator DeviceMap passes (Mapping/Mapping.cc:
 * 311-325): hashEntries (NumBuckets + NumExcess HashEntry), voxelBlocks
 * (NumSdfBlocks * 512 Voxel of 8 bytes; the precision form's FP16 TSDF
 * widened), heapMem (NumSdfBlocks int), heapCounter and entryPtr (one int
 * each).  The library keeps its map in its own layout; code that reads
 * Mapping's buffers directly (System::WriteMapToDisk, Core/System.cc:195-231)
 * calls this first.  The sizes must be the session's. */
FB_API int fb_map_export_reference(fb_session* s, void* hash_entries, size_t n_entries, void* voxels,
                                   size_t n_voxels, int32_t* heap, size_t n_heap, int32_t* heap_counter,
                                   int32_t* entry_ptr, void* stream);

/* Replaces: CreateRenderingBlocks + Raycast (Mapping/RenderScene.cu:199-276,
 * 447-489) as called by Mapping::RayTrace (Mapping/Mapping.cc:98-109): z
 * ranges of the visible blocks, then the raycast into vmap/nmap (float4,
 * camera frame).  Returns with *rendered = 0 and the maps untouched when no
 * rendering rectangle was produced. */
FB_API int fb_raycast(fb_session* s, fb_image* vmap, fb_image* nmap, const float Rview[9],
               const float RviewInv[9], const float tview[3], const float K[4], int* rendered,
               void* stream);

/* Headless rendering (no graphics API; the image is device memory).
 * fb_render_image replaces RenderImage (Tracking/Reduction.h:44-46,
 * Tracking/Pyrdown.cu:322-380): Phong shading of a raycast vertex/normal map
 * (camera frame) lit from `light`, RGBA8, a gradient where there is no
 * vertex.  fb_depth_to_image replaces DepthToImage (Reduction.h:48-49,
 * Pyrdown.cu:382-405), fb_rgb_to_rgba RgbImageToRgba (Reduction.h:51-52,
 * Pyrdown.cu:407-428).  rgba: uchar4 per pixel. */
FB_API int fb_render_image(const fb_image* vmap, const fb_image* nmap, const float light[3], fb_image* rgba,
                           void* stream);
FB_API int fb_depth_to_image(const fb_image* depth, fb_image* rgba, void* stream);
FB_API int fb_rgb_to_rgba(const fb_image* rgb, fb_image* rgba, void* stream);

/* Replaces: System::WriteMapToDisk (Core/System.cc:195-236, with
 * Mapping::DownloadToRAM, Mapping/Mapping.cc:170-184): the map in the
 * reference's dump layout -- int sizes {NumSdfBlocks, NumBuckets, NumVoxels,
 * NumEntries}, heap counter, excess counter, visible count, free-block
 * stack, bucket locks, voxels (8 B), hash entries and visible entries
 * (32-byte HashEntry, ptr a voxel index), key-point locks and SURF entries
 * (none kept here: unlocked and zero).  Either form (the precision form's
 * TSDF is widened to float).  The reference reads a file whose sizes match
 * its compile-time constants (fb_default_config's). */
FB_API int fb_write_map_file(fb_session* s, const char* path);
/* Replaces: System::ReadMapFromDisk (Core/System.cc:238-271, with
 * Mapping::UploadFromRAM, Mapping.cc:186-200) for the map: loads a file in
 * that layout whose sizes equal the session's, rebuilds this library's
 * allocated list (in block order) and visible list, and, as the reference,
 * restarts the tracker and disables mapping (fb_session_set_mapping).  The
 * reference's CreateModel after loading is fb_mesh_scene, on demand. */
FB_API int fb_read_map_file(fb_session* s, const char* path);
/* Tracker::mappingDisabled (Tracking/Tracking.h) off (on = 1, the default)
 * or on (on = 0): frames then track and raycast against the map, refreshing
 * the visible blocks first, without fusing (System.cc:109-118). */
FB_API int fb_session_set_mapping(fb_session* s, int on);

/* ------------------------------------------------------------ key points
 * The reference's SURF path (OpenCV CUDA SURF, absent here; this library's
 * own detector and descriptor follow the published SURF method): key points
 * of every frame with a 3-D point (Frame::ExtractKeyPoints, Core/Frame.cc:
 * 165-212), the bootstrap pose from matches with the last frame before ICP
 * (Tracker::TrackLastFrame, Tracking/Tracking.cc:169-204), keyframes with
 * observation counts (Tracking.cc:75-85, 113-148, 208-234), the key map they
 * are fused into (Mapping::FuseKeyFrame, Mapping/Mapping.cc:220-275) and
 * relocalisation against it when the camera is lost (Tracker::Relocalise,
 * Tracking.cc:411-470).  Off by default (the rest of this library runs the
 * reference's loop as it runs without key points); sessions with key points
 * on are stepped by fb_grab_frame only (not in batches).  The RANSAC solver
 * (Solver::PoseEstimate) draws its samples from a seeded sequence instead of
 * the clock. */
typedef struct fb_keypoint_stats {
    uint32_t keys;          /* key points with a 3-D point in the last frame */
    uint32_t matches;       /* ratio-test matches of its bootstrap or relocalisation */
    int32_t bootstrap;      /* TrackLastFrame: 1 pose found, 0 not, -1 not run */
    int32_t relocalised;    /* Relocalise: 1 pose found, 0 not, -1 not run */
    uint32_t keyframes;     /* keyframes created */
    uint32_t map_keys;      /* keys in the key map */
} fb_keypoint_stats;
FB_API int fb_session_set_keypoints(fb_session* s, int on);
FB_API int fb_session_keypoint_stats(fb_session* s, fb_keypoint_stats* out);
/* The key points of the last (which = 0) or next (1) frame, host arrays:
 * kp {x, y, scale, angle}, pts {x, y, z, 1} camera space, nrm (float4),
 * desc 64 floats each; any may be NULL.  *n = keys (at most capacity
 * written). */
FB_API int fb_download_keypoints(fb_session* s, int which, float* kp, float* pts, float* nrm, float* desc,
                                 uint32_t capacity, uint32_t* n);
/* Brute-force two-nearest-neighbour matching (cv::cuda BFMatcher knnMatch,
 * L2, k = 2) of nq query descriptors against nt train descriptors (64
 * floats each, device pointers): best (nq x 2 int: nearest, second nearest,
 * -1 when missing) and dist (nq x 2 float, L2 distances), device pointers.
 * Synchronous. */
FB_API int fb_match_descriptors(const float* query, uint32_t nq, const float* train, uint32_t nt, int32_t* best,
                                float* dist, void* stream);
/* Replaces: Solver::PoseEstimate (Optimization/Solver.cc:6-186), host
 * arrays: n matched points src / ref (3 doubles each); T (4x4 row-major)
 * maps ref onto src; inlier[i] = 1 for the final inliers (may be NULL).
 * Returns FB_OK with *ok = 1 when a pose was accepted.  Host only. */
FB_API int fb_pose_estimate(const double* src, const double* ref, uint32_t n, int iterations, int check_angle,
                            uint64_t seed, double T[16], uint8_t* inlier, int* ok);

/* Replaces: System::RenderTopDown (Core/System.cc:75-90): the model seen
 * from `dist` metres above the origin looking down (+y), the depth range
 * shifted by `dist`: visibility for a 640 x 480 camera (as the reference's
 * Mapping::UpdateVisibility), z ranges, raycast into vmap/nmap (float4,
 * camera frame, the frame's fx, fy and the image centre), then Phong shading
 * into rgba (uchar4, light at the camera).  All images one size, at most the
 * session's.  Replaces the session's visible-block list, as the reference
 * does.  *rendered = 0 when no block was in view: vmap/nmap are then left
 * as they were and rgba is shaded from them, as in the reference.
 * Synchronous. */
FB_API int fb_render_top_down(fb_session* s, float dist, fb_image* vmap, fb_image* nmap, fb_image* rgba,
                              int* rendered, void* stream);

/* Replaces: MeshScene (Mapping/MeshScene.cu:306-355) as called by
 * Mapping::CreateModel (Mapping/Mapping.cc:131-140): marching cubes over every
 * voxel of every allocated block.  Triangle soup, three vertices per
 * triangle: vertex and normal float3 (metres, unit gradient normals), color
 * uchar3, device pointers.  *no_triangles = all triangles the map holds; the
 * first min(that, max_triangles) are written, in a deterministic order
 * (blocks in allocation order, voxels in index order).  vertex = normal =
 * color = NULL counts only.  The vertices are the reference's, bit for bit;
 * the triangles over them come from this library's case table
 * (fb_mesh_case_table), which keeps ambiguous faces consistent between
 * neighbouring cubes.  Synchronous. */
FB_API int fb_mesh_scene(fb_session* s, float* vertex, float* normal, uint8_t* color, uint64_t max_triangles,
                         uint64_t* no_triangles, void* stream);
/* The marching-cubes case table fb_mesh_scene uses (the role of the
 * reference's triangleTableHost / vertexTableHost, Mapping/Constant.h): for
 * each of the 256 cases (bit i set: corner i has sdf < 0, corners in
 * MeshScene.cu's order) up to 5 triangles as edge triples, -1 filled;
 * counts[case] = triangles.  tri: 256 x 16.  Host only. */
FB_API int fb_mesh_case_table(int8_t* tri, int32_t* counts);
/* Replaces the file writing of System::WriteMeshToDisk (Core/System.cc:
 * 140-193): ASCII PLY with the reference's header and number formatting,
 * one PLY vertex per triangle corner.  Host pointers.  Synchronous. */
FB_API int fb_write_ply(const char* path, const float* vertex, const float* normal, const uint8_t* color,
                        uint64_t no_triangles);
/* System::WriteMeshToDisk as one call: fb_mesh_scene into temporary device
 * memory, download, fb_write_ply to `path`.  *no_triangles may be NULL. */
FB_API int fb_save_mesh(fb_session* s, const char* path, uint64_t* no_triangles);


#ifdef __cplusplus
}
#endif

#endif /* FUSION_B200_H */
