// Internal interfaces between the session units of libfusion_b200.so:
// session.cu (session objects, frame issue, frame graphs, the session's C
// entry points), keyframe_track.cu (key-point tracking steps),
// stage_api.cu (the per-stage C entry points), persist.cu (snapshots and
// the reference's map file) and batch_step.cu (batched steps).
#ifndef FB_SESSION_INTERNAL_H
#define FB_SESSION_INTERNAL_H

#include <cstdio>
#include <map>
#include <tuple>
#include <vector>

#include "../../include/fusion_b200.h"
#include "fb_fused.cuh"
#include "fb_internal.h"

// Returns FB_ECUDA from the calling function when a CUDA call fails.
#define FB_CUDA(call)                          \
    do {                                       \
        if (!cuda_ok(call)) return FB_ECUDA;   \
    } while (0)

namespace fb {

// The calling thread's last error text (fb_last_error).
extern thread_local char g_last_error[256];
// Records e's text as the last error; true when e is cudaSuccess.
bool cuda_ok(cudaError_t e);
// The last launch error as a status.
int check_launch();

// Compact result gathered on the device at the end of a frame.
struct FrameOut {
    double pose[16];
    int failed;
    float icp_error, icp_count, rgb_error, rgb_count;
    int n_alloc, n_visible, n_new, n_tiles;
    unsigned err;
    int heap_counter, entry_ptr, seq_path;
};

// What one frame does, decided on the host before it is issued.
struct FramePlan {
    int state;      // tracker state at this frame: 1 init, 0 tracking, -1 lost
    bool init, track, fuse, render;
    int after;      // frames_after_reloc after this frame
    int mode;       // 0 init, 1 track, 2 lost (graph key)
};

struct FrameBuf {
    uint16_t* depth_in;
    uint8_t* rgb;
    float* raw;
    float* depth[3];
    float4* vmap[3];
    float4* nmap[3];
    uint8_t* gray[3];
    int16_t* dx[3];
    int16_t* dy[3];
    uint8_t* rgbok[3];     // pose-independent photometric eligibility per level
};

constexpr int kStages = 8;   // resize, pyramid, tracking, allocation, visibility, integration, z ranges, raycast

// Key points of a session (fb_session_set_keypoints): the reference's SURF
// path -- Frame::ExtractKeyPoints on every frame, Tracker::TrackLastFrame's
// bootstrap, keyframes with observation counts, the key map
// (Mapping::FuseKeyFrame) and Tracker::Relocalise.
constexpr int kKeyMapCap = 500000;   // KeyMap::maxEntries
struct HostKeyFrame {
    double pose[16];
    int n = 0;
    std::vector<float> pts, nrm;   // 4 per key, camera space
    std::vector<int> obs;
};
struct KeyState {
    void* mem = nullptr;
    KeyScratch ks;
    KeySet set[2];                 // per frame buffer
    int n[2] = {0, 0};
    std::vector<float> pts[2], nrm[2];
    int* d_n = nullptr;
    int2* m_idx = nullptr;         // match results (queries = one frame's keys)
    float2* m_dist = nullptr;
    float* kf_desc = nullptr;      // the reference keyframe's descriptors
    HostKeyFrame kf;
    bool has_kf = false;
    float* map_desc = nullptr;     // the key map (KeyMap): descriptors ...
    int map_n = 0;
    std::vector<float> map_pos;    // ... world positions (3 per key)
    std::map<std::tuple<int, int, int>, int> map_cells;   // 1 cm grid cell -> key
    fb_keypoint_stats stats{};
};

// Frames staged by fb_stage_frame: host-to-device copies on their own
// stream into two buffers outside the arena, consumed in order by
// fb_grab_frame.
struct StagedInput {
    cudaStream_t copy = nullptr;
    uint16_t* depth[2] = {nullptr, nullptr};
    uint8_t* rgb[2] = {nullptr, nullptr};
    cudaEvent_t ready[2] = {nullptr, nullptr};   // copy done (copy stream)
    cudaEvent_t freed[2] = {nullptr, nullptr};   // taken into the frame (session stream)
    int head = 0, count = 0;
};


// The tracker's starting pose of a frame (the key-point bootstrap's).
struct Pose16 {
    double m[16];
};

}  // namespace fb

using namespace fb;

struct fb_session {
    fb_config cfg;
    cudaStream_t stream;
    bool own_stream;
    StagedInput* staged = nullptr;
    int W[3], H[3];
    Intr K[3];
    FrameBuf fr[2];
    int next;                  // index of NextFrame in fr
    TrackState* st;
    float* partials;
    unsigned int* tickets;
    int2* residual;            // per-block photometric correspondence segments
    int* counts;               // entries per segment
    MapView map;
    MapCounters* ctr;
    DevPose* scratch_pose;
    FrameOut* d_out;
    FrameOut* h_out;           // pinned
    FrameOut* h_out_dev;       // h_out's device address (cudaHostGetDevicePointer), null if none
    void* arena;               // one stream-ordered device allocation
    size_t arena_size, arena_used;
    bool sizing;               // dalloc only adds up sizes
    // Tracker / System host state (Tracking.cc:19-23, System.cc:72)
    int state, last_state, no_missed, frames_after_reloc;
    uint64_t frame_id;
    double pose[16];
    // tracing: CUDA events around each stage (off by default)
    bool profile;
    cudaEvent_t ev[kStages + 1];
    double stage_ms[kStages];
    uint64_t stage_calls[kStages];
    uint64_t launches;          // kernels launched by this session
    // CUDA graphs of whole frames, keyed by (mode, fuse, which frame is next);
    // mode 0 init, 1 track, 2 lost
    bool use_graphs;
    // ... and by whether the GPU is shared with other sessions' frames
    cudaGraphExec_t graph[3][2][2][2];
    int graph_kernels[3][2][2][2];
    int rc_bx, rc_by;          // raycast tile
    int integ_cps;             // integration CTAs per SM (0: the form's default)
    bool shared_gpu;           // frames run beside other sessions (batch steps of more than three)
    // Tracker::mappingDisabled (set by System::ReadMapFromDisk): frames track
    // and render against the map without fusing into it
    bool mapping_disabled;
    KeyState* keys;            // key points on (fb_session_set_keypoints), else null
};

namespace fb {

// All device buffers of a session are carved out of one stream-ordered
// allocation (the arena): a sizing pass adds up the sizes, a second pass
// hands out 256-byte aligned pieces.  Creating and destroying sessions while
// other sessions run then costs one cudaMallocAsync / cudaFreeAsync, neither
// of which waits for the device.
template <class T>
bool dalloc(fb_session* s, T** p, size_t n) {
    const size_t bytes = (sizeof(T) * (n ? n : 1) + 255) & ~(size_t)255;
    if (s->sizing) {
        s->arena_size += bytes;
        *p = nullptr;
        return true;
    }
    if (s->arena_used + bytes > s->arena_size) return false;
    *p = (T*)((char*)s->arena + s->arena_used);
    s->arena_used += bytes;
    return true;
}

// ---- session.cu
void* take_out_slot(size_t bytes);
void give_out_slot(void* p);
float half_bits_to_float(uint16_t h);
bool valid_config(const fb_config* c);
MapGeom make_geom(const fb_config& c);
TrackLevel level_view(const fb_session* s, int l);
void drop_graphs(fb_session* s);
void free_staged(fb_session* s);
void free_session(fb_session* s);
bool carve_session(fb_session* s, const fb_config* cfg);
int reset_session(fb_session* s);
int issue_frame(fb_session* s, bool track, bool fuse, bool render, bool init, unsigned* ran, int part = 0,
                const double* start = nullptr);
// The relocalised frame's pose into the tracker state (it becomes the last
// frame) and, after the caller's launches, the frame result.
void launch_track_reloc(fb_session* s, const double* T, cudaStream_t st);
void launch_commit(fb_session* s, int tracked_path, cudaStream_t st);
// The frame result from the device into the session's pinned h_out by a
// kernel (the fused batch step's replacement of the per-session copy).
void launch_result_out(fb_session* s, cudaStream_t st);
int image_ok(const fb_image* im, size_t elem);
cudaStream_t as_stream(void* s);
DevPose pose_from(const float R[9], const float Rinv[9], const float t[3]);
Intr intr_from(const float K[4]);
// The 29 sums of a normal-equation pass (FP64 on the device) as the
// reference's float sums (Reduction.cu:369-371) unpacked into the symmetric
// 6x6 A (row-major) and b (CreateMatrix<6,7>, Reduction.cu:6-16).
void unpack_sums(const double* s, double* A, double* b);
int copy_frame_in(fb_session* s, const uint16_t* depth, size_t depth_pitch, const uint8_t* rgb, size_t rgb_pitch,
                  int on_device, cudaStream_t st);
FramePlan plan_frame(fb_session* s);
int capture_frame(fb_session* s, const FramePlan& p, cudaStream_t st);
int enqueue_frame(fb_session* s, const FramePlan& p, cudaStream_t st, unsigned* ran);
void finish_frame(fb_session* s, const FramePlan& p, fb_frame_result* out);
int read_counters(fb_session* s, MapCounters* c);

// ---- stage_api.cu
// Scratch of the single-pass normal-equation entry points: block partials,
// completion counters, the FP64 sums and one correspondence per pixel.
struct StepScratch {
    float* partials;
    unsigned int* tickets;
    double* out;
    int* residual;
};
// The argument checks of fb_rgb_step (FB_OK or FB_EINVAL) and its body on a
// given scratch (synchronous: the sums are on the host when it returns).
int rgb_step_check(const fb_image* gcurr, const fb_image* glast, const fb_image* vcurr, const fb_image* vlast,
                   const fb_image* dx, const fb_image* dy, const float* Rcurr, const float* RcurrInv,
                   const float* Rlast, const float* RlastInv, const float* tcurr, const float* tlast, const float* K,
                   const float* residual, const double* A, const double* b);
int rgb_step_run(const fb_image* gcurr, const fb_image* glast, const fb_image* vcurr, const fb_image* vlast,
                 const fb_image* dx, const fb_image* dy, const float* Rcurr, const float* RcurrInv,
                 const float* Rlast, const float* RlastInv, const float* tcurr, const float* tlast, const float* K,
                 const StepScratch& sc, float* residual, double* A, double* b, cudaStream_t st);

// ---- keyframe_track.cu
int alloc_keys(fb_session* s);
void free_keys(fb_session* s);
int grab_with_keys(fb_session* s, fb_frame_result* out);

}  // namespace fb

#endif
