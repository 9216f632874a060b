// Session objects and the C ABI of libfusion_b200.so (include/fusion_b200.h).
//
// A session holds, in device memory, the two frames the reference's Tracker
// swaps (NextFrame / LastFrame, Core/Frame.h:61-70), the tracker state and the
// voxel-block map (Mapping::Create, Mapping/Mapping.cc:11-51).  fb_grab_frame
// issues the whole frame -- pyramid, 19 Gauss-Newton iterations with their
// on-device solves, allocation, visibility, integration, z ranges and raycast
// -- as one stream of kernels with no host round trip in between; the kernels
// after tracking read the device's tracking verdict and do nothing when the
// frame was not tracked.  One small device-to-host copy at the end returns the
// frame result, and the host then advances the reference's tracking state
// machine (Tracking/Tracking.cc:58-112) and swaps the frames.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <tuple>
#include <vector>
#include <cmath>

#include <cuda_fp16.h>

#include "../../include/fusion_b200.h"
#include "fb_internal.h"

using namespace fb;

namespace {

thread_local char g_last_error[256] = "";

bool cuda_ok(cudaError_t e) {
    if (e == cudaSuccess) return true;
    snprintf(g_last_error, sizeof g_last_error, "%s", cudaGetErrorString(e));
    return false;
}

#define FB_CUDA(call)                          \
    do {                                       \
        if (!cuda_ok(call)) return FB_ECUDA;   \
    } while (0)

// Kernels launched through the launchers report errors here.
int check_launch() {
    cudaError_t e = cudaGetLastError();
    return cuda_ok(e) ? FB_OK : FB_ECUDA;
}

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

__global__ void k_init_poses(TrackState* st) {
    for (int i = 0; i < 16; ++i) st->pose[i] = st->last_pose[i] = st->init_pose[i] = (i % 5 == 0) ? 1.0 : 0.0;
    st->cur = make_dev_pose_d(st->pose);
    st->last = st->cur;
    st->failed = 0;
    st->icp_error = st->rgb_error = qnan();
    st->icp_count = st->rgb_count = 0;
}

// After the frame: a tracked frame becomes the last frame (SwapFrame).  A
// timed-out device wait (err) counts as a tracking failure.
__global__ void k_commit(TrackState* st, MapCounters* c, FrameOut* out, int tracked_path, const int* err) {
    if (*err) {
        for (int i = 0; i < 16; ++i) st->pose[i] = st->last_pose[i];
        st->failed = 1;
        c->err |= kErrTimeout;
    }
    if (tracked_path && !st->failed) {
        for (int i = 0; i < 16; ++i) st->last_pose[i] = st->pose[i];
        st->last = st->cur;
    }
    for (int i = 0; i < 16; ++i) out->pose[i] = st->pose[i];
    out->failed = st->failed;
    out->icp_error = st->icp_error;
    out->icp_count = st->icp_count;
    out->rgb_error = st->rgb_error;
    out->rgb_count = st->rgb_count;
    out->n_alloc = c->n_alloc;
    out->n_visible = c->n_visible;
    out->n_new = c->n_new;
    out->n_tiles = c->n_tiles;
    out->err = c->err;
    out->heap_counter = c->heap_counter;
    out->entry_ptr = c->entry_ptr;
    out->seq_path = c->seq_path;
}

__global__ void k_set_pose(DevPose* dst, DevPose p) { *dst = p; }

__global__ void k_reset_barrier(unsigned int* bar, int* err) {
    bar[0] = 0;
    *err = 0;
}

// Export of the hash table in the reference's field order, ptr as voxel index.
__global__ void k_export_entries(const HEntry* e, int n, int* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        HEntry h = e[i];
        out[5 * i + 0] = h.x;
        out[5 * i + 1] = h.y;
        out[5 * i + 2] = h.z;
        out[5 * i + 3] = h.ptr >= 0 ? h.ptr * 512 : -1;
        out[5 * i + 4] = h.offset;
    }
}

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

}  // namespace

void fb_set_error_text(const char* msg) { snprintf(g_last_error, sizeof g_last_error, "%s", msg); }

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
    unsigned int* bar;         // grid barrier of the persistent tracking kernel
    int* err;                  // its timeout flag
    int2* residual;            // per-block photometric correspondence segments
    int* counts;               // entries per segment
    MapView map;
    MapCounters* ctr;
    DevPose* scratch_pose;
    FrameOut* d_out;
    FrameOut* h_out;           // pinned
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
    bool persistent;           // tracking as one cooperative kernel per frame
    // ... and by whether the GPU is shared with other sessions' frames
    cudaGraphExec_t graph[3][2][2][2];
    int graph_kernels[3][2][2][2];
    int rc_bx, rc_by;          // raycast tile
    bool shared_gpu;           // frames run beside other sessions (batch steps of more than three)
    // Tracker::mappingDisabled (set by System::ReadMapFromDisk): frames track
    // and render against the map without fusing into it
    bool mapping_disabled;
    KeyState* keys;            // key points on (fb_session_set_keypoints), else null
};

namespace {

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

// Pinned host slots for the per-frame results, recycled between sessions
// (freeing pinned memory may wait for the device).
std::mutex g_out_lock;
std::vector<void*> g_out_free;

void* take_out_slot(size_t bytes) {
    std::lock_guard<std::mutex> guard(g_out_lock);
    if (g_out_free.empty()) {
        // 1024 slots at a time: page-locking host memory is slow and may
        // wait for the device, so it happens rarely (normally once)
        const size_t stride = (bytes + 255) & ~(size_t)255;
        char* chunk = nullptr;
        if (cudaMallocHost((void**)&chunk, 1024 * stride) != cudaSuccess) return nullptr;
        for (int i = 1023; i >= 0; --i) g_out_free.push_back(chunk + (size_t)i * stride);
    }
    void* p = g_out_free.back();
    g_out_free.pop_back();
    return p;
}

void give_out_slot(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> guard(g_out_lock);
    g_out_free.push_back(p);
}

size_t next_pow2(size_t v) {
    size_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

// IEEE binary16 bits -> float (host; exact for every value incl. NaN, inf,
// subnormals).
float half_bits_to_float(uint16_t h) {
    const uint32_t sign = (uint32_t)(h >> 15) << 31;
    const int exp = (h >> 10) & 31;
    uint32_t mant = h & 1023;
    uint32_t bits;
    if (exp == 31) {
        bits = sign | 0x7f800000u | (mant << 13);
    } else if (exp == 0) {
        if (!mant) {
            bits = sign;
        } else {   // subnormal: normalise
            int e = -1;
            do {
                ++e;
                mant <<= 1;
            } while (!(mant & 1024));
            bits = sign | (uint32_t)(127 - 15 - e) << 23 | ((mant & 1023) << 13);
        }
    } else {
        bits = sign | (uint32_t)(exp - 15 + 127) << 23 | (mant << 13);
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

bool valid_config(const fb_config* c) {
    if (!c || c->width < 16 || c->height < 16 || c->width > 4096 || c->height > 2048) return false;
    if ((size_t)c->width * c->height >= (1u << 22)) return false;  // packed RGB correspondences
    if (!(c->fx > 0) || !(c->fy > 0) || !(c->depth_scale > 0) || !(c->voxel_size > 0) || !(c->trunc_dist > 0))
        return false;
    if (c->num_buckets <= 0 || c->num_excess < 0 || c->num_blocks <= 0) return false;
    if (c->form != FB_FORM_REFERENCE && c->form != FB_FORM_PRECISION) return false;
    if ((size_t)c->num_blocks * 512 >= ((size_t)1 << 40)) return false;
    for (int i = 0; i < 3; ++i)
        if (c->iters[i] < 0 || c->iters[i] > 1000) return false;
    return true;
}

MapGeom make_geom(const fb_config& c) {
    MapGeom g;
    g.voxel_size = c.voxel_size;
    // the reference's constexpr expressions (Mapping/DeviceMap.h:148-151)
    g.voxel_size_inv = (float)(1.0 / (double)c.voxel_size);
    g.trunc_dist = c.trunc_dist;
    g.step_scale = (float)(0.5 * (double)c.trunc_dist * (double)g.voxel_size_inv);
    g.block_width = c.voxel_size * 8.0f;
    g.depth_min = c.depth_min;
    g.depth_max = c.depth_max;
    return g;
}

TrackLevel level_view(const fb_session* s, int l) {
    const FrameBuf& N = s->fr[s->next];
    const FrameBuf& L = s->fr[1 - s->next];
    TrackLevel t;
    t.W = s->W[l];
    t.H = s->H[l];
    t.vp = t.gp = t.sp = t.W;
    t.k = s->K[l];
    t.vcurr = N.vmap[l];
    t.ncurr = N.nmap[l];
    t.vlast = L.vmap[l];
    t.nlast = L.nmap[l];
    t.gcurr = N.gray[l];
    t.glast = L.gray[l];
    t.dx = N.dx[l];
    t.dy = N.dy[l];
    t.rgbok = N.rgbok[l];
    return t;
}

void free_keys(fb_session* s) {
    if (!s->keys) return;
    if (s->keys->mem) cudaFree(s->keys->mem);
    delete s->keys;
    s->keys = nullptr;
}

void drop_graphs(fb_session* s);

void free_staged(fb_session* s) {
    StagedInput* g = s->staged;
    if (!g) return;
    if (g->copy) cudaStreamSynchronize(g->copy);
    for (int i = 0; i < 2; ++i) {
        if (g->depth[i]) cudaFree(g->depth[i]);
        if (g->rgb[i]) cudaFree(g->rgb[i]);
        if (g->ready[i]) cudaEventDestroy(g->ready[i]);
        if (g->freed[i]) cudaEventDestroy(g->freed[i]);
    }
    if (g->copy) cudaStreamDestroy(g->copy);
    delete g;
    s->staged = nullptr;
}

void free_session(fb_session* s) {
    free_keys(s);
    free_staged(s);
    drop_graphs(s);
    for (int i = 0; i <= kStages; ++i)
        if (s->ev[i]) cudaEventDestroy(s->ev[i]);
    if (s->arena) cudaFreeAsync(s->arena, s->stream);
    give_out_slot(s->h_out);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

// The device buffers of a session (see dalloc): frames, tracker, map.
bool carve_session(fb_session* s, const fb_config* cfg) {
    bool ok = true;
    for (int f = 0; f < 2 && ok; ++f) {
        FrameBuf& F = s->fr[f];
        size_t n0 = (size_t)s->W[0] * s->H[0];
        ok = ok && dalloc(s, &F.depth_in, n0) && dalloc(s, &F.rgb, 3 * n0) && dalloc(s, &F.raw, n0);
        for (int l = 0; l < 3 && ok; ++l) {
            size_t n = (size_t)s->W[l] * s->H[l];
            ok = dalloc(s, &F.depth[l], n) && dalloc(s, &F.vmap[l], n) && dalloc(s, &F.nmap[l], n) &&
                 dalloc(s, &F.gray[l], n) && dalloc(s, &F.dx[l], n) && dalloc(s, &F.dy[l], n) &&
                 dalloc(s, &F.rgbok[l], n);
        }
    }
    ok = ok && dalloc(s, &s->st, 1) && dalloc(s, &s->partials, (size_t)2 * kTrackMaxBlocks * 32) &&
         dalloc(s, &s->tickets, 4) && dalloc(s, &s->bar, 2) && dalloc(s, &s->err, 1) && dalloc(s, &s->residual, track_list_capacity(s->W[0] * s->H[0])) &&
         dalloc(s, &s->counts, (size_t)kTrackMaxBlocks * kTrackWarps) &&
         dalloc(s, &s->scratch_pose, 1) && dalloc(s, &s->d_out, 1);
    MapView& m = s->map;
    if (ok) {
        m.NB = cfg->num_buckets;
        m.nb_mask = (m.NB & (m.NB - 1)) == 0 ? (uint32_t)(m.NB - 1) : 0u;
        m.NE = cfg->num_excess;
        m.NS = cfg->num_blocks;
        // new blocks of one frame: at least kMinNewBlocks whatever the pool
        // size, so that a frame needing more blocks than the pool still lists
        // all of them and the exhaustion is handled by the exact sequential path
        m.newcap = m.NS > kMinNewBlocks ? m.NS : kMinNewBlocks;
        m.reqcap = (int)next_pow2((size_t)2 * m.newcap);
        m.nchunks = (m.NB + kScanChunk - 1) / kScanChunk;
        // dense raycast index: 16 cells per pool block, 64 K to 4 M cells
        {
            const size_t cap = (size_t)16 * m.NS;
            m.grid_cap = (int)(cap < ((size_t)1 << 16) ? ((size_t)1 << 16) : cap > ((size_t)1 << 22) ? ((size_t)1 << 22) : cap);
        }
        m.zc = (cfg->width + 7) / 8;
        m.zr = (cfg->height + 7) / 8;
        m.g = make_geom(*cfg);
        ok = dalloc(s, &m.entries, (size_t)m.NB + m.NE) && dalloc(s, &m.heap, m.NS) &&
             (cfg->form == FB_FORM_PRECISION ? dalloc(s, &m.cvox, (size_t)m.NS * kCBlockBytes)
                                             : dalloc(s, &m.voxels, (size_t)m.NS * 512)) &&
             dalloc(s, &m.ctr, 1) && dalloc(s, &m.alloc_list, m.NS) &&
             dalloc(s, &m.visible, m.NS) && dalloc(s, &m.vis_blocks, m.NS) && dalloc(s, &m.reqset, m.reqcap) &&
             dalloc(s, &m.newblk, m.newcap) &&
             dalloc(s, &m.order, m.newcap) && dalloc(s, &m.arrival, m.newcap) &&
             dalloc(s, &m.bucket_cnt, m.NB) && dalloc(s, &m.bucket_start, m.NB) && dalloc(s, &m.bucket_x, m.NB) &&
             dalloc(s, &m.chunk_sums, 2 * (size_t)m.nchunks) && dalloc(s, &m.zmin, (size_t)m.zc * m.zr) &&
             dalloc(s, &m.grid, (size_t)m.grid_cap) &&
             dalloc(s, &m.zmax, (size_t)m.zc * m.zr);
        s->ctr = m.ctr;
    }
    return ok;
}

int reset_session(fb_session* s) {
    launch_map_reset(s->map, s->stream);
    k_init_poses<<<1, 1, 0, s->stream>>>(s->st);
    FB_CUDA(cudaMemsetAsync(s->tickets, 0, 4 * sizeof(unsigned), s->stream));
    FB_CUDA(cudaMemsetAsync(s->bar, 0, 2 * sizeof(unsigned), s->stream));
    FB_CUDA(cudaMemsetAsync(s->err, 0, sizeof(int), s->stream));
    for (int f = 0; f < 2; ++f)
        for (int l = 0; l < 3; ++l) {
            size_t n = (size_t)s->W[l] * s->H[l];
            FB_CUDA(cudaMemsetAsync(s->fr[f].vmap[l], 0xff, n * sizeof(float4), s->stream));
            FB_CUDA(cudaMemsetAsync(s->fr[f].nmap[l], 0xff, n * sizeof(float4), s->stream));
        }
    FB_CUDA(cudaStreamSynchronize(s->stream));
    if (check_launch()) return FB_ECUDA;
    s->state = s->last_state = 1;
    s->no_missed = 0;
    s->frames_after_reloc = 10;
    s->frame_id = 0;
    s->next = 0;
    for (int i = 0; i < 16; ++i) s->pose[i] = (i % 5 == 0);
    return FB_OK;
}

// The tracker's starting pose of a frame (the key-point bootstrap's).
struct Pose16 {
    double m[16];
};

__global__ void k_track_start(TrackState* st, Pose16 T) {
    for (int i = 0; i < 16; ++i) st->pose[i] = st->init_pose[i] = T.m[i];
    st->cur = make_dev_pose_d(st->pose);
}

// A relocalised frame: its pose is the solver's, and it becomes the last frame.
__global__ void k_track_reloc(TrackState* st, Pose16 T) {
    for (int i = 0; i < 16; ++i) st->pose[i] = st->last_pose[i] = st->init_pose[i] = T.m[i];
    st->cur = st->last = make_dev_pose_d(st->pose);
    st->failed = 0;
}

// The frame's kernels after the input has reached fr[next].  Returns the
// number of kernels launched and which stages ran (bit k = stage k).
// part 0: the whole frame; 1: ResizeImages + FillImages only; 2: the rest.
// start: the tracker's starting pose when not the last pose.
int issue_frame(fb_session* s, bool track, bool fuse, bool render, bool init, unsigned* ran, int part = 0,
                const double* start = nullptr) {
    cudaStream_t st = s->stream;
    FrameBuf& N = s->fr[s->next];
    FrameBuf& L = s->fr[1 - s->next];
    const fb_config& c = s->cfg;
    int n = 0;
    *ran = 0;
    auto mark = [&](int k) {
        if (s->profile) cudaEventRecord(s->ev[k], st);
    };
    if (part != 2) {
        // Tracker::GrabFrame (Tracking.cc:236-243): LastFrame->ResizeImages ...
        mark(0);
        for (int l = 1; l < 3; ++l)
            n += launch_resize(L.vmap[l - 1], L.nmap[l - 1], s->W[l - 1], s->W[l - 1], s->H[l - 1], L.vmap[l], L.nmap[l],
                               s->W[l], st);
        *ran |= 1u << 0;
        // ... NextFrame->FillImages (Core/Frame.cc:59-78)
        mark(1);
        n += launch_level0(N.depth_in, s->W[0], N.rgb, 3 * s->W[0], s->W[0], s->H[0], c.depth_scale, c.depth_cutoff,
                           N.raw, s->W[0], N.depth[0], s->W[0], N.gray[0], s->W[0], st);
        for (int l = 1; l < 3; ++l)
            n += launch_pyrdown(N.depth[l - 1], s->W[l - 1], N.gray[l - 1], s->W[l - 1], s->W[l - 1], s->H[l - 1],
                                N.depth[l], s->W[l], N.gray[l], s->W[l], st);
        for (int l = 0; l < 3; ++l)
            n += launch_maps(N.depth[l], s->W[l], N.gray[l], s->W[l], s->W[l], s->H[l], s->K[l], c.depth_cutoff,
                             N.vmap[l], s->W[l], N.nmap[l], s->W[l], N.dx[l], N.dy[l], s->W[l], st, N.rgbok[l]);
        *ran |= 1u << 1;
        if (part == 1) return n;
    }
    mark(2);
    const int* skip = nullptr;
    if (init) {
        k_init_poses<<<1, 1, 0, st>>>(s->st);
        n += 1;
    } else if (track) {
        // Tracker::ComputeSE3 (Tracking.cc:296-409)
        static const int min_count[3] = {2000, 1000, 100};   // MIN_ICP_COUNT, Tracking.h:102
        n += launch_track_begin(s->st, st);
        if (start) {
            Pose16 T;
            std::memcpy(T.m, start, sizeof T.m);
            k_track_start<<<1, 1, 0, st>>>(s->st, T);
            n += 1;
        }
        k_reset_barrier<<<1, 1, 0, st>>>(s->bar, s->err);
        n += 1;
        int last_level = -1;
        for (int l = 2; l >= 0; --l)
            if (c.iters[l] > 0) last_level = l;
        const int grid = s->persistent ? track_frame_grid() : 0;
        if (grid > 0) {
            // all levels and iterations in one cooperative launch
            TrackFrame F;
            for (int l = 0; l < 3; ++l) {
                F.L[l] = level_view(s, l);
                F.iters[l] = c.iters[l];
                F.min_count[l] = min_count[l];
            }
            F.last_level = last_level;
            F.st = s->st;
            F.partials = s->partials;
            F.residual = (int*)s->residual;
            F.bar = s->bar;
            F.err = s->err;
            n += launch_track_frame(F, grid, st);
        } else {
            for (int l = 2; l >= 0; --l) {
                TrackLevel lv = level_view(s, l);
                for (int it = 0; it < c.iters[l]; ++it)
                    n += launch_track_iter(lv, s->st, s->tickets, s->residual, s->counts,
                                           min_count[l], l == last_level && it == c.iters[l] - 1, st,
                                           s->shared_gpu, c.form == FB_FORM_PRECISION);
            }
        }
        skip = &s->st->failed;
        *ran |= 1u << 2;
    }
    const DevPose* pose = &s->st->cur;
    mark(3);
    if (fuse) {
        // Mapping::FuseColor(LastFrame) after the swap (Mapping.cc:76-90):
        // raw depth, colour and level-0 normals of the frame just tracked
        n += launch_allocate(s->map, N.raw, s->W[0], s->W[0], s->H[0], s->K[0], pose, skip, st);
        mark(4);
        n += launch_visibility(s->map, s->W[0], s->H[0], s->K[0], pose, skip, st);
        mark(5);
        n += launch_integrate(s->map, N.raw, s->W[0], N.rgb, 3 * s->W[0], N.nmap[0], s->W[0], s->W[0], s->H[0],
                              s->K[0], pose, skip, st);
        *ran |= 7u << 3;
    } else {
        mark(4);
        mark(5);
    }
    mark(6);
    if (render) {
        // with mapping disabled, System::GrabImage refreshes the visible
        // blocks first (Mapping::UpdateVisibility, System.cc:116-118)
        if (!fuse && s->mapping_disabled) n += launch_visibility(s->map, s->W[0], s->H[0], s->K[0], pose, skip, st);
        // Mapping::RayTrace (Mapping.cc:92-109) into the frame's level-0 maps
        n += launch_zrange(s->map, s->K[0], pose, skip, st);
        mark(7);
        n += launch_raycast(s->map, N.vmap[0], N.nmap[0], s->W[0], s->W[0], s->H[0], s->K[0], pose, skip, st,
                            s->rc_bx, s->rc_by);
        *ran |= 3u << 6;
    } else {
        mark(7);
    }
    mark(8);
    k_commit<<<1, 1, 0, st>>>(s->st, s->ctr, s->d_out, track || init, s->err);
    return n + 1;
}

// A pitch must hold a row; for the word-sized element types the kernels index
// rows in elements, so it must also be a multiple of the element.  RGB8
// (3-byte) rows are indexed in bytes: cudaMallocPitch's pitch of a uchar3
// image (a multiple of 512 bytes, not of 3) is valid.
int image_ok(const fb_image* im, size_t elem) {
    return im && im->data && im->cols > 0 && im->rows > 0 && im->pitch >= elem * (size_t)im->cols &&
           (elem == 3 || im->pitch % elem == 0);
}

cudaStream_t as_stream(void* s) { return (cudaStream_t)s; }

DevPose pose_from(const float R[9], const float Rinv[9], const float t[3]) {
    DevPose p;
    p.R.r0 = {R[0], R[1], R[2]};
    p.R.r1 = {R[3], R[4], R[5]};
    p.R.r2 = {R[6], R[7], R[8]};
    p.Rinv.r0 = {Rinv[0], Rinv[1], Rinv[2]};
    p.Rinv.r1 = {Rinv[3], Rinv[4], Rinv[5]};
    p.Rinv.r2 = {Rinv[6], Rinv[7], Rinv[8]};
    p.t = {t[0], t[1], t[2]};
    p.pad = 0;
    return p;
}

Intr intr_from(const float K[4]) {
    Intr k;
    k.fx = K[0];
    k.fy = K[1];
    k.cx = K[2];
    k.cy = K[3];
    k.invfx = (float)(1.0 / (double)k.fx);
    k.invfy = (float)(1.0 / (double)k.fy);
    return k;
}

}  // namespace

namespace {

// Frame-graph executables of closed sessions (and of dropped graphs) are
// kept for reuse: a later graph of the same shape is written into one with
// cudaGraphExecUpdate instead of being instantiated.  Instantiating while
// other sessions' frames run stalled the calling thread for up to 80 ms on
// B200 once a thousand executables had been made; an update only rewrites
// node parameters.  An update that the driver refuses falls back to
// instantiation.
using ExecKey = std::tuple<int, int, int, int, int, int, int, int, int, int, int>;
std::mutex g_exec_lock;
std::multimap<ExecKey, cudaGraphExec_t> g_exec_pool;
constexpr size_t kExecPoolMax = 4096;
std::atomic<long long> g_exec_updated{0}, g_exec_instantiated{0};

ExecKey exec_key(const fb_session* s, int mode, int fuse, int shared) {
    int dev = 0;
    cudaGetDevice(&dev);
    return ExecKey(dev, s->W[0], s->H[0], s->cfg.form, mode, fuse, shared, s->persistent ? 1 : 0, s->rc_bx, s->rc_by,
                   s->mapping_disabled ? 1 : 0);
}

void release_exec(const fb_session* s, int mode, int fuse, int shared, cudaGraphExec_t g) {
    std::lock_guard<std::mutex> guard(g_exec_lock);
    if (g_exec_pool.size() < kExecPoolMax)
        g_exec_pool.emplace(exec_key(s, mode, fuse, shared), g);
    else
        cudaGraphExecDestroy(g);
}

cudaGraphExec_t take_exec(const ExecKey& key) {
    std::lock_guard<std::mutex> guard(g_exec_lock);
    auto it = g_exec_pool.find(key);
    if (it == g_exec_pool.end()) return nullptr;
    cudaGraphExec_t g = it->second;
    g_exec_pool.erase(it);
    return g;
}

// Cached frame graphs are released (rebuilt on next use).
void drop_graphs(fb_session* s) {
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 2; ++b)
            for (int c = 0; c < 2; ++c)
                for (int d = 0; d < 2; ++d)
                    if (s->graph[a][b][c][d]) {
                        release_exec(s, a, b, d, s->graph[a][b][c][d]);
                        s->graph[a][b][c][d] = nullptr;
                    }
}

// Host input -> the device input buffers of fr[next].
int copy_frame_in(fb_session* s, const uint16_t* depth, size_t depth_pitch, const uint8_t* rgb, size_t rgb_pitch,
                  int on_device, cudaStream_t st) {
    const int W = s->W[0], H = s->H[0];
    if (depth_pitch < (size_t)W * 2 || rgb_pitch < (size_t)W * 3) return FB_EINVAL;
    FrameBuf& N = s->fr[s->next];
    cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    FB_CUDA(cudaMemcpy2DAsync(N.depth_in, (size_t)W * 2, depth, depth_pitch, (size_t)W * 2, H, kind, st));
    FB_CUDA(cudaMemcpy2DAsync(N.rgb, (size_t)W * 3, rgb, rgb_pitch, (size_t)W * 3, H, kind, st));
    return FB_OK;
}

// Tracker::Track (Tracking.cc:58-112): the state is known on the host;
// whether tracking succeeds is decided on the device.
FramePlan plan_frame(fb_session* s) {
    FramePlan p;
    std::swap(s->state, s->last_state);
    p.state = s->state;
    p.init = p.state == 1;
    p.track = p.state == 0;
    // System::GrabImage (System.cc:98-115): frames_after_reloc is updated from
    // the tracker state, which does not depend on this frame's outcome
    p.after = s->frames_after_reloc;
    if (p.state == 0) p.after++;
    if (p.state == -1) p.after = 0;
    p.fuse = !s->mapping_disabled && (p.init || p.track) && p.after >= 10;
    p.render = p.init || p.track;
    p.mode = p.init ? 0 : p.track ? 1 : 2;
    return p;
}

// Captures the graph of a frame of plan p for the session's current frame
// parity and shared-GPU flag, unless it is cached already.  The capture runs
// on stream st (nothing executes).
int capture_frame(fb_session* s, const FramePlan& p, cudaStream_t st) {
    const int sh = s->shared_gpu ? 1 : 0;
    cudaGraphExec_t& g = s->graph[p.mode][p.fuse ? 1 : 0][s->next][sh];
    if (g) return FB_OK;
    cudaGraph_t graph = nullptr;
    cudaStream_t keep = s->stream;
    s->stream = st;
    unsigned ran = 0;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    int nk = 0;
    if (e == cudaSuccess) {
        nk = issue_frame(s, p.track, p.fuse, p.render, p.init, &ran);
        e = cudaStreamEndCapture(st, &graph);
    }
    s->stream = keep;
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) {
        cudaGraphExec_t r = take_exec(exec_key(s, p.mode, p.fuse ? 1 : 0, sh));
        if (r) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(r, graph, &info) == cudaSuccess) {
                g = r;
                g_exec_updated.fetch_add(1);
            } else {
                cudaGetLastError();
                cudaGraphExecDestroy(r);
            }
        }
        if (!g) {
            e = cudaGraphInstantiate(&g, graph, 0);
            g_exec_instantiated.fetch_add(1);
        }
    }
    // upload now, so that the frame that first launches it does not wait
    if (e == cudaSuccess) e = cudaGraphUpload(g, st);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        g = nullptr;
        cuda_ok(e);
        return FB_ECUDA;
    }
    s->graph_kernels[p.mode][p.fuse ? 1 : 0][s->next][sh] = nk;
    return FB_OK;
}

// The frame's kernels on stream `st`: the session's cached graph of this
// (mode, fuse, next, shared) when graphs are on and profiling is off
// (captured on first use), else direct launches.
int enqueue_frame(fb_session* s, const FramePlan& p, cudaStream_t st, unsigned* ran) {
    *ran = 0;
    if (s->use_graphs && !s->profile) {
        const int sh = s->shared_gpu ? 1 : 0;
        int rc = capture_frame(s, p, st);
        if (rc) return rc;
        cudaGraphExec_t g = s->graph[p.mode][p.fuse ? 1 : 0][s->next][sh];
        FB_CUDA(cudaGraphLaunch(g, st));
        s->launches += (uint64_t)s->graph_kernels[p.mode][p.fuse ? 1 : 0][s->next][sh];
        *ran = 0;
        return FB_OK;
    }
    cudaStream_t keep = s->stream;
    s->stream = st;
    s->launches += (uint64_t)issue_frame(s, p.track, p.fuse, p.render, p.init, ran);
    s->stream = keep;
    return check_launch();
}

// After the frame's result has reached h_out: the reference's tracking state
// machine (Tracking.cc:58-112) and SwapFrame, and the caller's result.
void finish_frame(fb_session* s, const FramePlan& p, fb_frame_result* out) {
    const FrameOut& o = *s->h_out;
    bool valid = false;
    if (p.init) {
        s->next = 1 - s->next;  // SwapFrame
        s->last_state = 0;
        valid = true;
    } else if (p.track) {
        if (!o.failed) {
            s->no_missed = 0;
            if (s->last_state != -1) {
                s->last_state = 0;
                s->next = 1 - s->next;
                valid = true;
            } else {
                s->last_state = 0;
            }
        } else {
            s->last_state = 0;
            if (++s->no_missed > 9) s->last_state = -1;
        }
    } else {
        s->last_state = -1;
    }
    s->frames_after_reloc = p.after;
    std::memcpy(s->pose, o.pose, sizeof s->pose);
    if (out) {
        out->status = valid ? FB_OK : FB_ETRACK_LOST;
        out->tracked = valid;
        out->tracker_state = p.state;
        out->fused = p.fuse && valid;
        out->no_visible = (p.fuse && valid) ? (uint32_t)o.n_visible : 0;
        out->no_allocated = (uint32_t)o.n_alloc;
        out->no_new = (p.fuse && valid) ? (uint32_t)o.n_new : 0;
        out->error_flags = o.err;
        out->icp_error = o.icp_error;
        out->icp_count = o.icp_count;
        out->rgb_error = o.rgb_error;
        out->rgb_count = o.rgb_count;
        std::memcpy(out->pose, o.pose, sizeof out->pose);
        out->frame_id = s->frame_id;
    }
    s->frame_id++;
}

// ------------------------------------------------------------- key points

int alloc_keys(fb_session* s) {
    KeyState* K = new (std::nothrow) KeyState();
    if (!K) return FB_ENOMEM;
    const int W = s->W[0], H = s->H[0];
    const size_t scratch = key_scratch_bytes(W, H);
    const int cap = W * H / 100;
    const size_t per_set = (size_t)cap * (3 * 16 + 4 * kKeyDesc) + 4 * 256;
    const size_t bytes = scratch + 2 * per_set + (size_t)cap * (4 * kKeyDesc + 16) + 2048 +
                         (size_t)kKeyMapCap * 4 * kKeyDesc;
    if (cudaMalloc(&K->mem, bytes) != cudaSuccess) {
        cudaGetLastError();
        delete K;
        return FB_ENOMEM;
    }
    char* p = (char*)K->mem;
    auto take = [&](size_t n) {
        char* q = p;
        p += (n + 255) & ~(size_t)255;
        return q;
    };
    int rc = key_scratch_carve(take(scratch), scratch, W, H, K->ks);
    for (int f = 0; f < 2; ++f) {
        KeySet& ks = K->set[f];
        ks.cap = cap;
        ks.kp = (float4*)take((size_t)cap * 16);
        ks.pt = (float4*)take((size_t)cap * 16);
        ks.nrm = (float4*)take((size_t)cap * 16);
        ks.desc = (float*)take((size_t)cap * 4 * kKeyDesc);
    }
    K->m_idx = (int2*)take((size_t)cap * 8);
    K->m_dist = (float2*)take((size_t)cap * 8);
    K->kf_desc = (float*)take((size_t)cap * 4 * kKeyDesc);
    K->d_n = (int*)take(256);
    K->map_desc = (float*)take((size_t)kKeyMapCap * 4 * kKeyDesc);
    if (rc != FB_OK || (size_t)(p - (char*)K->mem) > bytes) {
        cudaFree(K->mem);
        delete K;
        return FB_ENOMEM;
    }
    K->stats.bootstrap = K->stats.relocalised = -1;
    s->keys = K;
    return FB_OK;
}

// Frame::ExtractKeyPoints (Core/Frame.cc:165-212) of frame buffer f:
// detection on the level-0 gray image (SURF_CUDA(20)), then the key points
// with a depth and a normal; their points and normals also on the host.
int extract_keys(fb_session* s, int f) {
    KeyState& K = *s->keys;
    cudaStream_t st = s->stream;
    int nk = 0;
    int rc = launch_surf(s->fr[f].gray[0], s->W[0], 20.f, K.ks, &nk, st);
    if (rc) return rc;
    K.n[f] = 0;
    if (nk > 0) {
        rc = launch_backproject(K.ks, nk, s->fr[f].depth[0], s->W[0], s->fr[f].nmap[0], s->W[0], s->K[0],
                                s->cfg.depth_cutoff, K.set[f], K.d_n, st);
        if (rc) return rc;
        FB_CUDA(cudaMemcpyAsync(&K.n[f], K.d_n, 4, cudaMemcpyDeviceToHost, st));
        FB_CUDA(cudaStreamSynchronize(st));
    }
    const int n = K.n[f];
    K.pts[f].resize((size_t)4 * n);
    K.nrm[f].resize((size_t)4 * n);
    if (n) {
        FB_CUDA(cudaMemcpyAsync(K.pts[f].data(), K.set[f].pt, 16 * (size_t)n, cudaMemcpyDeviceToHost, st));
        FB_CUDA(cudaMemcpyAsync(K.nrm[f].data(), K.set[f].nrm, 16 * (size_t)n, cudaMemcpyDeviceToHost, st));
        FB_CUDA(cudaStreamSynchronize(st));
    }
    s->launches += 14;
    return FB_OK;
}

// knnMatch(query, train, 2): nearest and second-nearest train per query.
int match_keys(fb_session* s, const float* q, int nq, const float* t, int nt, std::vector<int2>& idx,
               std::vector<float2>& dist) {
    KeyState& K = *s->keys;
    idx.assign(nq, make_int2(-1, -1));
    dist.assign(nq, make_float2(INFINITY, INFINITY));
    if (nq <= 0 || nt <= 0) return FB_OK;
    int rc = launch_match2(q, nq, t, nt, K.m_idx, K.m_dist, s->stream);
    if (rc) return rc;
    FB_CUDA(cudaMemcpyAsync(idx.data(), K.m_idx, 8 * (size_t)nq, cudaMemcpyDeviceToHost, s->stream));
    FB_CUDA(cudaMemcpyAsync(dist.data(), K.m_dist, 8 * (size_t)nq, cudaMemcpyDeviceToHost, s->stream));
    FB_CUDA(cudaStreamSynchronize(s->stream));
    s->launches += 1;
    return FB_OK;
}

void rigid_inv(const double* A, double* B) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) B[4 * i + j] = A[4 * j + i];
    for (int i = 0; i < 3; ++i) B[4 * i + 3] = -(B[4 * i] * A[3] + B[4 * i + 1] * A[7] + B[4 * i + 2] * A[11]);
    B[12] = B[13] = B[14] = 0;
    B[15] = 1;
}

void mat4_mul(const double* A, const double* B, double* C) {
    double T[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double v = 0;
            for (int k = 0; k < 4; ++k) v += A[4 * i + k] * B[4 * k + j];
            T[4 * i + j] = v;
        }
    std::memcpy(C, T, sizeof T);
}

// Matched pairs (query i, train j) passing the ratio test d1 < ratio d2.
std::vector<std::pair<int, int>> ratio_pairs(const std::vector<int2>& idx, const std::vector<float2>& dist,
                                             float ratio) {
    std::vector<std::pair<int, int>> out;
    for (size_t i = 0; i < idx.size(); ++i)
        if (idx[i].x >= 0 && idx[i].y >= 0 && dist[i].x < ratio * dist[i].y) out.push_back({(int)i, idx[i].x});
    return out;
}

uint64_t key_seed(fb_session* s, uint64_t purpose) { return (s->frame_id + 1) * 0x9E3779B97F4A7C15ull ^ purpose; }

// Mapping::FuseKeyFrame (Mapping.cc:220-275) of the reference keyframe: its
// observed keys in world coordinates into the key map, one key per 1 cm cell
// (KeyMap::InsertKey keeps the key already in a cell).
int fuse_keyframe(fb_session* s) {
    KeyState& K = *s->keys;
    HostKeyFrame& kf = K.kf;
    if (kf.n == 0) return FB_OK;
    std::vector<float> desc((size_t)kf.n * kKeyDesc);
    FB_CUDA(cudaStreamSynchronize(s->stream));
    FB_CUDA(cudaMemcpy(desc.data(), K.kf_desc, 4 * desc.size(), cudaMemcpyDeviceToHost));
    float R[9], t[3];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) R[3 * i + j] = (float)kf.pose[4 * i + j];
        t[i] = (float)kf.pose[4 * i + 3];
    }
    std::vector<float> add;
    const int first = K.map_n;
    for (int i = 0; i < kf.n && K.map_n < kKeyMapCap; ++i) {
        if (kf.obs[i] <= 0) continue;
        const float* p = &kf.pts[4 * (size_t)i];
        float w[3];
        for (int r = 0; r < 3; ++r) w[r] = R[3 * r] * p[0] + R[3 * r + 1] * p[1] + R[3 * r + 2] * p[2] + t[r];
        const auto cell = std::make_tuple((int)(w[0] / 0.01f), (int)(w[1] / 0.01f), (int)(w[2] / 0.01f));
        if (K.map_cells.count(cell)) continue;
        K.map_cells[cell] = K.map_n++;
        K.map_pos.insert(K.map_pos.end(), w, w + 3);
        add.insert(add.end(), desc.begin() + (size_t)i * kKeyDesc, desc.begin() + (size_t)(i + 1) * kKeyDesc);
    }
    if (!add.empty())
        FB_CUDA(cudaMemcpy(K.map_desc + (size_t)first * kKeyDesc, add.data(), 4 * add.size(), cudaMemcpyHostToDevice));
    return FB_OK;
}

// Tracker::CreateKeyFrame (Tracking.cc:222-227): the reference keyframe is
// fused into the key map and frame f becomes the reference keyframe.
int create_keyframe(fb_session* s, int f, const double* pose) {
    KeyState& K = *s->keys;
    if (K.has_kf) {
        int rc = fuse_keyframe(s);
        if (rc) return rc;
    }
    HostKeyFrame& kf = K.kf;
    kf.n = K.n[f];
    std::memcpy(kf.pose, pose, sizeof kf.pose);
    kf.pts = K.pts[f];
    kf.nrm = K.nrm[f];
    kf.obs.assign(kf.n, 0);
    if (kf.n)
        FB_CUDA(cudaMemcpyAsync(K.kf_desc, K.set[f].desc, 4 * (size_t)kf.n * kKeyDesc, cudaMemcpyDeviceToDevice,
                                s->stream));
    K.has_kf = true;
    K.stats.keyframes++;
    return FB_OK;
}

// the reference works on float poses here (Matrix4f)
void pose_f(const double* T, float* F) {
    for (int i = 0; i < 16; ++i) F[i] = (float)T[i];
}

void rigid_inv_f(const float* A, float* B) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) B[4 * i + j] = A[4 * j + i];
    for (int i = 0; i < 3; ++i) B[4 * i + 3] = -(B[4 * i] * A[3] + B[4 * i + 1] * A[7] + B[4 * i + 2] * A[11]);
    B[12] = B[13] = B[14] = 0.f;
    B[15] = 1.f;
}

void mat4_mul_f(const float* A, const float* B, float* C) {
    float T[16];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            float v = 0.f;
            for (int k = 0; k < 4; ++k) v += A[4 * i + k] * B[4 * k + j];
            T[4 * i + j] = v;
        }
    std::memcpy(C, T, sizeof T);
}

// Tracker::NeedKeyFrame (Tracking.cc:208-220)
bool need_keyframe(fb_session* s, const double* pose) {
    if (s->mapping_disabled) return false;
    float P[16], K[16], Ki[16], d[16];
    pose_f(pose, P);
    pose_f(s->keys->kf.pose, K);
    rigid_inv_f(K, Ki);
    mat4_mul_f(P, Ki, d);
    const double a = std::atan2(-(double)d[6], (double)d[10]);
    const double b = std::atan2((double)d[2], std::sqrt((double)d[0] * d[0] + (double)d[1] * d[1]));
    const double c = std::atan2(-(double)d[1], (double)d[0]);
    const float sa = (float)std::sin(a), sb = (float)std::sin(b), sc = (float)std::sin(c);
    const float an = std::sqrt(sa * sa + sb * sb + sc * sc);
    const float tn = std::sqrt(d[3] * d[3] + d[7] * d[7] + d[11] * d[11]);
    return an > 0.1f || tn > 0.1f;
}

// Tracker::CheckOutliers (Tracking.cc:113-135): nearest keyframe key of
// every key of frame f; a match consistent with the relative pose within
// 5 cm counts as an observation of the keyframe's key.
int check_outliers(fb_session* s, int f, const double* pose) {
    KeyState& K = *s->keys;
    if (!K.has_kf) return FB_OK;
    std::vector<int2> idx;
    std::vector<float2> dist;
    int rc = match_keys(s, K.set[f].desc, K.n[f], K.kf_desc, K.kf.n, idx, dist);
    if (rc) return rc;
    float P[16], Kp[16], Ki[16], d[16];
    pose_f(pose, P);
    pose_f(K.kf.pose, Kp);
    rigid_inv_f(Kp, Ki);
    mat4_mul_f(Ki, P, d);
    for (int i = 0; i < K.n[f]; ++i) {
        const int j = idx[i].x;
        if (j < 0) continue;
        const float* src = &K.pts[f][4 * (size_t)i];
        const float* ref = &K.kf.pts[4 * (size_t)j];
        float e2 = 0.f;
        for (int r = 0; r < 3; ++r) {
            const float e = src[r] - (d[4 * r] * ref[0] + d[4 * r + 1] * ref[1] + d[4 * r + 2] * ref[2] + d[4 * r + 3]);
            e2 += e * e;
        }
        if (std::sqrt((double)e2) <= 0.05f) K.kf.obs[j]++;
    }
    return FB_OK;
}

// Relocalised frame: the solver's pose, the visible blocks and the model
// raycast from it (System::GrabImage's lost-state branch, System.cc:116-118).
int issue_reloc(fb_session* s, const double* T) {
    cudaStream_t st = s->stream;
    FrameBuf& N = s->fr[s->next];
    Pose16 P;
    std::memcpy(P.m, T, sizeof P.m);
    k_track_reloc<<<1, 1, 0, st>>>(s->st, P);
    const DevPose* pose = &s->st->cur;
    int n = 1;
    n += launch_visibility(s->map, s->W[0], s->H[0], s->K[0], pose, nullptr, st);
    n += launch_zrange(s->map, s->K[0], pose, nullptr, st);
    n += launch_raycast(s->map, N.vmap[0], N.nmap[0], s->W[0], s->W[0], s->H[0], s->K[0], pose, nullptr, st, s->rc_bx,
                        s->rc_by);
    k_commit<<<1, 1, 0, st>>>(s->st, s->ctr, s->d_out, 1, s->err);
    s->launches += (uint64_t)n + 1;
    return check_launch();
}

// One frame with key points (System::GrabImage with Tracker::Track's key
// point steps; Tracking.cc:58-112, 150-204, 411-470).
int grab_with_keys(fb_session* s, fb_frame_result* out) {
    KeyState& K = *s->keys;
    const FramePlan p = plan_frame(s);
    const int nx = s->next, lx = 1 - s->next;
    unsigned ran = 0;
    s->launches += (uint64_t)issue_frame(s, false, false, false, false, &ran, 1);
    int rc = check_launch();
    if (rc) return rc;
    rc = extract_keys(s, nx);
    if (rc) return rc;
    K.stats.keys = (uint32_t)K.n[nx];
    K.stats.matches = 0;
    K.stats.bootstrap = K.stats.relocalised = -1;
    double start[16], reloc[16];
    bool have_start = false, relocalised = false;
    std::vector<int2> idx;
    std::vector<float2> dist;
    std::vector<double> src, ref;
    std::vector<uint8_t> outl;
    if (p.track) {
        // TrackLastFrame: next-frame keys against last-frame keys, ratio 0.8,
        // then Solver::PoseEstimate (35 iterations, motion check)
        rc = match_keys(s, K.set[nx].desc, K.n[nx], K.set[lx].desc, K.n[lx], idx, dist);
        if (rc) return rc;
        const auto pairs = ratio_pairs(idx, dist, 0.8f);
        K.stats.matches = (uint32_t)pairs.size();
        K.stats.bootstrap = 0;
        if (pairs.size() >= 3) {
            for (const auto& m : pairs)
                for (int r = 0; r < 3; ++r) {
                    src.push_back(K.pts[nx][4 * (size_t)m.first + r]);
                    ref.push_back(K.pts[lx][4 * (size_t)m.second + r]);
                }
            outl.assign(pairs.size(), 1);
            double delta[16], dinv[16];
            if (pose_estimate(src.data(), ref.data(), (int)pairs.size(), 35, true, key_seed(s, 1), delta, outl.data())) {
                rigid_inv(delta, dinv);
                mat4_mul(dinv, s->pose, start);   // nextPose = delta^-1 * LastFrame->pose
                have_start = true;
                K.stats.bootstrap = 1;
            }
        }
    } else if (!p.init) {
        // Relocalise: next-frame keys against the key map, ratio 0.9, then
        // Solver::PoseEstimate (100 iterations, no motion check)
        K.stats.relocalised = 0;
        if (K.map_n > 0) {
            rc = match_keys(s, K.set[nx].desc, K.n[nx], K.map_desc, K.map_n, idx, dist);
            if (rc) return rc;
            const auto pairs = ratio_pairs(idx, dist, 0.9f);
            K.stats.matches = (uint32_t)pairs.size();
            if (pairs.size() >= 3) {
                for (const auto& m : pairs)
                    for (int r = 0; r < 3; ++r) {
                        src.push_back(K.pts[nx][4 * (size_t)m.first + r]);
                        ref.push_back(K.map_pos[3 * (size_t)m.second + r]);
                    }
                outl.assign(pairs.size(), 1);
                double delta[16];
                if (pose_estimate(src.data(), ref.data(), (int)pairs.size(), 100, false, key_seed(s, 2), delta,
                                  outl.data())) {
                    rigid_inv(delta, reloc);   // NextFrame->pose = delta^-1
                    relocalised = true;
                    K.stats.relocalised = 1;
                }
            }
        }
    }
    if (relocalised) {
        rc = issue_reloc(s, reloc);
    } else {
        s->launches += (uint64_t)issue_frame(s, p.track, p.fuse, p.render, p.init, &ran, 2,
                                             have_start ? start : nullptr);
        rc = check_launch();
    }
    if (rc) return rc;
    FB_CUDA(cudaMemcpyAsync(s->h_out, s->d_out, sizeof(FrameOut), cudaMemcpyDeviceToHost, s->stream));
    FB_CUDA(cudaStreamSynchronize(s->stream));
    if (relocalised) {
        // case -1 of Tracker::Track: lastState = 0, SwapFrame
        s->next = 1 - s->next;
        s->last_state = 0;
        s->frames_after_reloc = p.after;
        std::memcpy(s->pose, s->h_out->pose, sizeof s->pose);
        if (out) {
            std::memset(out, 0, sizeof *out);
            out->status = FB_OK;
            out->tracked = 1;
            out->tracker_state = p.state;
            out->no_allocated = (uint32_t)s->h_out->n_alloc;
            out->error_flags = s->h_out->err;
            std::memcpy(out->pose, s->h_out->pose, sizeof out->pose);
            out->frame_id = s->frame_id;
        }
        s->frame_id++;
        return FB_OK;
    }
    fb_frame_result local;
    fb_frame_result* r = out ? out : &local;
    finish_frame(s, p, r);
    if (p.init) {
        // InitTracking: ResetTracking, then CreateKeyFrame (Tracking.cc:229-234)
        return create_keyframe(s, nx, r->pose);
    }
    if (p.track && r->tracked) {
        // a tracked frame after a tracked one (Tracking.cc:75-85)
        if (need_keyframe(s, r->pose)) return create_keyframe(s, nx, r->pose);
        return check_outliers(s, nx, r->pose);
    }
    return FB_OK;
}

}  // namespace

extern "C" {

void fb_default_config(fb_config* c, int width, int height) {
    std::memset(c, 0, sizeof *c);
    c->width = width;
    c->height = height;
    c->fx = c->fy = 525.0f * width / 640.0f;
    c->cx = width * 0.5f;
    c->cy = height * 0.5f;
    c->depth_scale = 1000.0f;
    c->depth_cutoff = 3.0f;
    c->voxel_size = 0.006f;
    c->trunc_dist = 0.006f * 8;
    c->depth_min = 0.1f;
    c->depth_max = 3.0f;
    c->num_buckets = 1000000;
    c->num_excess = 500000;
    c->num_blocks = 700000;
    c->iters[0] = 10;
    c->iters[1] = 5;
    c->iters[2] = 3;
}

const char* fb_status_string(int st) {
    switch (st) {
    case FB_OK: return "ok";
    case FB_EINVAL: return "invalid argument";
    case FB_ENOMEM: return "out of memory";
    case FB_ECUDA: return "CUDA error";
    case FB_ETRACK_LOST: return "frame not tracked";
    default: return "unknown status";
    }
}

const char* fb_last_error(void) { return g_last_error; }

void fb_graph_exec_stats(long long* pooled, long long* updated, long long* instantiated) {
    {
        std::lock_guard<std::mutex> guard(g_exec_lock);
        if (pooled) *pooled = (long long)g_exec_pool.size();
    }
    if (updated) *updated = g_exec_updated.load();
    if (instantiated) *instantiated = g_exec_instantiated.load();
}

size_t fb_session_bytes(const fb_config* c) {
    if (!valid_config(c)) return 0;
    // the sizing pass of fb_session_create
    fb_session* s = new (std::nothrow) fb_session();
    if (!s) return 0;
    for (int l = 0; l < 3; ++l) {
        s->W[l] = c->width >> l;
        s->H[l] = c->height >> l;
    }
    s->sizing = true;
    carve_session(s, c);
    const size_t n = s->arena_size;
    delete s;
    return n;
}

int fb_session_create(const fb_config* cfg, void* stream, fb_session** out) {
    if (!out || !valid_config(cfg)) return FB_EINVAL;
    *out = nullptr;
    fb_session* s = new (std::nothrow) fb_session();
    if (!s) return FB_ENOMEM;
    s->cfg = *cfg;
    s->h_out = nullptr;
    s->profile = false;
    for (int i = 0; i <= kStages; ++i) s->ev[i] = nullptr;
    for (int i = 0; i < kStages; ++i) {
        s->stage_ms[i] = 0;
        s->stage_calls[i] = 0;
    }
    s->launches = 0;
    s->use_graphs = true;
    s->persistent = false;   // measured slower than graph-launched kernels on B200
    s->rc_bx = 16;
    s->rc_by = 8;
    s->shared_gpu = false;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 2; ++b)
            for (int c = 0; c < 2; ++c)
                for (int d = 0; d < 2; ++d) {
                    s->graph[a][b][c][d] = nullptr;
                    s->graph_kernels[a][b][c][d] = 0;
                }
    s->own_stream = stream == nullptr;
    s->stream = (cudaStream_t)stream;
    // an owned stream is a blocking one: it orders after work the caller put
    // on the legacy default stream (e.g. the copies that filled its inputs)
    if (s->own_stream && !cuda_ok(cudaStreamCreate(&s->stream))) {
        s->stream = nullptr;
        free_session(s);
        return FB_ECUDA;
    }
    for (int l = 0; l < 3; ++l) {
        s->W[l] = cfg->width >> l;
        s->H[l] = cfg->height >> l;
        s->K[l] = make_intr(cfg->fx, cfg->fy, cfg->cx, cfg->cy, l);
    }
    // sizes first, then one allocation, then the pieces
    s->arena = nullptr;
    s->arena_size = s->arena_used = 0;
    s->sizing = true;
    carve_session(s, cfg);
    s->sizing = false;
    bool ok = cuda_ok(cudaMallocAsync(&s->arena, s->arena_size, s->stream));
    if (!ok) s->arena = nullptr;
    ok = ok && carve_session(s, cfg);
    if (ok) {
        s->h_out = (FrameOut*)take_out_slot(sizeof(FrameOut));
        ok = s->h_out != nullptr;
    }
    for (int i = 0; i <= kStages && ok; ++i) ok = cuda_ok(cudaEventCreate(&s->ev[i]));
    if (!ok) {
        free_session(s);
        return FB_ENOMEM;
    }
    int rc = reset_session(s);
    if (rc) {
        free_session(s);
        return rc;
    }
    *out = s;
    return FB_OK;
}

int fb_session_destroy(fb_session* s) {
    if (!s) return FB_EINVAL;
    cudaStreamSynchronize(s->stream);
    free_session(s);
    return FB_OK;
}

int fb_session_reset(fb_session* s) {
    if (!s) return FB_EINVAL;
    return reset_session(s);
}

// The oldest staged frame into NextFrame's input buffers, on the session
// stream once its copy has landed.
int take_staged(fb_session* s) {
    StagedInput* g = s->staged;
    if (!g || g->count == 0) return FB_EINVAL;
    const int k = g->head, W = s->W[0], H = s->H[0];
    FrameBuf& N = s->fr[s->next];
    FB_CUDA(cudaStreamWaitEvent(s->stream, g->ready[k], 0));
    FB_CUDA(cudaMemcpyAsync(N.depth_in, g->depth[k], (size_t)W * H * 2, cudaMemcpyDeviceToDevice, s->stream));
    FB_CUDA(cudaMemcpyAsync(N.rgb, g->rgb[k], (size_t)W * H * 3, cudaMemcpyDeviceToDevice, s->stream));
    FB_CUDA(cudaEventRecord(g->freed[k], s->stream));
    g->head ^= 1;
    --g->count;
    return FB_OK;
}

int fb_stage_frame(fb_session* s, const uint16_t* depth, size_t depth_pitch, const uint8_t* rgb, size_t rgb_pitch) {
    if (!s || !depth || !rgb) return FB_EINVAL;
    const int W = s->W[0], H = s->H[0];
    if (depth_pitch < (size_t)W * 2 || rgb_pitch < (size_t)W * 3) return FB_EINVAL;
    if (!s->staged) {
        StagedInput* g = new (std::nothrow) StagedInput;
        if (!g) return FB_ENOMEM;
        s->staged = g;
        cudaError_t e = cudaStreamCreateWithFlags(&g->copy, cudaStreamNonBlocking);
        for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
            e = cudaMalloc(&g->depth[i], (size_t)W * H * 2);
            if (e == cudaSuccess) e = cudaMalloc(&g->rgb[i], (size_t)W * H * 3);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->ready[i], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->freed[i], cudaEventDisableTiming);
        }
        if (e != cudaSuccess) {
            free_staged(s);
            cudaGetLastError();
            return e == cudaErrorMemoryAllocation ? FB_ENOMEM : (cuda_ok(e) ? FB_OK : FB_ECUDA);
        }
    }
    StagedInput* g = s->staged;
    if (g->count == 2) return FB_EINVAL;   // two frames are waiting already
    const int k = (g->head + g->count) & 1;
    FB_CUDA(cudaStreamWaitEvent(g->copy, g->freed[k], 0));   // its previous frame has been taken
    FB_CUDA(cudaMemcpy2DAsync(g->depth[k], (size_t)W * 2, depth, depth_pitch, (size_t)W * 2, H, cudaMemcpyHostToDevice,
                              g->copy));
    FB_CUDA(cudaMemcpy2DAsync(g->rgb[k], (size_t)W * 3, rgb, rgb_pitch, (size_t)W * 3, H, cudaMemcpyHostToDevice,
                              g->copy));
    FB_CUDA(cudaEventRecord(g->ready[k], g->copy));
    ++g->count;
    return FB_OK;
}

int fb_grab_frame(fb_session* s, const uint16_t* depth, size_t depth_pitch, const uint8_t* rgb, size_t rgb_pitch,
                  int on_device, fb_frame_result* out) {
    if (!s || (!depth) != (!rgb)) return FB_EINVAL;
    int rc = depth ? copy_frame_in(s, depth, depth_pitch, rgb, rgb_pitch, on_device, s->stream) : take_staged(s);
    if (rc) return rc;
    if (s->keys) return grab_with_keys(s, out);
    const FramePlan p = plan_frame(s);
    unsigned ran = 0;
    rc = enqueue_frame(s, p, s->stream, &ran);
    if (rc) return rc;
    FB_CUDA(cudaMemcpyAsync(s->h_out, s->d_out, sizeof(FrameOut), cudaMemcpyDeviceToHost, s->stream));
    FB_CUDA(cudaStreamSynchronize(s->stream));
    if (s->profile)
        for (int k = 0; k < kStages; ++k) {
            if (!(ran & (1u << k))) continue;
            float ms = 0;
            FB_CUDA(cudaEventElapsedTime(&ms, s->ev[k], s->ev[k + 1]));
            s->stage_ms[k] += ms;
            s->stage_calls[k] += 1;
        }
    finish_frame(s, p, out);
    return FB_OK;
}

int fb_session_prepare_some(fb_session* s, int shared, int max_graphs, int* remaining) {
    if (!s || max_graphs < 0) return FB_EINVAL;
    if (remaining) *remaining = 0;
    if (!s->use_graphs) return FB_OK;
    const bool keep_shared = s->shared_gpu;
    const int keep_next = s->next;
    s->shared_gpu = shared != 0;
    const int sh = s->shared_gpu ? 1 : 0;
    int rc = FB_OK, done = 0, left = 0;
    for (int mode = 0; mode < 3 && rc == FB_OK; ++mode)
        for (int fuse = 0; fuse < (mode == 2 ? 1 : 2) && rc == FB_OK; ++fuse)
            for (int next = 0; next < 2 && rc == FB_OK; ++next) {
                if (s->graph[mode][fuse][next][sh]) continue;
                if (done == max_graphs) {
                    ++left;
                    continue;
                }
                FramePlan p;
                p.state = mode == 0 ? 1 : mode == 1 ? 0 : -1;
                p.init = mode == 0;
                p.track = mode == 1;
                p.fuse = fuse != 0;
                p.render = p.init || p.track;
                p.after = 0;
                p.mode = mode;
                s->next = next;
                rc = capture_frame(s, p, s->stream);
                ++done;
            }
    s->next = keep_next;
    s->shared_gpu = keep_shared;
    if (remaining) *remaining = left;
    return rc;
}

int fb_session_prepare(fb_session* s, int shared) { return fb_session_prepare_some(s, shared, 1 << 30, nullptr); }

int fb_session_set_raycast_tile(fb_session* s, int bx, int by) {
    const bool pooled = bx == 0 && by == 0;
    if (!s || (!pooled && (bx < 1 || by < 1 || bx * by > 128 || (bx * by) % 32 != 0))) return FB_EINVAL;
    if (bx == s->rc_bx && by == s->rc_by) return FB_OK;
    drop_graphs(s);
    s->rc_bx = bx;
    s->rc_by = by;
    return FB_OK;
}

int fb_session_set_keypoints(fb_session* s, int on) {
    if (!s) return FB_EINVAL;
    if ((on != 0) == (s->keys != nullptr)) return FB_OK;
    FB_CUDA(cudaStreamSynchronize(s->stream));
    if (!on) {
        free_keys(s);
        return FB_OK;
    }
    return alloc_keys(s);
}

int fb_session_keypoint_stats(fb_session* s, fb_keypoint_stats* out) {
    if (!s || !out) return FB_EINVAL;
    if (!s->keys) {
        std::memset(out, 0, sizeof *out);
        out->bootstrap = out->relocalised = -1;
        return FB_OK;
    }
    *out = s->keys->stats;
    out->map_keys = (uint32_t)s->keys->map_n;
    return FB_OK;
}

int fb_download_keypoints(fb_session* s, int which, float* kp, float* pts, float* nrm, float* desc, uint32_t capacity,
                          uint32_t* n) {
    if (!s || !n || (which != 0 && which != 1)) return FB_EINVAL;
    *n = 0;
    if (!s->keys) return FB_OK;
    const int f = which ? s->next : 1 - s->next;
    const KeySet& ks = s->keys->set[f];
    const uint32_t k = (uint32_t)s->keys->n[f];
    *n = k;
    const size_t m = std::min(k, capacity);
    FB_CUDA(cudaStreamSynchronize(s->stream));
    if (m && kp) FB_CUDA(cudaMemcpy(kp, ks.kp, 16 * m, cudaMemcpyDeviceToHost));
    if (m && pts) FB_CUDA(cudaMemcpy(pts, ks.pt, 16 * m, cudaMemcpyDeviceToHost));
    if (m && nrm) FB_CUDA(cudaMemcpy(nrm, ks.nrm, 16 * m, cudaMemcpyDeviceToHost));
    if (m && desc) FB_CUDA(cudaMemcpy(desc, ks.desc, 4 * kKeyDesc * m, cudaMemcpyDeviceToHost));
    return FB_OK;
}

int fb_match_descriptors(const float* query, uint32_t nq, const float* train, uint32_t nt, int32_t* best, float* dist,
                         void* stream) {
    if ((nq && (!query || !best || !dist)) || (nt && !train) || nq > (1u << 24) || nt > (1u << 24)) return FB_EINVAL;
    cudaStream_t st = as_stream(stream);
    if (nq == 0) return FB_OK;
    if (nt == 0) {
        FB_CUDA(cudaMemsetAsync(best, 0xff, 8 * (size_t)nq, st));
        FB_CUDA(cudaMemsetAsync(dist, 0x7f, 8 * (size_t)nq, st));
        FB_CUDA(cudaStreamSynchronize(st));
        return FB_OK;
    }
    const int rc = launch_match2(query, (int)nq, train, (int)nt, (int2*)best, (float2*)dist, st);
    if (rc) return rc;
    FB_CUDA(cudaStreamSynchronize(st));
    return FB_OK;
}

int fb_pose_estimate(const double* src, const double* ref, uint32_t n, int iterations, int check_angle, uint64_t seed,
                     double T[16], uint8_t* inlier, int* ok) {
    if (!src || !ref || !T || !ok || iterations < 0 || n > (1u << 24)) return FB_EINVAL;
    std::vector<uint8_t> outl(n ? n : 1, 1);
    *ok = pose_estimate(src, ref, (int)n, iterations, check_angle != 0, seed, T, outl.data()) ? 1 : 0;
    if (inlier)
        for (uint32_t i = 0; i < n; ++i) inlier[i] = outl[i] ? 0 : 1;
    return FB_OK;
}

int fb_session_set_mapping(fb_session* s, int on) {
    if (!s) return FB_EINVAL;
    if (s->mapping_disabled == (on != 0)) drop_graphs(s);   // cached graphs hold the other variant
    s->mapping_disabled = on == 0;
    return FB_OK;
}

int fb_session_set_graphs(fb_session* s, int on) {
    if (!s) return FB_EINVAL;
    s->use_graphs = on != 0;
    return FB_OK;
}

int fb_session_set_persistent(fb_session* s, int on) {
    if (!s) return FB_EINVAL;
    if (s->persistent != (on != 0)) drop_graphs(s);   // cached graphs hold the other tracking variant
    s->persistent = on != 0;
    return FB_OK;
}

int fb_session_set_profiling(fb_session* s, int on) {
    if (!s) return FB_EINVAL;
    s->profile = on != 0;
    for (int i = 0; i < kStages; ++i) {
        s->stage_ms[i] = 0;
        s->stage_calls[i] = 0;
    }
    return FB_OK;
}

int fb_session_stage_times(fb_session* s, double* ms, uint64_t* calls, int n) {
    if (!s || n < 0) return FB_EINVAL;
    for (int i = 0; i < n && i < kStages; ++i) {
        if (ms) ms[i] = s->stage_ms[i];
        if (calls) calls[i] = s->stage_calls[i];
    }
    return FB_OK;
}

int fb_session_launch_count(fb_session* s, uint64_t* launches) {
    if (!s || !launches) return FB_EINVAL;
    *launches = s->launches;
    return FB_OK;
}

int fb_frame_transfer_bytes(const fb_config* c, size_t* h2d, size_t* d2h) {
    if (!valid_config(c)) return FB_EINVAL;
    if (h2d) *h2d = (size_t)c->width * c->height * (sizeof(uint16_t) + 3);
    if (d2h) *d2h = sizeof(FrameOut);
    return FB_OK;
}

int fb_get_pose(fb_session* s, double pose[16]) {
    if (!s || !pose) return FB_EINVAL;
    std::memcpy(pose, s->pose, sizeof s->pose);
    return FB_OK;
}

int fb_download_level(fb_session* s, int which, int l, float* vmap, float* nmap, float* depth, uint8_t* gray,
                      int16_t* dx, int16_t* dy) {
    if (!s || which < 0 || which > 1 || l < 0 || l > 2) return FB_EINVAL;
    const FrameBuf& F = s->fr[which ? s->next : 1 - s->next];
    size_t n = (size_t)s->W[l] * s->H[l];
    cudaStream_t st = s->stream;
    if (vmap) FB_CUDA(cudaMemcpyAsync(vmap, F.vmap[l], 16 * n, cudaMemcpyDeviceToHost, st));
    if (nmap) FB_CUDA(cudaMemcpyAsync(nmap, F.nmap[l], 16 * n, cudaMemcpyDeviceToHost, st));
    if (depth) FB_CUDA(cudaMemcpyAsync(depth, F.depth[l], 4 * n, cudaMemcpyDeviceToHost, st));
    if (gray) FB_CUDA(cudaMemcpyAsync(gray, F.gray[l], n, cudaMemcpyDeviceToHost, st));
    if (dx) FB_CUDA(cudaMemcpyAsync(dx, F.dx[l], 2 * n, cudaMemcpyDeviceToHost, st));
    if (dy) FB_CUDA(cudaMemcpyAsync(dy, F.dy[l], 2 * n, cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaStreamSynchronize(st));
    return FB_OK;
}

int fb_download_raw(fb_session* s, int which, float* raw) {
    if (!s || !raw || which < 0 || which > 1) return FB_EINVAL;
    const FrameBuf& F = s->fr[which ? s->next : 1 - s->next];
    FB_CUDA(cudaMemcpyAsync(raw, F.raw, 4 * (size_t)s->W[0] * s->H[0], cudaMemcpyDeviceToHost, s->stream));
    FB_CUDA(cudaStreamSynchronize(s->stream));
    return FB_OK;
}

int fb_map_get_stats(fb_session* s, fb_map_stats* out) {
    if (!s || !out) return FB_EINVAL;
    MapCounters c;
    FB_CUDA(cudaMemcpyAsync(&c, s->ctr, sizeof c, cudaMemcpyDeviceToHost, s->stream));
    FB_CUDA(cudaStreamSynchronize(s->stream));
    out->heap_counter = c.heap_counter;
    out->entry_ptr = c.entry_ptr;
    out->no_allocated = (uint32_t)c.n_alloc;
    out->no_visible = (uint32_t)c.n_visible;
    out->no_new = (uint32_t)c.n_new;
    out->no_tiles = (uint32_t)c.n_tiles;
    out->error_flags = c.err;
    out->sequential = c.seq_path;
    return FB_OK;
}

int fb_map_download_entries(fb_session* s, int32_t* entries) {
    if (!s || !entries) return FB_EINVAL;
    const int n = s->map.NB + s->map.NE;
    int* tmp = nullptr;
    FB_CUDA(cudaMallocAsync((void**)&tmp, sizeof(int) * 5 * (size_t)n, s->stream));
    k_export_entries<<<592, 256, 0, s->stream>>>(s->map.entries, n, tmp);
    cudaError_t e = cudaMemcpyAsync(entries, tmp, sizeof(int) * 5 * (size_t)n, cudaMemcpyDeviceToHost, s->stream);
    cudaFreeAsync(tmp, s->stream);
    FB_CUDA(e);
    FB_CUDA(cudaStreamSynchronize(s->stream));
    return FB_OK;
}

int fb_map_download_blocks(fb_session* s, const int32_t* ptrs, int n, float* sdf, uint8_t* weight, uint8_t* rgb) {
    if (!s || (n > 0 && !ptrs) || n < 0) return FB_EINVAL;
    std::vector<Voxel> tmp(512);
    std::vector<uint8_t> cb(kCBlockBytes);
    for (int i = 0; i < n; ++i) {
        if (ptrs[i] < 0 || ptrs[i] % 512 || ptrs[i] / 512 >= s->map.NS) return FB_EINVAL;
        if (s->map.cvox) {
            // precision form: FP16 TSDF widened to float, weight and colour as stored
            FB_CUDA(cudaMemcpyAsync(cb.data(), s->map.cvox + (size_t)(ptrs[i] / 512) * kCBlockBytes, kCBlockBytes,
                                    cudaMemcpyDeviceToHost, s->stream));
            FB_CUDA(cudaStreamSynchronize(s->stream));
            for (int v = 0; v < 512; ++v) {
                uint16_t h;
                std::memcpy(&h, cb.data() + 2 * v, 2);
                tmp[v].sdf = half_bits_to_float(h);
                tmp[v].weight = cb[kCWeight + v];
                tmp[v].r = cb[kCRed + v];
                tmp[v].g = cb[kCGreen + v];
                tmp[v].b = cb[kCBlue + v];
            }
        } else {
            FB_CUDA(cudaMemcpyAsync(tmp.data(), s->map.voxels + ptrs[i], 512 * sizeof(Voxel), cudaMemcpyDeviceToHost,
                                    s->stream));
            FB_CUDA(cudaStreamSynchronize(s->stream));
        }
        for (int v = 0; v < 512; ++v) {
            size_t o = (size_t)i * 512 + v;
            if (sdf) sdf[o] = tmp[v].sdf;
            if (weight) weight[o] = tmp[v].weight;
            if (rgb) {
                rgb[3 * o] = tmp[v].r;
                rgb[3 * o + 1] = tmp[v].g;
                rgb[3 * o + 2] = tmp[v].b;
            }
        }
    }
    return FB_OK;
}

int fb_map_download_visible(fb_session* s, int32_t* slots, uint32_t capacity, uint32_t* n) {
    if (!s || !n) return FB_EINVAL;
    MapCounters c;
    FB_CUDA(cudaMemcpyAsync(&c, s->ctr, sizeof c, cudaMemcpyDeviceToHost, s->stream));
    FB_CUDA(cudaStreamSynchronize(s->stream));
    uint32_t nv = (uint32_t)(c.n_visible < s->map.NS ? c.n_visible : s->map.NS);
    *n = nv;
    if (slots && capacity) {
        uint32_t k = nv < capacity ? nv : capacity;
        FB_CUDA(cudaMemcpyAsync(slots, s->map.visible, 4 * (size_t)k, cudaMemcpyDeviceToHost, s->stream));
        FB_CUDA(cudaStreamSynchronize(s->stream));
    }
    return FB_OK;
}

// ---------------------------------------------------------- per-stage entries

int fb_filter_depth(const fb_image* depth, fb_image* raw, fb_image* filtered, float depth_scale, float depth_cutoff,
                    void* stream) {
    if (!image_ok(depth, 2) || !image_ok(raw, 4) || !image_ok(filtered, 4)) return FB_EINVAL;
    if (raw->cols < depth->cols || raw->rows < depth->rows || filtered->cols < depth->cols ||
        filtered->rows < depth->rows || !(depth_scale > 0))
        return FB_EINVAL;
    launch_level0((const uint16_t*)depth->data, (int)(depth->pitch / 2), nullptr, 0, depth->cols, depth->rows,
                  depth_scale, depth_cutoff, (float*)raw->data, (int)(raw->pitch / 4), (float*)filtered->data,
                  (int)(filtered->pitch / 4), nullptr, 0, as_stream(stream));
    return check_launch();
}

int fb_image_to_intensity(const fb_image* rgb, fb_image* gray, void* stream) {
    if (!image_ok(rgb, 3) || !image_ok(gray, 1) || gray->cols < rgb->cols || gray->rows < rgb->rows) return FB_EINVAL;
    // gray only: the level-0 kernel with no depth outputs reads no depth
    launch_level0(nullptr, 0, (const uint8_t*)rgb->data, (int)rgb->pitch, rgb->cols, rgb->rows, 1.0f, 0.0f,
                  nullptr, 0, nullptr, 0, (uint8_t*)gray->data, (int)gray->pitch, as_stream(stream));
    return check_launch();
}

int fb_pyrdown_gauss_f32(const fb_image* src, fb_image* dst, void* stream) {
    if (!image_ok(src, 4) || !image_ok(dst, 4) || dst->cols < src->cols / 2 || dst->rows < src->rows / 2)
        return FB_EINVAL;
    launch_pyrdown((const float*)src->data, (int)(src->pitch / 4), nullptr, 0, src->cols, src->rows,
                   (float*)dst->data, (int)(dst->pitch / 4), nullptr, 0, as_stream(stream));
    return check_launch();
}

int fb_pyrdown_gauss_u8(const fb_image* src, fb_image* dst, void* stream) {
    if (!image_ok(src, 1) || !image_ok(dst, 1) || dst->cols < src->cols / 2 || dst->rows < src->rows / 2)
        return FB_EINVAL;
    launch_pyrdown(nullptr, 0, (const uint8_t*)src->data, (int)src->pitch, src->cols, src->rows, nullptr, 0,
                   (uint8_t*)dst->data, (int)dst->pitch, as_stream(stream));
    return check_launch();
}

int fb_compute_vmap(const fb_image* depth, fb_image* vmap, float fx, float fy, float cx, float cy, float depth_cutoff,
                    void* stream) {
    if (!image_ok(depth, 4) || !image_ok(vmap, 16) || vmap->cols < depth->cols || vmap->rows < depth->rows)
        return FB_EINVAL;
    if (!(fx > 0) || !(fy > 0)) return FB_EINVAL;
    Intr k;
    k.fx = fx;
    k.fy = fy;
    k.cx = cx;
    k.cy = cy;
    k.invfx = (float)(1.0 / (double)fx);
    k.invfy = (float)(1.0 / (double)fy);
    launch_maps((const float*)depth->data, (int)(depth->pitch / 4), nullptr, 0, depth->cols, depth->rows, k,
                depth_cutoff, (float4*)vmap->data, (int)(vmap->pitch / 16), nullptr, 0, nullptr, nullptr, 0,
                as_stream(stream));
    return check_launch();
}

int fb_compute_nmap(const fb_image* vmap, fb_image* nmap, void* stream) {
    if (!image_ok(vmap, 16) || !image_ok(nmap, 16) || nmap->cols < vmap->cols || nmap->rows < vmap->rows)
        return FB_EINVAL;
    launch_nmap((const float4*)vmap->data, (int)(vmap->pitch / 16), vmap->cols, vmap->rows, (float4*)nmap->data,
                (int)(nmap->pitch / 16), as_stream(stream));
    return check_launch();
}

int fb_compute_derivative_image(const fb_image* gray, fb_image* dx, fb_image* dy, void* stream) {
    if (!image_ok(gray, 1) || !image_ok(dx, 2) || !image_ok(dy, 2) || dx->pitch != dy->pitch ||
        dx->cols < gray->cols || dx->rows < gray->rows)
        return FB_EINVAL;
    Intr k{};
    launch_maps(nullptr, 0, (const uint8_t*)gray->data, (int)gray->pitch, gray->cols, gray->rows, k, 0.f, nullptr, 0,
                nullptr, 0, (int16_t*)dx->data, (int16_t*)dy->data, (int)(dx->pitch / 2), as_stream(stream));
    return check_launch();
}

int fb_resize_map(const fb_image* vsrc, const fb_image* nsrc, fb_image* vdst, fb_image* ndst, void* stream) {
    if (!image_ok(vsrc, 16) || !image_ok(nsrc, 16) || !image_ok(vdst, 16) || !image_ok(ndst, 16)) return FB_EINVAL;
    if (vsrc->pitch != nsrc->pitch || vdst->pitch != ndst->pitch || vdst->cols < vsrc->cols / 2 ||
        vdst->rows < vsrc->rows / 2)
        return FB_EINVAL;
    launch_resize((const float4*)vsrc->data, (const float4*)nsrc->data, (int)(vsrc->pitch / 16), vsrc->cols,
                  vsrc->rows, (float4*)vdst->data, (float4*)ndst->data, (int)(vdst->pitch / 16), as_stream(stream));
    return check_launch();
}

size_t fb_step_scratch_bytes(int cols, int rows) {
    if (cols <= 0 || rows <= 0) return 0;
    // partials | tickets | out sums (32 doubles) | per-pixel correspondences
    return (size_t)kTrackMaxBlocks * 32 * 4 + 256 + 32 * 8 + (size_t)cols * rows * 4;
}

namespace {
struct StepScratch {
    float* partials;
    unsigned int* tickets;
    double* out;
    int* residual;
};
bool carve(void* scratch, size_t bytes, int cols, int rows, StepScratch& s) {
    if (!scratch || bytes < fb_step_scratch_bytes(cols, rows) || ((uintptr_t)scratch & 15)) return false;
    char* p = (char*)scratch;
    s.partials = (float*)p;
    p += (size_t)kTrackMaxBlocks * 32 * 4;
    s.tickets = (unsigned int*)p;
    p += 256;
    s.out = (double*)p;
    p += 32 * 8;
    s.residual = (int*)p;
    return true;
}
void unpack(const double* s, double* A, double* b) {
    int n = 0;
    for (int i = 0; i < 6; ++i)
        for (int j = i; j < 7; ++j) {
            double v = (double)(float)s[n++];  // the reference's sums are floats (Reduction.cu:369-371)
            if (j == 6)
                b[i] = v;
            else
                A[j * 6 + i] = A[i * 6 + j] = v;
        }
}
}  // namespace

int fb_icp_step(const fb_image* vcurr, const fb_image* vlast, const fb_image* ncurr, const fb_image* nlast,
                const float Rcurr[9], const float tcurr[3], const float Rlast[9], const float RlastInv[9],
                const float tlast[3], const float K[4], void* scratch, size_t scratch_bytes, float residual[2],
                double A[36], double b[6], void* stream) {
    if (!image_ok(vcurr, 16) || !image_ok(vlast, 16) || !image_ok(ncurr, 16) || !image_ok(nlast, 16)) return FB_EINVAL;
    if (!Rcurr || !tcurr || !Rlast || !RlastInv || !tlast || !K || !residual || !A || !b) return FB_EINVAL;
    const int W = vcurr->cols, H = vcurr->rows;
    if (vlast->cols != W || vlast->rows != H || ncurr->cols != W || nlast->cols != W || ncurr->rows != H ||
        nlast->rows != H || vcurr->pitch != vlast->pitch || vcurr->pitch != ncurr->pitch ||
        vcurr->pitch != nlast->pitch)
        return FB_EINVAL;
    StepScratch sc;
    if (!carve(scratch, scratch_bytes, W, H, sc)) return FB_EINVAL;
    cudaStream_t st = as_stream(stream);
    TrackLevel L{};
    L.W = W;
    L.H = H;
    L.vp = (int)(vcurr->pitch / 16);
    L.k = intr_from(K);
    L.vcurr = (const float4*)vcurr->data;
    L.vlast = (const float4*)vlast->data;
    L.ncurr = (const float4*)ncurr->data;
    L.nlast = (const float4*)nlast->data;
    float Rt[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Rt[i * 3 + j] = Rcurr[j * 3 + i];
    DevPose cur = pose_from(Rcurr, Rt, tcurr), last = pose_from(Rlast, RlastInv, tlast);
    FB_CUDA(cudaMemsetAsync(sc.tickets, 0, 16, st));
    launch_step_icp(L, cur, last, sc.partials, sc.tickets, sc.out, st);
    if (check_launch()) return FB_ECUDA;
    double host[32];
    FB_CUDA(cudaMemcpyAsync(host, sc.out, 29 * 8, cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaStreamSynchronize(st));
    unpack(host, A, b);
    residual[0] = (float)host[27];
    residual[1] = (float)host[28];
    return FB_OK;
}

int fb_rgb_step(const fb_image* gcurr, const fb_image* glast, const fb_image* vcurr, const fb_image* vlast,
                const fb_image* dx, const fb_image* dy, const float Rcurr[9], const float RcurrInv[9],
                const float Rlast[9], const float RlastInv[9], const float tcurr[3], const float tlast[3],
                const float K[4], void* scratch, size_t scratch_bytes, float residual[2], double A[36], double b[6],
                void* stream) {
    if (!image_ok(gcurr, 1) || !image_ok(glast, 1) || !image_ok(vcurr, 16) || !image_ok(vlast, 16) ||
        !image_ok(dx, 2) || !image_ok(dy, 2))
        return FB_EINVAL;
    if (!Rcurr || !RcurrInv || !Rlast || !RlastInv || !tcurr || !tlast || !K || !residual || !A || !b)
        return FB_EINVAL;
    const int W = gcurr->cols, H = gcurr->rows;
    if (glast->cols != W || glast->rows != H || vcurr->cols != W || vcurr->rows != H || vlast->cols != W ||
        vlast->rows != H || dx->cols != W || dy->cols != W || dx->rows != H || dy->rows != H ||
        gcurr->pitch != glast->pitch || vcurr->pitch != vlast->pitch || dx->pitch != dy->pitch)
        return FB_EINVAL;
    StepScratch sc;
    if (!carve(scratch, scratch_bytes, W, H, sc)) return FB_EINVAL;
    cudaStream_t st = as_stream(stream);
    TrackLevel L{};
    L.W = W;
    L.H = H;
    L.vp = (int)(vcurr->pitch / 16);
    L.gp = (int)gcurr->pitch;
    L.sp = (int)(dx->pitch / 2);
    L.k = intr_from(K);
    L.vcurr = (const float4*)vcurr->data;
    L.vlast = (const float4*)vlast->data;
    L.gcurr = (const uint8_t*)gcurr->data;
    L.glast = (const uint8_t*)glast->data;
    L.dx = (const int16_t*)dx->data;
    L.dy = (const int16_t*)dy->data;
    DevPose cur = pose_from(Rcurr, RcurrInv, tcurr), last = pose_from(Rlast, RlastInv, tlast);
    FB_CUDA(cudaMemsetAsync(sc.tickets, 0, 16, st));
    launch_step_rgb(L, cur, last, sc.partials, sc.tickets, sc.residual, sc.out, st);
    if (check_launch()) return FB_ECUDA;
    double host[32];
    FB_CUDA(cudaMemcpyAsync(host, sc.out, 32 * 8, cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaStreamSynchronize(st));
    unpack(host, A, b);
    residual[0] = (float)host[27];
    residual[1] = (float)host[28];
    return FB_OK;
}

int fb_reset_map(fb_session* s) {
    if (!s) return FB_EINVAL;
    launch_map_reset(s->map, s->stream);
    if (check_launch()) return FB_ECUDA;
    FB_CUDA(cudaStreamSynchronize(s->stream));
    return FB_OK;
}

int fb_fuse_map_color(fb_session* s, const fb_image* depth, const fb_image* rgb, const fb_image* nmap,
                      const float Rview[9], const float RviewInv[9], const float tview[3], const float K[4],
                      uint32_t* no_visible, void* stream) {
    if (!s || !image_ok(depth, 4) || !image_ok(rgb, 3) || !image_ok(nmap, 16) || !Rview || !RviewInv || !tview || !K)
        return FB_EINVAL;
    const int W = depth->cols, H = depth->rows;
    if (rgb->cols < W || rgb->rows < H || nmap->cols < W || nmap->rows < H) return FB_EINVAL;
    if ((W + 7) / 8 > s->map.zc || (H + 7) / 8 > s->map.zr) return FB_EINVAL;
    cudaStream_t st = stream ? as_stream(stream) : s->stream;
    k_set_pose<<<1, 1, 0, st>>>(s->scratch_pose, pose_from(Rview, RviewInv, tview));
    const Intr k = intr_from(K);
    launch_allocate(s->map, (const float*)depth->data, (int)(depth->pitch / 4), W, H, k, s->scratch_pose, nullptr, st);
    launch_visibility(s->map, W, H, k, s->scratch_pose, nullptr, st);
    launch_integrate(s->map, (const float*)depth->data, (int)(depth->pitch / 4), (const uint8_t*)rgb->data,
                     (int)rgb->pitch, (const float4*)nmap->data, (int)(nmap->pitch / 16), W, H, k, s->scratch_pose,
                     nullptr, st);
    if (check_launch()) return FB_ECUDA;
    FB_CUDA(cudaStreamSynchronize(st));
    if (no_visible) {
        MapCounters c;
        FB_CUDA(cudaMemcpy(&c, s->ctr, sizeof c, cudaMemcpyDeviceToHost));
        *no_visible = (uint32_t)c.n_visible;
    }
    return FB_OK;
}

int fb_check_block_visibility(fb_session* s, const float Rview[9], const float RviewInv[9], const float tview[3],
                              int cols, int rows, const float K[4], uint32_t* no_visible, void* stream) {
    if (!s || !Rview || !RviewInv || !tview || !K || cols <= 0 || rows <= 0) return FB_EINVAL;
    cudaStream_t st = stream ? as_stream(stream) : s->stream;
    k_set_pose<<<1, 1, 0, st>>>(s->scratch_pose, pose_from(Rview, RviewInv, tview));
    launch_visibility(s->map, cols, rows, intr_from(K), s->scratch_pose, nullptr, st);
    if (check_launch()) return FB_ECUDA;
    FB_CUDA(cudaStreamSynchronize(st));
    if (no_visible) {
        MapCounters c;
        FB_CUDA(cudaMemcpy(&c, s->ctr, sizeof c, cudaMemcpyDeviceToHost));
        *no_visible = (uint32_t)c.n_visible;
    }
    return FB_OK;
}

int fb_raycast(fb_session* s, fb_image* vmap, fb_image* nmap, const float Rview[9], const float RviewInv[9],
               const float tview[3], const float K[4], int* rendered, void* stream) {
    if (!s || !image_ok(vmap, 16) || !image_ok(nmap, 16) || vmap->pitch != nmap->pitch || !Rview || !RviewInv ||
        !tview || !K)
        return FB_EINVAL;
    const int W = vmap->cols, H = vmap->rows;
    if (nmap->cols != W || nmap->rows != H || (W + 7) / 8 > s->map.zc || (H + 7) / 8 > s->map.zr) return FB_EINVAL;
    cudaStream_t st = stream ? as_stream(stream) : s->stream;
    k_set_pose<<<1, 1, 0, st>>>(s->scratch_pose, pose_from(Rview, RviewInv, tview));
    const Intr k = intr_from(K);
    launch_zrange(s->map, k, s->scratch_pose, nullptr, st);
    launch_raycast(s->map, (float4*)vmap->data, (float4*)nmap->data, (int)(vmap->pitch / 16), W, H, k,
                   s->scratch_pose, nullptr, st);
    if (check_launch()) return FB_ECUDA;
    FB_CUDA(cudaStreamSynchronize(st));
    if (rendered) {
        MapCounters c;
        FB_CUDA(cudaMemcpy(&c, s->ctr, sizeof c, cudaMemcpyDeviceToHost));
        *rendered = c.n_tiles > 0;
    }
    return FB_OK;
}

int fb_render_top_down(fb_session* s, float dist, fb_image* vmap, fb_image* nmap, fb_image* rgba, int* rendered,
                       void* stream) {
    if (!s || !image_ok(vmap, 16) || !image_ok(nmap, 16) || !image_ok(rgba, 4) || vmap->pitch != nmap->pitch ||
        !(dist >= 0.f))
        return FB_EINVAL;
    const int W = vmap->cols, H = vmap->rows;
    if (nmap->cols != W || nmap->rows != H || rgba->cols != W || rgba->rows != H || (W + 7) / 8 > s->map.zc ||
        (H + 7) / 8 > s->map.zr)
        return FB_EINVAL;
    cudaStream_t st = stream ? as_stream(stream) : s->stream;
    // Eigen::AngleAxisd(M_PI / 2, -UnitX).toRotationMatrix() rounded to float
    // (System.cc:77-81): c I + s [a]x + (1 - c) a a^T with a = -x, s = 1 and
    // c = cos(pi / 2) = 6.1e-17, which float keeps
    const float c = (float)std::cos(M_PI / 2);
    const float R[9] = {1.f, 0.f, 0.f, 0.f, c, 1.f, 0.f, -1.f, c};
    const float Rinv[9] = {1.f, 0.f, 0.f, 0.f, c, -1.f, 0.f, 1.f, c};
    const float t[3] = {0.f, -dist, 0.f};
    // Frame::fx(0), Frame::fy(0) and the image centre in whole pixels
    const float K[4] = {s->K[0].fx, s->K[0].fy, (float)(W / 2), (float)(H / 2)};
    MapView m = s->map;
    m.g.depth_min = dist + s->map.g.depth_min;
    m.g.depth_max = dist + s->map.g.depth_max;
    k_set_pose<<<1, 1, 0, st>>>(s->scratch_pose, pose_from(R, Rinv, t));
    const Intr k = intr_from(K);
    // Mapping::UpdateVisibility (Mapping.cc:68-74) scans for a 640 x 480
    // camera whatever the image size
    launch_visibility(m, 640, 480, k, s->scratch_pose, nullptr, st);
    launch_zrange(m, k, s->scratch_pose, nullptr, st);
    launch_raycast(m, (float4*)vmap->data, (float4*)nmap->data, (int)(vmap->pitch / 16), W, H, k, s->scratch_pose,
                   nullptr, st);
    if (check_launch()) return FB_ECUDA;
    MapCounters ctr;
    FB_CUDA(cudaMemcpyAsync(&ctr, s->ctr, sizeof ctr, cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaStreamSynchronize(st));
    const float light[3] = {0.f, 0.f, 0.f};
    const int rc = fb_render_image(vmap, nmap, light, rgba, st);
    if (rc != FB_OK) return rc;
    if (rendered) *rendered = ctr.n_tiles > 0;
    return FB_OK;
}

int fb_mesh_scene(fb_session* s, float* vertex, float* normal, uint8_t* color, uint64_t max_triangles,
                  uint64_t* no_triangles, void* stream) {
    if (!s || !no_triangles) return FB_EINVAL;
    const bool any = vertex || normal || color;
    if (any && !(vertex && normal && color)) return FB_EINVAL;
    cudaStream_t st = stream ? as_stream(stream) : s->stream;
    MapCounters c;
    FB_CUDA(cudaMemcpyAsync(&c, s->ctr, sizeof c, cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaStreamSynchronize(st));
    unsigned long long total = 0;
    const int rc = launch_mesh(s->map, c.n_alloc, vertex, normal, color, any ? max_triangles : 0, &total, st);
    if (rc != FB_OK) return rc;
    s->launches += any ? 3 : 2;
    *no_triangles = total;
    return FB_OK;
}

int fb_save_mesh(fb_session* s, const char* path, uint64_t* no_triangles) {
    if (!s || !path) return FB_EINVAL;
    uint64_t n = 0;
    int rc = fb_mesh_scene(s, nullptr, nullptr, nullptr, 0, &n, nullptr);
    if (rc != FB_OK) return rc;
    std::vector<float> V(n * 9), N(n * 9);
    std::vector<uint8_t> C(n * 9);
    if (n) {
        float* dv = nullptr;
        FB_CUDA(cudaMallocAsync((void**)&dv, n * 9 * (2 * sizeof(float) + 1), s->stream));
        float* dn = dv + n * 9;
        uint8_t* dc = (uint8_t*)(dn + n * 9);
        uint64_t m = 0;
        rc = fb_mesh_scene(s, dv, dn, dc, n, &m, nullptr);
        cudaError_t e = cudaSuccess;
        if (rc == FB_OK) {
            e = cudaMemcpyAsync(V.data(), dv, n * 9 * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(N.data(), dn, n * 9 * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(C.data(), dc, n * 9, cudaMemcpyDeviceToHost, s->stream);
        }
        cudaFreeAsync(dv, s->stream);
        const cudaError_t se = cudaStreamSynchronize(s->stream);
        if (rc != FB_OK) return rc;
        if (e != cudaSuccess || se != cudaSuccess) {
            fb_set_error_text(cudaGetErrorString(e != cudaSuccess ? e : se));
            return FB_ECUDA;
        }
    }
    if (no_triangles) *no_triangles = n;
    return fb_write_ply(path, V.data(), N.data(), C.data(), n);
}

}  // extern "C"

// ---------------------------------------------------------------- snapshots
//
// A snapshot holds everything a session needs to continue exactly where it
// was: the tracker's host state, the device tracker state, both frames, and
// the map -- counters, the whole hash table, the free-block stack, the
// allocated and visible lists and the used prefix of the voxel pool.  Blocks
// are taken from the free stack in order and never given back, so the used
// blocks are exactly the pool prefix [0, NumBlocks - 1 - heap_counter); the
// rest of the pool is in its reset state and is not stored.  The reference
// dumps its whole device map (System::WriteMapToDisk, Core/System.cc:195-236);
// this is the same idea with the unused pool left out and the tracker added.

namespace {

constexpr char kSnapMagic[8] = {'F', 'B', 'S', 'N', 'A', 'P', '0', '1'};

struct SnapHeader {
    char magic[8];
    fb_config cfg;
    int next, state, last_state, no_missed, frames_after_reloc, used_blocks;
    uint64_t frame_id;
    double pose[16];
    MapCounters ctr;
    uint64_t total_bytes;
};

int clamp_count(int v, int hi) { return v < 0 ? 0 : v > hi ? hi : v; }

// The byte ranges of a session's state in snapshot order (device pointer,
// size), after the header.
std::vector<std::pair<void*, size_t>> snapshot_ranges(fb_session* s, const MapCounters& c) {
    std::vector<std::pair<void*, size_t>> r;
    const MapView& m = s->map;
    const int used = clamp_count(m.NS - 1 - c.heap_counter, m.NS);
    const int na = clamp_count(c.n_alloc, m.NS);
    const int nv = clamp_count(c.n_visible, m.NS);
    r.push_back({m.entries, ((size_t)m.NB + m.NE) * sizeof(HEntry)});
    r.push_back({m.heap, (size_t)m.NS * sizeof(int)});
    r.push_back({m.alloc_list, (size_t)na * sizeof(int)});
    r.push_back({m.visible, (size_t)nv * sizeof(int)});
    r.push_back({m.vis_blocks, (size_t)nv * sizeof(HEntry)});
    if (m.cvox)
        r.push_back({m.cvox, (size_t)used * kCBlockBytes});
    else
        r.push_back({m.voxels, (size_t)used * 512 * sizeof(Voxel)});
    r.push_back({s->st, sizeof(TrackState)});
    for (int f = 0; f < 2; ++f) {
        FrameBuf& F = s->fr[f];
        const size_t n0 = (size_t)s->W[0] * s->H[0];
        r.push_back({F.depth_in, n0 * 2});
        r.push_back({F.rgb, n0 * 3});
        r.push_back({F.raw, n0 * 4});
        for (int l = 0; l < 3; ++l) {
            const size_t n = (size_t)s->W[l] * s->H[l];
            r.push_back({F.depth[l], n * 4});
            r.push_back({F.vmap[l], n * 16});
            r.push_back({F.nmap[l], n * 16});
            r.push_back({F.gray[l], n});
            r.push_back({F.dx[l], n * 2});
            r.push_back({F.dy[l], n * 2});
            r.push_back({F.rgbok[l], n});
        }
    }
    return r;
}

int read_counters(fb_session* s, MapCounters* c) {
    FB_CUDA(cudaMemcpyAsync(c, s->ctr, sizeof *c, cudaMemcpyDeviceToHost, s->stream));
    FB_CUDA(cudaStreamSynchronize(s->stream));
    return FB_OK;
}

}  // namespace

extern "C" {

int fb_snapshot_bytes(fb_session* s, size_t* bytes) {
    if (!s || !bytes) return FB_EINVAL;
    MapCounters c;
    int rc = read_counters(s, &c);
    if (rc) return rc;
    size_t n = sizeof(SnapHeader);
    for (auto& r : snapshot_ranges(s, c)) n += r.second;
    *bytes = n;
    return FB_OK;
}

int fb_snapshot(fb_session* s, void* buf, size_t capacity, size_t* written) {
    if (!s || !buf) return FB_EINVAL;
    SnapHeader h;
    std::memset(&h, 0, sizeof h);
    int rc = read_counters(s, &h.ctr);
    if (rc) return rc;
    const auto ranges = snapshot_ranges(s, h.ctr);
    size_t total = sizeof h;
    for (auto& r : ranges) total += r.second;
    if (capacity < total) {
        fb_set_error_text("fb_snapshot: buffer smaller than fb_snapshot_bytes");
        return FB_EINVAL;
    }
    std::memcpy(h.magic, kSnapMagic, 8);
    h.cfg = s->cfg;
    h.next = s->next;
    h.state = s->state;
    h.last_state = s->last_state;
    h.no_missed = s->no_missed;
    h.frames_after_reloc = s->frames_after_reloc;
    h.frame_id = s->frame_id;
    std::memcpy(h.pose, s->pose, sizeof h.pose);
    h.used_blocks = clamp_count(s->map.NS - 1 - h.ctr.heap_counter, s->map.NS);
    h.total_bytes = total;
    char* out = (char*)buf;
    std::memcpy(out, &h, sizeof h);
    size_t o = sizeof h;
    for (auto& r : ranges) {
        if (r.second) FB_CUDA(cudaMemcpyAsync(out + o, r.first, r.second, cudaMemcpyDeviceToHost, s->stream));
        o += r.second;
    }
    FB_CUDA(cudaStreamSynchronize(s->stream));
    if (written) *written = total;
    return FB_OK;
}

int fb_restore(fb_session* s, const void* buf, size_t size) {
    if (!s || !buf || size < sizeof(SnapHeader)) return FB_EINVAL;
    SnapHeader h;
    std::memcpy(&h, buf, sizeof h);
    if (std::memcmp(h.magic, kSnapMagic, 8) != 0 || h.total_bytes != size) {
        fb_set_error_text("fb_restore: not a snapshot of this format");
        return FB_EINVAL;
    }
    if (std::memcmp(&h.cfg, &s->cfg, sizeof h.cfg) != 0) {
        fb_set_error_text("fb_restore: the snapshot was taken with another configuration");
        return FB_EINVAL;
    }
    // the unused pool and the per-frame scratch in their reset state first
    launch_map_reset(s->map, s->stream);
    if (check_launch()) return FB_ECUDA;
    const auto ranges = snapshot_ranges(s, h.ctr);
    size_t o = sizeof h;
    for (auto& r : ranges) {
        if (o + r.second > size) return FB_EINVAL;
        if (r.second)
            FB_CUDA(cudaMemcpyAsync(r.first, (const char*)buf + o, r.second, cudaMemcpyHostToDevice, s->stream));
        o += r.second;
    }
    FB_CUDA(cudaMemcpyAsync(s->ctr, &h.ctr, sizeof h.ctr, cudaMemcpyHostToDevice, s->stream));
    FB_CUDA(cudaStreamSynchronize(s->stream));
    s->next = h.next;
    s->state = h.state;
    s->last_state = h.last_state;
    s->no_missed = h.no_missed;
    s->frames_after_reloc = h.frames_after_reloc;
    s->frame_id = h.frame_id;
    std::memcpy(s->pose, h.pose, sizeof s->pose);
    return FB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- map files
//
// System::WriteMapToDisk / ReadMapFromDisk (Core/System.cc:195-271, through
// Mapping::DownloadToRAM / UploadFromRAM, Mapping/Mapping.cc:153-213): the
// reference's dump of its device map, in its byte layout -- four int sizes
// (NumSdfBlocks, NumBuckets, NumVoxels, NumEntries), the heap counter, the
// excess-list counter and the visible count, the free-block stack, the
// bucket locks, every voxel (8 bytes: sdf, weight, rgb), every hash entry,
// the visible-entry list (32-byte HashEntry: int3 pos, ptr as a voxel index,
// offset, padding), then the key-point map (an int lock per key and a
// 288-byte SURF per entry).  This library keeps no key points: it writes
// them unlocked (-1) and zero, and skips them when reading.  A file loads
// into a session whose sizes match the file's.

namespace {

struct RefEntry {
    int32_t x, y, z, ptr, offset, pad[3];
};
static_assert(sizeof(RefEntry) == 32, "the reference's __align__(16) HashEntry");
static_assert(sizeof(Voxel) == 8, "the reference's Voxel");
constexpr size_t kKeyLocks = 100000;    // KeyMap::MaxKeys (Mapping/DeviceMap.h)
constexpr size_t kKeyEntries = 500000;  // KeyMap::maxEntries = MaxKeys * nBuckets
constexpr size_t kSurfBytes = 288;      // sizeof(SURF): bool, float3, float4 (16-aligned), float[64]
constexpr int kFileChunkBlocks = 4096;  // voxel blocks per host staging chunk

struct FileCloser {
    FILE* f;
    ~FileCloser() {
        if (f) std::fclose(f);
    }
};

bool put(FILE* f, const void* p, size_t n) { return std::fwrite(p, 1, n, f) == n; }
bool get(FILE* f, void* p, size_t n) { return std::fread(p, 1, n, f) == n; }

bool put_fill(FILE* f, int32_t value, size_t count) {
    std::vector<int32_t> buf(std::min(count, (size_t)1 << 18), value);
    for (size_t done = 0; done < count;) {
        const size_t k = std::min(buf.size(), count - done);
        if (!put(f, buf.data(), k * 4)) return false;
        done += k;
    }
    return true;
}

bool skip(FILE* f, size_t bytes) {
    std::vector<char> buf(std::min(bytes, (size_t)1 << 22));
    for (size_t done = 0; done < bytes;) {
        const size_t k = std::min(buf.size(), bytes - done);
        if (!get(f, buf.data(), k)) return false;
        done += k;
    }
    return true;
}

RefEntry to_ref(const HEntry& e) {
    RefEntry r{};
    r.x = e.x;
    r.y = e.y;
    r.z = e.z;
    r.ptr = e.ptr >= 0 ? e.ptr * 512 : -1;
    r.offset = e.offset;
    return r;
}

int file_error(const char* what) {
    fb_set_error_text(what);
    return FB_EINVAL;
}

}  // namespace

extern "C" {

int fb_write_map_file(fb_session* s, const char* path) {
    if (!s || !path) return FB_EINVAL;
    const MapView& m = s->map;
    const size_t NE_all = (size_t)m.NB + m.NE;
    if ((size_t)m.NS * 512 > (size_t)INT32_MAX || NE_all > (size_t)INT32_MAX)
        return file_error("fb_write_map_file: the map is too large for the file's int sizes");
    FB_CUDA(cudaStreamSynchronize(s->stream));
    MapCounters c;
    FB_CUDA(cudaMemcpy(&c, s->ctr, sizeof c, cudaMemcpyDeviceToHost));
    FileCloser fc{std::fopen(path, "wb")};
    if (!fc.f) return file_error("fb_write_map_file: cannot open the file");
    FILE* f = fc.f;
    const int32_t head[4] = {m.NS, m.NB, m.NS * 512, (int32_t)NE_all};
    const uint32_t nvis = (uint32_t)std::max(c.n_visible, 0);
    bool ok = put(f, head, sizeof head) && put(f, &c.heap_counter, 4) && put(f, &c.entry_ptr, 4) && put(f, &nvis, 4);
    std::vector<int32_t> heap(m.NS);
    FB_CUDA(cudaMemcpy(heap.data(), m.heap, 4 * heap.size(), cudaMemcpyDeviceToHost));
    ok = ok && put(f, heap.data(), 4 * heap.size()) && put_fill(f, -1, m.NB);   // locks: EntryAvailable
    std::vector<Voxel> vox((size_t)kFileChunkBlocks * 512);
    std::vector<uint8_t> cb(m.cvox ? (size_t)kFileChunkBlocks * kCBlockBytes : 0);
    for (int b0 = 0; ok && b0 < m.NS; b0 += kFileChunkBlocks) {
        const int nb = std::min(kFileChunkBlocks, m.NS - b0);
        if (m.cvox) {
            FB_CUDA(cudaMemcpy(cb.data(), m.cvox + (size_t)b0 * kCBlockBytes, (size_t)nb * kCBlockBytes,
                               cudaMemcpyDeviceToHost));
            for (int b = 0; b < nb; ++b) {
                const uint8_t* blk = cb.data() + (size_t)b * kCBlockBytes;
                for (int v = 0; v < 512; ++v) {
                    uint16_t h;
                    std::memcpy(&h, blk + 2 * v, 2);
                    Voxel& o = vox[(size_t)b * 512 + v];
                    o.sdf = half_bits_to_float(h);
                    o.weight = blk[kCWeight + v];
                    o.r = blk[kCRed + v];
                    o.g = blk[kCGreen + v];
                    o.b = blk[kCBlue + v];
                }
            }
        } else {
            FB_CUDA(cudaMemcpy(vox.data(), m.voxels + (size_t)b0 * 512, (size_t)nb * 512 * sizeof(Voxel),
                               cudaMemcpyDeviceToHost));
        }
        ok = put(f, vox.data(), (size_t)nb * 512 * sizeof(Voxel));
    }
    std::vector<HEntry> ent(NE_all);
    FB_CUDA(cudaMemcpy(ent.data(), m.entries, sizeof(HEntry) * NE_all, cudaMemcpyDeviceToHost));
    std::vector<RefEntry> ref(NE_all);
    for (size_t i = 0; i < NE_all; ++i) ref[i] = to_ref(ent[i]);
    ok = ok && put(f, ref.data(), sizeof(RefEntry) * NE_all);
    // the visible-entry list, the rest of its array zero
    const size_t nv = std::min<size_t>(nvis, (size_t)m.NS);
    std::vector<HEntry> vis(nv);
    if (nv) FB_CUDA(cudaMemcpy(vis.data(), m.vis_blocks, sizeof(HEntry) * nv, cudaMemcpyDeviceToHost));
    std::fill(ref.begin(), ref.end(), RefEntry{});
    for (size_t i = 0; i < nv; ++i) ref[i] = to_ref(vis[i]);
    ok = ok && put(f, ref.data(), sizeof(RefEntry) * NE_all);
    ok = ok && put_fill(f, -1, kKeyLocks) && put_fill(f, 0, kKeyEntries * kSurfBytes / 4);
    if (!ok || std::fflush(f) != 0) return file_error("fb_write_map_file: write failed");
    return FB_OK;
}

int fb_read_map_file(fb_session* s, const char* path) {
    if (!s || !path) return FB_EINVAL;
    const MapView& m = s->map;
    const size_t NE_all = (size_t)m.NB + m.NE;
    FileCloser fc{std::fopen(path, "rb")};
    if (!fc.f) return file_error("fb_read_map_file: cannot open the file");
    FILE* f = fc.f;
    int32_t head[4], hc, ep;
    uint32_t nvis;
    if (!get(f, head, sizeof head) || !get(f, &hc, 4) || !get(f, &ep, 4) || !get(f, &nvis, 4))
        return file_error("fb_read_map_file: truncated header");
    if (head[0] != m.NS || head[1] != m.NB || (int64_t)head[2] != (int64_t)m.NS * 512 || (size_t)head[3] != NE_all)
        return file_error("fb_read_map_file: the file's map sizes differ from the session's");
    std::vector<int32_t> heap(m.NS);
    if (!get(f, heap.data(), 4 * heap.size()) || !skip(f, 4 * (size_t)m.NB))
        return file_error("fb_read_map_file: truncated file");
    for (int32_t v : heap)
        if (v < -1 || v >= m.NS) return file_error("fb_read_map_file: free-block stack out of range");
    // reset first: the per-frame scratch and anything not in the file
    FB_CUDA(cudaStreamSynchronize(s->stream));
    launch_map_reset(s->map, s->stream);
    if (check_launch()) return FB_ECUDA;
    FB_CUDA(cudaStreamSynchronize(s->stream));
    FB_CUDA(cudaMemcpy(m.heap, heap.data(), 4 * heap.size(), cudaMemcpyHostToDevice));
    std::vector<Voxel> vox((size_t)kFileChunkBlocks * 512);
    std::vector<uint8_t> cb(m.cvox ? (size_t)kFileChunkBlocks * kCBlockBytes : 0);
    for (int b0 = 0; b0 < m.NS; b0 += kFileChunkBlocks) {
        const int nb = std::min(kFileChunkBlocks, m.NS - b0);
        if (!get(f, vox.data(), (size_t)nb * 512 * sizeof(Voxel))) return file_error("fb_read_map_file: truncated voxels");
        if (m.cvox) {
            // precision form: TSDF rounded to FP16, weight and colour as stored
            for (int b = 0; b < nb; ++b) {
                uint8_t* blk = cb.data() + (size_t)b * kCBlockBytes;
                for (int v = 0; v < 512; ++v) {
                    const Voxel& x = vox[(size_t)b * 512 + v];
                    const __half h = __float2half_rn(x.sdf);
                    std::memcpy(blk + 2 * v, &h, 2);
                    blk[kCWeight + v] = x.weight;
                    blk[kCRed + v] = x.r;
                    blk[kCGreen + v] = x.g;
                    blk[kCBlue + v] = x.b;
                }
            }
            FB_CUDA(cudaMemcpy(m.cvox + (size_t)b0 * kCBlockBytes, cb.data(), (size_t)nb * kCBlockBytes,
                               cudaMemcpyHostToDevice));
        } else {
            FB_CUDA(cudaMemcpy(m.voxels + (size_t)b0 * 512, vox.data(), (size_t)nb * 512 * sizeof(Voxel),
                               cudaMemcpyHostToDevice));
        }
    }
    std::vector<RefEntry> ref(NE_all);
    if (!get(f, ref.data(), sizeof(RefEntry) * NE_all)) return file_error("fb_read_map_file: truncated hash table");
    std::vector<HEntry> ent(NE_all);
    std::vector<std::pair<int, int>> alloc;   // (block, slot)
    int holes = 0;
    for (size_t i = 0; i < NE_all; ++i) {
        const RefEntry& r = ref[i];
        if (r.ptr != -1 && (r.ptr < 0 || r.ptr % 512 || r.ptr / 512 >= m.NS))
            return file_error("fb_read_map_file: hash entry with a bad voxel pointer");
        if (r.offset > m.NE) return file_error("fb_read_map_file: hash entry with a bad link");
        HEntry& e = ent[i];
        if (r.ptr >= 0) {
            if (r.x < -32767 || r.x > 32767 || r.y < -32767 || r.y > 32767 || r.z < -32767 || r.z > 32767)
                return file_error("fb_read_map_file: block coordinates beyond +-32767");
            e.x = (short)r.x;
            e.y = (short)r.y;
            e.z = (short)r.z;
            alloc.push_back({r.ptr / 512, (int)i});
        } else {
            const bool fits = r.x >= -32767 && r.x <= 32767 && r.y >= -32767 && r.y <= 32767 && r.z >= -32767 &&
                              r.z <= 32767;
            e.x = fits ? (short)r.x : 0;
            e.y = fits ? (short)r.y : 0;
            e.z = fits ? (short)r.z : 0;
            // an empty slot a chain passes through -- a bucket head with a
            // link or a used excess slot -- means the pool ran out once
            const bool linked_head = i < (size_t)m.NB && r.offset > 0;
            const bool used_excess = i >= (size_t)m.NB && i < (size_t)m.NB + (size_t)std::max(0, ep - 1);
            if (linked_head || used_excess) holes = 1;
        }
        e.pad = 0;
        e.ptr = r.ptr >= 0 ? r.ptr / 512 : -1;
        e.offset = std::max(r.offset, 0);   // the reference ends a chain at any offset <= 0
    }
    if (alloc.size() > (size_t)m.NS) return file_error("fb_read_map_file: more allocated entries than blocks");
    FB_CUDA(cudaMemcpy(m.entries, ent.data(), sizeof(HEntry) * NE_all, cudaMemcpyHostToDevice));
    // the allocated list in block order (this library allocates blocks in
    // list order, so its own maps come back in their original order)
    std::sort(alloc.begin(), alloc.end());
    std::vector<int> alloc_slots(alloc.size());
    for (size_t i = 0; i < alloc.size(); ++i) alloc_slots[i] = alloc[i].second;
    if (!alloc_slots.empty())
        FB_CUDA(cudaMemcpy(m.alloc_list, alloc_slots.data(), 4 * alloc_slots.size(), cudaMemcpyHostToDevice));
    // the visible list: the entries' slots found through the hash chains
    if (nvis > NE_all) return file_error("fb_read_map_file: visible count out of range");
    if (!get(f, ref.data(), sizeof(RefEntry) * NE_all)) return file_error("fb_read_map_file: truncated visible list");
    std::vector<int> vis_slots;
    std::vector<HEntry> vis_entries;
    for (uint32_t i = 0; i < nvis && vis_slots.size() < (size_t)m.NS; ++i) {
        const RefEntry& r = ref[i];
        size_t b = bucket_of(r.x, r.y, r.z, (uint32_t)m.NB);
        for (int guard = 0; guard <= m.NE; ++guard) {
            const HEntry& e = ent[b];
            if (e.ptr >= 0 && e.x == r.x && e.y == r.y && e.z == r.z) {
                vis_slots.push_back((int)b);
                vis_entries.push_back(e);
                break;
            }
            if (e.offset <= 0) break;
            b = (size_t)m.NB + e.offset - 1;
        }
    }
    if (!vis_slots.empty()) {
        FB_CUDA(cudaMemcpy(m.visible, vis_slots.data(), 4 * vis_slots.size(), cudaMemcpyHostToDevice));
        FB_CUDA(cudaMemcpy(m.vis_blocks, vis_entries.data(), sizeof(HEntry) * vis_entries.size(),
                           cudaMemcpyHostToDevice));
    }
    if (!skip(f, 4 * kKeyLocks + kKeyEntries * kSurfBytes)) return file_error("fb_read_map_file: truncated key map");
    MapCounters c;
    FB_CUDA(cudaMemcpy(&c, s->ctr, sizeof c, cudaMemcpyDeviceToHost));
    c.heap_counter = hc;
    c.entry_ptr = ep;
    c.holes = holes;
    c.n_alloc = (int)alloc_slots.size();
    c.n_visible = (int)vis_slots.size();
    c.err = 0;
    FB_CUDA(cudaMemcpy(s->ctr, &c, sizeof c, cudaMemcpyHostToDevice));
    // System::ReadMapFromDisk: the tracker restarts and the map is no longer fused
    s->state = s->last_state = 1;
    if (!s->mapping_disabled) drop_graphs(s);
    s->mapping_disabled = true;
    return FB_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ batches

struct fb_batch {
    cudaStream_t origin = nullptr;
    bool own_origin = false;
    int mode = 0;
    cudaEvent_t fork = nullptr;
    std::vector<cudaStream_t> slots;
    std::vector<cudaEvent_t> done;
    // mode 1: one graph per composition
    std::map<std::vector<uint64_t>, std::pair<cudaGraphExec_t, int>> cache;
    uint64_t steps = 0, captures = 0;
};

namespace {

constexpr size_t kBatchCacheMax = 32;

void clear_cache(fb_batch* b) {
    for (auto& kv : b->cache) cudaGraphExecDestroy(kv.second.first);
    b->cache.clear();
}

// Slot streams of a batch: a fixed set, created with the batch.  Creating a
// stream while frames run can take tens of milliseconds (the driver
// serialises it with the device's work), so a step never creates one; beyond
// kBatchSlots sessions, sessions share slots round-robin (their frames then
// run one after the other on that slot, with the same results).
constexpr int kBatchSlots = 32;
// Steps of at most this many sessions run each frame as a session alone
// (served p50 at 64 clients on B200: 2.50 ms with 1, 2.25 with 2, 1.67 with 3).
constexpr int kBatchSharedMin = 3;

int ensure_slots(fb_batch* b, int n) {
    while ((int)b->slots.size() < n) {
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        FB_CUDA(cudaStreamCreate(&st));
        if (!cuda_ok(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming))) {
            cudaStreamDestroy(st);
            return FB_ECUDA;
        }
        b->slots.push_back(st);
        b->done.push_back(ev);
    }
    return FB_OK;
}

// The frames of a step on the slot streams (session i on slot i mod
// kBatchSlots), forked from and joined back into the origin stream.  With
// capture on, the same calls record one graph.  direct: launch each session's
// cached frame graph (mode 0), else issue its kernels (captured into the
// composite graph, mode 1).
int issue_step(fb_batch* b, fb_session* const* ss, int n, const FramePlan* plans, bool direct, int* kernels) {
    FB_CUDA(cudaEventRecord(b->fork, b->origin));
    *kernels = 0;
    const int used = std::min(n, kBatchSlots);
    for (int k = 0; k < used; ++k) FB_CUDA(cudaStreamWaitEvent(b->slots[k], b->fork, 0));
    for (int i = 0; i < n; ++i) {
        fb_session* s = ss[i];
        cudaStream_t st = b->slots[i % kBatchSlots];
        if (direct) {
            unsigned ran = 0;
            int rc = enqueue_frame(s, plans[i], st, &ran);
            if (rc) return rc;
        } else {
            unsigned ran = 0;
            cudaStream_t keep = s->stream;
            s->stream = st;
            *kernels += issue_frame(s, plans[i].track, plans[i].fuse, plans[i].render, plans[i].init, &ran);
            s->stream = keep;
        }
        FB_CUDA(cudaMemcpyAsync(s->h_out, s->d_out, sizeof(FrameOut), cudaMemcpyDeviceToHost, st));
    }
    for (int k = 0; k < used; ++k) {
        FB_CUDA(cudaEventRecord(b->done[k], b->slots[k]));
        FB_CUDA(cudaStreamWaitEvent(b->origin, b->done[k], 0));
    }
    return check_launch();
}

}  // namespace

extern "C" {

int fb_batch_create(void* stream, fb_batch** out) {
    if (!out) return FB_EINVAL;
    fb_batch* b = new (std::nothrow) fb_batch();
    if (!b) return FB_ENOMEM;
    b->origin = (cudaStream_t)stream;
    if (!b->origin) {
        if (!cuda_ok(cudaStreamCreate(&b->origin))) {
            delete b;
            return FB_ECUDA;
        }
        b->own_origin = true;
    }
    if (!cuda_ok(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming))) {
        if (b->own_origin) cudaStreamDestroy(b->origin);
        delete b;
        return FB_ECUDA;
    }
    if (ensure_slots(b, kBatchSlots) != FB_OK) {
        fb_batch_destroy(b);
        return FB_ECUDA;
    }
    // sessions come and go beside running ones: keep the memory of destroyed
    // sessions in the device's default pool for the next ones
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    *out = b;
    return FB_OK;
}

int fb_batch_destroy(fb_batch* b) {
    if (!b) return FB_EINVAL;
    cudaStreamSynchronize(b->origin);
    clear_cache(b);
    for (size_t i = 0; i < b->slots.size(); ++i) {
        cudaStreamSynchronize(b->slots[i]);
        cudaStreamDestroy(b->slots[i]);
        cudaEventDestroy(b->done[i]);
    }
    cudaEventDestroy(b->fork);
    if (b->own_origin) cudaStreamDestroy(b->origin);
    delete b;
    return FB_OK;
}

int fb_batch_reserve(fb_batch* b, size_t bytes) {
    if (!b) return FB_EINVAL;
    if (!bytes) return FB_OK;
    void* p = nullptr;
    FB_CUDA(cudaMallocAsync(&p, bytes, b->origin));
    FB_CUDA(cudaFreeAsync(p, b->origin));
    FB_CUDA(cudaStreamSynchronize(b->origin));
    return FB_OK;
}

int fb_batch_set_mode(fb_batch* b, int mode) {
    if (!b || mode < 0 || mode > 1) return FB_EINVAL;
    b->mode = mode;
    return FB_OK;
}

int fb_batch_stats(fb_batch* b, uint64_t* steps, uint64_t* captures) {
    if (!b) return FB_EINVAL;
    if (steps) *steps = b->steps;
    if (captures) *captures = b->captures;
    return FB_OK;
}

int fb_batch_step(fb_batch* b, fb_session* const* ss, int n, const fb_frame_input* in, fb_frame_result* out) {
    if (!b || !ss || !in || n <= 0) return FB_EINVAL;
    for (int i = 0; i < n; ++i) {
        if (!ss[i] || !in[i].depth || !in[i].rgb || ss[i]->keys) return FB_EINVAL;
        if (in[i].depth_pitch < (size_t)ss[i]->W[0] * 2 || in[i].rgb_pitch < (size_t)ss[i]->W[0] * 3)
            return FB_EINVAL;
        for (int j = 0; j < i; ++j)
            if (ss[j] == ss[i]) return FB_EINVAL;
    }
    int rc = FB_OK;
    // inputs first (on the origin stream; the frames fork after them)
    for (int i = 0; i < n; ++i) {
        rc = copy_frame_in(ss[i], in[i].depth, in[i].depth_pitch, in[i].rgb, in[i].rgb_pitch, in[i].on_device,
                           b->origin);
        if (rc) return rc;
    }
    // sessions of a step of more than kBatchSharedMin sessions run the
    // tracking forms that leave room for the other sessions' frames (their
    // frame graphs are the ones fb_session_prepare(s, 1) captures); smaller
    // steps run the forms of a session alone (fb_session_prepare(s, 0)),
    // which finish sooner.  Both give the same results.
    const bool shared = n > kBatchSharedMin;
    for (int i = 0; i < n; ++i) ss[i]->shared_gpu = shared;
    std::vector<FramePlan> plans(n);
    for (int i = 0; i < n; ++i) plans[i] = plan_frame(ss[i]);
    if (b->mode == 1) {
        std::vector<uint64_t> key;
        key.reserve(2 * n);
        for (int i = 0; i < n; ++i) {
            const fb_session* s = ss[i];
            key.push_back((uint64_t)(uintptr_t)s);
            key.push_back((uint64_t)plans[i].mode | (uint64_t)plans[i].fuse << 2 | (uint64_t)s->next << 3 |
                          (uint64_t)s->persistent << 4 | (uint64_t)s->shared_gpu << 5 |
                          (uint64_t)s->mapping_disabled << 6 | (uint64_t)s->rc_bx << 8 |
                          (uint64_t)s->rc_by << 20);
        }
        auto it = b->cache.find(key);
        if (it == b->cache.end()) {
            if (b->cache.size() >= kBatchCacheMax) clear_cache(b);
            cudaGraph_t graph = nullptr;
            cudaGraphExec_t exec = nullptr;
            int kernels = 0;
            FB_CUDA(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
            rc = issue_step(b, ss, n, plans.data(), false, &kernels);
            cudaError_t e = cudaStreamEndCapture(b->origin, &graph);
            if (rc == FB_OK && e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (rc) return rc;
            FB_CUDA(e);
            it = b->cache.emplace(key, std::make_pair(exec, kernels)).first;
            b->captures++;
        }
        FB_CUDA(cudaGraphLaunch(it->second.first, b->origin));
        // kernels per session are not separated in a composite graph: count
        // them on the first session
        ss[0]->launches += (uint64_t)it->second.second;
    } else {
        int kernels = 0;
        rc = issue_step(b, ss, n, plans.data(), true, &kernels);
        if (rc) return rc;
    }
    FB_CUDA(cudaStreamSynchronize(b->origin));
    for (int i = 0; i < n; ++i) {
        finish_frame(ss[i], plans[i], out ? &out[i] : nullptr);
        ss[i]->shared_gpu = false;
    }
    b->steps++;
    return FB_OK;
}

}  // extern "C"
