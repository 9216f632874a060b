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

#include "session_internal.h"

using namespace fb;

namespace fb {

thread_local char g_last_error[256] = "";

bool cuda_ok(cudaError_t e) {
    if (e == cudaSuccess) return true;
    snprintf(g_last_error, sizeof g_last_error, "%s", cudaGetErrorString(e));
    return false;
}

// Kernels launched through the launchers report errors here.
int check_launch() {
    cudaError_t e = cudaGetLastError();
    return cuda_ok(e) ? FB_OK : FB_ECUDA;
}

}  // namespace fb

namespace {








__device__ __forceinline__ void init_poses_body(const BlockCtx&, TrackState* st) {
    for (int i = 0; i < 16; ++i) st->pose[i] = st->last_pose[i] = st->init_pose[i] = (i % 5 == 0) ? 1.0 : 0.0;
    st->cur = make_dev_pose_d(st->pose);
    st->last = st->cur;
    st->failed = 0;
    st->icp_error = st->rgb_error = qnan();
    st->icp_count = st->rgb_count = 0;
}
__global__ void k_init_poses(TrackState* st) { init_poses_body(own_ctx(), st); }
FB_FUSED_KERNEL(k_init_poses, init_poses_body, 32)

// After the frame: a tracked frame becomes the last frame (SwapFrame).
__device__ __forceinline__ void commit_body(const BlockCtx&, TrackState* st, MapCounters* c, FrameOut* out,
                                            int tracked_path) {
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
__global__ void k_commit(TrackState* st, MapCounters* c, FrameOut* out, int tracked_path) {
    commit_body(own_ctx(), st, c, out, tracked_path);
}
FB_FUSED_KERNEL(k_commit, commit_body, 32)

// The frame result into the caller's pinned host memory (device-accessible
// through unified addressing): the fused batch step reads every session's
// result this way instead of one copy per session.
__device__ __forceinline__ void result_out_body(const BlockCtx&, const FrameOut* d, FrameOut* h) {
    static_assert(sizeof(FrameOut) % 4 == 0, "FrameOut is copied in words");
    const int n = (int)(sizeof(FrameOut) / 4);
    for (int i = threadIdx.x; i < n; i += blockDim.x) ((int*)h)[i] = ((const int*)d)[i];
}
__global__ void k_result_out(const FrameOut* d, FrameOut* h) { result_out_body(own_ctx(), d, h); }
FB_FUSED_KERNEL(k_result_out, result_out_body, 64)


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


__device__ __forceinline__ void track_start_body(const BlockCtx&, TrackState* st, Pose16 T) {
    for (int i = 0; i < 16; ++i) st->pose[i] = st->init_pose[i] = T.m[i];
    st->cur = make_dev_pose_d(st->pose);
}
__global__ void k_track_start(TrackState* st, Pose16 T) { track_start_body(own_ctx(), st, T); }
FB_FUSED_KERNEL(k_track_start, track_start_body, 32)

// A relocalised frame: its pose is the solver's, and it becomes the last frame.
__global__ void k_track_reloc(TrackState* st, Pose16 T) {
    for (int i = 0; i < 16; ++i) st->pose[i] = st->last_pose[i] = st->init_pose[i] = T.m[i];
    st->cur = st->last = make_dev_pose_d(st->pose);
    st->failed = 0;
}

}  // namespace

void fb_set_error_text(const char* msg) { snprintf(g_last_error, sizeof g_last_error, "%s", msg); }

namespace fb {


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
         dalloc(s, &s->tickets, 4) &&
         dalloc(s, &s->residual, track_list_capacity(s->W[0] * s->H[0])) &&
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
        m.rc_cap = raycast_tile_cap(cfg->width, cfg->height);
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
             dalloc(s, &m.zmax, (size_t)m.zc * m.zr) && dalloc(s, &m.frec, (size_t)64 * m.zc * m.zr) &&
             dalloc(s, &m.fcol, (size_t)64 * m.zc * m.zr) && dalloc(s, &m.rc_cost, (size_t)m.rc_cap) &&
             dalloc(s, &m.rc_order, (size_t)m.rc_cap + 1);
        s->ctr = m.ctr;
    }
    return ok;
}

int reset_session(fb_session* s) {
    launch_map_reset(s->map, s->stream);
    k_init_poses<<<1, 1, 0, s->stream>>>(s->st);
    FB_CUDA(cudaMemsetAsync(s->tickets, 0, 4 * sizeof(unsigned), s->stream));
    FB_CUDA(cudaMemsetAsync(s->map.rc_cost, 0, (size_t)s->map.rc_cap * sizeof(uint32_t), s->stream));
    FB_CUDA(cudaMemsetAsync(s->map.rc_order, 0, sizeof(int), s->stream));   // no order yet: blocks in grid order
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




// The frame's kernels after the input has reached fr[next].  Returns the
// number of kernels launched and which stages ran (bit k = stage k).
// part 0: the whole frame; 1: ResizeImages + FillImages only; 2: the rest.
// start: the tracker's starting pose when not the last pose.
int issue_frame(fb_session* s, bool track, bool fuse, bool render, bool init, unsigned* ran, int part,
                const double* start) {
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
        // Tracker::GrabFrame (Tracking.cc:236-243): LastFrame->ResizeImages and
        // NextFrame->FillImages (Core/Frame.cc:59-84) in four launches whose
        // roles do not depend on each other: {level 0, resize 0 -> 1},
        // {pyrdown 0 -> 1, maps 0, resize 1 -> 2}, {pyrdown 1 -> 2, maps 1},
        // {maps 2} (the resize's time is counted in the pyramid's)
        mark(0);
        *ran |= 1u << 0;
        mark(1);
        launch_slot(kSlotPyramid);
        auto maps = [&](PreLaunch& P, int l) {
            // level 0 also makes the frame's fusion records
            FuseRecDst fr{N.raw,          s->W[0],      N.rgb, 3 * s->W[0], c.depth_min, c.depth_max, s->map.frec,
                          s->map.fcol, s->map.cvox ? 1 : 0};
            pre_maps(P, N.depth[l], s->W[l], N.gray[l], s->W[l], s->W[l], s->H[l], s->K[l], c.depth_cutoff, N.vmap[l],
                     s->W[l], N.nmap[l], s->W[l], N.dx[l], N.dy[l], s->W[l], N.rgbok[l], l == 0 ? &fr : nullptr);
        };
        auto resize = [&](PreLaunch& P, int l) {
            pre_resize(P, L.vmap[l - 1], L.nmap[l - 1], s->W[l - 1], s->W[l - 1], s->H[l - 1], L.vmap[l], L.nmap[l],
                       s->W[l]);
        };
        auto pyrdown = [&](PreLaunch& P, int l) {
            pre_pyrdown(P, N.depth[l - 1], s->W[l - 1], N.gray[l - 1], s->W[l - 1], s->W[l - 1], s->H[l - 1],
                        N.depth[l], s->W[l], N.gray[l], s->W[l]);
        };
        {
            PreLaunch P{};
            pre_level0(P, N.depth_in, s->W[0], N.rgb, 3 * s->W[0], s->W[0], s->H[0], c.depth_scale, c.depth_cutoff,
                       N.raw, s->W[0], N.depth[0], s->W[0], N.gray[0], s->W[0]);
            resize(P, 1);
            n += launch_pre(P, st);
        }
        {
            PreLaunch P{};
            pyrdown(P, 1);
            maps(P, 0);
            resize(P, 2);
            n += launch_pre(P, st);
        }
        {
            PreLaunch P{};
            pyrdown(P, 2);
            maps(P, 1);
            n += launch_pre(P, st);
        }
        {
            PreLaunch P{};
            maps(P, 2);
            n += launch_pre(P, st);
        }
        *ran |= 1u << 1;
        if (part == 1) return n;
    }
    mark(2);
    const int* skip = nullptr;
    launch_slot(kSlotTrackInit);
    if (init) {
        fb_launch(k_init_poses, (const void*)k_init_poses_fused, 1, 1, 0, st, s->st);
        n += 1;
    } else if (track) {
        // Tracker::ComputeSE3 (Tracking.cc:296-409)
        static const int min_count[3] = {2000, 1000, 100};   // MIN_ICP_COUNT, Tracking.h:102
        n += launch_track_begin(s->st, st);
        if (start) {
            Pose16 T;
            std::memcpy(T.m, start, sizeof T.m);
            fb_launch(k_track_start, (const void*)k_track_start_fused, 1, 1, 0, st, s->st, T);
            n += 1;
        }
        int last_level = -1;
        for (int l = 2; l >= 0; --l)
            if (c.iters[l] > 0) last_level = l;
        for (int l = 2; l >= 0; --l) {
            TrackLevel lv = level_view(s, l);
            for (int it = 0; it < c.iters[l]; ++it) {
                launch_slot(kSlotTrack, 2 - l, it);
                n += launch_track_iter(lv, s->st, s->tickets, s->residual, s->counts, min_count[l],
                                       l == last_level && it == c.iters[l] - 1, st, s->shared_gpu,
                                       c.form == FB_FORM_PRECISION);
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
        launch_slot(kSlotAllocate);
        n += launch_allocate(s->map, N.raw, s->W[0], s->W[0], s->H[0], s->K[0], pose, skip, st);
        mark(4);
        launch_slot(kSlotVisibility);
        n += launch_visibility(s->map, s->W[0], s->H[0], s->K[0], pose, skip, st, true);
        mark(5);
        launch_slot(kSlotIntegrate);
        n += launch_integrate(s->map, s->W[0], s->H[0], s->K[0], pose, skip, st, s->integ_cps);
        *ran |= 7u << 3;
    } else {
        mark(4);
        mark(5);
    }
    mark(6);
    if (render) {
        // with mapping disabled, System::GrabImage refreshes the visible
        // blocks first (Mapping::UpdateVisibility, System.cc:116-118)
        if (!fuse && s->mapping_disabled) {
            launch_slot(kSlotRenderVisibility);
            n += launch_visibility(s->map, s->W[0], s->H[0], s->K[0], pose, skip, st);
        }
        // Mapping::RayTrace (Mapping.cc:92-109) into the frame's level-0 maps
        launch_slot(kSlotZRange);
        n += launch_zrange(s->map, s->K[0], pose, skip, st, raycast_tiles(s->W[0], s->H[0], s->rc_bx, s->rc_by));
        mark(7);
        launch_slot(kSlotRaycast);
        n += launch_raycast(s->map, N.vmap[0], N.nmap[0], s->W[0], s->W[0], s->H[0], s->K[0], pose, skip, st,
                            s->rc_bx, s->rc_by);
        *ran |= 3u << 6;
    } else {
        mark(7);
    }
    mark(8);
    launch_slot(kSlotCommit);
    launch_commit(s, track || init, st);
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

void unpack_sums(const double* s, double* A, double* b) {
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


int read_counters(fb_session* s, MapCounters* c) {
    FB_CUDA(cudaMemcpyAsync(c, s->ctr, sizeof *c, cudaMemcpyDeviceToHost, s->stream));
    FB_CUDA(cudaStreamSynchronize(s->stream));
    return FB_OK;
}

void launch_track_reloc(fb_session* s, const double* T, cudaStream_t st) {
    Pose16 P;
    std::memcpy(P.m, T, sizeof P.m);
    k_track_reloc<<<1, 1, 0, st>>>(s->st, P);
}

LaunchRecorder*& launch_recorder() {
    static thread_local LaunchRecorder* r = nullptr;
    return r;
}

void launch_result_out(fb_session* s, cudaStream_t st) {
    fb_launch(k_result_out, (const void*)k_result_out_fused, 1, 64, 0, st, s->d_out, s->h_out_dev);
}

void launch_commit(fb_session* s, int tracked_path, cudaStream_t st) {
    fb_launch(k_commit, (const void*)k_commit_fused, 1, 1, 0, st, s->st, s->ctr, s->d_out, tracked_path);
}

}  // namespace fb

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
    return ExecKey(dev, s->W[0], s->H[0], s->cfg.form, mode, fuse, shared, s->integ_cps, s->rc_bx, s->rc_by,
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

}  // namespace

namespace fb {

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

}  // namespace fb

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
    s->h_out_dev = nullptr;
    s->profile = false;
    for (int i = 0; i <= kStages; ++i) s->ev[i] = nullptr;
    for (int i = 0; i < kStages; ++i) {
        s->stage_ms[i] = 0;
        s->stage_calls[i] = 0;
    }
    s->launches = 0;
    s->use_graphs = true;
    s->rc_bx = 16;
    s->rc_by = 8;
    s->integ_cps = 0;
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
        // the device address of the pinned result (fused batch steps write it
        // from a kernel); without one the session cannot take fused steps
        if (ok && cudaHostGetDevicePointer((void**)&s->h_out_dev, s->h_out, 0) != cudaSuccess) {
            s->h_out_dev = nullptr;
            cudaGetLastError();
        }
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

int fb_session_set_integration_grid(fb_session* s, int ctas_per_sm) {
    if (!s || ctas_per_sm < 0 || ctas_per_sm > 32) return FB_EINVAL;
    if (ctas_per_sm == s->integ_cps) return FB_OK;
    drop_graphs(s);
    s->integ_cps = ctas_per_sm;
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
                tmp[v].weight = cb[c_weight(v)];
                tmp[v].r = cb[c_red(v)];
                tmp[v].g = cb[c_green(v)];
                tmp[v].b = cb[c_blue(v)];
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

}  // extern "C"
