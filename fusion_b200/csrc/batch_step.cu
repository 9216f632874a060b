// Batched steps (fb_batch_*): one frame of each of n independent sessions
// with all frames in flight together -- each session's cached frame graph on
// its own stream of the batch (mode 0), one composite graph per composition
// (mode 1), or fused launches (mode 2): every stage kernel runs once for all
// sessions of the step, as one launch whose grid is the concatenation of the
// sessions' grids (fb_fused.cuh), captured as one graph per composition.
#include <algorithm>
#include <cstring>
#include <tuple>
#include <map>
#include <new>
#include <vector>

#include "session_internal.h"

// ------------------------------------------------------------------ batches

// One merged launch of a fused step: the fused kernel over n parts (one per
// session that issued this launch, at most kFusedMaxParts), with its
// parameter (FusedParams: parts and argument tuples) at a byte offset of the
// plan's parameter bytes.
struct FusedLaunch {
    const void* fused;
    dim3 block;
    size_t smem;
    int n, blocks;
    int lane;               // the stream (lane) it runs on
    size_t param_off;
};

// The fused launches of one composition, their parameters and, once the
// composition repeats, their graph.
struct FusedPlan {
    std::vector<unsigned char> params;
    int lanes = 1;
    std::vector<FusedLaunch> launches;
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;      // per-session kernel launches the merged ones replace
    uint64_t uses = 0;
};

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
    // mode 2: fused plans by composition, the recorders of a step's frames
    std::map<std::vector<uint64_t>, FusedPlan> fused;
    std::vector<LaunchRecorder> recs;
    int lanes = 4;
    // the step in flight between fb_batch_submit and fb_batch_collect
    bool pending = false;
    std::vector<fb_session*> pend_ss;
    std::vector<FramePlan> pend_plans;
    cudaEvent_t pend_done = nullptr;                             // fb_batch_set_lanes
    int last_launches = 0, last_kernels = 0;   // of the last fused step
};

namespace {

constexpr size_t kBatchCacheMax = 32;

void clear_cache(fb_batch* b) {
    for (auto& kv : b->cache) cudaGraphExecDestroy(kv.second.first);
    b->cache.clear();
}

constexpr size_t kFusedCacheMax = 64;

// Slot streams of a batch: a fixed set, created with the batch.  Creating a
// stream while frames run can take tens of milliseconds (the driver
// serialises it with the device's work), so a step never creates one; beyond
// kBatchSlots sessions, sessions share slots round-robin (their frames then
// run one after the other on that slot, with the same results).  Fused steps
// use the first slots as their lanes.
constexpr int kBatchSlots = 32;

void clear_fused(fb_batch* b) {
    if (b->fused.empty()) return;
    cudaStreamSynchronize(b->origin);
    for (auto& kv : b->fused)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    b->fused.clear();
}

// The composition of a step: each session with what decides its launches
// (tracker mode, fusion, frame parity, map form options, raycast tile).
std::vector<uint64_t> composition(fb_session* const* ss, int n, const FramePlan* plans) {
    std::vector<uint64_t> key;
    key.reserve(2 * n);
    for (int i = 0; i < n; ++i) {
        const fb_session* s = ss[i];
        key.push_back((uint64_t)(uintptr_t)s);
        key.push_back((uint64_t)plans[i].mode | (uint64_t)plans[i].fuse << 2 | (uint64_t)s->next << 3 |
                      (uint64_t)s->shared_gpu << 5 | (uint64_t)s->mapping_disabled << 6 |
                      (uint64_t)s->rc_bx << 8 | (uint64_t)s->rc_by << 20 | (uint64_t)s->integ_cps << 32);
    }
    return key;
}

// Lanes of a fused step: the sessions split into `lanes` groups of about
// equal pixel counts (largest first into the lightest lane).  Each lane's
// fused launches run on a stream of their own, so one lane's latency-bound
// tracking overlaps another lane's raycast or integration.
std::vector<int> assign_lanes(fb_session* const* ss, int n, int lanes) {
    std::vector<int> order(n), lane(n, 0);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int c) { return ss[a]->W[0] * ss[a]->H[0] > ss[c]->W[0] * ss[c]->H[0]; });
    std::vector<long long> load(lanes, 0);
    for (int i : order) {
        int best = 0;
        for (int l = 1; l < lanes; ++l)
            if (load[l] < load[best]) best = l;
        lane[i] = best;
        load[best] += (long long)ss[i]->W[0] * ss[i]->H[0];
    }
    return lane;
}

// Records every session's frame (and its result read-back), merges the
// launches of the same lane, slot and kernel across sessions (up to
// kFusedMaxParts sessions per launch), and lays out each merged launch's
// parameter.
int build_fused(fb_batch* b, fb_session* const* ss, int n, const FramePlan* plans, FusedPlan& out) {
    if ((int)b->recs.size() < n) b->recs.resize(n);
    int kernels = 0;
    for (int i = 0; i < n; ++i)
        if (!ss[i]->h_out_dev) {
            fb_set_error_text("fused batch step: a session's pinned result has no device address");
            return FB_ECUDA;
        }
    for (int i = 0; i < n; ++i) {
        fb_session* s = ss[i];
        LaunchRecorder& r = b->recs[i];
        r.clear();
        const bool prof = s->profile;
        s->profile = false;   // no stage events inside fused launches
        launch_recorder() = &r;
        unsigned ran = 0;
        const int issued = issue_frame(s, plans[i].track, plans[i].fuse, plans[i].render, plans[i].init, &ran);
        launch_slot(kSlotOut);
        launch_result_out(s, b->origin);
        launch_recorder() = nullptr;
        s->profile = prof;
        // every kernel of the frame went through the recorder, in slot order
        if ((int)r.recs.size() != issued + 1) {
            fb_set_error_text("fused batch step: a frame kernel was not recorded");
            return FB_ECUDA;
        }
        for (size_t k = 1; k < r.recs.size(); ++k)
            if (r.recs[k].slot <= r.recs[k - 1].slot) {
                fb_set_error_text("fused batch step: frame launches out of slot order");
                return FB_ECUDA;
            }
        kernels += (int)r.recs.size();
    }
    // (lane, slot, kernel, block shape, shared memory, session): launches of
    // one lane, slot and kernel merge; the sessions' parts keep session order
    const std::vector<int> lane = assign_lanes(ss, n, out.lanes);
    using Ent = std::tuple<int, uint64_t, uintptr_t, unsigned, unsigned, size_t, int, int>;
    std::vector<Ent> ents;
    ents.reserve((size_t)kernels);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < (int)b->recs[i].recs.size(); ++k) {
            const LaunchRec& r = b->recs[i].recs[k];
            if (r.grid.z != 1 || r.block.z != 1) {
                fb_set_error_text("fused batch step: 3-D grid");
                return FB_ECUDA;
            }
            ents.emplace_back(lane[i], r.slot, (uintptr_t)r.fused, r.block.x, r.block.y, r.smem, i, k);
        }
    std::sort(ents.begin(), ents.end());
    std::vector<FusedLaunch> launches;
    std::vector<std::pair<size_t, size_t>> groups;   // [first, last) in ents
    size_t bytes = 0;
    for (size_t e = 0; e < ents.size();) {
        size_t f = e + 1;
        while (f < ents.size() && f - e < (size_t)kFusedMaxParts && std::get<0>(ents[f]) == std::get<0>(ents[e]) &&
               std::get<1>(ents[f]) == std::get<1>(ents[e]) && std::get<2>(ents[f]) == std::get<2>(ents[e]) &&
               std::get<3>(ents[f]) == std::get<3>(ents[e]) && std::get<4>(ents[f]) == std::get<4>(ents[e]) &&
               std::get<5>(ents[f]) == std::get<5>(ents[e]))
            ++f;
        const LaunchRec& r0 = b->recs[std::get<6>(ents[e])].recs[std::get<7>(ents[e])];
        FusedLaunch L;
        L.fused = r0.fused;
        L.block = r0.block;
        L.smem = r0.smem;
        L.n = (int)(f - e);
        L.lane = std::get<0>(ents[e]);
        L.blocks = 0;
        L.param_off = bytes;
        bytes += fused_param_bytes(r0.size);
        launches.push_back(L);
        groups.emplace_back(e, f);
        e = f;
    }
    out.params.assign(bytes, 0);
    for (size_t g = 0; g < launches.size(); ++g) {
        FusedLaunch& L = launches[g];
        unsigned char* prm = out.params.data() + L.param_off;
        FusedPart* parts = (FusedPart*)prm;
        size_t size0 = 0;
        for (size_t e = groups[g].first; e < groups[g].second; ++e) {
            const LaunchRec& r = b->recs[std::get<6>(ents[e])].recs[std::get<7>(ents[e])];
            if (e == groups[g].first) size0 = r.size;
            if (r.size != size0) {
                fb_set_error_text("fused batch step: argument tuples of one kernel differ in size");
                return FB_ECUDA;
            }
            const int j = (int)(e - groups[g].first);
            const long long nb = (long long)r.grid.x * r.grid.y;
            if (nb <= 0 || L.blocks + nb > 0x7fffffffLL) {
                fb_set_error_text("fused batch step: grid too large");
                return FB_ECUDA;
            }
            parts[j] = FusedPart{L.blocks, (int)r.grid.x, (int)r.grid.y, 0};
            L.blocks += (int)nb;
            const unsigned char* src = b->recs[std::get<6>(ents[e])].bytes.data() + r.off;
            std::memcpy(prm + kFusedArgsOffset + (size_t)j * r.size, src, r.size);
        }
        std::memcpy(prm + kFusedNOffset, &L.n, sizeof(int));
    }
    out.launches = std::move(launches);
    out.kernels = kernels;
    return FB_OK;
}

// The plan's launches: lane l on slot stream l, forked from and joined back
// into the origin stream (one lane: on the origin stream itself).
int launch_fused(fb_batch* b, const FusedPlan& p) {
    const bool fork = p.lanes > 1;
    if (fork) {
        FB_CUDA(cudaEventRecord(b->fork, b->origin));
        for (int l = 0; l < p.lanes; ++l) FB_CUDA(cudaStreamWaitEvent(b->slots[l], b->fork, 0));
    }
    for (const FusedLaunch& L : p.launches) {
        void* kargs[] = {(void*)(p.params.data() + L.param_off)};
        cudaStream_t st = fork ? b->slots[L.lane] : b->origin;
        FB_CUDA(cudaLaunchKernel(L.fused, dim3((unsigned)L.blocks), L.block, kargs, L.smem, st));
    }
    if (fork)
        for (int l = 0; l < p.lanes; ++l) {
            FB_CUDA(cudaEventRecord(b->done[l], b->slots[l]));
            FB_CUDA(cudaStreamWaitEvent(b->origin, b->done[l], 0));
        }
    return FB_OK;
}

// One fused step: the plan of this composition (built on first sight), its
// graph from the second use on (a composition seen once is launched
// directly: no instantiation for one-off mixes of the served form).
int fused_step(fb_batch* b, fb_session* const* ss, int n, const FramePlan* plans) {
    std::vector<uint64_t> key = composition(ss, n, plans);
    const int lanes = std::max(1, std::min(std::min(b->lanes, n), kBatchSlots));
    key.push_back((uint64_t)lanes);
    auto it = b->fused.find(key);
    if (it == b->fused.end()) {
        if (b->fused.size() >= kFusedCacheMax) clear_fused(b);
        FusedPlan p;
        p.lanes = lanes;
        if (int rc = build_fused(b, ss, n, plans, p)) return rc;
        it = b->fused.emplace(std::move(key), std::move(p)).first;
    }
    FusedPlan& p = it->second;
    if (p.uses > 0 && !p.exec) {
        cudaGraph_t graph = nullptr;
        FB_CUDA(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
        int rc = launch_fused(b, p);
        cudaError_t e = cudaStreamEndCapture(b->origin, &graph);
        if (rc == FB_OK && e == cudaSuccess) e = cudaGraphInstantiate(&p.exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (rc) return rc;
        FB_CUDA(e);
        b->captures++;
    }
    if (p.exec)
        FB_CUDA(cudaGraphLaunch(p.exec, b->origin));
    else if (int rc = launch_fused(b, p))
        return rc;
    p.uses++;
    b->last_launches = (int)p.launches.size();
    b->last_kernels = p.kernels;
    ss[0]->launches += (uint64_t)p.launches.size();
    return check_launch();
}


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
    if (b->pend_done) cudaEventDestroy(b->pend_done);
    clear_cache(b);
    clear_fused(b);
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
    if (!b || mode < 0 || mode > 2) return FB_EINVAL;
    b->mode = mode;
    return FB_OK;
}

int fb_batch_set_lanes(fb_batch* b, int lanes) {
    if (!b || lanes < 1 || lanes > kBatchSlots) return FB_EINVAL;
    b->lanes = lanes;
    return FB_OK;
}

int fb_batch_launch_stats(fb_batch* b, int* launches, int* kernels) {
    if (!b) return FB_EINVAL;
    if (launches) *launches = b->last_launches;
    if (kernels) *kernels = b->last_kernels;
    return FB_OK;
}

int fb_batch_stats(fb_batch* b, uint64_t* steps, uint64_t* captures) {
    if (!b) return FB_EINVAL;
    if (steps) *steps = b->steps;
    if (captures) *captures = b->captures;
    return FB_OK;
}

int fb_batch_step(fb_batch* b, fb_session* const* ss, int n, const fb_frame_input* in, fb_frame_result* out) {
    int rc = fb_batch_submit(b, ss, n, in);
    if (rc) return rc;
    return fb_batch_collect(b, out);
}

int fb_batch_submit(fb_batch* b, fb_session* const* ss, int n, const fb_frame_input* in) {
    if (!b || !ss || !in || n <= 0 || b->pending) return FB_EINVAL;
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
    // fused steps always run the group forms (clusters do not span the parts
    // of a fused grid)
    const bool shared = n > kBatchSharedMin || b->mode == 2;
    for (int i = 0; i < n; ++i) ss[i]->shared_gpu = shared;
    std::vector<FramePlan> plans(n);
    for (int i = 0; i < n; ++i) plans[i] = plan_frame(ss[i]);
    if (b->mode == 2) {
        rc = fused_step(b, ss, n, plans.data());
        if (rc) {
            for (int i = 0; i < n; ++i) ss[i]->shared_gpu = false;
            return rc;
        }
    } else if (b->mode == 1) {
        std::vector<uint64_t> key = composition(ss, n, plans.data());
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
    if (!b->pend_done) FB_CUDA(cudaEventCreateWithFlags(&b->pend_done, cudaEventDisableTiming));
    FB_CUDA(cudaEventRecord(b->pend_done, b->origin));
    b->pend_ss.assign(ss, ss + n);
    b->pend_plans = std::move(plans);
    b->pending = true;
    return FB_OK;
}

int fb_batch_collect(fb_batch* b, fb_frame_result* out) {
    if (!b || !b->pending) return FB_EINVAL;
    b->pending = false;
    FB_CUDA(cudaEventSynchronize(b->pend_done));
    const int n = (int)b->pend_ss.size();
    for (int i = 0; i < n; ++i) {
        finish_frame(b->pend_ss[i], b->pend_plans[i], out ? &out[i] : nullptr);
        b->pend_ss[i]->shared_gpu = false;
    }
    b->steps++;
    return FB_OK;
}

}  // extern "C"
