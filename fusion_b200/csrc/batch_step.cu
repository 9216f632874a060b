// Batched steps (fb_batch_*): one frame of each of n independent sessions
// with all frames in flight together, each session's cached frame graph on
// its own stream of the batch, or one composite graph per composition.
#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "session_internal.h"

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
                          (uint64_t)s->shared_gpu << 5 |
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
