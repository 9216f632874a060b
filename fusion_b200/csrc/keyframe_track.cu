// Key points in the session's frames (fb_session_set_keypoints): the
// reference's SURF path -- Frame::ExtractKeyPoints on every frame,
// Tracker::TrackLastFrame's bootstrap pose, keyframes with observation
// counts, the key map (Mapping::FuseKeyFrame) and Tracker::Relocalise --
// over this library's own detector, descriptor, matcher and pose solver
// (keypoints.cu).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "session_internal.h"

namespace fb {

void free_keys(fb_session* s) {
    if (!s->keys) return;
    if (s->keys->mem) cudaFree(s->keys->mem);
    delete s->keys;
    s->keys = nullptr;
}

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
    launch_track_reloc(s, T, st);
    const DevPose* pose = &s->st->cur;
    int n = 1;
    n += launch_visibility(s->map, s->W[0], s->H[0], s->K[0], pose, nullptr, st);
    n += launch_zrange(s->map, s->K[0], pose, nullptr, st, raycast_tiles(s->W[0], s->H[0], s->rc_bx, s->rc_by));
    n += launch_raycast(s->map, N.vmap[0], N.nmap[0], s->W[0], s->W[0], s->H[0], s->K[0], pose, nullptr, st, s->rc_bx,
                        s->rc_by);
    launch_commit(s, 1, st);
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

}  // namespace fb

extern "C" {

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

}  // extern "C"
