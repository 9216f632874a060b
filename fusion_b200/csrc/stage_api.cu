// The per-stage C entry points: one call per free function of the
// reference's boundary (Tracking/Reduction.h:18-83, Mapping/RenderScene.h:3-52)
// over plain pointer + pitch images, the map functions on a session's map,
// the top-down view and mesh extraction.
#include <cmath>
#include <cstring>

#include "session_internal.h"

namespace {

__global__ void k_set_pose(DevPose* dst, DevPose p) { *dst = p; }

}  // namespace

extern "C" {

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

int fb_track_reduction_grid(int pixels) {
    if (pixels <= 0) return 0;
    return track_cluster_grid(pixels);
}

size_t fb_step_scratch_bytes(int cols, int rows) {
    if (cols <= 0 || rows <= 0) return 0;
    // partials | tickets | out sums (32 doubles) | per-pixel correspondences
    return (size_t)kTrackMaxBlocks * 32 * 4 + 256 + 32 * 8 + (size_t)cols * rows * 4;
}

namespace {
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
}  // namespace

}  // extern "C"

namespace fb {

int rgb_step_check(const fb_image* gcurr, const fb_image* glast, const fb_image* vcurr, const fb_image* vlast,
                   const fb_image* dx, const fb_image* dy, const float* Rcurr, const float* RcurrInv,
                   const float* Rlast, const float* RlastInv, const float* tcurr, const float* tlast, const float* K,
                   const float* residual, const double* A, const double* b) {
    if (!image_ok(gcurr, 1) || !image_ok(glast, 1) || !image_ok(vcurr, 16) || !image_ok(vlast, 16) ||
        !image_ok(dx, 2) || !image_ok(dy, 2))
        return FB_EINVAL;
    if (!Rcurr || !RcurrInv || !Rlast || !RlastInv || !tcurr || !tlast || !K || !residual || !A || !b)
        return FB_EINVAL;
    const int W = gcurr->cols, H = gcurr->rows;
    if (W > 4096 || H > 2048) return FB_EINVAL;   // packed correspondences: 12-bit column, 11-bit row
    if (glast->cols != W || glast->rows != H || vcurr->cols != W || vcurr->rows != H || vlast->cols != W ||
        vlast->rows != H || dx->cols != W || dy->cols != W || dx->rows != H || dy->rows != H ||
        gcurr->pitch != glast->pitch || vcurr->pitch != vlast->pitch || dx->pitch != dy->pitch)
        return FB_EINVAL;
    return FB_OK;
}

int rgb_step_run(const fb_image* gcurr, const fb_image* glast, const fb_image* vcurr, const fb_image* vlast,
                 const fb_image* dx, const fb_image* dy, const float* Rcurr, const float* RcurrInv,
                 const float* Rlast, const float* RlastInv, const float* tcurr, const float* tlast, const float* K,
                 const StepScratch& sc, float* residual, double* A, double* b, cudaStream_t st) {
    TrackLevel L{};
    L.W = gcurr->cols;
    L.H = gcurr->rows;
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
    // the completion counters must start at zero; everything else in the
    // scratch is written by the kernels before it is read
    FB_CUDA(cudaMemsetAsync(sc.tickets, 0, 16, st));
    launch_step_rgb(L, cur, last, sc.partials, sc.tickets, sc.residual, sc.out, st);
    if (check_launch()) return FB_ECUDA;
    double host[32];
    FB_CUDA(cudaMemcpyAsync(host, sc.out, 32 * 8, cudaMemcpyDeviceToHost, st));
    FB_CUDA(cudaStreamSynchronize(st));
    unpack_sums(host, A, b);
    residual[0] = (float)host[27];
    residual[1] = (float)host[28];
    return FB_OK;
}

}  // namespace fb

extern "C" {

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
    unpack_sums(host, A, b);
    residual[0] = (float)host[27];
    residual[1] = (float)host[28];
    return FB_OK;
}

int fb_rgb_step(const fb_image* gcurr, const fb_image* glast, const fb_image* vcurr, const fb_image* vlast,
                const fb_image* dx, const fb_image* dy, const float Rcurr[9], const float RcurrInv[9],
                const float Rlast[9], const float RlastInv[9], const float tcurr[3], const float tlast[3],
                const float K[4], void* scratch, size_t scratch_bytes, float residual[2], double A[36], double b[6],
                void* stream) {
    int rc = rgb_step_check(gcurr, glast, vcurr, vlast, dx, dy, Rcurr, RcurrInv, Rlast, RlastInv, tcurr, tlast, K,
                            residual, A, b);
    if (rc) return rc;
    StepScratch sc;
    if (!carve(scratch, scratch_bytes, gcurr->cols, gcurr->rows, sc)) return FB_EINVAL;
    return rgb_step_run(gcurr, glast, vcurr, vlast, dx, dy, Rcurr, RcurrInv, Rlast, RlastInv, tcurr, tlast, K, sc,
                        residual, A, b, as_stream(stream));
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
    launch_fuse_records(s->map, (const float*)depth->data, (int)(depth->pitch / 4), (const uint8_t*)rgb->data,
                        (int)rgb->pitch, (const float4*)nmap->data, (int)(nmap->pitch / 16), W, H, st);
    launch_integrate(s->map, W, H, k, s->scratch_pose, nullptr, st);
    if (check_launch()) return FB_ECUDA;
    FB_CUDA(cudaStreamSynchronize(st));
    MapCounters c;
    FB_CUDA(cudaMemcpy(&c, s->ctr, sizeof c, cudaMemcpyDeviceToHost));
    if (no_visible) *no_visible = (uint32_t)c.n_visible;
    if (c.err & kErrNormalW) {
        fb_set_error_text("fb_fuse_map_color: a valid normal's w lane is not 1 (ComputeNMap writes 1)");
        return FB_EINVAL;
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

int fb_create_rendering_blocks(fb_session* s, const float RviewInv[9], const float tview[3], const float K[4],
                               fb_image* zmin, fb_image* zmax, uint32_t* no_tiles, void* stream) {
    if (!s || !RviewInv || !tview || !K || !image_ok(zmin, 4) || !image_ok(zmax, 4)) return FB_EINVAL;
    const MapView& m = s->map;
    if (zmin->cols < m.zc || zmin->rows < m.zr || zmax->cols < m.zc || zmax->rows < m.zr) return FB_EINVAL;
    // the view's rotation is the transpose of RviewInv
    const float R[9] = {RviewInv[0], RviewInv[3], RviewInv[6], RviewInv[1], RviewInv[4],
                        RviewInv[7], RviewInv[2], RviewInv[5], RviewInv[8]};
    cudaStream_t st = stream ? as_stream(stream) : s->stream;
    k_set_pose<<<1, 1, 0, st>>>(s->scratch_pose, pose_from(R, RviewInv, tview));
    launch_zrange(m, intr_from(K), s->scratch_pose, nullptr, st);
    if (check_launch()) return FB_ECUDA;
    FB_CUDA(cudaMemcpy2DAsync(zmin->data, zmin->pitch, m.zmin, (size_t)m.zc * 4, (size_t)m.zc * 4, m.zr,
                              cudaMemcpyDeviceToDevice, st));
    FB_CUDA(cudaMemcpy2DAsync(zmax->data, zmax->pitch, m.zmax, (size_t)m.zc * 4, (size_t)m.zc * 4, m.zr,
                              cudaMemcpyDeviceToDevice, st));
    FB_CUDA(cudaStreamSynchronize(st));
    if (no_tiles) {
        MapCounters c;
        FB_CUDA(cudaMemcpy(&c, s->ctr, sizeof c, cudaMemcpyDeviceToHost));
        *no_tiles = (uint32_t)c.n_tiles;
    }
    return FB_OK;
}

int fb_map_export_visible(fb_session* s, void* entries, uint32_t capacity, uint32_t* n, void* stream) {
    if (!s || (capacity && !entries) || ((uintptr_t)entries & 15)) return FB_EINVAL;
    cudaStream_t st = stream ? as_stream(stream) : s->stream;
    if (capacity) launch_export_visible(s->map, entries, (int)(capacity > (uint32_t)INT32_MAX ? INT32_MAX : capacity), st);
    if (check_launch()) return FB_ECUDA;
    FB_CUDA(cudaStreamSynchronize(st));
    MapCounters c;
    FB_CUDA(cudaMemcpy(&c, s->ctr, sizeof c, cudaMemcpyDeviceToHost));
    const uint32_t nv = (uint32_t)(c.n_visible < 0 ? 0 : c.n_visible < s->map.NS ? c.n_visible : s->map.NS);
    if (n) *n = nv;
    if (nv > capacity) {
        fb_set_error_text("fb_map_export_visible: more visible entries than the destination holds");
        return FB_EINVAL;
    }
    return FB_OK;
}

int fb_map_export_reference(fb_session* s, void* hash_entries, size_t n_entries, void* voxels, size_t n_voxels,
                            int32_t* heap, size_t n_heap, int32_t* heap_counter, int32_t* entry_ptr, void* stream) {
    if (!s || !hash_entries || !voxels || !heap || !heap_counter || !entry_ptr) return FB_EINVAL;
    const MapView& m = s->map;
    if (n_entries != (size_t)m.NB + m.NE || n_voxels != (size_t)m.NS * 512 || n_heap != (size_t)m.NS ||
        ((uintptr_t)hash_entries & 15) || ((uintptr_t)voxels & 7)) {
        fb_set_error_text("fb_map_export_reference: the buffers' sizes differ from the session's map");
        return FB_EINVAL;
    }
    cudaStream_t st = stream ? as_stream(stream) : s->stream;
    launch_export_reference(m, hash_entries, voxels, heap_counter, entry_ptr, st);
    if (check_launch()) return FB_ECUDA;
    if (!m.cvox)
        FB_CUDA(cudaMemcpyAsync(voxels, m.voxels, n_voxels * sizeof(Voxel), cudaMemcpyDeviceToDevice, st));
    FB_CUDA(cudaMemcpyAsync(heap, m.heap, n_heap * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    FB_CUDA(cudaStreamSynchronize(st));
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