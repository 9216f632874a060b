// Depth/intensity pyramid of one frame (the reference's Frame::FillImages,
// Core/Frame.cc:59-78, and the kernels of Tracking/Pyrdown.cu), plus the 2x2
// reduction of raycast maps (Frame::ResizeImages, Core/Frame.cc:80-84).
//
// Fusion: level 0 computes raw depth, the bilateral filter and the gray image
// in one pass; each coarser level computes depth and gray together; each level
// then computes vertex map, normal map and both Sobel derivatives in one pass
// (the neighbour vertices the normal needs are recomputed from depth instead
// of being re-read from a separate vertex-map pass).  All kernels are
// elementwise over pixels with small stencils served from L1.
#include "fb_fused.cuh"
#include "fb_internal.h"

namespace fb {

__constant__ float c_gauss[25] = {1, 4, 6, 4, 1, 4, 16, 24, 16, 4, 6, 24, 36,
                                  24, 6, 4, 16, 24, 16, 4, 1, 4, 6, 4, 1};

// FilterDepthKernel (Tracking/Pyrdown.cu:3-41) + ImageToIntensityKernel
// (Pyrdown.cu:183-193) for one level-0 pixel.
__device__ __forceinline__ void level0_body(const BlockCtx& ctx, const uint16_t* __restrict__ depth, int dpitch,
                                            const uint8_t* __restrict__ rgb, int rgbpitch, int W, int H, float inv,
                                            float cutoff, float* __restrict__ raw, int rawpitch,
                                            float* __restrict__ filt, int fpitch, uint8_t* __restrict__ gray,
                                            int gpitch) {
    const int x = ctx.bx * blockDim.x + threadIdx.x;
    const int y = ctx.by * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    if (gray) {
        const uint8_t* px = rgb + (size_t)y * rgbpitch + 3 * x;
        // double arithmetic, truncated (uchar3 lanes x, y, z = R, G, B)
        double v = da(da(dm(0.2125, (double)px[1]), dm(0.7154, (double)px[0])), dm(0.0721, (double)px[2]));
        gray[(size_t)y * gpitch + x] = (uint8_t)(int)v;
    }
    if (!depth) return;
    const float sigSpace = 0.03125f, sigRange = 2.0f;  // 0.5/(4*4), 0.5/(0.5*0.5)
    const float center = fm((float)depth[(size_t)y * dpitch + x], inv);
    if (raw) raw[(size_t)y * rawpitch + x] = center < cutoff ? center : qnan();
    if (!filt) return;
    const int tx = min(x + 3, W - 1), ty = min(y + 3, H - 1);
    float sum1 = 0.f, sum2 = 0.f;
    for (int cy = max(y - 2, 0); cy < ty; ++cy) {
        const uint16_t* row = depth + (size_t)cy * dpitch;
        for (int cx = max(x - 2, 0); cx < tx; ++cx) {
            float val = fm((float)row[cx], inv);
            float space2 = (float)((x - cx) * (x - cx) + (y - cy) * (y - cy));
            float dz = fs(center, val);
            float color2 = fm(dz, dz);
            float weight = expf(-fa(fm(space2, sigSpace), fm(color2, sigRange)));
            sum1 = fa(sum1, fm(val, weight));
            sum2 = fa(sum2, weight);
        }
    }
    float fin = fd(sum1, sum2);
    filt[(size_t)y * fpitch + x] = fin < cutoff ? fin : qnan();
}

__global__ void k_level0(const uint16_t* __restrict__ depth, int dpitch, const uint8_t* __restrict__ rgb,
                         int rgbpitch, int W, int H, float inv, float cutoff, float* __restrict__ raw,
                         int rawpitch, float* __restrict__ filt, int fpitch, uint8_t* __restrict__ gray,
                         int gpitch) {
    level0_body(own_ctx(), depth, dpitch, rgb, rgbpitch, W, H, inv, cutoff, raw, rawpitch, filt, fpitch, gray, gpitch);
}
FB_FUSED_KERNEL(k_level0, level0_body, 256)

// PyrDownGaussKernel<float> and <uchar> (Tracking/Pyrdown.cu:134-158) for one
// destination pixel: window clipped to [max(0, 2x-2), min(2x+3, cols-1)),
// kernel indexed from the clipped end, NaN taps skipped, truncating cast.
template <class T>
__device__ __forceinline__ T pyr_pixel(const T* __restrict__ src, int spitch, int SW, int SH, int x, int y) {
    const int tx = min(2 * x + 3, SW - 1), ty = min(2 * y + 3, SH - 1);
    float sum = 0.f;
    int count = 0;
    for (int cy = max(0, 2 * y - 2); cy < ty; ++cy)
        for (int cx = max(0, 2 * x - 2); cx < tx; ++cx) {
            float s = (float)src[(size_t)cy * spitch + cx];
            if (!isnan(s)) {
                float k = c_gauss[(ty - cy - 1) * 5 + (tx - cx - 1)];
                sum = fa(sum, fm(s, k));
                count += (int)k;
            }
        }
    return (T)fd(sum, (float)count);
}

__device__ __forceinline__ void pyrdown_body(const BlockCtx& ctx, const float* __restrict__ sd, int sdp,
                                             const uint8_t* __restrict__ sg, int sgp, int SW, int SH,
                                             float* __restrict__ dd, int ddp, uint8_t* __restrict__ dg, int dgp) {
    const int x = ctx.bx * blockDim.x + threadIdx.x;
    const int y = ctx.by * blockDim.y + threadIdx.y;
    if (x >= SW / 2 || y >= SH / 2) return;
    if (dd) dd[(size_t)y * ddp + x] = pyr_pixel<float>(sd, sdp, SW, SH, x, y);
    if (dg) dg[(size_t)y * dgp + x] = pyr_pixel<uint8_t>(sg, sgp, SW, SH, x, y);
}

__global__ void k_pyrdown(const float* __restrict__ sd, int sdp, const uint8_t* __restrict__ sg, int sgp,
                          int SW, int SH, float* __restrict__ dd, int ddp, uint8_t* __restrict__ dg,
                          int dgp) {
    pyrdown_body(own_ctx(), sd, sdp, sg, sgp, SW, SH, dd, ddp, dg, dgp);
}
FB_FUSED_KERNEL(k_pyrdown, pyrdown_body, 256)

// ComputeVMapKernel (Tracking/Pyrdown.cu:56-78) for one pixel; invalid
// vertices get NaN in x (the reference leaves y and w unset; NaN here).
__device__ __forceinline__ float4 vertex(const float* __restrict__ depth, int dp, int x, int y,
                                         const Intr& k, float cutoff) {
    float z = depth[(size_t)y * dp + x];
    if (!isnan(z) && (double)z > 0.1 && z < cutoff) {
        float vx = fm(fm(z, fs((float)x, k.cx)), k.invfx);
        float vy = fm(fm(z, fs((float)y, k.cy)), k.invfy);
        return make_float4(vx, vy, z, 1.0f);
    }
    return make_float4(qnan(), qnan(), z, qnan());
}

// ComputeNMapKernel (Tracking/Pyrdown.cu:93-114) from three vertices
__device__ __forceinline__ float4 normal_of(float4 c, float4 r, float4 d) {
    if (!isnan(c.x) && !isnan(r.x) && !isnan(d.x)) {
        f3 a = mk3(fs(r.x, c.x), fs(r.y, c.y), fs(r.z, c.z));
        f3 b = mk3(fs(d.x, c.x), fs(d.y, c.y), fs(d.z, c.z));
        f3 nn = normalised3(cross3(a, b));
        return make_float4(nn.x, nn.y, nn.z, 1.0f);
    }
    return make_float4(qnan(), qnan(), qnan(), qnan());
}

// Normal map of a given vertex map (the reference's ComputeNMap).
__global__ void k_nmap(const float4* __restrict__ vmap, int vp, int W, int H, float4* __restrict__ nmap, int np) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    float4 n = make_float4(qnan(), qnan(), qnan(), qnan());
    if (x != W - 1 && y != H - 1)
        n = normal_of(vmap[(size_t)y * vp + x], vmap[(size_t)y * vp + x + 1], vmap[(size_t)(y + 1) * vp + x]);
    nmap[(size_t)y * np + x] = n;
}

// Vertex map, normal map (ComputeNMapKernel, Pyrdown.cu:93-114) and Sobel
// derivatives (ComputeDerivativeImageKernel, Pyrdown.cu:207-237) of one level.
__device__ __forceinline__ void maps_body(const BlockCtx& ctx, const float* __restrict__ depth, int dp,
                                          const uint8_t* __restrict__ gray, int gp, int W, int H, Intr k,
                                          float cutoff, float4* __restrict__ vmap, int vp, float4* __restrict__ nmap,
                                          int np, int16_t* __restrict__ dxo, int16_t* __restrict__ dyo, int sp,
                                          uint8_t* __restrict__ rgbok, FuseRecDst fr) {
    const int x = ctx.bx * blockDim.x + threadIdx.x;
    const int y = ctx.by * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    if (vmap) {
        float4 c = vertex(depth, dp, x, y, k, cutoff);
        vmap[(size_t)y * vp + x] = c;
        if (nmap) {
            float4 n = make_float4(qnan(), qnan(), qnan(), qnan());
            if (x != W - 1 && y != H - 1) {
                float4 r = vertex(depth, dp, x + 1, y, k, cutoff);
                float4 d = vertex(depth, dp, x, y + 1, k, cutoff);
                n = normal_of(c, r, d);
            }
            nmap[(size_t)y * np + x] = n;
            // the fusion record of this pixel (level 0 of a frame that may be fused)
            if (fr.rec) {
                const float dp = fr.raw[(size_t)y * fr.rp + x];
                const uint8_t* c3 = fr.rgb + (size_t)y * fr.cp + 3 * x;
                if (fr.packed)
                    fuse_record_packed(dp, n, c3, fr.dmin, fr.dmax, (uint4*)fr.rec + (size_t)y * W + x);
                else
                    fuse_record(dp, n, c3, fr.dmin, fr.dmax, fr.rec + (size_t)y * W + x, fr.col + (size_t)y * W + x);
            }
        }
    }
    if (dxo) {
        // kernel index runs 8 -> 0 over the clipped window; integer sums are
        // exact, as the reference's float sums of small integers are
        const int sx[9] = {1, 0, -1, 2, 0, -2, 1, 0, -1};
        const int sy[9] = {1, 2, 1, 0, 0, 0, -1, -2, -1};
        int gx = 0, gy = 0, idx = 8;
        for (int j = max(y - 1, 0); j <= min(y + 1, H - 1); ++j)
            for (int i = max(x - 1, 0); i <= min(x + 1, W - 1); ++i) {
                int v = gray[(size_t)j * gp + i];
                gx += v * sx[idx];
                gy += v * sy[idx];
                --idx;
            }
        dxo[(size_t)y * sp + x] = (int16_t)gx;
        dyo[(size_t)y * sp + x] = (int16_t)gy;
        if (rgbok) {
            // the pose-independent part of RGBReduction::FindCorresp
            // (Tracking/Reduction.cu:413-425): 5-pixel border, gray > 0 over
            // the window y-2..y+1, x-2..x+1, nonzero gradient
            bool ok = x >= 5 && x < W - 5 && y >= 5 && y < H - 5 && ((int16_t)gx != 0 || (int16_t)gy != 0);
            if (ok)
                for (int u = y - 2; u < y + 2 && ok; ++u)
                    for (int v = x - 2; v < x + 2; ++v)
                        if (gray[(size_t)u * gp + v] == 0) {
                            ok = false;
                            break;
                        }
            rgbok[(size_t)y * sp + x] = ok ? 1 : 0;
        }
    }
}

__global__ void k_maps(const float* __restrict__ depth, int dp, const uint8_t* __restrict__ gray, int gp,
                       int W, int H, Intr k, float cutoff, float4* __restrict__ vmap, int vp,
                       float4* __restrict__ nmap, int np, int16_t* __restrict__ dxo, int16_t* __restrict__ dyo,
                       int sp, uint8_t* __restrict__ rgbok, FuseRecDst fr) {
    maps_body(own_ctx(), depth, dp, gray, gp, W, H, k, cutoff, vmap, vp, nmap, np, dxo, dyo, sp, rgbok, fr);
}
FB_FUSED_KERNEL(k_maps, maps_body, 256)

// ResizeMapKernel (Tracking/Pyrdown.cu:251-279): 2x2 means; the normal mean
// is normalised over all four lanes.  Bounds are the destination size (the
// reference checks the source size and writes past short destinations).
__device__ __forceinline__ void resize_body(const BlockCtx& ctx, const float4* __restrict__ vs,
                                            const float4* __restrict__ ns, int sp, int SW, int SH,
                                            float4* __restrict__ vd, float4* __restrict__ nd, int dp) {
    const int x = ctx.bx * blockDim.x + threadIdx.x;
    const int y = ctx.by * blockDim.y + threadIdx.y;
    if (x >= SW / 2 || y >= SH / 2) return;
    const size_t i00 = (size_t)(2 * y) * sp + 2 * x, i10 = i00 + sp;
    float4 v00 = vs[i00], v01 = vs[i00 + 1], v10 = vs[i10], v11 = vs[i10 + 1];
    float4 o;
    if (isnan(v00.x) || isnan(v01.x) || isnan(v10.x) || isnan(v11.x)) {
        o = make_float4(qnan(), qnan(), qnan(), qnan());
    } else {
        o.x = fd(fa(fa(fa(v00.x, v01.x), v10.x), v11.x), 4.f);
        o.y = fd(fa(fa(fa(v00.y, v01.y), v10.y), v11.y), 4.f);
        o.z = fd(fa(fa(fa(v00.z, v01.z), v10.z), v11.z), 4.f);
        o.w = fd(fa(fa(fa(v00.w, v01.w), v10.w), v11.w), 4.f);
    }
    vd[(size_t)y * dp + x] = o;
    float4 n00 = ns[i00], n01 = ns[i00 + 1], n10 = ns[i10], n11 = ns[i10 + 1];
    if (isnan(n00.x) || isnan(n01.x) || isnan(n10.x) || isnan(n11.x)) {
        o = make_float4(qnan(), qnan(), qnan(), qnan());
    } else {
        float mx = fd(fa(fa(fa(n00.x, n01.x), n10.x), n11.x), 4.f);
        float my = fd(fa(fa(fa(n00.y, n01.y), n10.y), n11.y), 4.f);
        float mz = fd(fa(fa(fa(n00.z, n01.z), n10.z), n11.z), 4.f);
        float mw = fd(fa(fa(fa(n00.w, n01.w), n10.w), n11.w), 4.f);
        float nn = fsq(fa(fa(fa(fm(mx, mx), fm(my, my)), fm(mz, mz)), fm(mw, mw)));
        o = make_float4(fd(mx, nn), fd(my, nn), fd(mz, nn), fd(mw, nn));
    }
    nd[(size_t)y * dp + x] = o;
}

__global__ void k_resize(const float4* __restrict__ vs, const float4* __restrict__ ns, int sp, int SW, int SH,
                         float4* __restrict__ vd, float4* __restrict__ nd, int dp) {
    resize_body(own_ctx(), vs, ns, sp, SW, SH, vd, nd, dp);
}
FB_FUSED_KERNEL(k_resize, resize_body, 256)

// A launch of up to four roles (PreLaunch): each block finds its role and
// runs that role's body with its coordinates in the role's own grid.
__device__ __forceinline__ void pre_body(const BlockCtx& ctx, const PreLaunch& P) {
    int b = ctx.bx;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int n = P.gx[r] * P.gy[r];
        if (b < n) {
            const BlockCtx c{b % P.gx[r], b / P.gx[r], P.gx[r], P.gy[r]};
            if (r == 0) {
                const Level0Args& a = P.l0;
                level0_body(c, a.depth, a.dpitch, a.rgb, a.rgbpitch, a.W, a.H, a.inv, a.cutoff, a.raw, a.rawpitch,
                            a.filt, a.fpitch, a.gray, a.gpitch);
            } else if (r == 1) {
                const ResizeArgs& a = P.rs;
                resize_body(c, a.vs, a.ns, a.sp, a.SW, a.SH, a.vd, a.nd, a.dp);
            } else if (r == 2) {
                const PyrArgs& a = P.py;
                pyrdown_body(c, a.sd, a.sdp, a.sg, a.sgp, a.SW, a.SH, a.dd, a.ddp, a.dg, a.dgp);
            } else {
                const MapsArgs& a = P.mp;
                maps_body(c, a.depth, a.dp, a.gray, a.gp, a.W, a.H, a.k, a.cutoff, a.vmap, a.vp, a.nmap, a.np,
                          a.dxo, a.dyo, a.sp, a.rgbok, a.fr);
            }
            return;
        }
        b -= n;
    }
}

__global__ void __launch_bounds__(256) k_pre(PreLaunch P) { pre_body(own_ctx(), P); }
FB_FUSED_KERNEL(k_pre, pre_body, 256)

static inline dim3 grid2d(int W, int H, dim3 b) { return dim3((W + b.x - 1) / b.x, (H + b.y - 1) / b.y); }

static void set_role(PreLaunch& P, int r, int W, int H) {
    const dim3 g = grid2d(W, H, dim3(32, 8));
    P.gx[r] = W > 0 && H > 0 ? (int)g.x : 0;
    P.gy[r] = W > 0 && H > 0 ? (int)g.y : 0;
}

void pre_level0(PreLaunch& P, const uint16_t* depth, int dpitch, const uint8_t* rgb, int rgbpitch, int W, int H,
                float depth_scale, float cutoff, float* raw, int rawpitch, float* filt, int fpitch, uint8_t* gray,
                int gpitch) {
    // FilterDepth passes 1.0 / depthScale computed in double (Pyrdown.cu:50)
    P.l0 = Level0Args{depth, dpitch, rgb, rgbpitch, W, H, (float)(1.0 / (double)depth_scale), cutoff, raw,
                      rawpitch, filt, fpitch, gray, gpitch};
    set_role(P, 0, W, H);
}

void pre_resize(PreLaunch& P, const float4* vs, const float4* ns, int sp, int SW, int SH, float4* vd, float4* nd,
                int dp) {
    P.rs = ResizeArgs{vs, ns, sp, SW, SH, vd, nd, dp};
    set_role(P, 1, SW / 2, SH / 2);
}

void pre_pyrdown(PreLaunch& P, const float* sd, int sdp, const uint8_t* sg, int sgp, int SW, int SH, float* dd,
                 int ddp, uint8_t* dg, int dgp) {
    P.py = PyrArgs{sd, sdp, sg, sgp, SW, SH, dd, ddp, dg, dgp};
    set_role(P, 2, SW / 2, SH / 2);
}

void pre_maps(PreLaunch& P, const float* depth, int dp, const uint8_t* gray, int gp, int W, int H, const Intr& k,
              float cutoff, float4* vmap, int vp, float4* nmap, int np, int16_t* dx, int16_t* dy, int sp,
              uint8_t* rgbok, const FuseRecDst* fr) {
    const FuseRecDst none{};
    P.mp = MapsArgs{depth, dp, gray, gp, W, H, k, cutoff, vmap, vp, nmap, np, dx, dy, sp, rgbok, fr ? *fr : none};
    set_role(P, 3, W, H);
}

int launch_pre(const PreLaunch& P, cudaStream_t st) {
    int blocks = 0;
    for (int r = 0; r < 4; ++r) blocks += P.gx[r] * P.gy[r];
    if (blocks == 0) return 0;
    fb_launch(k_pre, (const void*)k_pre_fused, blocks, dim3(32, 8), 0, st, P);
    return 1;
}

// ---- launchers (pitches in elements) ----

int launch_level0(const uint16_t* depth, int dpitch, const uint8_t* rgb, int rgbpitch, int W, int H,
                   float depth_scale, float cutoff, float* raw, int rawpitch, float* filt, int fpitch,
                   uint8_t* gray, int gpitch, cudaStream_t st) {
    dim3 b(32, 8);
    // FilterDepth passes 1.0 / depthScale computed in double (Pyrdown.cu:50)
    float inv = (float)(1.0 / (double)depth_scale);
    fb_launch(k_level0, (const void*)k_level0_fused, grid2d(W, H, b), b, 0, st, depth, dpitch, rgb, rgbpitch, W, H,
              inv, cutoff, raw, rawpitch, filt, fpitch, gray, gpitch);
    return 1;
}

int launch_pyrdown(const float* sd, int sdp, const uint8_t* sg, int sgp, int SW, int SH, float* dd,
                    int ddp, uint8_t* dg, int dgp, cudaStream_t st) {
    dim3 b(32, 8);
    fb_launch(k_pyrdown, (const void*)k_pyrdown_fused, grid2d(SW / 2, SH / 2, b), b, 0, st, sd, sdp, sg, sgp, SW, SH,
              dd, ddp, dg, dgp);
    return 1;
}

int launch_maps(const float* depth, int dp, const uint8_t* gray, int gp, int W, int H, const Intr& k,
                 float cutoff, float4* vmap, int vp, float4* nmap, int np, int16_t* dx, int16_t* dy,
                 int sp, cudaStream_t st, uint8_t* rgbok, const FuseRecDst* fr) {
    dim3 b(32, 8);
    const FuseRecDst none{};
    fb_launch(k_maps, (const void*)k_maps_fused, grid2d(W, H, b), b, 0, st, depth, dp, gray, gp, W, H, k, cutoff, vmap,
              vp, nmap, np, dx, dy, sp, rgbok, fr ? *fr : none);
    return 1;
}

int launch_nmap(const float4* vmap, int vp, int W, int H, float4* nmap, int np, cudaStream_t st) {
    dim3 b(32, 8);
    k_nmap<<<grid2d(W, H, b), b, 0, st>>>(vmap, vp, W, H, nmap, np);
    return 1;
}

int launch_resize(const float4* vs, const float4* ns, int sp, int SW, int SH, float4* vd, float4* nd,
                   int dp, cudaStream_t st) {
    dim3 b(32, 8);
    fb_launch(k_resize, (const void*)k_resize_fused, grid2d(SW / 2, SH / 2, b), b, 0, st, vs, ns, sp, SW, SH, vd, nd,
              dp);
    return 1;
}

}  // namespace fb
