// Headless rendering of the model: Phong shading of a raycast vertex/normal
// map into an RGBA8 image (RenderImage, Tracking/Pyrdown.cu:322-380), and the
// two display conversions of the reference's frame loop (DepthToImage,
// Pyrdown.cu:382-405; RgbImageToRgba, Pyrdown.cu:407-428).  No graphics API:
// the image is device memory the caller reads back or writes to a file.
#include "../../include/fusion_b200.h"
#include "fb_internal.h"

namespace fb {

// RenderImageDevice: background gradient where the vertex is missing, else
// ambient + diffuse + specular (Ka 0.3, Kd 0.5, Ks 0.2, power 20) of a white
// light at `light`, viewed from the camera origin; the reference's
// expressions in its order, with its fast __powf.
__global__ void k_render_image(const float4* __restrict__ vmap, const float4* __restrict__ nmap, int vp, float3 light,
                               uchar4* __restrict__ dst, int dp, int W, int H) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const float4 v = vmap[(size_t)y * vp + x];
    float cx, cy, cz;
    if (isnan(v.x)) {
        const float w = (float)y / H;
        cx = 4.f / 255.f * (1 - w) + 236.f / 255.f * w;
        cy = 2.f / 255.f * (1 - w) + 120.f / 255.f * w;
        cz = 2.f / 255.f * (1 - w) + 120.f / 255.f * w;
    } else {
        const float4 n4 = nmap[(size_t)y * vp + x];
        const f3 P = mk3(v.x, v.y, v.z), N = mk3(n4.x, n4.y, n4.z);
        const f3 L = normalised3(mk3(light.x - P.x, light.y - P.y, light.z - P.z));
        const f3 V = normalised3(mk3(0.f - P.x, 0.f - P.y, 0.f - P.z));
        const float nl = N.x * L.x + N.y * L.y + N.z * L.z;
        const f3 R = normalised3(mk3(2 * N.x * nl - L.x, 2 * N.y * nl - L.y, 2 * N.z * nl - L.z));
        const float rv = R.x * V.x + R.y * V.y + R.z * V.z;
        const float I = 1.f * 0.3f * 1.f + 1.f * 0.5f * 1.f * fmaxf(0.f, nl) +
                        1.f * 0.2f * 1.f * __powf(fmaxf(0.f, rv), 20.f);
        cx = cy = cz = I;
    }
    uchar4 o;
    o.x = (unsigned char)(__saturatef(cx) * 255.f);
    o.y = (unsigned char)(__saturatef(cy) * 255.f);
    o.z = (unsigned char)(__saturatef(cz) * 255.f);
    o.w = 255;
    dst[(size_t)y * dp + x] = o;
}

// depthToImageKernel: depth / 3 m as gray, NaN black.
__global__ void k_depth_to_image(const float* __restrict__ depth, int sp, uchar4* __restrict__ dst, int dp, int W,
                                 int H) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const float d = (float)((double)depth[(size_t)y * sp + x] / 3.0);
    int g = __float2int_rd(d * 255);
    g = g > 255 ? 255 : g;
    if (isnan(d)) g = 0;
    dst[(size_t)y * dp + x] = make_uchar4((unsigned char)g, (unsigned char)g, (unsigned char)g, 255);
}

// rgbImageToRgbaKernel
__global__ void k_rgb_to_rgba(const uint8_t* __restrict__ rgb, int sp, uchar4* __restrict__ dst, int dp, int W, int H) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const uint8_t* p = rgb + (size_t)y * sp + 3 * x;
    dst[(size_t)y * dp + x] = make_uchar4(p[0], p[1], p[2], 255);
}

}  // namespace fb

using namespace fb;

namespace {

int ok_image(const fb_image* im, size_t elem) {
    return im && im->data && im->cols > 0 && im->rows > 0 && im->pitch >= elem * (size_t)im->cols &&
           im->pitch % elem == 0;
}

int finish(cudaStream_t st) {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        fb_set_error_text(cudaGetErrorString(e));
        return FB_ECUDA;
    }
    return FB_OK;
}

}  // namespace

extern "C" {

int fb_render_image(const fb_image* vmap, const fb_image* nmap, const float light[3], fb_image* rgba, void* stream) {
    if (!ok_image(vmap, 16) || !ok_image(nmap, 16) || !ok_image(rgba, 4) || !light) return FB_EINVAL;
    const int W = rgba->cols, H = rgba->rows;
    if (vmap->cols < W || vmap->rows < H || nmap->cols < W || nmap->rows < H || vmap->pitch != nmap->pitch)
        return FB_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    dim3 b(32, 8), g((W + 31) / 32, (H + 7) / 8);
    k_render_image<<<g, b, 0, st>>>((const float4*)vmap->data, (const float4*)nmap->data, (int)(vmap->pitch / 16),
                                    make_float3(light[0], light[1], light[2]), (uchar4*)rgba->data,
                                    (int)(rgba->pitch / 4), W, H);
    return finish(st);
}

int fb_depth_to_image(const fb_image* depth, fb_image* rgba, void* stream) {
    if (!ok_image(depth, 4) || !ok_image(rgba, 4)) return FB_EINVAL;
    const int W = rgba->cols, H = rgba->rows;
    if (depth->cols < W || depth->rows < H) return FB_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    dim3 b(32, 8), g((W + 31) / 32, (H + 7) / 8);
    k_depth_to_image<<<g, b, 0, st>>>((const float*)depth->data, (int)(depth->pitch / 4), (uchar4*)rgba->data,
                                      (int)(rgba->pitch / 4), W, H);
    return finish(st);
}

int fb_rgb_to_rgba(const fb_image* rgb, fb_image* rgba, void* stream) {
    if (!ok_image(rgb, 1) || !ok_image(rgba, 4) || rgb->pitch < (size_t)3 * rgb->cols) return FB_EINVAL;
    const int W = rgba->cols, H = rgba->rows;
    if (rgb->cols < W || rgb->rows < H) return FB_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    dim3 b(32, 8), g((W + 31) / 32, (H + 7) / 8);
    k_rgb_to_rgba<<<g, b, 0, st>>>((const uint8_t*)rgb->data, (int)rgb->pitch, (uchar4*)rgba->data,
                                   (int)(rgba->pitch / 4), W, H);
    return finish(st);
}

}  // extern "C"
