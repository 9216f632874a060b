// Key points: detection, description, back-projection, matching and the
// RANSAC pose solver.
//
// The reference extracts SURF key points from every frame's level-0 gray
// image with OpenCV's CUDA SURF (Frame::ExtractKeyPoints, Core/Frame.cc:
// 165-212; SURF_CUDA(20): Hessian threshold 20, 4 octaves of 4 filter sizes,
// 64-value descriptors with orientation, at most 1 % of the pixels as key
// points), keeps those with a valid interpolated depth and normal as 3-D
// points, and matches descriptors by brute force (cv::cuda BFMatcher, L2,
// two nearest neighbours and a ratio test; Tracking.cc:169-204, 411-458).
// OpenCV is not part of this library; the detector and descriptor here are
// this library's own implementation of the published SURF method (Bay, Ess,
// Tuytelaars, Van Gool, "Speeded-Up Robust Features (SURF)", CVIU 110(3),
// 2008): box-filter Hessian determinants on an integral image, 3x3x3
// non-maximum suppression on the two middle filter sizes of each octave,
// quadratic sub-sample refinement, the dominant orientation of Gaussian-
// weighted Haar responses in a sliding pi/3 window, and 4 x 4 subregions of
// (sum dx, sum dy, sum |dx|, sum |dy|) Haar responses, normalised.
//
// Everything is deterministic: box sums are integer, candidates are ranked
// by (response, sample index) with a total order, and every reduction has a
// fixed order.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/fusion_b200.h"
#include "fb_internal.h"

namespace fb {

// ---------------------------------------------------------------- geometry

__host__ __device__ constexpr int surf_filter(int octave, int layer) {
    // filter side 3 (2^(octave + 1) (layer + 1) + 1): 9 15 21 27 | 15 27 39 51 | ...
    return 3 * ((2 << octave) * (layer + 1) + 1);
}

__host__ __device__ inline int surf_margin(int octave) {
    // the largest filter of the octave fits around a sample at this distance
    return surf_filter(octave, kSurfLayers - 1) / 2 + 1;
}

size_t key_scratch_bytes(int W, int H) {
    size_t b = 0;
    b += (size_t)(W + 1) * (H + 1) * 4;                                                  // integral image
    for (int o = 0; o < kSurfOctaves; ++o) b += (size_t)kSurfLayers * (W >> o) * (H >> o) * 4;   // responses
    b += (size_t)kSurfMaxCand * 16 + (size_t)kSurfMaxCand * 8;                           // candidates, keys
    for (int o = 0; o < kSurfOctaves; ++o) b += (size_t)(kSurfLayers - 2) * (W >> o) * (H >> o) * 4;   // slot map
    b += 64;                                                                              // counter
    b += (size_t)(W * H / 100) * (16 + 4 * kKeyDesc) + 1024;                              // selected key points
    return b + 16 * 256;                                                                  // alignment
}

// ----------------------------------------------------------- integral image

// Row prefix sums: one CTA of 256 threads per row (block scan of uint32).
__global__ void __launch_bounds__(256) k_integral_rows(const uint8_t* __restrict__ img, int ip, int W, int H,
                                                       uint32_t* __restrict__ I) {
    const int y = blockIdx.x;
    if (y >= H) return;
    __shared__ uint32_t warp_tot[8];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    uint32_t* row = I + (size_t)(y + 1) * (W + 1);
    if (threadIdx.x == 0) row[0] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int x0 = 0; x0 < W; x0 += 256) {
        const int x = x0 + threadIdx.x;
        uint32_t v = x < W ? img[(size_t)y * ip + x] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += t;
        }
        if (lane == 31) warp_tot[w] = v;
        __syncthreads();
        uint32_t before = carry;
        for (int k = 0; k < w; ++k) before += warp_tot[k];
        if (x < W) row[x + 1] = before + v;
        __syncthreads();
        if (threadIdx.x == 255) carry = before + v;
        __syncthreads();
    }
}

// Column prefix sums in place (row 0 is zero): a CTA of 32 x 16 threads per
// 32 columns; thread (c, g) adds rows [g R, (g + 1) R) of its column, the 16
// segment sums are scanned in shared memory, then the segment is rewritten
// with its offset (coalesced across the 32 columns).
__global__ void __launch_bounds__(512) k_integral_cols(uint32_t* __restrict__ I, int W, int H) {
    __shared__ uint32_t seg[16][33];
    const int x = blockIdx.x * 32 + threadIdx.x, g = threadIdx.y;
    const int R = (H + 15) / 16, y0 = 1 + g * R, y1 = min(H + 1, y0 + R);
    const int s = W + 1;
    uint32_t t = 0;
    if (x <= W)
        for (int y = y0; y < y1; ++y) t += I[(size_t)y * s + x];
    seg[g][threadIdx.x] = t;
    __syncthreads();
    uint32_t off = 0;
    for (int q = 0; q < g; ++q) off += seg[q][threadIdx.x];
    if (x <= W) {
        if (g == 0) I[x] = 0;
        uint32_t acc = off;
        for (int y = y0; y < y1; ++y) {
            acc += I[(size_t)y * s + x];
            I[(size_t)y * s + x] = acc;
        }
    }
}

struct Integral {
    const uint32_t* I;
    int W, H;
    // sum over the half-open box [x0, x1) x [y0, y1), clipped to the image
    __device__ __forceinline__ int box(int x0, int y0, int x1, int y1) const {
        x0 = min(max(x0, 0), W);
        x1 = min(max(x1, 0), W);
        y0 = min(max(y0, 0), H);
        y1 = min(max(y1, 0), H);
        if (x1 <= x0 || y1 <= y0) return 0;
        const int s = W + 1;
        return (int)(I[(size_t)y1 * s + x1] - I[(size_t)y0 * s + x1] - I[(size_t)y1 * s + x0] + I[(size_t)y0 * s + x0]);
    }
};

// ------------------------------------------------------------------ Hessian

// det(H) of the box-filter approximation at pixel (x, y), filter side L:
// Dxx, Dyy over a (2l - 1) x 3l region (lobes +1, -2, +1), Dxy over four
// l x l squares around the centre, each normalised by L^2; Dxy weighted 0.9.
// One rounding per operation (no contraction), so a CPU restatement
// reproduces every response.
__device__ __forceinline__ float hessian_det(const Integral& it, int x, int y, int L) {
    const int l = L / 3, h = (3 * l - 1) / 2, m = (l - 1) / 2;
    const int dyy = it.box(x - (l - 1), y - h, x + l, y + h + 1) - 3 * it.box(x - (l - 1), y - m, x + l, y + m + 1);
    const int dxx = it.box(x - h, y - (l - 1), x + h + 1, y + l) - 3 * it.box(x - m, y - (l - 1), x + m + 1, y + l);
    const int dxy = it.box(x - l, y - l, x, y) + it.box(x + 1, y + 1, x + l + 1, y + l + 1) -
                    it.box(x + 1, y - l, x + l + 1, y) - it.box(x - l, y + 1, x, y + l + 1);
    const float inv = fd(1.0f, fm((float)L, (float)L));
    const float fxx = fm((float)dxx, inv), fyy = fm((float)dyy, inv), fxy = fm((float)dxy, inv);
    return fs(fm(fxx, fyy), fm(fm(0.81f, fxy), fxy));
}

// All layers of one octave at its samples (pixel = sample << o); zero where
// the octave's largest filter does not fit.  map: [layer][oh][ow].
__global__ void k_hessian(Integral it, float* __restrict__ map, int ow, int oh, int o) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= ow || j >= oh) return;
    const int x = i << o, y = j << o, mg = surf_margin(o);
    const bool in = x >= mg && y >= mg && x < it.W - mg && y < it.H - mg;
#pragma unroll
    for (int l = 0; l < kSurfLayers; ++l)
        map[((size_t)l * oh + j) * ow + i] = in ? hessian_det(it, x, y, surf_filter(o, l)) : 0.f;
}

// Candidates of one octave: samples of the middle layers above the threshold
// and above their 26 neighbours, refined by a quadratic fit (offsets below
// half a sample).  cand = {x, y, scale, response}; key = response bits << 32
// | sample index over all octaves' middle layers (unique: a total order, as
// responses are positive); slotmap[sample index] = the candidate's slot.
__global__ void k_extrema(const float* __restrict__ M, int ow, int oh, int o, int code0, float threshold,
                          float4* __restrict__ cand, unsigned long long* __restrict__ keys, int* __restrict__ slotmap,
                          int* __restrict__ counter, int cap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    const int mg = (surf_margin(o) + (1 << o) - 1) >> o;   // margin in samples
    if (i < mg + 1 || j < mg + 1 || i >= ow - mg - 1 || j >= oh - mg - 1) return;
    auto at = [&](int l, int jj, int ii) { return M[((size_t)l * oh + jj) * ow + ii]; };
    for (int l = 1; l < kSurfLayers - 1; ++l) {
        const float v = at(l, j, i);
        if (!(v > threshold)) continue;
        bool peak = true;
        for (int dl = -1; dl <= 1 && peak; ++dl)
            for (int dj = -1; dj <= 1 && peak; ++dj)
                for (int di = -1; di <= 1; ++di) {
                    if (!dl && !dj && !di) continue;
                    if (!(v > at(l + dl, j + dj, i + di))) {
                        peak = false;
                        break;
                    }
                }
        if (!peak) continue;
        // gradient and Hessian by central differences in (x, y, layer)
        const float gx = 0.5f * (at(l, j, i + 1) - at(l, j, i - 1));
        const float gy = 0.5f * (at(l, j + 1, i) - at(l, j - 1, i));
        const float gs = 0.5f * (at(l + 1, j, i) - at(l - 1, j, i));
        const float hxx = at(l, j, i + 1) + at(l, j, i - 1) - 2.f * v;
        const float hyy = at(l, j + 1, i) + at(l, j - 1, i) - 2.f * v;
        const float hss = at(l + 1, j, i) + at(l - 1, j, i) - 2.f * v;
        const float hxy = 0.25f * (at(l, j + 1, i + 1) - at(l, j + 1, i - 1) - at(l, j - 1, i + 1) + at(l, j - 1, i - 1));
        const float hxs = 0.25f * (at(l + 1, j, i + 1) - at(l + 1, j, i - 1) - at(l - 1, j, i + 1) + at(l - 1, j, i - 1));
        const float hys = 0.25f * (at(l + 1, j + 1, i) - at(l + 1, j - 1, i) - at(l - 1, j + 1, i) + at(l - 1, j - 1, i));
        // H d = -g by Cramer's rule in double
        const double a = hxx, b = hxy, c = hxs, d = hyy, e = hys, f = hss;
        const double det = a * (d * f - e * e) - b * (b * f - e * c) + c * (b * e - d * c);
        if (!(fabs(det) > 1e-30)) continue;
        const double rx = -gx, ry = -gy, rs = -gs;
        const double ox = (rx * (d * f - e * e) - b * (ry * f - e * rs) + c * (ry * e - d * rs)) / det;
        const double oy = (a * (ry * f - e * rs) - rx * (b * f - e * c) + c * (b * rs - ry * c)) / det;
        const double os = (a * (d * rs - ry * e) - b * (b * rs - ry * c) + rx * (b * e - d * c)) / det;
        if (!(fabs(ox) < 0.5 && fabs(oy) < 0.5 && fabs(os) < 0.5)) continue;
        const float step = (float)(1 << o);
        const float L = (float)surf_filter(o, l) + (float)os * (float)(surf_filter(o, l + 1) - surf_filter(o, l));
        const int slot = atomicAdd(counter, 1);
        if (slot < cap) {
            cand[slot] = make_float4(((float)i + (float)ox) * step, ((float)j + (float)oy) * step, 1.2f * L / 9.f, v);
            const unsigned code = (unsigned)(code0 + ((l - 1) * oh + j) * ow + i);
            keys[slot] = (unsigned long long)__float_as_uint(v) << 32 | code;
            slotmap[code] = slot;
        }
    }
}

// Descending bitonic sort of n (a power of two, <= kSurfMaxCand) keys, one
// CTA, in shared memory; entries past count are zero (they sort last).
__global__ void __launch_bounds__(1024) k_sort_keys(unsigned long long* __restrict__ keys, int count, int n) {
    extern __shared__ unsigned long long sk[];
    for (int t = threadIdx.x; t < n; t += blockDim.x) sk[t] = t < count ? keys[t] : 0ull;
    __syncthreads();
    for (int k = 2; k <= n; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int t = threadIdx.x; t < n; t += blockDim.x) {
                const int p = t ^ j;
                if (p > t) {
                    const bool desc = (t & k) == 0;
                    const unsigned long long a = sk[t], b = sk[p];
                    if (desc ? (a < b) : (a > b)) {
                        sk[t] = b;
                        sk[p] = a;
                    }
                }
            }
            __syncthreads();
        }
    for (int t = threadIdx.x; t < n; t += blockDim.x) keys[t] = sk[t];
}

// ------------------------------------------------------ orientation, descriptor

__device__ __forceinline__ void haar(const Integral& it, int x, int y, int h, float& dx, float& dy) {
    const int r = h / 2;
    dx = (float)(it.box(x, y - r, x + r, y + r) - it.box(x - r, y - r, x, y + r));
    dy = (float)(it.box(x - r, y, x + r, y + r) - it.box(x - r, y - r, x + r, y));
}

__device__ __forceinline__ int even_size(float v) { return max(2, 2 * __float2int_rn(0.5f * v)); }

// One warp per selected key point: orientation, then the 64 descriptor
// values.  kp out: {x, y, scale, angle}.
__global__ void __launch_bounds__(256) k_describe(Integral it, const float4* __restrict__ cand,
                                                  const unsigned long long* __restrict__ keys,
                                                  const int* __restrict__ slotmap, int n, float4* __restrict__ kp,
                                                  float* __restrict__ desc) {
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int k = blockIdx.x * 8 + wib;
    if (k >= n) return;
    __shared__ float s_dx[8][112], s_dy[8][112], s_ang[8][112];
    const int slot = slotmap[(unsigned)(keys[k] & 0xffffffffull)];
    const float4 c = cand[slot];
    const float x = c.x, y = c.y, s = c.z;
    // orientation: Haar responses of side 4s within radius 6s, step s,
    // Gaussian sigma 2s
    const int h4 = even_size(4.f * s);
    int m = 0;
    for (int b = -5; b <= 5; ++b)
        for (int a = -5; a <= 5; ++a) {
            if (a * a + b * b >= 36) continue;
            if ((m & 31) == lane) {
                float dx, dy;
                haar(it, __float2int_rn(x + a * s), __float2int_rn(y + b * s), h4, dx, dy);
                const float g = expf(-(float)(a * a + b * b) / 8.f);
                dx *= g;
                dy *= g;
                float ang = atan2f(dy, dx);
                if (ang < 0.f) ang += 6.2831853f;
                s_dx[wib][m] = dx;
                s_dy[wib][m] = dy;
                s_ang[wib][m] = ang;
            }
            ++m;
        }
    __syncwarp();
    // 72 windows of pi/3 starting every 5 degrees; the longest summed vector
    float best = -1.f, bx = 0.f, by = 0.f;
    int bw = 0;
    for (int w = lane; w < 72; w += 32) {
        const float start = (float)w * (6.2831853f / 72.f);
        float sx = 0.f, sy = 0.f;
        for (int q = 0; q < m; ++q) {
            float d = s_ang[wib][q] - start;
            if (d < 0.f) d += 6.2831853f;
            if (d < 1.0471976f) {
                sx += s_dx[wib][q];
                sy += s_dy[wib][q];
            }
        }
        const float mag = sx * sx + sy * sy;
        if (mag > best) {
            best = mag;
            bx = sx;
            by = sy;
            bw = w;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, best, off);
        const float ox = __shfl_xor_sync(0xffffffffu, bx, off);
        const float oy = __shfl_xor_sync(0xffffffffu, by, off);
        const int ow = __shfl_xor_sync(0xffffffffu, bw, off);
        if (ob > best || (ob == best && ow < bw)) {
            best = ob;
            bx = ox;
            by = oy;
            bw = ow;
        }
    }
    const float theta = atan2f(by, bx);
    const float co = cosf(theta), si = sinf(theta);
    // descriptor: 20 x 20 samples at step s over a 20s square turned by
    // theta, Haar side 2s, Gaussian sigma 3.3s; lanes 2q and 2q + 1 share
    // subregion q (alternate samples)
    const int h2 = even_size(2.f * s);
    const int sub = lane >> 1, sr = sub >> 2, sc = sub & 3;
    float sdx = 0.f, sdy = 0.f, sax = 0.f, say = 0.f;
    for (int t = lane & 1; t < 25; t += 2) {
        const int kk = sc * 5 + t % 5, mm = sr * 5 + t / 5;
        const float u = ((float)kk - 9.5f) * s, v = ((float)mm - 9.5f) * s;
        const int px = __float2int_rn(x + u * co - v * si), py = __float2int_rn(y + u * si + v * co);
        float dx, dy;
        haar(it, px, py, h2, dx, dy);
        const float du = (float)kk - 9.5f, dv = (float)mm - 9.5f;
        const float g = expf(-(du * du + dv * dv) / (2.f * 3.3f * 3.3f));
        const float rx = g * (dx * co + dy * si), ry = g * (-dx * si + dy * co);
        sdx += rx;
        sdy += ry;
        sax += fabsf(rx);
        say += fabsf(ry);
    }
    sdx += __shfl_xor_sync(0xffffffffu, sdx, 1);
    sdy += __shfl_xor_sync(0xffffffffu, sdy, 1);
    sax += __shfl_xor_sync(0xffffffffu, sax, 1);
    say += __shfl_xor_sync(0xffffffffu, say, 1);
    float sq = (lane & 1) ? 0.f : sdx * sdx + sdy * sdy + sax * sax + say * say;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, off);
    const float inv = sq > 0.f ? 1.f / sqrtf(sq) : 0.f;
    if (!(lane & 1)) {
        float* dst = desc + (size_t)k * kKeyDesc + 4 * sub;
        dst[0] = sdx * inv;
        dst[1] = sdy * inv;
        dst[2] = sax * inv;
        dst[3] = say * inv;
    }
    if (lane == 0) kp[k] = make_float4(x, y, s, theta);
}

// --------------------------------------------------------- back-projection

// Frame::InterpDepth (Core/Frame.cc:93-129), including its bounds test with
// rows and columns exchanged (plus a test that keeps the reads in the image).
__device__ float interp_depth(const float* d, int dp, int W, int H, float x, float y, float cutoff) {
    const float nan = qnan();
    if (x <= 1 || y <= 1 || y >= (float)(W - 1) || x >= (float)(H - 1)) return nan;
    const float cx = fs(x, floorf(x)), cy = fs(y, floorf(y));
    const int x0 = (int)floorf(x), x1 = (int)ceilf(x), y0 = (int)floorf(y), y1 = (int)ceilf(y);
    if (x1 >= W || y1 >= H) return nan;
    auto ok = [&](float v) { return !(isnan(v) || v < 0.3 || v > cutoff); };
    const float d00 = d[(size_t)y0 * dp + x0];
    if (!ok(d00)) return nan;
    const float d10 = d[(size_t)y1 * dp + x0];
    if (!ok(d10)) return nan;
    const float d01 = d[(size_t)y0 * dp + x1];
    if (!ok(d01)) return nan;
    const float d11 = d[(size_t)y1 * dp + x1];
    if (!ok(d11)) return nan;
    const float d0 = fa(fm(d01, cx), fm(d00, fs(1.f, cx)));
    const float d1 = fa(fm(d11, cx), fm(d10, fs(1.f, cx)));
    const float fin = fa(fm(fs(1.f, cy), d0), fm(cy, d1));
    return fabsf(fs(fin, d00)) <= 0.005 ? fin : nan;
}

// Frame::InterpNormal (Core/Frame.cc:131-163), the same bounds test.
__device__ float4 interp_normal(const float4* n, int np, int W, int H, float x, float y) {
    const float nan = qnan();
    if (x <= 1 || y <= 1 || y >= (float)(W - 1) || x >= (float)(H - 1)) return make_float4(nan, nan, nan, nan);
    const float cx = fs(x, floorf(x)), cy = fs(y, floorf(y));
    const int x0 = (int)floorf(x), x1 = (int)ceilf(x), y0 = (int)floorf(y), y1 = (int)ceilf(y);
    if (x1 >= W || y1 >= H) return make_float4(nan, nan, nan, nan);
    const float4 d00 = n[(size_t)y0 * np + x0], d10 = n[(size_t)y1 * np + x0];
    const float4 d01 = n[(size_t)y0 * np + x1], d11 = n[(size_t)y1 * np + x1];
    const float ocx = fs(1.f, cx), ocy = fs(1.f, cy);
    auto lerp4 = [&](float4 a, float wa, float4 b, float wb) {
        return make_float4(fa(fm(a.x, wa), fm(b.x, wb)), fa(fm(a.y, wa), fm(b.y, wb)), fa(fm(a.z, wa), fm(b.z, wb)),
                           fa(fm(a.w, wa), fm(b.w, wb)));
    };
    const float4 d0 = lerp4(d01, cx, d00, ocx), d1 = lerp4(d11, cx, d10, ocx);
    const float4 f = lerp4(d0, ocy, d1, cy);
    const float ex = fs(f.x, d00.x), ey = fs(f.y, d00.y), ez = fs(f.z, d00.z), ew = fs(f.w, d00.w);
    const float nn = fsq(fa(fa(fa(fm(ex, ex), fm(ey, ey)), fm(ez, ez)), fm(ew, ew)));
    return (double)nn <= 0.1 ? f : make_float4(nan, nan, nan, nan);
}

// Frame::ExtractKeyPoints' filter (Core/Frame.cc:186-205): keeps the key
// points with a depth in (0.3, cutoff) and a normal, as camera-space
// points, in key-point order (one CTA).
__global__ void __launch_bounds__(1024) k_backproject(const float4* __restrict__ kp, const float* __restrict__ kdesc,
                                                      int n, const float* __restrict__ depth, int dp,
                                                      const float4* __restrict__ nmap, int np, int W, int H, Intr k,
                                                      float cutoff, KeySet out, int* __restrict__ n_out) {
    __shared__ int warp_tot[32];
    __shared__ int base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k0 = 0; k0 < n; k0 += 1024) {
        const int i = k0 + threadIdx.x;
        bool keep = false;
        float4 pt = make_float4(0.f, 0.f, 0.f, 1.f), nl = pt;
        float4 key = make_float4(0.f, 0.f, 0.f, 0.f);
        if (i < n) {
            key = kp[i];
            const float d = interp_depth(depth, dp, W, H, key.x, key.y, cutoff);
            if (!isnan(d) && d > 0.3 && d < cutoff) {
                nl = interp_normal(nmap, np, W, H, key.x, key.y);
                if (!isnan(nl.x)) {
                    keep = true;
                    pt = make_float4(fd(fm(d, fs(key.x, k.cx)), k.fx), fd(fm(d, fs(key.y, k.cy)), k.fy), d, 1.f);
                }
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) warp_tot[w] = __popc(bal);
        __syncthreads();
        int before = base;
        for (int q = 0; q < w; ++q) before += warp_tot[q];
        const int o = before + __popc(bal & ((1u << lane) - 1u));
        if (keep && o < out.cap) {
            out.kp[o] = key;
            out.pt[o] = pt;
            out.nrm[o] = nl;
            for (int q = 0; q < kKeyDesc; ++q) out.desc[(size_t)o * kKeyDesc + q] = kdesc[(size_t)i * kKeyDesc + q];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int q = 0; q < 32; ++q) t += warp_tot[q];
            base += t;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *n_out = min(base, out.cap);
}

// ----------------------------------------------------------------- matching

// Two nearest train descriptors of each query by L2 distance (BFMatcher
// knnMatch with k = 2).  One CTA of 256 threads per 32 queries: train tiles
// of 64 descriptors in shared memory, 8 threads per query each taking every
// 8th train of the tile, best two merged in a fixed order.  Distances are
// square roots of the sums of squares in descriptor order; ties go to the
// lower train index.
__global__ void __launch_bounds__(256) k_match2(const float* __restrict__ Q, int nq, const float* __restrict__ T,
                                                int nt, int2* __restrict__ idx, float2* __restrict__ dist) {
    __shared__ float sq[32][kKeyDesc + 1];
    __shared__ float st[64][kKeyDesc + 1];
    const int q0 = blockIdx.x * 32;
    for (int t = threadIdx.x; t < 32 * kKeyDesc; t += 256) {
        const int r = t / kKeyDesc, c = t % kKeyDesc;
        sq[r][c] = (q0 + r < nq) ? Q[(size_t)(q0 + r) * kKeyDesc + c] : 0.f;
    }
    const int qi = threadIdx.x >> 3, part = threadIdx.x & 7;
    float b1 = INFINITY, b2 = INFINITY;
    int i1 = -1, i2 = -1;
    for (int t0 = 0; t0 < nt; t0 += 64) {
        __syncthreads();
        for (int t = threadIdx.x; t < 64 * kKeyDesc; t += 256) {
            const int r = t / kKeyDesc, c = t % kKeyDesc;
            st[r][c] = (t0 + r < nt) ? T[(size_t)(t0 + r) * kKeyDesc + c] : 0.f;
        }
        __syncthreads();
        for (int r = part; r < 64 && t0 + r < nt; r += 8) {
            float acc = 0.f;
#pragma unroll 16
            for (int c = 0; c < kKeyDesc; ++c) {
                const float d = sq[qi][c] - st[r][c];
                acc = fmaf(d, d, acc);
            }
            const int ti = t0 + r;
            if (acc < b1) {
                b2 = b1;
                i2 = i1;
                b1 = acc;
                i1 = ti;
            } else if (acc < b2) {
                b2 = acc;
                i2 = ti;
            }
        }
    }
    // merge the 8 partial results of each query (xor tree: fixed order)
    auto less = [](float a, int ia, float b, int ib) { return a < b || (a == b && ia >= 0 && (ib < 0 || ia < ib)); };
#pragma unroll
    for (int off = 1; off < 8; off <<= 1) {
        const float ob1 = __shfl_xor_sync(0xffffffffu, b1, off), ob2 = __shfl_xor_sync(0xffffffffu, b2, off);
        const int oi1 = __shfl_xor_sync(0xffffffffu, i1, off), oi2 = __shfl_xor_sync(0xffffffffu, i2, off);
        float c1, c2;
        int j1, j2;
        if (less(b1, i1, ob1, oi1)) {
            c1 = b1;
            j1 = i1;
            if (less(b2, i2, ob1, oi1)) {
                c2 = b2;
                j2 = i2;
            } else {
                c2 = ob1;
                j2 = oi1;
            }
        } else {
            c1 = ob1;
            j1 = oi1;
            if (less(b1, i1, ob2, oi2)) {
                c2 = b1;
                j2 = i1;
            } else {
                c2 = ob2;
                j2 = oi2;
            }
        }
        b1 = c1;
        i1 = j1;
        b2 = c2;
        i2 = j2;
    }
    if (part == 0 && q0 + qi < nq) {
        idx[q0 + qi] = make_int2(i1, i2);
        dist[q0 + qi] = make_float2(sqrtf(b1), sqrtf(b2));
    }
}

// ------------------------------------------------------------------ launch

int key_scratch_carve(void* base, size_t bytes, int W, int H, KeyScratch& ks) {
    char* p = (char*)base;
    char* end = p + bytes;
    auto take = [&](size_t n) -> char* {
        char* q = p;
        p += (n + 255) & ~(size_t)255;
        return q;
    };
    ks.W = W;
    ks.H = H;
    ks.integral = (uint32_t*)take((size_t)(W + 1) * (H + 1) * 4);
    for (int o = 0; o < kSurfOctaves; ++o) {
        ks.ow[o] = W >> o;
        ks.oh[o] = H >> o;
        ks.det[o] = (float*)take((size_t)kSurfLayers * ks.ow[o] * ks.oh[o] * 4);
    }
    ks.cand = (float4*)take((size_t)kSurfMaxCand * 16);
    ks.keys = (unsigned long long*)take((size_t)kSurfMaxCand * 8);
    size_t codes = 0;
    for (int o = 0; o < kSurfOctaves; ++o) codes += (size_t)(kSurfLayers - 2) * ks.ow[o] * ks.oh[o];
    ks.slotmap = (int*)take(codes * 4);
    ks.counter = (int*)take(64);
    ks.max_keys = W * H / 100;
    ks.kp = (float4*)take((size_t)ks.max_keys * 16);
    ks.desc = (float*)take((size_t)ks.max_keys * 4 * kKeyDesc + 4);
    return p <= end ? FB_OK : FB_ENOMEM;
}

int launch_surf(const uint8_t* gray, int gp, float threshold, const KeyScratch& ks, int* n_keys, cudaStream_t st) {
    const int W = ks.W, H = ks.H;
    *n_keys = 0;
    k_integral_rows<<<H, 256, 0, st>>>(gray, gp, W, H, ks.integral);
    k_integral_cols<<<(W + 1 + 31) / 32, dim3(32, 16), 0, st>>>(ks.integral, W, H);
    const Integral it{ks.integral, W, H};
    int code0[kSurfOctaves], code = 0;
    for (int o = 0; o < kSurfOctaves; ++o) {
        code0[o] = code;
        code += (kSurfLayers - 2) * ks.ow[o] * ks.oh[o];
        dim3 b(32, 8), g((ks.ow[o] + 31) / 32, (ks.oh[o] + 7) / 8);
        k_hessian<<<g, b, 0, st>>>(it, ks.det[o], ks.ow[o], ks.oh[o], o);
    }
    // candidates; a set larger than the buffer is found again with a doubled
    // threshold (which candidates are kept must not depend on arrival order)
    int count = 0;
    float thr = threshold;
    for (int attempt = 0; attempt < 8; ++attempt) {
        if (cudaMemsetAsync(ks.counter, 0, 4, st) != cudaSuccess) return FB_ECUDA;
        for (int o = 0; o < kSurfOctaves; ++o) {
            dim3 b(32, 8), g((ks.ow[o] + 31) / 32, (ks.oh[o] + 7) / 8);
            k_extrema<<<g, b, 0, st>>>(ks.det[o], ks.ow[o], ks.oh[o], o, code0[o], thr, ks.cand, ks.keys, ks.slotmap,
                                       ks.counter, kSurfMaxCand);
        }
        if (cudaMemcpyAsync(&count, ks.counter, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) return FB_ECUDA;
        if (cudaStreamSynchronize(st) != cudaSuccess) return FB_ECUDA;
        if (count <= kSurfMaxCand) break;
        thr *= 2.f;
    }
    if (count > kSurfMaxCand) count = kSurfMaxCand;
    if (count == 0) return cudaGetLastError() == cudaSuccess ? FB_OK : FB_ECUDA;
    int n = 1;
    while (n < count) n <<= 1;
    // the sort's shared memory beyond the default limit: once per device
    {
        static std::mutex lock;
        static bool done[64] = {};
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return FB_ECUDA;
        std::lock_guard<std::mutex> guard(lock);
        if (!done[dev]) {
            if (cudaFuncSetAttribute(k_sort_keys, cudaFuncAttributeMaxDynamicSharedMemorySize, kSurfMaxCand * 8) !=
                cudaSuccess)
                return FB_ECUDA;
            done[dev] = true;
        }
    }
    k_sort_keys<<<1, 1024, (size_t)n * 8, st>>>(ks.keys, count, n);
    const int nk = count < ks.max_keys ? count : ks.max_keys;
    k_describe<<<(nk + 7) / 8, 256, 0, st>>>(it, ks.cand, ks.keys, ks.slotmap, nk, ks.kp, ks.desc);
    *n_keys = nk;
    return cudaGetLastError() == cudaSuccess ? FB_OK : FB_ECUDA;
}

int launch_backproject(const KeyScratch& ks, int n, const float* depth, int dp, const float4* nmap, int np,
                       const Intr& k, float cutoff, const KeySet& out, int* d_n, cudaStream_t st) {
    k_backproject<<<1, 1024, 0, st>>>(ks.kp, ks.desc, n, depth, dp, nmap, np, ks.W, ks.H, k, cutoff, out, d_n);
    return cudaGetLastError() == cudaSuccess ? FB_OK : FB_ECUDA;
}

int launch_match2(const float* q, int nq, const float* t, int nt, int2* idx, float2* dist, cudaStream_t st) {
    if (nq <= 0) return FB_OK;
    k_match2<<<(nq + 31) / 32, 256, 0, st>>>(q, nq, t, nt, idx, dist);
    return cudaGetLastError() == cudaSuccess ? FB_OK : FB_ECUDA;
}

// ------------------------------------------------------------- pose solver
//
// Solver::PoseEstimate (Optimization/Solver.cc:6-186): RANSAC over triples
// of matched 3-D points, each hypothesis the least-squares rotation and
// translation of the triple (Kabsch: R = U V^T from the SVD U S V^T of the
// cross-covariance), inliers within 5 cm, a refit on the inliers of every
// better hypothesis, early exit after 20 iterations at 95 % confidence, a
// final refit whose rotation must be proper, and (checkAngle) the reference's
// plausibility test of the motion.  The reference seeds rand() from the
// clock; here the sample stream is a splitmix64 sequence from the caller's
// seed, so a call is reproducible.

namespace {

uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Eigenvalues (descending) and eigenvectors (columns of V) of a symmetric
// 3x3 matrix by cyclic Jacobi rotations.
void jacobi_eig3(const double S[3][3], double w[3], double V[3][3]) {
    double A[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            A[i][j] = S[i][j];
            V[i][j] = i == j;
        }
    for (int sweep = 0; sweep < 64; ++sweep) {
        const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        const double diag = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
        if (off <= 1e-30 * diag || off == 0.0) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (A[p][q] == 0.0) continue;
                const double theta = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    const double akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - s * akq;
                    A[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    const double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - s * aqk;
                    A[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
    int order[3] = {0, 1, 2};
    for (int i = 0; i < 3; ++i)
        for (int j = i + 1; j < 3; ++j)
            if (A[order[j]][order[j]] > A[order[i]][order[i]]) std::swap(order[i], order[j]);
    double Vs[3][3];
    for (int c = 0; c < 3; ++c) {
        w[c] = A[order[c]][order[c]];
        for (int r = 0; r < 3; ++r) Vs[r][c] = V[r][order[c]];
    }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) V[r][c] = Vs[r][c];
}

void cross3d(const double a[3], const double b[3], double o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// R = U V^T from the SVD of H.  The singular vectors of a singular value
// below 1e-12 of the largest are completed as cross products, so a rank-2 H
// -- any three points -- gives a proper rotation.
void kabsch(const double H[3][3], double R[3][3]) {
    double HtH[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) HtH[i][j] = H[0][i] * H[0][j] + H[1][i] * H[1][j] + H[2][i] * H[2][j];
    double w[3], V[3][3];
    jacobi_eig3(HtH, w, V);
    double v[3][3], u[3][3];
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) v[c][r] = V[r][c];
    const double s0 = std::sqrt(std::max(w[0], 0.0));
    for (int c = 0; c < 3; ++c) {
        const double sc = std::sqrt(std::max(w[c], 0.0));
        if (c < 2 || sc > 1e-12 * s0) {
            if (!(sc > 1e-300)) {
                // rank below 2: no unique rotation; the identity
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) R[i][j] = i == j;
                return;
            }
            for (int r = 0; r < 3; ++r) u[c][r] = (H[r][0] * v[c][0] + H[r][1] * v[c][1] + H[r][2] * v[c][2]) / sc;
        } else {
            cross3d(u[0], u[1], u[2]);
            cross3d(v[0], v[1], v[2]);
        }
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[i][j] = u[0][i] * v[0][j] + u[1][i] * v[1][j] + u[2][i] * v[2][j];
}

double det3(const double R[3][3]) {
    return R[0][0] * (R[1][1] * R[2][2] - R[1][2] * R[2][1]) - R[0][1] * (R[1][0] * R[2][2] - R[1][2] * R[2][0]) +
           R[0][2] * (R[1][0] * R[2][1] - R[1][1] * R[2][0]);
}

// the norm of the sines of Eigen's eulerAngles(0, 1, 2) of R (the same for
// either of the two equivalent angle triples)
double euler_sin_norm3(const double R[3][3]) {
    const double a = std::atan2(-R[1][2], R[2][2]);
    const double b = std::atan2(R[0][2], std::sqrt(R[0][0] * R[0][0] + R[0][1] * R[0][1]));
    const double c = std::atan2(-R[0][1], R[0][0]);
    const double sa = std::sin(a), sb = std::sin(b), sc = std::sin(c);
    return std::sqrt(sa * sa + sb * sb + sc * sc);
}

// R, t fitted to the points with outlier[i] == 0; false when there are none
bool fit_inliers(const double* src, const double* ref, int n, const uint8_t* outlier, double R[3][3], double t[3]) {
    double sm[3] = {0, 0, 0}, rm[3] = {0, 0, 0};
    int N = 0;
    for (int i = 0; i < n; ++i)
        if (!outlier[i]) {
            for (int k = 0; k < 3; ++k) {
                sm[k] += src[3 * i + k];
                rm[k] += ref[3 * i + k];
            }
            ++N;
        }
    if (N == 0) return false;
    for (int k = 0; k < 3; ++k) {
        sm[k] /= N;
        rm[k] /= N;
    }
    double H[3][3] = {};
    for (int i = 0; i < n; ++i)
        if (!outlier[i])
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) H[a][b] += (src[3 * i + a] - sm[a]) * (ref[3 * i + b] - rm[b]);
    kabsch(H, R);
    for (int k = 0; k < 3; ++k) t[k] = sm[k] - (R[k][0] * rm[0] + R[k][1] * rm[1] + R[k][2] * rm[2]);
    return true;
}

}  // namespace

bool pose_estimate(const double* src, const double* ref, int n, int iterations, bool check_angle, uint64_t seed,
                   double T[16], uint8_t* outlier) {
    double Rb[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, tb[3] = {0, 0, 0};
    int best = 0, it = 0;
    float ratio = 0.f, confidence = 0.f;
    const float thresh_inlier = 0.05f;
    for (int i = 0; i < 16; ++i) T[i] = i % 5 == 0;
    if (n < 3) return false;
    for (int i = 0; i < n; ++i) outlier[i] = 1;
    uint64_t rng = seed;
    int attempts = 0;
    while (it < iterations && attempts++ < 64 * iterations) {
        int sidx[3];
        for (int k = 0; k < 3; ++k) sidx[k] = (int)(splitmix64(rng) % (uint64_t)n);
        const bool bad = sidx[0] == sidx[1] || sidx[1] == sidx[2] || sidx[2] == sidx[0];
        const double* sa = src + 3 * sidx[0];
        const double* sb = src + 3 * sidx[1];
        const double* sc = src + 3 * sidx[2];
        const double* ra = ref + 3 * sidx[0];
        const double* rb = ref + 3 * sidx[1];
        const double* rc = ref + 3 * sidx[2];
        double u[3], v[3], w[3];
        for (int k = 0; k < 3; ++k) {
            u[k] = sb[k] - sa[k];
            v[k] = sa[k] - sc[k];
        }
        cross3d(u, v, w);
        const float src_d = (float)std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        for (int k = 0; k < 3; ++k) {
            u[k] = rb[k] - ra[k];
            v[k] = ra[k] - rc[k];
        }
        cross3d(u, v, w);
        const float ref_d = (float)std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        if (bad || src_d < 1e-6 || ref_d < 1e-6) {
            ++it;
            continue;
        }
        double sm[3], rm[3], H[3][3] = {};
        for (int k = 0; k < 3; ++k) {
            sm[k] = (sa[k] + sb[k] + sc[k]) / 3;
            rm[k] = (ra[k] + rb[k] + rc[k]) / 3;
        }
        const double* S3[3] = {sa, sb, sc};
        const double* R3[3] = {ra, rb, rc};
        for (int q = 0; q < 3; ++q)
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) H[a][b] += (S3[q][a] - sm[a]) * (R3[q][b] - rm[b]);
        double R[3][3], t[3];
        kabsch(H, R);
        if (det3(R) < 0) continue;   // as the reference: not counted as an iteration
        for (int k = 0; k < 3; ++k) t[k] = sm[k] - (R[k][0] * rm[0] + R[k][1] * rm[1] + R[k][2] * rm[2]);
        int inl = 0;
        for (int i = 0; i < n; ++i) {
            const double* p = src + 3 * i;
            const double* q = ref + 3 * i;
            double d2 = 0;
            for (int k = 0; k < 3; ++k) {
                const double e = p[k] - (R[k][0] * q[0] + R[k][1] * q[1] + R[k][2] * q[2] + t[k]);
                d2 += e * e;
            }
            outlier[i] = !(std::sqrt(d2) <= thresh_inlier);
            inl += !outlier[i];
        }
        if (inl > best) {
            fit_inliers(src, ref, n, outlier, Rb, tb);
            best = inl;
            ratio = (float)inl / n;
            confidence = 1.f - (float)std::pow(1.0 - std::pow((double)ratio, 3.0), (double)(it + 1));
            if (it >= 20 && confidence >= 0.95f) break;
        }
        ++it;
    }
    // the loop's best pose is the result (Solver.cc:136-137) ...
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) T[4 * r + c] = Rb[r][c];
        T[4 * r + 3] = tb[r];
    }
    // ... checked by a refit on its inliers (added to the last hypothesis'
    // flags, Solver.cc:139-176) that must be a proper rotation
    for (int i = 0; i < n; ++i) {
        const double* p = src + 3 * i;
        const double* q = ref + 3 * i;
        double d2 = 0;
        for (int k = 0; k < 3; ++k) {
            const double e = p[k] - (Rb[k][0] * q[0] + Rb[k][1] * q[1] + Rb[k][2] * q[2] + tb[k]);
            d2 += e * e;
        }
        if (std::sqrt(d2) <= thresh_inlier) outlier[i] = 0;
    }
    double Rf[3][3], tf[3];
    if (!fit_inliers(src, ref, n, outlier, Rf, tf)) return true;   // no inliers: the reference's checks see NaN
    if (det3(Rf) < 0) return false;
    if (check_angle && confidence < 0.8f) {
        const double tn = std::sqrt(tf[0] * tf[0] + tf[1] * tf[1] + tf[2] * tf[2]);
        if (euler_sin_norm3(Rf) >= 0.2 || tn >= 0.1) return false;
    }
    return true;
}

}  // namespace fb
