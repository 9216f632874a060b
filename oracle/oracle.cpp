// ORACLE / TEST INFRASTRUCTURE ONLY -- see oracle.hpp for what this file is,
// its two precisions, and who may use it.  Each function cites the reference
// code it restates.  Storage between stages uses the reference's types (float
// maps, u8 images, float TSDF voxels); arithmetic inside a stage uses R.
#include "oracle.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <tuple>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "se3.hpp"

namespace {

const float kNaN = std::numeric_limits<float>::quiet_NaN();

template <class R> struct V3 { R x, y, z; };
template <class R> struct V4 { R x, y, z, w; };
template <class R> struct M3 { V3<R> r0, r1, r2; };

// VectorMath.h:191-205 -- float3*float3 and float3*float4 dot over xyz,
// float4*float4 over all four lanes, float4*float3 adds a.w.
template <class R> inline R dot3(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline R dot4(V4<R> a, V4<R> b) {
    return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}
template <class R> inline V3<R> xyz(V4<R> a) { return {a.x, a.y, a.z}; }
template <class R> inline V3<R> add(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> sub(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> mul(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline V3<R> mul(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> inline V3<R> divs(V3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> inline V3<R> neg(V3<R> a) { return {-a.x, -a.y, -a.z}; }
// VectorMath.h:308-312
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> inline R norm3(V3<R> a) { return std::sqrt(dot3(a, a)); }
template <class R> inline R norm4(V4<R> a) { return std::sqrt(dot4(a, a)); }
template <class R> inline V3<R> normalised3(V3<R> a) { return divs(a, norm3(a)); }
template <class R> inline V4<R> normalised4(V4<R> a) {
    R n = norm4(a);
    return {a.x / n, a.y / n, a.z / n, a.w / n};
}
// Matrix3f * float3 / float4 (VectorMath.h:364-370): row dots over xyz
template <class R> inline V3<R> mv(const M3<R>& m, V3<R> a) {
    return {dot3(m.r0, a), dot3(m.r1, a), dot3(m.r2, a)};
}
template <class R> inline bool isnan_(R v) { return std::isnan(v); }

// Frame::GpuRotation / GpuInvRotation / GpuTranslation (Core/Frame.cc:275-294):
// double pose entries rounded to float.
template <class R> M3<R> rot(const double* T) {
    return {{(R)(float)T[0], (R)(float)T[1], (R)(float)T[2]},
            {(R)(float)T[4], (R)(float)T[5], (R)(float)T[6]},
            {(R)(float)T[8], (R)(float)T[9], (R)(float)T[10]}};
}
template <class R> M3<R> rot_inv(const double* T) {
    return {{(R)(float)T[0], (R)(float)T[4], (R)(float)T[8]},
            {(R)(float)T[1], (R)(float)T[5], (R)(float)T[9]},
            {(R)(float)T[2], (R)(float)T[6], (R)(float)T[10]}};
}
template <class R> V3<R> trans(const double* T) {
    return {(R)(float)T[3], (R)(float)T[7], (R)(float)T[11]};
}

inline V4<float> ld4(const float* p, size_t i) { return {p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]}; }
template <class R> inline V4<R> cv4(V4<float> a) { return {(R)a.x, (R)a.y, (R)a.z, (R)a.w}; }
inline void st4(float* p, size_t i, float x, float y, float z, float w) {
    p[4 * i] = x; p[4 * i + 1] = y; p[4 * i + 2] = z; p[4 * i + 3] = w;
}

// ---------------------------------------------------------------- pyramid --

// FilterDepthKernel (Tracking/Pyrdown.cu:3-41; host Pyrdown.cu:43-54)
template <class R>
void filter_depth(int W, int H, const uint16_t* d, float scale, float cutoff, float* raw,
                  float* filt) {
    const R inv = (R)(float)(1.0 / (double)scale);
    const R sigSpace = (R)(float)(0.5 / (4 * 4)), sigRange = (R)(float)(0.5 / (0.5 * 0.5));
    const R cut = (R)cutoff;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            R center = (R)d[y * W + x] * inv;
            raw[y * W + x] = center < cut ? (float)center : kNaN;
            if (isnan_(center)) { filt[y * W + x] = kNaN; continue; }
            int tx = std::min(x - 2 + 5, W - 1), ty = std::min(y - 2 + 5, H - 1);
            R sum1 = 0, sum2 = 0;
            for (int cy = std::max(y - 2, 0); cy < ty; ++cy)
                for (int cx = std::max(x - 2, 0); cx < tx; ++cx) {
                    R val = (R)d[cy * W + cx] * inv;
                    R space2 = (R)((x - cx) * (x - cx) + (y - cy) * (y - cy));
                    R color2 = (center - val) * (center - val);
                    R weight = std::exp(-(space2 * sigSpace + color2 * sigRange));
                    sum1 += val * weight;
                    sum2 += weight;
                }
            R fin = sum1 / sum2;
            filt[y * W + x] = fin < cut ? (float)fin : kNaN;
        }
}

// ImageToIntensityKernel (Tracking/Pyrdown.cu:183-193): double arithmetic,
// truncated; uchar3 lanes are (x, y, z) = (R, G, B)
void intensity(int W, int H, const uint8_t* rgb, uint8_t* gray) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < W * H; ++i) {
        const uint8_t* v = rgb + 3 * i;
        int value = (int)(0.2125 * v[1] + 0.7154 * v[0] + 0.0721 * v[2]);
        gray[i] = (uint8_t)value;
    }
}

// gaussKernel (Tracking/Pyrdown.cu:127-133)
const float kGauss[25] = {1, 4, 6, 4, 1, 4, 16, 24, 16, 4, 6, 24, 36, 24, 6,
                          4, 16, 24, 16, 4, 1, 4, 6, 4, 1};

// PyrDownGaussKernel (Tracking/Pyrdown.cu:134-158): 5x5 window clipped at
// [max(0,2x-2), min(2x+3, cols-1)), weights indexed mirrored from the clipped
// end, NaN taps skipped, integer weight count, cast truncates.
template <class R, class T>
void pyrdown(int W, int H, const T* src, T* dst) {
    const int w2 = W / 2, h2 = H / 2;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h2; ++y)
        for (int x = 0; x < w2; ++x) {
            int tx = std::min(2 * x - 2 + 5, W - 1), ty = std::min(2 * y - 2 + 5, H - 1);
            R sum = 0;
            int count = 0;
            for (int cy = std::max(0, 2 * y - 2); cy < ty; ++cy)
                for (int cx = std::max(0, 2 * x - 2); cx < tx; ++cx) {
                    float s = (float)src[cy * W + cx];
                    if (!std::isnan(s)) {
                        float k = kGauss[(ty - cy - 1) * 5 + (tx - cx - 1)];
                        sum += (R)src[cy * W + cx] * (R)k;
                        count += (int)k;
                    }
                }
            R q = sum / (R)count;
            dst[y * w2 + x] = (T)q;
        }
}

// ComputeVMapKernel (Tracking/Pyrdown.cu:56-91); invalid pixels keep z and
// get NaN in x (the reference leaves y and w unset; NaN is written here).
template <class R>
void vmap(int W, int H, const float* depth, float fx, float fy, float cx, float cy, float cutoff,
          float* out) {
    const R invfx = (R)(float)(1.0 / (double)fx), invfy = (R)(float)(1.0 / (double)fy);
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            float zf = depth[y * W + x];
            R z = (R)zf;
            if (!std::isnan(zf) && (double)zf > 0.1 && zf < cutoff) {
                R vx = z * ((R)x - (R)cx) * invfx;
                R vy = z * ((R)y - (R)cy) * invfy;
                st4(out, y * W + x, (float)vx, (float)vy, zf, 1.0f);
            } else {
                st4(out, y * W + x, kNaN, kNaN, zf, kNaN);
            }
        }
}

// ComputeNMapKernel (Tracking/Pyrdown.cu:93-114)
template <class R>
void nmap(int W, int H, const float* vm, float* out) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            size_t i = (size_t)y * W + x;
            if (x == W - 1 || y == H - 1) { st4(out, i, kNaN, kNaN, kNaN, kNaN); continue; }
            V4<R> c = cv4<R>(ld4(vm, i)), r = cv4<R>(ld4(vm, i + 1)), d = cv4<R>(ld4(vm, i + W));
            if (!isnan_(c.x) && !isnan_(r.x) && !isnan_(d.x)) {
                V3<R> a = {r.x - c.x, r.y - c.y, r.z - c.z};
                V3<R> b = {d.x - c.x, d.y - c.y, d.z - c.z};
                V3<R> n = normalised3(cross(a, b));
                st4(out, i, (float)n.x, (float)n.y, (float)n.z, 1.0f);
            } else {
                st4(out, i, kNaN, kNaN, kNaN, kNaN);
            }
        }
}

// ComputeDerivativeImageKernel (Tracking/Pyrdown.cu:207-237): 3x3 Sobel with
// the kernel index running 8 -> 0 over the clipped window
void derivative(int W, int H, const uint8_t* img, int16_t* dx, int16_t* dy) {
    static const float sx[9] = {1, 0, -1, 2, 0, -2, 1, 0, -1};
    static const float sy[9] = {1, 2, 1, 0, 0, 0, -1, -2, -1};
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            float dxv = 0, dyv = 0;
            int k = 8;
            for (int j = std::max(y - 1, 0); j <= std::min(y + 1, H - 1); ++j)
                for (int i = std::max(x - 1, 0); i <= std::min(x + 1, W - 1); ++i) {
                    dxv += img[j * W + i] * sx[k];
                    dyv += img[j * W + i] * sy[k];
                    --k;
                }
            dx[y * W + x] = (int16_t)dxv;
            dy[y * W + x] = (int16_t)dyv;
        }
}

// ResizeMapKernel (Tracking/Pyrdown.cu:251-279): 2x2 means; the normal mean is
// normalised over all four lanes (w = 1 included).  Written for the
// destination size only (the reference checks the source size).
template <class R>
void resize_map(int W, int H, const float* vs, const float* ns, float* vd, float* nd) {
    const int w2 = W / 2, h2 = H / 2;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h2; ++y)
        for (int x = 0; x < w2; ++x) {
            size_t i00 = (size_t)(2 * y) * W + 2 * x, i01 = i00 + 1, i10 = i00 + W, i11 = i10 + 1;
            size_t o = (size_t)y * w2 + x;
            V4<R> v00 = cv4<R>(ld4(vs, i00)), v01 = cv4<R>(ld4(vs, i01)), v10 = cv4<R>(ld4(vs, i10)),
                  v11 = cv4<R>(ld4(vs, i11));
            if (isnan_(v00.x) || isnan_(v01.x) || isnan_(v10.x) || isnan_(v11.x)) {
                st4(vd, o, kNaN, kNaN, kNaN, kNaN);
            } else {
                R f = 4;
                st4(vd, o, (float)((v00.x + v01.x + v10.x + v11.x) / f),
                    (float)((v00.y + v01.y + v10.y + v11.y) / f),
                    (float)((v00.z + v01.z + v10.z + v11.z) / f),
                    (float)((v00.w + v01.w + v10.w + v11.w) / f));
            }
            V4<R> n00 = cv4<R>(ld4(ns, i00)), n01 = cv4<R>(ld4(ns, i01)), n10 = cv4<R>(ld4(ns, i10)),
                  n11 = cv4<R>(ld4(ns, i11));
            if (isnan_(n00.x) || isnan_(n01.x) || isnan_(n10.x) || isnan_(n11.x)) {
                st4(nd, o, kNaN, kNaN, kNaN, kNaN);
            } else {
                R f = 4;
                V4<R> m = {(n00.x + n01.x + n10.x + n11.x) / f, (n00.y + n01.y + n10.y + n11.y) / f,
                           (n00.z + n01.z + n10.z + n11.z) / f, (n00.w + n01.w + n10.w + n11.w) / f};
                V4<R> n = normalised4(m);
                st4(nd, o, (float)n.x, (float)n.y, (float)n.z, (float)n.w);
            }
        }
}

// ------------------------------------------------------- normal equations --

template <class R> inline void add_products(const R row[7], double* s) {
    int k = 0;
    for (int i = 0; i < 7; ++i)
        for (int j = i; j < 7; ++j) s[k++] += (double)(row[i] * row[j]);
}

// Per-row partial sums combined in row order: deterministic for any thread count.
template <class F>
void reduce_rows(int H, int nsum, double* out, F&& row_fn) {
    std::vector<double> part((size_t)H * nsum, 0.0);
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < H; ++y) row_fn(y, part.data() + (size_t)y * nsum);
    for (int k = 0; k < nsum; ++k) out[k] = 0;
    for (int y = 0; y < H; ++y)
        for (int k = 0; k < nsum; ++k) out[k] += part[(size_t)y * nsum + k];
}

// ICPReduce::searchPoint / getRow (Tracking/Reduction.cu:227-286) of pixel
// (x, y): the 7-wide point-to-plane row, or false without a correspondence
// (ICPStep's angleThresh 0.6 and distThresh 0.1, Reduction.cu:319-375).
template <class R>
bool icp_pixel(int W, int H, const float* vc, const float* vl, const float* nc, const float* nl, const M3<R>& Rc,
               const M3<R>& Rl, const M3<R>& RlInv, const V3<R>& tc, const V3<R>& tl, float fx, float fy, float cx,
               float cy, int x, int y, R row[7]) {
    const R angleThresh = (R)0.6f, distThresh = (R)0.1f;
    size_t i = (size_t)y * W + x;
    V3<R> vcurr_c = xyz(cv4<R>(ld4(vc, i)));
    if (isnan_(vcurr_c.x) || (double)vcurr_c.z < 1e-3) return false;
    V3<R> vcurr_g = add(mv(Rc, vcurr_c), tc);
    V3<R> vcurr_p = mv(RlInv, sub(vcurr_g, tl));
    R invz = (R)(1.0 / (double)vcurr_p.z);
    int u = (int)((double)(vcurr_p.x * invz * (R)fx + (R)cx) + 0.5);
    int v = (int)((double)(vcurr_p.y * invz * (R)fy + (R)cy) + 0.5);
    if (u < 0 || v < 0 || u >= W || v >= H) return false;
    size_t j = (size_t)v * W + u;
    V3<R> vlast_c = xyz(cv4<R>(ld4(vl, j)));
    V3<R> vlast_g = add(mv(Rl, vlast_c), tl);
    V3<R> ncurr_c = xyz(cv4<R>(ld4(nc, i)));
    V3<R> ncurr_g = mv(Rc, ncurr_c);
    V3<R> nlast_c = xyz(cv4<R>(ld4(nl, j)));
    V3<R> nlast_g = mv(Rl, nlast_c);
    R dist = norm3(sub(vlast_g, vcurr_g));
    R sine = norm3(cross(ncurr_g, nlast_g));
    if (!(sine < angleThresh && dist <= distThresh && !isnan_(ncurr_c.x) && !isnan_(nlast_c.x))) return false;
    V3<R> nlast = mv(RlInv, nlast_g);
    V3<R> vcurr = mv(RlInv, sub(vcurr_g, tl));
    V3<R> vlast = mv(RlInv, sub(vlast_g, tl));
    V3<R> a = neg(nlast), b = cross(nlast, vlast);
    row[0] = a.x; row[1] = a.y; row[2] = a.z; row[3] = b.x; row[4] = b.y; row[5] = b.z;
    row[6] = dot3(neg(nlast), sub(vcurr, vlast));
    return true;
}

// ICPStep (Reduction.cu:319-375): the 29 sums of all pixels' rows.
template <class R>
void icp_step(int W, int H, const float* vc, const float* vl, const float* nc, const float* nl,
              const double* Tc, const double* Tl, float fx, float fy, float cx, float cy,
              double* sums) {
    const M3<R> Rc = rot<R>(Tc), Rl = rot<R>(Tl), RlInv = rot_inv<R>(Tl);
    const V3<R> tc = trans<R>(Tc), tl = trans<R>(Tl);
    reduce_rows(H, 29, sums, [&](int y, double* s) {
        for (int x = 0; x < W; ++x) {
            R row[7];
            if (!icp_pixel<R>(W, H, vc, vl, nc, nl, Rc, Rl, RlInv, tc, tl, fx, fy, cx, cy, x, y, row)) continue;
            add_products(row, s);
            s[28] += 1;
        }
    });
}

// RGBReduction::FindCorresp (Tracking/Reduction.cu:404-451) of pixel (x, y):
// the last-frame pixel and the intensity difference, or false.
struct RgbCorr { int diff; int cx, cy, lx, ly; };

template <class R>
bool rgb_corresp(int W, int H, const uint8_t* gc, const uint8_t* gl, const float* vc, const float* vl,
                 const int16_t* dxm, const int16_t* dym, const M3<R>& Rc, const M3<R>& RlInv, const V3<R>& tc,
                 const V3<R>& tl, float fx, float fy, float cx, float cy, int x, int y, RgbCorr& r) {
    size_t k = (size_t)y * W + x;
    if (!(x >= 5 && x < W - 5 && y >= 5 && y < H - 5)) return false;
    for (int u = std::max(y - 2, 0); u < std::min(y + 2, H); ++u)
        for (int v = std::max(x - 2, 0); v < std::min(x + 2, W); ++v)
            if (!(gc[u * W + v] > 0)) return false;
    int gx = dxm[k], gy = dym[k];
    if (!(std::sqrt((float)(gx * gx + gy * gy)) > 0)) return false;
    V4<R> vcurr = cv4<R>(ld4(vc, k));
    if (isnan_(vcurr.x)) return false;
    V3<R> vcurr_g = add(mv(Rc, xyz(vcurr)), tc);
    V3<R> vcl = mv(RlInv, sub(vcurr_g, tl));
    R pu = (R)fx * vcl.x / vcl.z + (R)cx;
    R pv = (R)fy * vcl.y / vcl.z + (R)cy;
    int u = (int)std::floor((R)((double)pu + 0.5));
    int v = (int)std::floor((R)((double)pv + 0.5));
    if (!(u >= 0 && v >= 0 && u < W && v < H)) return false;
    size_t j = (size_t)v * W + u;
    V4<R> vlast = cv4<R>(ld4(vl, j));
    V4<R> dd = {vlast.x - vcurr.x, vlast.y - vcurr.y, vlast.z - vcurr.z, vlast.w - vcurr.w};
    if (!(!isnan_(vlast.x) && (double)norm4(dd) < 0.1 && gl[j] != 0)) return false;
    r.diff = (int)gc[k] - (int)gl[j];
    r.cx = x; r.cy = y; r.lx = u; r.ly = v;
    return true;
}

// RGBReduction::GetRow (Reduction.cu:471-508) of one correspondence.
template <class R>
void rgb_row(int W, const float* vl, const int16_t* dxm, const int16_t* dym, const M3<R>& RcInv, const M3<R>& Rl,
             const V3<R>& tc, const V3<R>& tl, float fx, float fy, float sigma, const RgbCorr& r, R row[7]) {
    R w = (R)sigma + (R)std::abs(r.diff);
    w = (double)w < 1e-3 ? (R)1 : (R)1 / w;
    if ((double)sigma < 1e-6) w = 1;
    V3<R> vlast = xyz(cv4<R>(ld4(vl, (size_t)r.ly * W + r.lx)));
    V3<R> point = mv(RcInv, sub(add(mv(Rl, vlast), tl), tc));
    R gx = (R)(float)((double)(float)dxm[(size_t)r.cy * W + r.cx] / 9.0);
    R gy = (R)(float)((double)(float)dym[(size_t)r.cy * W + r.cx] / 9.0);
    R invz = (R)1 / point.z;
    V3<R> left;
    left.x = gx * (R)fx * invz;
    left.y = gy * (R)fy * invz;
    left.z = -(left.x * point.x + left.y * point.y) * invz;
    V3<R> a = mul(w, left), b = mul(w, cross(point, left));
    row[0] = a.x; row[1] = a.y; row[2] = a.z; row[3] = b.x; row[4] = b.y; row[5] = b.z;
    row[6] = -w * (R)r.diff;
}

// RGBStep (Reduction.cu:547-627).  The two integer sums are kept in 64 bits
// (the reference sums diff^2 in int32 and would wrap beyond 2^31).
template <class R>
void rgb_step(int W, int H, const uint8_t* gc, const uint8_t* gl, const float* vc,
              const float* vl, const int16_t* dxm, const int16_t* dym, const double* Tc,
              const double* Tl, float fx, float fy, float cx, float cy, double* sums,
              int64_t* res2) {
    const M3<R> Rc = rot<R>(Tc), RcInv = rot_inv<R>(Tc), Rl = rot<R>(Tl), RlInv = rot_inv<R>(Tl);
    const V3<R> tc = trans<R>(Tc), tl = trans<R>(Tl);
    std::vector<RgbCorr> res((size_t)W * H);
    std::vector<unsigned char> valid((size_t)W * H, 0);
    std::vector<int64_t> rc((size_t)H * 2, 0);
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            size_t k = (size_t)y * W + x;
            RgbCorr r;
            if (!rgb_corresp<R>(W, H, gc, gl, vc, vl, dxm, dym, Rc, RlInv, tc, tl, fx, fy, cx, cy, x, y, r))
                continue;
            res[k] = r;
            valid[k] = 1;
            rc[(size_t)y * 2] += 1;
            rc[(size_t)y * 2 + 1] += (int64_t)r.diff * r.diff;
        }
    }
    res2[0] = res2[1] = 0;
    for (int y = 0; y < H; ++y) { res2[0] += rc[(size_t)y * 2]; res2[1] += rc[(size_t)y * 2 + 1]; }
    // sigma = sqrt((float) sum / count), both sums as the reference's int sums
    float sigma = std::sqrt((float)res2[1] / (float)(res2[0] == 0 ? 1 : res2[0]));
    reduce_rows(H, 29, sums, [&](int y, double* s) {
        for (int x = 0; x < W; ++x) {
            size_t k = (size_t)y * W + x;
            if (!valid[k]) continue;
            R row[7];
            rgb_row<R>(W, vl, dxm, dym, RcInv, Rl, tc, tl, fx, fy, sigma, res[k], row);
            add_products(row, s);
            s[28] += 1;
        }
    });
}

// ------------------------------------------- the GPU kernels' summation order
//
// Reference precision only.  The library's tracking kernels sum the 29
// normal-equation values in a fixed order that depends only on the grid size
// G (a multiple of 4 blocks of 256 threads; fb_track_reduction_grid reports
// it per pyramid level):
//   pass A (ICP rows): thread t of block b visits pixels p = 256 b + t +
//     256 G k, k = 0, 1, ..., and adds each valid row's products into float
//     accumulators (product rounded, then added);
//   pass B (photometric rows): warp w of block b lists its correspondences in
//     pass A's visiting order (k, then lane); lane l of that warp then adds
//     the rows of entries l, l + 32, l + 64, ... in float;
//   each block: a transposed butterfly over the warp's 32 lanes (at distance
//     16, 8, 4, 2, 1 a lane keeps one half of its values and adds its
//     partner's copy of that half), then the 8 warp sums in warp order (float,
//     from 0);
//   each cluster of 4 consecutive blocks: the block sums in rank order (FP64,
//     from 0); then the NG = G / 4 cluster sums in four consecutive ranges of
//     ceil(NG / 4) clusters (FP64, from 0), and the ranges added as
//     ((r0 + r1) + r2) + r3.
// Summing in that order makes the oracle's sums equal the GPU's bit for bit,
// so the tracker can be compared bit for bit on every frame.
namespace gpuorder {

constexpr int kThreads = 256, kWarps = 8, kCluster = 4;

// One block's sums of thread accumulators acc[256][29] (float).
void block_sum(const float* acc, float* out) {
    float bs[kWarps][32];
    for (int w = 0; w < kWarps; ++w) {
        float a[32][32];
        int id[32][32];
        for (int l = 0; l < 32; ++l)
            for (int k = 0; k < 32; ++k) {
                a[l][k] = k < 29 ? acc[(size_t)(w * 32 + l) * 29 + k] : 0.f;
                id[l][k] = k;
            }
        for (int off = 16; off >= 1; off >>= 1) {
            float na[32][16];
            int nid[32][16];
            for (int l = 0; l < 32; ++l) {
                const bool up = (l & off) != 0;
                const int p = l ^ off;
                for (int k = 0; k < off; ++k) {
                    const int q = up ? k + off : k;
                    na[l][k] = a[l][q] + a[p][q];
                    nid[l][k] = id[l][q];
                }
            }
            for (int l = 0; l < 32; ++l)
                for (int k = 0; k < off; ++k) {
                    a[l][k] = na[l][k];
                    id[l][k] = nid[l][k];
                }
        }
        for (int l = 0; l < 32; ++l) bs[w][id[l][0]] = a[l][0];
    }
    for (int v = 0; v < 29; ++v) {
        float r = 0.f;
        for (int w = 0; w < kWarps; ++w) r += bs[w][v];
        out[v] = r;
    }
}

// The 29 sums of per-thread accumulators acc[G * 256][29].
void grid_sum(const std::vector<float>& acc, int G, double* sums) {
    std::vector<float> bsum((size_t)G * 29);
#pragma omp parallel for schedule(static)
    for (int b = 0; b < G; ++b) block_sum(&acc[(size_t)b * kThreads * 29], &bsum[(size_t)b * 29]);
    const int NG = G / kCluster, per = (NG + 3) / 4;
    for (int v = 0; v < 29; ++v) {
        double part[4];
        for (int q = 0; q < 4; ++q) {
            double t = 0;
            for (int g = q * per; g < std::min(NG, (q + 1) * per); ++g) {
                double c = 0;
                for (int r = 0; r < kCluster; ++r) c += (double)bsum[(size_t)(g * kCluster + r) * 29 + v];
                t += c;
            }
            part[q] = t;
        }
        sums[v] = ((part[0] + part[1]) + part[2]) + part[3];
    }
}

inline void add_row(const float row[7], float* acc) {
    int n = 0;
    for (int i = 0; i < 7; ++i)
        for (int j = i; j < 7; ++j) acc[n++] += row[i] * row[j];
    acc[28] += 1.0f;
}

void icp_step(int W, int H, const float* vc, const float* vl, const float* nc, const float* nl, const double* Tc,
              const double* Tl, float fx, float fy, float cx, float cy, int G, double* sums) {
    const M3<float> Rc = rot<float>(Tc), Rl = rot<float>(Tl), RlInv = rot_inv<float>(Tl);
    const V3<float> tc = trans<float>(Tc), tl = trans<float>(Tl);
    const int N = W * H, stride = G * kThreads, iters = (N + stride - 1) / stride;
    std::vector<float> acc((size_t)stride * 29, 0.f);
#pragma omp parallel for schedule(static)
    for (int th = 0; th < stride; ++th) {
        float* a = &acc[(size_t)th * 29];
        for (int k = 0; k < iters; ++k) {
            const int p = th + k * stride;
            if (p >= N) break;
            float row[7];
            if (icp_pixel<float>(W, H, vc, vl, nc, nl, Rc, Rl, RlInv, tc, tl, fx, fy, cx, cy, p % W, p / W, row))
                add_row(row, a);
        }
    }
    grid_sum(acc, G, sums);
}

void rgb_step(int W, int H, const uint8_t* gc, const uint8_t* gl, const float* vc, const float* vl,
              const int16_t* dxm, const int16_t* dym, const double* Tc, const double* Tl, float fx, float fy,
              float cx, float cy, int G, double* sums, int64_t* res2) {
    const M3<float> Rc = rot<float>(Tc), RcInv = rot_inv<float>(Tc), Rl = rot<float>(Tl),
                    RlInv = rot_inv<float>(Tl);
    const V3<float> tc = trans<float>(Tc), tl = trans<float>(Tl);
    const int N = W * H, stride = G * kThreads, iters = (N + stride - 1) / stride;
    const int nwarps = G * kWarps;
    std::vector<std::vector<RgbCorr>> seg(nwarps);
    std::vector<int64_t> cnt(nwarps, 0), sq(nwarps, 0);
#pragma omp parallel for schedule(static)
    for (int gw = 0; gw < nwarps; ++gw) {
        const int b = gw / kWarps, w = gw % kWarps;
        for (int k = 0; k < iters; ++k)
            for (int lane = 0; lane < 32; ++lane) {
                const int p = b * kThreads + w * 32 + lane + k * stride;
                if (p >= N) continue;
                RgbCorr r;
                if (!rgb_corresp<float>(W, H, gc, gl, vc, vl, dxm, dym, Rc, RlInv, tc, tl, fx, fy, cx, cy, p % W,
                                        p / W, r))
                    continue;
                seg[gw].push_back(r);
                cnt[gw] += 1;
                sq[gw] += (int64_t)r.diff * r.diff;
            }
    }
    res2[0] = res2[1] = 0;
    for (int gw = 0; gw < nwarps; ++gw) {
        res2[0] += cnt[gw];
        res2[1] += sq[gw];
    }
    const float sigma = std::sqrt((float)res2[1] / (float)(res2[0] == 0 ? 1 : res2[0]));
    std::vector<float> acc((size_t)stride * 29, 0.f);
#pragma omp parallel for schedule(static)
    for (int gw = 0; gw < nwarps; ++gw)
        for (int lane = 0; lane < 32; ++lane) {
            float* a = &acc[(size_t)(gw * 32 + lane) * 29];
            for (size_t i = lane; i < seg[gw].size(); i += 32) {
                float row[7];
                rgb_row<float>(W, vl, dxm, dym, RcInv, Rl, tc, tl, fx, fy, sigma, seg[gw][i], row);
                add_row(row, a);
            }
        }
    grid_sum(acc, G, sums);
}

}  // namespace gpuorder

// ------------------------------------------------------------------- map --

struct Entry { int x, y, z, ptr, offset; };
struct Voxel { float sdf; uint8_t weight; uint8_t rgb[3]; };

// Hash (Mapping/DeviceMap.cu:3-10).  NumBuckets is an unsigned constant, so
// the int XOR is converted to unsigned before the modulo.
inline uint32_t bucket_of(int x, int y, int z, uint32_t nb) {
    uint32_t h = ((uint32_t)x * 73856093u) ^ ((uint32_t)y * 19349669u) ^ ((uint32_t)z * 83492791u);
    return h % nb;
}

// voxelPosToBlockPos (DeviceMap.cu:150-161): floor division by 8
inline int block_of(int v) { return (v < 0 ? v - 7 : v) / 8; }
// voxelPosToLocalPos (DeviceMap.cu:167-178)
inline int local_of(int v) { int l = v % 8; return l < 0 ? l + 8 : l; }

struct Map {
    fbo_config cfg;
    int NB, NE, NS;
    std::vector<Entry> entries;
    std::vector<int> heap;
    int heapCounter, entryPtr;
    std::vector<Voxel> voxels;
    std::vector<int> visible;   // hash slots in ascending order

    explicit Map(const fbo_config& c) : cfg(c), NB(c.num_buckets), NE(c.num_excess), NS(c.num_blocks) {
        entries.resize((size_t)NB + NE);
        heap.resize(NS);
        voxels.resize((size_t)NS * 512);
        reset();
    }
    // ResetMap (Mapping/FuseMap.cu:321-364) on a zero-filled table
    void reset() {
        for (auto& e : entries) e = {0, 0, 0, -1, 0};
        for (int x = 0; x < NS; ++x) heap[x] = NS - x - 1;
        heapCounter = NS - 1;
        entryPtr = 1;
        for (auto& v : voxels) v = {kNaN, 0, {0, 0, 0}};
        visible.clear();
    }
    // derived constants, computed as the reference's constexpr expressions
    float voxelSizeInv() const { return (float)(1.0 / (double)cfg.voxel_size); }
    float blockWidth() const { return cfg.voxel_size * 8.0f; }
    float stepScale() const {
        return (float)(0.5 * (double)cfg.trunc_dist * (double)voxelSizeInv());
    }

    // FindEntry (DeviceMap.cu:122-135): slot index or -1
    int find(int x, int y, int z) const {
        int b = (int)bucket_of(x, y, z, (uint32_t)NB);
        const Entry* e = &entries[b];
        if (e->ptr != -1 && e->x == x && e->y == y && e->z == z) return b;
        while (e->offset > 0) {
            b = NB + e->offset - 1;
            e = &entries[b];
            if (e->x == x && e->y == y && e->z == z && e->ptr != -1) return b;
        }
        return -1;
    }
    // CreateEntry (DeviceMap.cu:12-21)
    Entry create_entry(int x, int y, int z, int offset) {
        int old = heapCounter--;
        if (old >= 0) {
            int ptr = heap[old];
            if (ptr != -1) return {x, y, z, ptr * 512, offset};
        }
        return {x, y, z, -1, 0};
    }
    // CreateBlock (DeviceMap.cu:23-62) without contention: the bucket lock
    // always succeeds.  Returns the slot written or -1.
    int create_block(int x, int y, int z) {
        int b = (int)bucket_of(x, y, z, (uint32_t)NB);
        Entry* e = &entries[b];
        Entry* eEmpty = nullptr;
        if (e->x == x && e->y == y && e->z == z && e->ptr != -1) return -1;
        if (e->ptr == -1 && !eEmpty) eEmpty = e;
        while (e->offset > 0) {
            int s = NB + e->offset - 1;
            e = &entries[s];
            if (e->x == x && e->y == y && e->z == z && e->ptr != -1) return -1;
            if (e->ptr == -1 && !eEmpty) eEmpty = e;
        }
        if (eEmpty) {
            *eEmpty = create_entry(x, y, z, e->offset);
            return (int)(eEmpty - entries.data());
        }
        int offset = entryPtr++;
        if (offset <= NE) {
            Entry* n = &entries[(size_t)NB + offset - 1];
            *n = create_entry(x, y, z, 0);
            e->offset = offset;
            return (int)(n - entries.data());
        }
        return -1;
    }
};

// Fusion::CreateBlocks (Mapping/FuseMap.cu:80-111) for every pixel, then the
// requested blocks that do not exist yet are inserted once each in canonical
// order: ascending (bucket, x, y, z).  This is the reference's allocation
// without its lock contention (which drops requests and can duplicate
// entries).  Returns the number of blocks requested that were new.
template <class R>
int allocate(Map& m, const float* depth, const double* T) {
    const fbo_config& c = m.cfg;
    const int W = c.width, H = c.height;
    const M3<R> Rv = rot<R>(T);
    const V3<R> tv = trans<R>(T);
    const R invfx = (R)(float)(1.0 / (double)c.fx), invfy = (R)(float)(1.0 / (double)c.fy);
    const R vinv = (R)m.voxelSizeInv();
    const R thresh = (R)(c.trunc_dist / 2);
    const R dmax = (R)c.depth_max, dmin = (R)c.depth_min;
    struct Req { uint32_t bucket; int x, y, z; };
    std::vector<std::vector<Req>> rows(H);
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < H; ++y) {
        std::vector<Req>& out = rows[y];
        for (int x = 0; x < W; ++x) {
            float zf = depth[y * W + x];
            R z = (R)zf;
            if (std::isnan(zf) || z < dmin || z > dmax) continue;
            R z_near = std::min(dmax, z - thresh);
            R z_far = std::min(dmax, z + thresh);
            if (z_near >= z_far) continue;
            auto unproject = [&](R zz) {
                V3<R> p = {zz * ((R)x - (R)c.cx) * invfx, zz * ((R)y - (R)c.cy) * invfy, zz};
                return add(mv(Rv, p), tv);
            };
            V3<R> pn = mul(unproject(z_near), vinv);
            V3<R> pf = mul(unproject(z_far), vinv);
            V3<R> dir = sub(pf, pn);
            R length = norm3(dir);
            int nSteps = (int)std::ceil(2.0 * (double)length);
            dir = divs(dir, (R)(float)(nSteps - 1));
            int px = 0, py = 0, pz = 0;
            bool have = false;
            for (int i = 0; i < nSteps; ++i) {
                // make_int3(float3) truncates toward zero (VectorMath.h:36-38)
                int bx = block_of((int)pn.x), by = block_of((int)pn.y), bz = block_of((int)pn.z);
                if (!have || bx != px || by != py || bz != pz) {
                    out.push_back({bucket_of(bx, by, bz, (uint32_t)m.NB), bx, by, bz});
                    px = bx; py = by; pz = bz; have = true;
                }
                pn = add(pn, dir);
            }
        }
    }
    std::vector<Req> all;
    for (auto& r : rows) all.insert(all.end(), r.begin(), r.end());
    auto key = [](const Req& a) { return std::make_tuple(a.bucket, a.x, a.y, a.z); };
    std::sort(all.begin(), all.end(), [&](const Req& a, const Req& b) { return key(a) < key(b); });
    all.erase(std::unique(all.begin(), all.end(),
                          [&](const Req& a, const Req& b) { return key(a) == key(b); }),
              all.end());
    std::vector<Req> fresh;
    for (auto& r : all)
        if (m.find(r.x, r.y, r.z) < 0) fresh.push_back(r);
    for (auto& r : fresh) m.create_block(r.x, r.y, r.z);
    return (int)fresh.size();
}

// Fusion::CheckVertexVisibility / CheckBlockVisibility (FuseMap.cu:36-78):
// the eight corners are visited by the reference's sequence of float adds.
template <class R>
bool block_visible(const Map& m, int bx, int by, int bz, const M3<R>& RvInv, V3<R> tv, R fx, R fy,
                   R cx, R cy) {
    const fbo_config& c = m.cfg;
    const R scale = (R)m.blockWidth();
    auto vis = [&](V3<R> p) {
        p = mv(RvInv, sub(p, tv));
        if (p.z < (R)1e-3f) return false;
        R u = fx * p.x / p.z + cx, v = fy * p.y / p.z + cy;
        return u >= 0 && v >= 0 && u < (R)c.width && v < (R)c.height && p.z >= (R)c.depth_min &&
               p.z <= (R)c.depth_max;
    };
    V3<R> k = {(R)bx * scale, (R)by * scale, (R)bz * scale};
    if (vis(k)) return true;
    k.z += scale; if (vis(k)) return true;
    k.y += scale; if (vis(k)) return true;
    k.x += scale; if (vis(k)) return true;
    k.z -= scale; if (vis(k)) return true;
    k.y -= scale; if (vis(k)) return true;
    k.x -= scale; k.y += scale; if (vis(k)) return true;
    k.x += scale; k.y -= scale; k.z += scale; if (vis(k)) return true;
    return false;
}

// CheckVisibleBlockKernel over every hash slot (FuseMap.cu:113-138)
template <class R>
void visibility(Map& m, const double* T) {
    const fbo_config& c = m.cfg;
    const M3<R> RvInv = rot_inv<R>(T);
    const V3<R> tv = trans<R>(T);
    const size_t n = m.entries.size();
    std::vector<unsigned char> flag(n, 0);
#pragma omp parallel for schedule(static)
    for (long long s = 0; s < (long long)n; ++s) {
        const Entry& e = m.entries[s];
        if (e.ptr != -1 &&
            block_visible<R>(m, e.x, e.y, e.z, RvInv, tv, (R)c.fx, (R)c.fy, (R)c.cx, (R)c.cy))
            flag[s] = 1;
    }
    m.visible.clear();
    for (size_t s = 0; s < n; ++s)
        if (flag[s]) m.visible.push_back((int)s);
}

// Fusion::integrateColor (FuseMap.cu:140-191) for every voxel of every
// visible block.
template <class R>
void integrate(Map& m, const float* depth, const uint8_t* rgb, const float* nmp, const double* T) {
    const fbo_config& c = m.cfg;
    const int W = c.width, H = c.height;
    const M3<R> RvInv = rot_inv<R>(T);
    const V3<R> tv = trans<R>(T);
    const R vs = (R)c.voxel_size, thresh = (R)c.trunc_dist;
    const R fx = (R)c.fx, fy = (R)c.fy, cx = (R)c.cx, cy = (R)c.cy;
#pragma omp parallel for schedule(dynamic, 16)
    for (long long b = 0; b < (long long)m.visible.size(); ++b) {
        const Entry& e = m.entries[m.visible[b]];
        for (int i = 0; i < 8; ++i)
            for (int ty = 0; ty < 8; ++ty)
                for (int tx = 0; tx < 8; ++tx) {
                    int locId = i * 64 + ty * 8 + tx;
                    V3<R> pos = {(R)(e.x * 8 + tx) * vs, (R)(e.y * 8 + ty) * vs, (R)(e.z * 8 + i) * vs};
                    pos = mv(RvInv, sub(pos, tv));
                    R pu = fx * pos.x / pos.z + cx, pv = fy * pos.y / pos.z + cy;
                    int u = (int)pu, v = (int)pv;   // make_int2(float2) truncates
                    if (u < 0 || v < 0 || u >= W || v >= H) continue;
                    float dpf = depth[v * W + u];
                    R dp = (R)dpf;
                    if (std::isnan(dpf) || dp > (R)c.depth_max || dp < (R)c.depth_min) continue;
                    R sdf = dp - pos.z;
                    if (!(sdf >= -thresh)) continue;
                    sdf = std::min((R)1, sdf / thresh);
                    V4<R> nl = cv4<R>(ld4(nmp, (size_t)v * W + u));
                    if (isnan_(nl.x)) continue;
                    R w = dot4(nl, normalised4(V4<R>{pos.x, pos.y, pos.z, (R)1}));
                    const uint8_t* px = rgb + 3 * ((size_t)v * W + u);
                    V3<R> val = {(R)px[0], (R)px[1], (R)px[2]};
                    Voxel& prev = m.voxels[(size_t)e.ptr + locId];
                    if (prev.weight == 0) {
                        prev.sdf = (float)sdf;
                        prev.weight = 1;
                        prev.rgb[0] = (uint8_t)(int)val.x;
                        prev.rgb[1] = (uint8_t)(int)val.y;
                        prev.rgb[2] = (uint8_t)(int)val.z;
                    } else {
                        val = divs(val, (R)255.f);
                        V3<R> old = divs(V3<R>{(R)prev.rgb[0], (R)prev.rgb[1], (R)prev.rgb[2]}, (R)255.f);
                        R a = w * (R)0.2f;
                        V3<R> res = mul(add(mul(a, val), mul((R)1 - a, old)), (R)255.f);
                        R W0 = (R)prev.weight;
                        prev.sdf = (float)(((R)prev.sdf * W0 + w * sdf) / (W0 + w));
                        prev.weight = (uint8_t)std::min(255, (int)prev.weight + 1);
                        prev.rgb[0] = (uint8_t)(int)res.x;
                        prev.rgb[1] = (uint8_t)(int)res.y;
                        prev.rgb[2] = (uint8_t)(int)res.z;
                    }
                }
    }
}

// ---------------------------------------------------------------- raycast --

template <class R> struct Cache { int x, y, z, ptr; bool set; };

// FindVoxel(float3, cache, valid) (DeviceMap.cu:97-114).  The reference's
// cache starts as HashEntry() -- pos (0,0,0), ptr -1 -- and trusts a position
// match without checking ptr, reading a wrong voxel when the first probe is
// in block (0,0,0); here the cache starts empty instead.
template <class R>
const Voxel* find_voxel(const Map& m, V3<R> p, Cache<R>& cache, bool& valid) {
    int vx = (int)p.x, vy = (int)p.y, vz = (int)p.z;
    int bx = block_of(vx), by = block_of(vy), bz = block_of(vz);
    int idx = local_of(vz) * 64 + local_of(vy) * 8 + local_of(vx);
    if (cache.set && bx == cache.x && by == cache.y && bz == cache.z) {
        valid = true;
        return &m.voxels[(size_t)cache.ptr + idx];
    }
    int s = m.find(bx, by, bz);
    if (s < 0) { valid = false; return nullptr; }
    valid = true;
    cache = {bx, by, bz, m.entries[s].ptr, true};
    return &m.voxels[(size_t)cache.ptr + idx];
}

template <class R> inline R vsdf(const Voxel* v) { return v ? (R)v->sdf : (R)kNaN; }

// Rendering::readSdf (RenderScene.cu:290-295)
template <class R> R read_sdf(const Map& m, V3<R> p, Cache<R>& c, bool& valid) {
    const Voxel* v = find_voxel(m, p, c, valid);
    if (!v || v->weight == 0) valid = false;
    return vsdf<R>(v);
}

// Rendering::readSdfInterped (RenderScene.cu:297-319)
template <class R> R read_sdf_interp(const Map& m, V3<R> pt, Cache<R>& c, bool& valid) {
    V3<R> f = {pt.x - std::floor(pt.x), pt.y - std::floor(pt.y), pt.z - std::floor(pt.z)};
    auto at = [&](R dx, R dy, R dz) {
        return vsdf<R>(find_voxel(m, V3<R>{pt.x + dx, pt.y + dy, pt.z + dz}, c, valid));
    };
    R s0 = at(0, 0, 0), s1 = at(1, 0, 0);
    R r0 = ((R)1 - f.x) * s0 + f.x * s1;
    s0 = at(0, 1, 0); s1 = at(1, 1, 0);
    R r1 = ((R)1 - f.x) * s0 + f.x * s1;
    R r2 = ((R)1 - f.y) * r0 + f.y * r1;
    s0 = at(0, 0, 1); s1 = at(1, 0, 1);
    r0 = ((R)1 - f.x) * s0 + f.x * s1;
    s0 = at(0, 1, 1); s1 = at(1, 1, 1);
    r1 = ((R)1 - f.x) * s0 + f.x * s1;
    R r3 = ((R)1 - f.y) * r0 + f.y * r1;
    return ((R)1 - f.z) * r2 + f.z * r3;
}

// Rendering::readNormal (RenderScene.cu:321-352)
template <class R>
bool read_normal(const Map& m, V3<R> pt, Cache<R>& c, const M3<R>& RvInv, V3<R>& n) {
    bool valid;
    R s[6];
    const R off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (int k = 0; k < 6; ++k) {
        s[k] = read_sdf_interp(m, V3<R>{pt.x + off[k][0], pt.y + off[k][1], pt.z + off[k][2]}, c, valid);
        if (isnan_(s[k]) || s[k] == (R)1 || !valid) return false;
    }
    n = normalised3(mv(RvInv, V3<R>{s[0] - s[1], s[2] - s[3], s[4] - s[5]}));
    return true;
}

// Projection::projectBlock + the tile fill of fillBlocksKernel
// (RenderScene.cu:54-104, 106-124, 156-179).  Because each tile's lower-right
// corner is taken from the block's upper-left corner (RenderScene.cu:115-116),
// only the first tile of a block covers pixels: [ul, min(ul + 15, lr)].
template <class R>
int zranges(const Map& m, const double* T, int zc, int zr, std::vector<float>& zmin,
            std::vector<float>& zmax) {
    int tiles = 0;
    const fbo_config& c = m.cfg;
    const M3<R> RvInv = rot_inv<R>(T);
    const V3<R> tv = trans<R>(T);
    const R fx = (R)c.fx, fy = (R)c.fy, cx = (R)c.cx, cy = (R)c.cy;
    zmin.assign((size_t)zc * zr, 100.f);
    zmax.assign((size_t)zc * zr, 0.f);
    for (int s : m.visible) {
        const Entry& e = m.entries[s];
        int ulx = zc, uly = zr, lrx = -1, lry = -1;
        R zx = (R)c.depth_max, zy = (R)c.depth_min;
        for (int k = 0; k < 8; ++k) {
            int tx = e.x + ((k & 1) ? 1 : 0), ty = e.y + ((k & 2) ? 1 : 0), tz = e.z + ((k & 4) ? 1 : 0);
            V3<R> p = {(R)(tx * 8) * (R)c.voxel_size, (R)(ty * 8) * (R)c.voxel_size,
                       (R)(tz * 8) * (R)c.voxel_size};
            p = mv(RvInv, sub(p, tv));
            if ((double)p.z < 2e-1) continue;
            R qx = (fx * p.x / p.z + cx) / (R)8, qy = (fy * p.y / p.z + cy) / (R)8;
            // upperLeft/lowerRight are short2 (RenderScene.cu:72-79)
            if ((R)ulx > std::floor(qx)) ulx = (short)(int)std::floor(qx);
            if ((R)lrx < std::ceil(qx)) lrx = (short)(int)std::ceil(qx);
            if ((R)uly > std::floor(qy)) uly = (short)(int)std::floor(qy);
            if ((R)lry < std::ceil(qy)) lry = (short)(int)std::ceil(qy);
            if (zx > p.z) zx = p.z;
            if (zy < p.z) zy = p.z;
        }
        if (ulx < 0) ulx = 0;
        if (uly < 0) uly = 0;
        if (lrx >= zc) lrx = zc - 1;
        if (lry >= zr) lry = zr - 1;
        if (ulx > lrx || uly > lry) continue;
        if (zx < (R)c.depth_min) zx = (R)c.depth_min;
        if (zy < (R)c.depth_min) continue;
        float fzx = (float)zx, fzy = (float)zy;
        ++tiles;
        int ex = std::min(ulx + 15, lrx), ey = std::min(uly + 15, lry);
        for (int y = uly; y <= ey; ++y)
            for (int x = ulx; x <= ex; ++x) {
                size_t i = (size_t)y * zc + x;
                zmin[i] = std::min(zmin[i], fzx);
                zmax[i] = std::max(zmax[i], fzy);
            }
    }
    return tiles;
}

// Rendering::operator() (RenderScene.cu:354-440)
template <class R>
void raycast(const Map& m, const double* T, const std::vector<float>& zmin,
             const std::vector<float>& zmax, int zc, float* vout, float* nout) {
    const fbo_config& c = m.cfg;
    const int W = c.width, H = c.height;
    const M3<R> Rv = rot<R>(T), RvInv = rot_inv<R>(T);
    const V3<R> tv = trans<R>(T);
    const R invfx = (R)(float)(1.0 / (double)c.fx), invfy = (R)(float)(1.0 / (double)c.fy);
    const R cx = (R)c.cx, cy = (R)c.cy;
    const R vinv = (R)m.voxelSizeInv(), vs = (R)c.voxel_size, stepScale = (R)m.stepScale();
#pragma omp parallel for schedule(dynamic, 2)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            size_t o = (size_t)y * W + x;
            st4(vout, o, kNaN, kNaN, kNaN, kNaN);
            st4(nout, o, kNaN, kNaN, kNaN, kNaN);
            int lx = (int)std::floor((float)x / 8.f), ly = (int)std::floor((float)y / 8.f);
            float zrx = zmin[(size_t)ly * zc + lx], zry = zmax[(size_t)ly * zc + lx];
            if (zry < 1e-3 || zrx < 1e-3 || std::isnan(zrx) || std::isnan(zry)) continue;
            R sdf = 1;
            V3<R> p;
            p.z = (R)zrx;
            p.x = p.z * ((R)x - cx) * invfx;
            p.y = p.z * ((R)y - cy) * invfy;
            R dist_s = norm3(p) * vinv;
            V3<R> block_s = mul(add(mv(Rv, p), tv), vinv);
            p.z = (R)zry;
            p.x = p.z * ((R)x - cx) * invfx;
            p.y = p.z * ((R)y - cy) * invfy;
            R dist_e = norm3(p) * vinv;
            V3<R> block_e = mul(add(mv(Rv, p), tv), vinv);
            V3<R> dir = normalised3(sub(block_e, block_s));
            V3<R> result = block_s;
            bool valid_sdf = false, found = false;
            R step;
            Cache<R> cache{0, 0, 0, -1, false};
            while (dist_s < dist_e) {
                sdf = read_sdf(m, result, cache, valid_sdf);
                if (!valid_sdf) {
                    step = 8;
                } else {
                    if (sdf <= (R)0.1f && sdf >= (R)-0.5f) sdf = read_sdf_interp(m, result, cache, valid_sdf);
                    if (sdf <= 0) break;
                    if (!isnan_(sdf))
                        step = std::max(sdf * stepScale, (R)1);
                    else
                        step = 8;
                }
                result = add(result, mul(step, dir));
                dist_s += step;
            }
            if (sdf <= 0) {
                step = sdf * stepScale;
                result = add(result, mul(step, dir));
                sdf = read_sdf_interp(m, result, cache, valid_sdf);
                step = sdf * stepScale;
                result = add(result, mul(step, dir));
                found = true;
            }
            if (found) {
                V3<R> n;
                if (read_normal(m, result, cache, RvInv, n)) {
                    V3<R> r = mv(RvInv, sub(mul(result, vs), tv));
                    st4(vout, o, (float)r.x, (float)r.y, (float)r.z, 1.0f);
                    st4(nout, o, (float)n.x, (float)n.y, (float)n.z, 1.0f);
                }
            }
        }
}

// ---------------------------------------------------------------- system --

struct Level { int W, H; std::vector<float> vmap, nmap, depth; std::vector<uint8_t> image;
               std::vector<int16_t> dx, dy; };
struct Frame {
    std::vector<float> range;
    std::vector<uint8_t> color;
    Level lv[3];
    double pose[16];
};

struct System {
    fbo_config cfg;
    Map map;
    Frame frames[2];
    Frame* next;
    Frame* last;
    int state = 1, lastState = 1, noMissedFrames = 0, numFramesAfterReloc = 10;
    double lastIcpError = NAN, lastRgbError = NAN, lastIcpCount = 0, lastRgbCount = 0;
    explicit System(const fbo_config& c) : cfg(c), map(c) {
        for (auto& f : frames) {
            f.range.resize((size_t)c.width * c.height);
            f.color.resize((size_t)c.width * c.height * 3);
            for (int i = 0; i < 3; ++i) {
                Level& l = f.lv[i];
                l.W = c.width >> i;
                l.H = c.height >> i;
                size_t n = (size_t)l.W * l.H;
                l.vmap.assign(4 * n, kNaN);
                l.nmap.assign(4 * n, kNaN);
                l.depth.assign(n, 0);
                l.image.assign(n, 0);
                l.dx.assign(n, 0);
                l.dy.assign(n, 0);
            }
            for (int i = 0; i < 16; ++i) f.pose[i] = (i % 5 == 0);
        }
        next = &frames[0];
        last = &frames[1];
    }
    float fx(int i) const { return cfg.fx / (1 << i); }
    float fy(int i) const { return cfg.fy / (1 << i); }
    float cx(int i) const { return cfg.cx / (1 << i); }
    float cy(int i) const { return cfg.cy / (1 << i); }
};

// Frame::FillImages (Core/Frame.cc:59-78)
template <class R>
void fill_images(System& s, Frame& f, const uint16_t* depth, const uint8_t* rgb) {
    const fbo_config& c = s.cfg;
    std::memcpy(f.color.data(), rgb, f.color.size());
    filter_depth<R>(c.width, c.height, depth, c.depth_scale, c.depth_cutoff, f.range.data(),
                    f.lv[0].depth.data());
    intensity(c.width, c.height, rgb, f.lv[0].image.data());
    for (int i = 1; i < 3; ++i) {
        pyrdown<R, float>(f.lv[i - 1].W, f.lv[i - 1].H, f.lv[i - 1].depth.data(), f.lv[i].depth.data());
        pyrdown<R, uint8_t>(f.lv[i - 1].W, f.lv[i - 1].H, f.lv[i - 1].image.data(), f.lv[i].image.data());
    }
    for (int i = 0; i < 3; ++i) {
        Level& l = f.lv[i];
        vmap<R>(l.W, l.H, l.depth.data(), s.fx(i), s.fy(i), s.cx(i), s.cy(i), c.depth_cutoff, l.vmap.data());
        nmap<R>(l.W, l.H, l.vmap.data(), l.nmap.data());
        derivative(l.W, l.H, l.image.data(), l.dx.data(), l.dy.data());
    }
}

// Frame::ResizeImages (Core/Frame.cc:80-84)
template <class R> void resize_images(Frame& f) {
    for (int i = 1; i < 3; ++i)
        resize_map<R>(f.lv[i - 1].W, f.lv[i - 1].H, f.lv[i - 1].vmap.data(), f.lv[i - 1].nmap.data(),
                      f.lv[i].vmap.data(), f.lv[i].nmap.data());
}

// Tracker::ComputeSE3(false, ITERATIONS_SE3, THRESH_ICP_SE3) (Tracking.cc:296-409).
// grid (reference precision only, else null): the library's tracking grid per
// pyramid level; the normal equations are then summed in its kernels' order
// (gpuorder above) and solved in its solver's order (pivot-free LDL^T, rigid
// inverses), so that the result equals the library's bit for bit.
template <class R> bool compute_se3(System& s, const int* grid = nullptr) {
    const int minCount[3] = {2000, 1000, 100};   // Tracking.h:102
    double lastPose[16], pose[16], delta[16];
    std::memcpy(lastPose, s.last->pose, sizeof lastPose);
    std::memcpy(pose, s.next->pose, sizeof pose);
    for (int i = 0; i < 16; ++i) delta[i] = (i % 5 == 0);
    float icpError = 0;
    for (int i = 2; i >= 0; --i) {
        Level &N = s.next->lv[i], &L = s.last->lv[i];
        for (int j = 0; j < s.cfg.iters[i]; ++j) {
            double sr[29], si[29], Ar[36], br[6], Ai[36], bi[6];
            int64_t res2[2];
            if (grid)
                gpuorder::rgb_step(N.W, N.H, N.image.data(), L.image.data(), N.vmap.data(), L.vmap.data(),
                                   N.dx.data(), N.dy.data(), s.next->pose, s.last->pose, s.fx(i), s.fy(i), s.cx(i),
                                   s.cy(i), grid[i], sr, res2);
            else
                rgb_step<R>(N.W, N.H, N.image.data(), L.image.data(), N.vmap.data(), L.vmap.data(),
                            N.dx.data(), N.dy.data(), s.next->pose, s.last->pose, s.fx(i), s.fy(i),
                            s.cx(i), s.cy(i), sr, res2);
            float r0 = (float)sr[27], r1 = (float)sr[28];
            float rgbError = std::sqrt(r0) / r1;
            s.lastRgbError = rgbError;
            s.lastRgbCount = r1;
            if (std::isnan(rgbError) || (int)r1 < minCount[i]) {
                std::memcpy(s.next->pose, lastPose, sizeof lastPose);
                return false;
            }
            if (grid)
                gpuorder::icp_step(N.W, N.H, N.vmap.data(), L.vmap.data(), N.nmap.data(), L.nmap.data(),
                                   s.next->pose, s.last->pose, s.fx(i), s.fy(i), s.cx(i), s.cy(i), grid[i], si);
            else
                icp_step<R>(N.W, N.H, N.vmap.data(), L.vmap.data(), N.nmap.data(), L.nmap.data(),
                            s.next->pose, s.last->pose, s.fx(i), s.fy(i), s.cx(i), s.cy(i), si);
            float q0 = (float)si[27], q1 = (float)si[28];
            icpError = std::sqrt(q0) / q1;
            s.lastIcpError = icpError;
            s.lastIcpCount = q1;
            if (std::isnan(icpError) || (int)q1 < minCount[i]) {
                std::memcpy(s.next->pose, lastPose, sizeof lastPose);
                return false;
            }
            fbo::unpack_29(sr, Ar, br);
            fbo::unpack_29(si, Ai, bi);
            double A[36], b[6], xi[6], dT[16], dinv[16];
            const float w = 1e-4f;
            for (int k = 0; k < 36; ++k) A[k] = Ar[k] * w + Ai[k];
            for (int k = 0; k < 6; ++k) b[k] = br[k] * w + bi[k];
            if (grid)
                fbo::ldlt_solve_nopivot(A, b, xi);
            else
                fbo::ldlt_solve(A, b, xi);
            fbo::se3_exp(xi, dT);
            fbo::mat4_mul(dT, delta, delta);
            if (grid)
                fbo::mat4_rigid_inv(delta, dinv);
            else
                fbo::mat4_inv(delta, dinv);
            fbo::mat4_mul(lastPose, dinv, s.next->pose);
        }
    }
    double pinv[16], p[16];
    if (grid)
        fbo::mat4_rigid_inv(pose, pinv);
    else
        fbo::mat4_inv(pose, pinv);
    fbo::mat4_mul(pinv, s.next->pose, p);
    double tn = std::sqrt(p[3] * p[3] + p[7] * p[7] + p[11] * p[11]);
    if (icpError < 0.0001f && fbo::euler_sin_norm(p) <= 0.1 && tn <= 0.1) return true;
    std::memcpy(s.next->pose, lastPose, sizeof lastPose);
    return false;
}

// Tracker::Track without SURF bootstrap / keyframes / relocalisation
// (Tracking.cc:58-112, 150-164)
template <class R> bool track(System& s) {
    std::swap(s.state, s.lastState);
    if (s.state == 1) {
        for (int i = 0; i < 16; ++i) s.next->pose[i] = s.last->pose[i] = (i % 5 == 0);
        std::swap(s.next, s.last);
        s.lastState = 0;
        return true;
    }
    if (s.state == 0) {
        std::memcpy(s.next->pose, s.last->pose, sizeof s.next->pose);
        bool valid = compute_se3<R>(s);
        if (valid) {
            s.noMissedFrames = 0;
            if (s.lastState != -1) {
                s.lastState = 0;
                std::swap(s.next, s.last);
                return true;
            }
            s.lastState = 0;
            return false;
        }
        s.lastState = 0;
        if (++s.noMissedFrames > 9) s.lastState = -1;
        return false;
    }
    s.lastState = -1;
    return false;
}

template <class R>
void fuse(Map& m, const float* raw, const uint8_t* rgb, const float* nmp, const double* T,
          uint32_t* nvis) {
    allocate<R>(m, raw, T);
    visibility<R>(m, T);
    integrate<R>(m, raw, rgb, nmp, T);
    if (nvis) *nvis = (uint32_t)m.visible.size();
}

// Mapping::RayTrace (Mapping/Mapping.cc:98-109): CreateRenderingBlocks
// returns false when there is nothing visible or no tile was produced
// (RenderScene.cu:214-215, 264-266) and the maps are then left unchanged.
// Returns the number of rendering tiles.
template <class R>
int raytrace(Map& m, const double* T, float* vm, float* nm, float* zminOut, float* zmaxOut) {
    if (m.visible.empty()) return 0;
    const int zc = (m.cfg.width + 7) / 8, zr = (m.cfg.height + 7) / 8;
    std::vector<float> zmin, zmax;
    int tiles = zranges<R>(m, T, zc, zr, zmin, zmax);
    if (zminOut) std::memcpy(zminOut, zmin.data(), zmin.size() * sizeof(float));
    if (zmaxOut) std::memcpy(zmaxOut, zmax.data(), zmax.size() * sizeof(float));
    if (tiles == 0) return 0;
    raycast<R>(m, T, zmin, zmax, zc, vm, nm);
    return tiles;
}

// System::GrabImage (Core/System.cc:92-138) without the viewer and meshing.
template <class R> int grab(System& s, const uint16_t* depth, const uint8_t* rgb, double* info) {
    s.lastIcpError = s.lastRgbError = NAN;
    s.lastIcpCount = s.lastRgbCount = 0;
    resize_images<R>(*s.last);
    fill_images<R>(s, *s.next, depth, rgb);
    bool state = track<R>(s);
    if (s.state == 0) s.numFramesAfterReloc++;
    if (s.state == -1) s.numFramesAfterReloc = 0;
    uint32_t noBlocks = 0;
    int fused = 0;
    if (state) {
        if (s.state != -1 && s.numFramesAfterReloc >= 10) {
            fuse<R>(s.map, s.last->range.data(), s.last->color.data(), s.last->lv[0].nmap.data(),
                    s.last->pose, &noBlocks);
            fused = 1;
        }
        if (s.state != -1)
            raytrace<R>(s.map, s.last->pose, s.last->lv[0].vmap.data(), s.last->lv[0].nmap.data(),
                        nullptr, nullptr);
    }
    if (info) {
        info[0] = state; info[1] = s.state; info[2] = noBlocks; info[3] = s.lastIcpError;
        info[4] = s.lastIcpCount; info[5] = s.lastRgbError; info[6] = s.lastRgbCount; info[7] = fused;
    }
    return 0;
}

// ------------------------------------------------------------------ mesh --
//
// MeshScene (Mapping/MeshScene.cu:20-295) restated on the CPU, driven by a
// case table given as an argument (the reference's Constant.h table or the
// library's own), over every entry with ptr >= 0 in slot order.  `fused`
// selects how the normal is rounded: 0 as written (n_a + val * (n_b - n_a),
// n . n left to right, each operation rounded), 1 with the multiply-adds
// fused (fma(val, n_b - n_a, n_a); fma(z, z, fma(y, y, x x))), the form a
// CUDA build contracts these expressions to.

struct MeshVox { float sdf; const uint8_t* rgb; };

// FindVoxel(int3) (DeviceMap.cu:78-84): Voxel() -- NaN, colour 0 -- where the
// block is missing
inline MeshVox mesh_voxel(const Map& m, int x, int y, int z) {
    static const uint8_t kBlack[3] = {0, 0, 0};
    const int slot = m.find(block_of(x), block_of(y), block_of(z));
    if (slot < 0) return {kNaN, kBlack};
    const Voxel& v = m.voxels[(size_t)m.entries[slot].ptr + local_of(z) * 64 + local_of(y) * 8 + local_of(x)];
    return {v.sdf, v.rgb};
}

// interp (MeshScene.cu:142-150): float operands, double thresholds
inline float mesh_interp(float v1, float v2) {
    if (std::fabs(0.f - v1) < 1e-6) return 0.f;
    if (std::fabs(0.f - v2) < 1e-6) return 1.f;
    if (std::fabs(v1 - v2) < 1e-6) return 0.f;
    return (0.f - v1) / (v2 - v1);
}

const int kMC[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
const int kME[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

uint64_t mesh_scene(const Map& m, const int8_t* tri, const int32_t* ntri, int fused, float* V, float* N,
                    uint8_t* C, uint64_t cap) {
    uint64_t count = 0;
    for (size_t slot = 0; slot < m.entries.size(); ++slot) {
        const Entry& e = m.entries[slot];
        if (e.ptr < 0) continue;
        for (int lz = 0; lz < 8; ++lz)
            for (int ly = 0; ly < 8; ++ly)
                for (int lx = 0; lx < 8; ++lx) {
                    const int px = e.x * 8 + lx, py = e.y * 8 + ly, pz = e.z * 8 + lz;
                    // readVertexAndColor (MeshScene.cu:105-140)
                    float sdf[8];
                    const uint8_t* col[8];
                    bool ok = true;
                    for (int i = 0; i < 8 && ok; ++i) {
                        MeshVox v = mesh_voxel(m, px + kMC[i][0], py + kMC[i][1], pz + kMC[i][2]);
                        sdf[i] = v.sdf;
                        col[i] = v.rgb;
                        ok = !(sdf[i] == 1.0 || std::isnan(sdf[i]));
                    }
                    if (!ok) continue;
                    // readNormal (MeshScene.cu:43-103): central differences
                    float nrm[8][3];
                    for (int i = 0; i < 8 && ok; ++i)
                        for (int a = 0; a < 3 && ok; ++a) {
                            int hi[3] = {px + kMC[i][0], py + kMC[i][1], pz + kMC[i][2]};
                            int lo[3] = {hi[0], hi[1], hi[2]};
                            hi[a] += 1;
                            lo[a] -= 1;
                            const float h = mesh_voxel(m, hi[0], hi[1], hi[2]).sdf;
                            const float l = mesh_voxel(m, lo[0], lo[1], lo[2]).sdf;
                            ok = !(std::isnan(h) || std::isnan(l));
                            nrm[i][a] = h - l;
                        }
                    if (!ok) continue;
                    int ci = 0;
                    for (int i = 0; i < 8; ++i)
                        if (sdf[i] < 0) ci |= 1 << i;
                    if (ci == 0 || ci == 255) continue;
                    // buildVertexList (MeshScene.cu:152-259) and MarchingCube's
                    // output (MeshScene.cu:277-293)
                    for (int t = 0; t < ntri[ci]; ++t, ++count) {
                        if (count >= cap) continue;
                        for (int k = 0; k < 3; ++k) {
                            const int ed = tri[ci * 16 + 3 * t + k];
                            const int a = kME[ed][0], b = kME[ed][1];
                            const float val = mesh_interp(sdf[a], sdf[b]);
                            float p[3];
                            for (int c = 0; c < 3; ++c) {
                                const int d = kMC[b][c] - kMC[a][c];
                                const float off = d > 0 ? val : (d < 0 ? 1.f - val : (float)kMC[a][c]);
                                const int base = c == 0 ? px : (c == 1 ? py : pz);
                                p[c] = ((float)base + off) * m.cfg.voxel_size;
                            }
                            float n[3];
                            for (int c = 0; c < 3; ++c)
                                n[c] = fused ? std::fmaf(val, nrm[b][c] - nrm[a][c], nrm[a][c])
                                             : nrm[a][c] + val * (nrm[b][c] - nrm[a][c]);
                            const float nn = fused ? std::fmaf(n[2], n[2], std::fmaf(n[1], n[1], n[0] * n[0]))
                                                   : n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
                            const float len = std::sqrt(nn);
                            const uint64_t o = (count * 3 + k) * 3;
                            const int iv = (int)val;
                            for (int c = 0; c < 3; ++c) {
                                V[o + c] = p[c];
                                N[o + c] = n[c] / len;
                                C[o + c] = (uint8_t)(col[a][c] + (uint8_t)((uint8_t)(col[b][c] - col[a][c]) * iv));
                            }
                        }
                    }
                }
    }
    return count;
}

}  // namespace

// ------------------------------------------------------------------ C API --
extern "C" {

#define DISPATCH(prec, call) ((prec) == 32 ? (call<float>) : (call<double>))

int fbo_filter_depth(int prec, int W, int H, const uint16_t* d, float s, float c, float* raw, float* f) {
    if (prec == 32) filter_depth<float>(W, H, d, s, c, raw, f); else filter_depth<double>(W, H, d, s, c, raw, f);
    return 0;
}
int fbo_intensity(int W, int H, const uint8_t* rgb, uint8_t* gray) { intensity(W, H, rgb, gray); return 0; }
int fbo_pyrdown_f32(int prec, int W, int H, const float* src, float* dst) {
    if (prec == 32) pyrdown<float, float>(W, H, src, dst); else pyrdown<double, float>(W, H, src, dst);
    return 0;
}
int fbo_pyrdown_u8(int prec, int W, int H, const uint8_t* src, uint8_t* dst) {
    if (prec == 32) pyrdown<float, uint8_t>(W, H, src, dst); else pyrdown<double, uint8_t>(W, H, src, dst);
    return 0;
}
int fbo_vmap(int prec, int W, int H, const float* d, float fx, float fy, float cx, float cy, float cut, float* out) {
    if (prec == 32) vmap<float>(W, H, d, fx, fy, cx, cy, cut, out); else vmap<double>(W, H, d, fx, fy, cx, cy, cut, out);
    return 0;
}
int fbo_nmap(int prec, int W, int H, const float* v, float* out) {
    if (prec == 32) nmap<float>(W, H, v, out); else nmap<double>(W, H, v, out);
    return 0;
}
int fbo_derivative(int W, int H, const uint8_t* g, int16_t* dx, int16_t* dy) { derivative(W, H, g, dx, dy); return 0; }
int fbo_resize_map(int prec, int W, int H, const float* vs, const float* ns, float* vd, float* nd) {
    if (prec == 32) resize_map<float>(W, H, vs, ns, vd, nd); else resize_map<double>(W, H, vs, ns, vd, nd);
    return 0;
}
int fbo_icp_step(int prec, int W, int H, const float* vc, const float* vl, const float* nc, const float* nl,
                 const double* Tc, const double* Tl, float fx, float fy, float cx, float cy, double* s) {
    if (prec == 32) icp_step<float>(W, H, vc, vl, nc, nl, Tc, Tl, fx, fy, cx, cy, s);
    else icp_step<double>(W, H, vc, vl, nc, nl, Tc, Tl, fx, fy, cx, cy, s);
    return 0;
}
int fbo_rgb_step(int prec, int W, int H, const uint8_t* gc, const uint8_t* gl, const float* vc, const float* vl,
                 const int16_t* dx, const int16_t* dy, const double* Tc, const double* Tl, float fx, float fy,
                 float cx, float cy, double* s, int64_t* r) {
    if (prec == 32) rgb_step<float>(W, H, gc, gl, vc, vl, dx, dy, Tc, Tl, fx, fy, cx, cy, s, r);
    else rgb_step<double>(W, H, gc, gl, vc, vl, dx, dy, Tc, Tl, fx, fy, cx, cy, s, r);
    return 0;
}

void* fbo_map_create(const fbo_config* c) { return new Map(*c); }
void fbo_map_destroy(void* m) { delete (Map*)m; }
void fbo_map_reset(void* m) { ((Map*)m)->reset(); }
int fbo_map_fuse(void* mp, const float* raw, const uint8_t* rgb, const float* nm, const double* T, uint32_t* nv) {
    Map& m = *(Map*)mp;
    if (m.cfg.precision == 32) fuse<float>(m, raw, rgb, nm, T, nv); else fuse<double>(m, raw, rgb, nm, T, nv);
    return 0;
}
int fbo_map_allocate(void* mp, const float* raw, const double* T, uint32_t* n_new) {
    Map& m = *(Map*)mp;
    int n = m.cfg.precision == 32 ? allocate<float>(m, raw, T) : allocate<double>(m, raw, T);
    if (n_new) *n_new = (uint32_t)n;
    return 0;
}
int fbo_map_raycast(void* mp, const double* T, float* vm, float* nm, float* zmin, float* zmax) {
    Map& m = *(Map*)mp;
    return m.cfg.precision == 32 ? raytrace<float>(m, T, vm, nm, zmin, zmax)
                                 : raytrace<double>(m, T, vm, nm, zmin, zmax);
}
int fbo_map_visibility(void* mp, const double* T, uint32_t* nv) {
    Map& m = *(Map*)mp;
    if (m.cfg.precision == 32)
        visibility<float>(m, T);
    else
        visibility<double>(m, T);
    if (nv) *nv = (uint32_t)m.visible.size();
    return 0;
}
int fbo_map_counters(void* mp, int32_t* hc, int32_t* ep, uint32_t* nv) {
    Map& m = *(Map*)mp;
    if (hc) *hc = m.heapCounter;
    if (ep) *ep = m.entryPtr;
    if (nv) *nv = (uint32_t)m.visible.size();
    return 0;
}
int fbo_map_entries(void* mp, int32_t* out) {
    Map& m = *(Map*)mp;
    for (size_t i = 0; i < m.entries.size(); ++i) {
        const Entry& e = m.entries[i];
        out[5 * i] = e.x; out[5 * i + 1] = e.y; out[5 * i + 2] = e.z; out[5 * i + 3] = e.ptr; out[5 * i + 4] = e.offset;
    }
    return 0;
}
int fbo_map_visible(void* mp, int32_t* slots) {
    Map& m = *(Map*)mp;
    for (size_t i = 0; i < m.visible.size(); ++i) slots[i] = m.visible[i];
    return 0;
}
int fbo_map_voxels(void* mp, const int32_t* ptrs, int n, double* sdf, uint8_t* w, uint8_t* rgb) {
    Map& m = *(Map*)mp;
    for (int i = 0; i < n; ++i)
        for (int v = 0; v < 512; ++v) {
            const Voxel& x = m.voxels[(size_t)ptrs[i] + v];
            size_t o = (size_t)i * 512 + v;
            if (sdf) sdf[o] = x.sdf;
            if (w) w[o] = x.weight;
            if (rgb) { rgb[3 * o] = x.rgb[0]; rgb[3 * o + 1] = x.rgb[1]; rgb[3 * o + 2] = x.rgb[2]; }
        }
    return 0;
}
int fbo_map_set_entries(void* mp, const int32_t* slots, const int32_t* ent, int n, int32_t hc,
                        int32_t ep) {
    Map& m = *(Map*)mp;
    for (auto& e : m.entries) e = {0, 0, 0, -1, 0};
    for (int i = 0; i < n; ++i)
        m.entries[slots[i]] = {ent[5 * i], ent[5 * i + 1], ent[5 * i + 2], ent[5 * i + 3], ent[5 * i + 4]};
    m.heapCounter = hc;
    m.entryPtr = ep;
    return 0;
}
int fbo_map_set_visible(void* mp, const int32_t* slots, int n) {
    Map& m = *(Map*)mp;
    m.visible.assign(slots, slots + n);
    return 0;
}
int fbo_map_load_blocks(void* mp, const int32_t* ptrs, int n, const double* sdf, const uint8_t* w,
                        const uint8_t* rgb) {
    Map& m = *(Map*)mp;
    for (int i = 0; i < n; ++i)
        for (int v = 0; v < 512; ++v) {
            Voxel& x = m.voxels[(size_t)ptrs[i] + v];
            size_t o = (size_t)i * 512 + v;
            x.sdf = (float)sdf[o];
            x.weight = w[o];
            for (int k = 0; k < 3; ++k) x.rgb[k] = rgb[3 * o + k];
        }
    return 0;
}

int fbo_map_mesh(void* mp, const int8_t* tri, const int32_t* ntri, int fused, float* V, float* N, uint8_t* C,
                 uint64_t cap, uint64_t* count) {
    *count = mesh_scene(*(Map*)mp, tri, ntri, fused, V, N, C, (V && N && C) ? cap : 0);
    return 0;
}

void* fbo_system_create(const fbo_config* c) { return new System(*c); }
void fbo_system_destroy(void* s) { delete (System*)s; }
int fbo_system_grab(void* sp, const uint16_t* d, const uint8_t* rgb, double* info) {
    System& s = *(System*)sp;
    return s.cfg.precision == 32 ? grab<float>(s, d, rgb, info) : grab<double>(s, d, rgb, info);
}
int fbo_system_pose(void* sp, int which, double* T) {
    System& s = *(System*)sp;
    std::memcpy(T, which ? s.next->pose : s.last->pose, 16 * sizeof(double));
    return 0;
}
void* fbo_system_map(void* sp) { return &((System*)sp)->map; }
int fbo_system_level(void* sp, int which, int lv, float* vm, float* nm, float* dp, uint8_t* im,
                     int16_t* dx, int16_t* dy) {
    System& s = *(System*)sp;
    Level& l = (which ? s.next : s.last)->lv[lv];
    size_t n = (size_t)l.W * l.H;
    if (vm) std::memcpy(vm, l.vmap.data(), 16 * n);
    if (nm) std::memcpy(nm, l.nmap.data(), 16 * n);
    if (dp) std::memcpy(dp, l.depth.data(), 4 * n);
    if (im) std::memcpy(im, l.image.data(), n);
    if (dx) std::memcpy(dx, l.dx.data(), 2 * n);
    if (dy) std::memcpy(dy, l.dy.data(), 2 * n);
    return 0;
}
int fbo_track(const fbo_config* c, const float* const* nv, const float* const* nn,
              const uint8_t* const* ng, const int16_t* const* ndx, const int16_t* const* ndy,
              const float* const* lv, const float* const* ln, const uint8_t* const* lg,
              const double* last_pose, double* out_pose, double* info) {
    fbo_config cc = *c;
    cc.num_buckets = 1;
    cc.num_excess = 0;
    cc.num_blocks = 1;
    System s(cc);
    for (int l = 0; l < 3; ++l) {
        Level &N = s.next->lv[l], &L = s.last->lv[l];
        size_t n = (size_t)N.W * N.H;
        std::memcpy(N.vmap.data(), nv[l], 16 * n);
        std::memcpy(N.nmap.data(), nn[l], 16 * n);
        std::memcpy(N.image.data(), ng[l], n);
        std::memcpy(N.dx.data(), ndx[l], 2 * n);
        std::memcpy(N.dy.data(), ndy[l], 2 * n);
        std::memcpy(L.vmap.data(), lv[l], 16 * n);
        std::memcpy(L.nmap.data(), ln[l], 16 * n);
        std::memcpy(L.image.data(), lg[l], n);
    }
    std::memcpy(s.last->pose, last_pose, 16 * sizeof(double));
    std::memcpy(s.next->pose, last_pose, 16 * sizeof(double));
    bool ok = c->precision == 32 ? compute_se3<float>(s) : compute_se3<double>(s);
    std::memcpy(out_pose, s.next->pose, 16 * sizeof(double));
    if (info) {
        info[0] = ok; info[1] = s.lastIcpError; info[2] = s.lastIcpCount; info[3] = s.lastRgbError;
        info[4] = s.lastRgbCount;
    }
    return 0;
}

// fbo_track in reference precision with the normal equations summed and
// solved in the order of the library's kernels for the tracking grid
// grid[level] (see gpuorder).
int fbo_track_gpu_order(const fbo_config* c, const int* grid, const float* const* nv, const float* const* nn,
                        const uint8_t* const* ng, const int16_t* const* ndx, const int16_t* const* ndy,
                        const float* const* lv, const float* const* ln, const uint8_t* const* lg,
                        const double* last_pose, double* out_pose, double* info) {
    fbo_config cc = *c;
    cc.num_buckets = 1;
    cc.num_excess = 0;
    cc.num_blocks = 1;
    System s(cc);
    for (int l = 0; l < 3; ++l) {
        if (c->iters[l] > 0 && (grid[l] <= 0 || grid[l] % gpuorder::kCluster)) return -1;
        Level &N = s.next->lv[l], &L = s.last->lv[l];
        size_t n = (size_t)N.W * N.H;
        std::memcpy(N.vmap.data(), nv[l], 16 * n);
        std::memcpy(N.nmap.data(), nn[l], 16 * n);
        std::memcpy(N.image.data(), ng[l], n);
        std::memcpy(N.dx.data(), ndx[l], 2 * n);
        std::memcpy(N.dy.data(), ndy[l], 2 * n);
        std::memcpy(L.vmap.data(), lv[l], 16 * n);
        std::memcpy(L.nmap.data(), ln[l], 16 * n);
        std::memcpy(L.image.data(), lg[l], n);
    }
    std::memcpy(s.last->pose, last_pose, 16 * sizeof(double));
    std::memcpy(s.next->pose, last_pose, 16 * sizeof(double));
    bool ok = compute_se3<float>(s, grid);
    std::memcpy(out_pose, s.next->pose, 16 * sizeof(double));
    if (info) {
        info[0] = ok; info[1] = s.lastIcpError; info[2] = s.lastIcpCount; info[3] = s.lastRgbError;
        info[4] = s.lastRgbCount;
    }
    return 0;
}

int fbo_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
