// Frame-to-model tracking: projective ICP + photometric normal equations
// (Tracking/Reduction.cu: ICPReduce 212-375, RGBReduction 377-627) and the
// coarse-to-fine Gauss-Newton loop of Tracker::ComputeSE3
// (Tracking/Tracking.cc:296-409), kept entirely on the device.
//
// One iteration is two kernels:
//   pass A: per pixel, the ICP row (point-to-plane, 7 wide) and the RGB
//           correspondence search; ICP products and the RGB count / sum of
//           squared differences are reduced.  The RGB correspondence of each
//           pixel is kept as one packed int (last-frame pixel + difference).
//           The current frame's per-pixel inputs are staged in shared memory
//           by bulk copies (PixelStage), two 256-pixel chunks ahead.
//   pass B: per pixel with a correspondence, the photometric row weighted by
//           the robust scale sigma from pass A; products reduced.  The last
//           block to finish also solves A x = b in FP64 (LDL^T), applies the
//           SE(3) exponential and writes the next pose for the following
//           iteration, with the reference's failure and acceptance tests.
// Reductions are deterministic: fixed per-thread pixel sets, warp shuffles,
// block sums in shared memory, then the blocks' partial sums are added in
// block order in FP64 by the last block (no atomics on values).
//
// The per-iteration kernels come in two instances of the same code: two
// resident blocks per SM (registers for latency: a session alone) and four
// (half the registers, some spilled: sessions sharing the GPU leave room for
// each other).  This file is compiled without contraction of multiplies and
// adds into FMAs, so both instances compute the same bits.
#include <cooperative_groups.h>

#include "fb_async.cuh"
#include "fb_fused.cuh"
#include "fb_internal.h"

namespace cg = cooperative_groups;

namespace fb {

// ------------------------------------------------------------ row builders
//
// The reference evaluates a few float expressions in double (Reduction.cu:
// (float)(1.0 / (double)z), (int)((double)f + 0.5), (float)((double)f + 0.5),
// (double)dx / 9.0, (double)x < c).  Their float equivalents below give the
// same bits for every float input:
//   - a quotient or sum of floats computed in double and rounded to float is
//     the IEEE float quotient or sum (double rounding is innocuous when the
//     wide format has at least 2p + 2 bits: 53 >= 50; f + 0.5 is exact in
//     double where it matters), hence __frcp_rn, __fdiv_rn, __fadd_rn;
//   - (int)((double)f + 0.5) truncates f + 0.5; the float sum rounded toward
//     zero lies between that integer and the exact sum, so it truncates to
//     the same integer (saturation and NaN -> 0 as the double conversion);
//   - (double)x < c for a double c that is not a float holds exactly when x
//     is below the smallest float above c.
__device__ __forceinline__ int trunc_half_up(float f) { return __float2int_rz(__fadd_rz(f, 0.5f)); }
constexpr float kBelow1em3 = 0.001f;   // (double)x < 1e-3  <=>  x < 0.001f
constexpr float kBelow0p1 = 0.1f;      // (double)x < 0.1   <=>  x < 0.1f
__device__ __forceinline__ float below_1em6() { return __int_as_float(0x358637be); }   // (double)x < 1e-6

// Photometric correspondences are packed in 32 bits: last-frame pixel
// (u, v) and the gray difference d (-254..255, as d + 255 in 1..510):
// v << 21 | u << 9 | (d + 255).  Images are at most 4096 x 2048; the low 9
// bits are never all ones, so -1 (all ones) marks "no correspondence".
// A correspondence list entry is {the pixel's Sobel derivatives (uint16) dx | dy << 16, pack_corr}.
__device__ __forceinline__ int pack_corr(int u, int v, int d255) {
    return (int)(((unsigned)v << 21) | ((unsigned)u << 9) | (unsigned)d255);
}
__device__ __forceinline__ int corr_u(int c) { return (int)(((unsigned)c >> 9) & 4095u); }
__device__ __forceinline__ int corr_v(int c) { return (int)((unsigned)c >> 21); }

// ICPReduce::searchPoint + getRow (Reduction.cu:227-286).  Returns false when
// the pixel has no correspondence.  Decisions use the order-exact float ops.
__device__ __forceinline__ bool icp_row(const TrackLevel& L, const DevPose& cur, const DevPose& last, int x,
                                        int y, float row[7]) {
    const size_t i = (size_t)y * L.vp + x;
    float4 vc4 = L.vcurr[i];
    f3 vcurr_c = xyz(vc4);
    if (isnan(vcurr_c.x) || vcurr_c.z < kBelow1em3) return false;
    f3 vcurr_g = add3(mv(cur.R, vcurr_c), cur.t);
    f3 vcurr_p = mv(last.Rinv, sub3(vcurr_g, last.t));
    float invz = __frcp_rn(vcurr_p.z);
    int u = trunc_half_up(fa(fm(fm(vcurr_p.x, invz), L.k.fx), L.k.cx));
    int v = trunc_half_up(fa(fm(fm(vcurr_p.y, invz), L.k.fy), L.k.cy));
    if (u < 0 || v < 0 || u >= L.W || v >= L.H) return false;
    const size_t j = (size_t)v * L.vp + u;
    f3 vlast_c = xyz(L.vlast[j]);
    f3 vlast_g = add3(mv(last.R, vlast_c), last.t);
    f3 ncurr_c = xyz(L.ncurr[i]);
    f3 ncurr_g = mv(cur.R, ncurr_c);
    f3 nlast_c = xyz(L.nlast[j]);
    f3 nlast_g = mv(last.R, nlast_c);
    float dist = norm3(sub3(vlast_g, vcurr_g));
    float sine = norm3(cross3(ncurr_g, nlast_g));
    if (!(sine < 0.6f && dist <= 0.1f && !isnan(ncurr_c.x) && !isnan(nlast_c.x))) return false;
    f3 nl = mv(last.Rinv, nlast_g);
    f3 vcl = mv(last.Rinv, sub3(vcurr_g, last.t));
    f3 vll = mv(last.Rinv, sub3(vlast_g, last.t));
    f3 c = cross3(nl, vll);
    row[0] = -nl.x;
    row[1] = -nl.y;
    row[2] = -nl.z;
    row[3] = c.x;
    row[4] = c.y;
    row[5] = c.z;
    row[6] = dot3(neg3(nl), sub3(vcl, vll));
    return true;
}

// RGBReduction::FindCorresp (Reduction.cu:404-451).  Returns the packed
// correspondence (pack_corr) of last-frame pixel (u, v), or -1.
__device__ __forceinline__ int rgb_corresp(const TrackLevel& L, const DevPose& cur, const DevPose& last, int x,
                                           int y) {
    const int W = L.W, H = L.H;
    if (L.rgbok) {
        // border, window and gradient tests precomputed per frame
        if (!L.rgbok[(size_t)y * L.sp + x]) return -1;
    } else {
        if (!(x >= 5 && x < W - 5 && y >= 5 && y < H - 5)) return -1;
        // the window is y-2..y+1, x-2..x+1 (Reduction.cu:416-417)
        for (int u = y - 2; u < y + 2; ++u)
            for (int v = x - 2; v < x + 2; ++v)
                if (L.gcurr[(size_t)u * L.gp + v] == 0) return -1;
        int gx = L.dx[(size_t)y * L.sp + x], gy = L.dy[(size_t)y * L.sp + x];
        if (gx == 0 && gy == 0) return -1;  // sqrtf(gx*gx + gy*gy) > 0
    }
    float4 vcurr = L.vcurr[(size_t)y * L.vp + x];
    if (isnan(vcurr.x)) return -1;
    f3 vcurr_g = add3(mv(cur.R, xyz(vcurr)), cur.t);
    f3 vcl = mv(last.Rinv, sub3(vcurr_g, last.t));
    float pu = fa(fd(fm(L.k.fx, vcl.x), vcl.z), L.k.cx);
    float pv = fa(fd(fm(L.k.fy, vcl.y), vcl.z), L.k.cy);
    int u = (int)floorf(__fadd_rn(pu, 0.5f));
    int v = (int)floorf(__fadd_rn(pv, 0.5f));
    if (!(u >= 0 && v >= 0 && u < W && v < H)) return -1;
    float4 vlast = L.vlast[(size_t)v * L.vp + u];
    if (isnan(vlast.x)) return -1;
    float ddx = fs(vlast.x, vcurr.x), ddy = fs(vlast.y, vcurr.y), ddz = fs(vlast.z, vcurr.z),
          ddw = fs(vlast.w, vcurr.w);
    float nd = fsq(fa(fa(fa(fm(ddx, ddx), fm(ddy, ddy)), fm(ddz, ddz)), fm(ddw, ddw)));
    if (!(nd < kBelow0p1)) return -1;
    int gl = L.glast[(size_t)v * L.gp + u];
    if (gl == 0) return -1;
    int diff = (int)L.gcurr[(size_t)y * L.gp + x] - gl;
    return pack_corr(u, v, diff + 255);
}

// The memory inputs of one photometric row: the last frame's vertex at the
// correspondence, the current pixel's derivatives and the packed value.
struct RgbIn {
    float4 vlast;
    int dx, dy, packed;
};

__device__ __forceinline__ RgbIn rgb_fetch(const TrackLevel& L, int x, int y, int packed) {
    RgbIn in;
    in.vlast = L.vlast[corr_v(packed) * L.vp + corr_u(packed)];
    const int k = y * L.sp + x;
    in.dx = L.dx[k];
    in.dy = L.dy[k];
    in.packed = packed;
    return in;
}

// The fetch of correspondence list entry e (the pixel's derivatives
// (uint16) dx | dy << 16, packed value): only the last vertex at the
// correspondence is gathered.
__device__ __forceinline__ RgbIn rgb_fetch_entry(const TrackLevel& L, int2 e) {
    RgbIn in;
    in.vlast = L.vlast[corr_v(e.y) * L.vp + corr_u(e.y)];
    in.dx = (int)(int16_t)(e.x & 0xffff);
    in.dy = e.x >> 16;
    in.packed = e.y;
    return in;
}

// RGBReduction::GetRow (Reduction.cu:471-508) from fetched inputs.
__device__ __forceinline__ void rgb_row_of(const RgbIn& in, const TrackLevel& L, const DevPose& cur,
                                           const DevPose& last, float sigma, float row[7]) {
    const int diff = (in.packed & 511) - 255;
    float w = sigma + (float)abs(diff);
    w = w < kBelow1em3 ? 1.0f : __frcp_rn(w);
    if (sigma < below_1em6()) w = 1.0f;
    f3 vlast = xyz(in.vlast);
    f3 point = mv(cur.Rinv, sub3(add3(mv(last.R, vlast), last.t), cur.t));
    float gx = __fdiv_rn((float)in.dx, 9.0f);
    float gy = __fdiv_rn((float)in.dy, 9.0f);
    float invz = __frcp_rn(point.z);
    f3 left;
    left.x = gx * L.k.fx * invz;
    left.y = gy * L.k.fy * invz;
    left.z = -(left.x * point.x + left.y * point.y) * invz;
    f3 c = cross3(point, left);
    row[0] = w * left.x;
    row[1] = w * left.y;
    row[2] = w * left.z;
    row[3] = w * c.x;
    row[4] = w * c.y;
    row[5] = w * c.z;
    row[6] = -w * (float)diff;
}

// RGBReduction::GetRow of the correspondence `packed` of pixel (x, y).
__device__ __forceinline__ void rgb_row(const TrackLevel& L, const DevPose& cur, const DevPose& last, int x, int y,
                                        int packed, float sigma, float row[7]) {
    rgb_row_of(rgb_fetch(L, x, y, packed), L, cur, last, sigma, row);
}

// Pose-independent inputs of one pixel for pass A (staged in shared memory
// by PixelStage).
struct PixelIn {
    float4 vc;      // current vertex
    float3 nc;      // current normal (xyz)
    int ok;         // photometric eligibility (border, window, gradient)
    int gc;         // current gray value
    int dxy;        // Sobel derivatives: (uint16) dx | dy << 16
};

// Pass A's current-frame inputs staged in shared memory by bulk copies
// (cp.async.bulk, this GPU's own memory, no multicast).  A chunk is one
// logical block's 256 consecutive pixels of one pass over the image (the
// frame buffers have pitch == width, so a chunk is one contiguous range of
// each map): vertices and normals (4 KB each), the Sobel derivatives
// (512 B each), photometric eligibility and gray (256 B each; the derivative
// and byte rows are rounded up to 16 B at the image's end, inside the
// allocations, which are 256-byte multiples).  Two buffers: chunk c + 2 is
// copied while chunk c + 1 is processed.
struct PixelStage {
    float4 v[2][256];
    float4 n[2][256];
    int16_t dx[2][256];
    int16_t dy[2][256];
    uint8_t ok[2][256];
    uint8_t g[2][256];
    uint64_t bar[2];
};

// Thread 0: copy the chunk of pixels [start, min(start + 256, N)) into
// buffer `buf`, completing on its barrier.
__device__ __forceinline__ void stage_chunk(PixelStage& S, int buf, const TrackLevel& L, int start, int N) {
    const int cnt = min(256, N - start);
    const uint32_t b16 = (uint32_t)cnt * 16u, b1 = ((uint32_t)cnt + 15u) & ~15u;
    const uint32_t b2 = ((uint32_t)cnt * 2u + 15u) & ~15u;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&S.bar[buf], 2u * b16 + 2u * b2 + 2u * b1);
    bulk_copy_g2s(S.v[buf], L.vcurr + start, b16, &S.bar[buf]);
    bulk_copy_g2s(S.n[buf], L.ncurr + start, b16, &S.bar[buf]);
    bulk_copy_g2s(S.dx[buf], L.dx + start, b2, &S.bar[buf]);
    bulk_copy_g2s(S.dy[buf], L.dy + start, b2, &S.bar[buf]);
    bulk_copy_g2s(S.ok[buf], L.rgbok + start, b1, &S.bar[buf]);
    bulk_copy_g2s(S.g[buf], L.gcurr + start, b1, &S.bar[buf]);
}

// Every thread: wait for buffer `buf`'s fill number `use` (bounded); then
// read pixel t of the chunk.  Returns false in every thread of the block
// when any thread's wait gave up.
__device__ __forceinline__ bool take_chunk(PixelStage& S, int buf, uint32_t use) {
    const bool ok = mbar_wait(&S.bar[buf], use & 1u);
    return !__syncthreads_or(!ok);
}

// The chunks of a group-form block in processing order: groups j of the
// block, the group's kTrackCluster logical blocks r, their passes k over the
// image while the chunk starts inside it.  start < 0: no chunk left.
struct ChunkCursor {
    int j, r, k, start;
    __device__ __forceinline__ int start_of(int bx, int gpc, int S) const {
        return ((bx * gpc + j) * kTrackCluster + r) * 256 + k * S;
    }
    // the first chunk at or after (j, r, k)
    __device__ __forceinline__ void settle(int bx, int gpc, int NG, int iters, int S, int N) {
        for (;;) {
            if (j >= gpc || bx * gpc + j >= NG) {
                start = -1;
                return;
            }
            if (k < iters) {
                start = start_of(bx, gpc, S);
                if (start < N) return;
            }
            k = 0;
            if (++r == kTrackCluster) {
                r = 0;
                ++j;
            }
            if (start_of(bx, gpc, S) >= N) {   // later logical blocks start later still
                start = -1;
                return;
            }
        }
    }
};

__device__ __forceinline__ PixelIn staged_pixel(const PixelStage& S, int buf, int t) {
    PixelIn in;
    in.vc = S.v[buf][t];
    const float4 n = S.n[buf][t];
    in.nc = make_float3(n.x, n.y, n.z);
    in.ok = S.ok[buf][t];
    in.gc = S.g[buf][t];
    in.dxy = (int)(uint16_t)S.dx[buf][t] | ((int)S.dy[buf][t] << 16);
    return in;
}

// icp_row and rgb_corresp of one pixel together (same arithmetic, same
// decisions), with the pose-independent loads done by the caller and the four
// pose-dependent gathers (last vertex and normal at the ICP projection, last
// vertex and gray value at the photometric projection) issued together.
// Needs L.rgbok.  Returns whether the ICP row is valid; *rgb = packed
// correspondence or -1.
__device__ __forceinline__ bool pixel_pass_a(const TrackLevel& L, const DevPose& cur, const DevPose& last,
                                             const PixelIn& in, float row[7], int* rgb) {
    const f3 vcurr_c = xyz(in.vc);
    const bool vnan = isnan(vcurr_c.x);
    const f3 vcurr_g = add3(mv(cur.R, vcurr_c), cur.t);
    // ICP projection (ICPReduce::searchPoint, Reduction.cu:227-250)
    int ju = -1;
    if (!vnan && !(vcurr_c.z < kBelow1em3)) {
        const f3 vcurr_p = mv(last.Rinv, sub3(vcurr_g, last.t));
        const float invz = __frcp_rn(vcurr_p.z);
        const int u = trunc_half_up(fa(fm(fm(vcurr_p.x, invz), L.k.fx), L.k.cx));
        const int v = trunc_half_up(fa(fm(fm(vcurr_p.y, invz), L.k.fy), L.k.cy));
        if (!(u < 0 || v < 0 || u >= L.W || v >= L.H)) ju = v * L.vp + u;
    }
    // photometric projection (RGBReduction::FindCorresp, Reduction.cu:404-451)
    int jr = -1, ur = 0, vr = 0;
    if (in.ok && !vnan) {
        const f3 vcl = mv(last.Rinv, sub3(vcurr_g, last.t));
        const float pu = fa(fd(fm(L.k.fx, vcl.x), vcl.z), L.k.cx);
        const float pv = fa(fd(fm(L.k.fy, vcl.y), vcl.z), L.k.cy);
        ur = (int)floorf(__fadd_rn(pu, 0.5f));
        vr = (int)floorf(__fadd_rn(pv, 0.5f));
        if (ur >= 0 && vr >= 0 && ur < L.W && vr < L.H) jr = vr * L.vp + ur;
    }
    const float nanf_ = qnan();
    const float4 vl4 = ju >= 0 ? L.vlast[ju] : make_float4(nanf_, nanf_, nanf_, nanf_);
    const float4 nl4 = ju >= 0 ? L.nlast[ju] : make_float4(nanf_, nanf_, nanf_, nanf_);
    const float4 vr4 = jr >= 0 ? L.vlast[jr] : make_float4(nanf_, nanf_, nanf_, nanf_);
    const int gl = jr >= 0 ? (int)L.glast[vr * L.gp + ur] : 0;
    // photometric residual
    *rgb = -1;
    if (jr >= 0 && !isnan(vr4.x)) {
        const float ddx = fs(vr4.x, in.vc.x), ddy = fs(vr4.y, in.vc.y), ddz = fs(vr4.z, in.vc.z),
                    ddw = fs(vr4.w, in.vc.w);
        const float nd = fsq(fa(fa(fa(fm(ddx, ddx), fm(ddy, ddy)), fm(ddz, ddz)), fm(ddw, ddw)));
        if (nd < kBelow0p1 && gl != 0) *rgb = pack_corr(ur, vr, in.gc - gl + 255);
    }
    // ICP row (ICPReduce::getRow, Reduction.cu:252-286)
    if (ju < 0) return false;
    const f3 vlast_c = xyz(vl4);
    const f3 vlast_g = add3(mv(last.R, vlast_c), last.t);
    const f3 ncurr_c = mk3(in.nc.x, in.nc.y, in.nc.z);
    const f3 ncurr_g = mv(cur.R, ncurr_c);
    const f3 nlast_c = xyz(nl4);
    const f3 nlast_g = mv(last.R, nlast_c);
    const float dist = norm3(sub3(vlast_g, vcurr_g));
    const float sine = norm3(cross3(ncurr_g, nlast_g));
    if (!(sine < 0.6f && dist <= 0.1f && !isnan(ncurr_c.x) && !isnan(nlast_c.x))) return false;
    const f3 nl = mv(last.Rinv, nlast_g);
    const f3 vcl = mv(last.Rinv, sub3(vcurr_g, last.t));
    const f3 vll = mv(last.Rinv, sub3(vlast_g, last.t));
    const f3 c = cross3(nl, vll);
    row[0] = -nl.x;
    row[1] = -nl.y;
    row[2] = -nl.z;
    row[3] = c.x;
    row[4] = c.y;
    row[5] = c.z;
    row[6] = dot3(neg3(nl), sub3(vcl, vll));
    return true;
}

__device__ __forceinline__ void add_products(const float row[7], float acc[29]) {
    int n = 0;
#pragma unroll
    for (int i = 0; i < 7; ++i)
#pragma unroll
        for (int j = i; j < 7; ++j) acc[n++] += row[i] * row[j];
    acc[28] += 1.0f;
}

// Pass B's rows of one warp segment (n entries): lane l adds the rows of
// entries l, l + 32, ... in that order.  The next entry's loads are issued
// before the current row is computed, so the list read and the dependent
// gathers of two entries overlap (the clustered forms, with registers to
// spare; the 64-register group forms add the rows one at a time,
// add_segment_rows_seq: 2 % faster there, the same sums).
// `a`: the fetch of entry `lane` (when lane < n), issued by the caller before
// the robust scale is known.
__device__ __forceinline__ void add_segment_rows(const TrackLevel& L, const DevPose& cur, const DevPose& last,
                                                 float sigma, const int2* seg, int n, int lane, float acc[29],
                                                 RgbIn a) {
    int i = lane;
    if (i >= n) return;
    for (; i < n; i += 32) {
        RgbIn b = a;
        if (i + 32 < n) b = rgb_fetch_entry(L, seg[i + 32]);
        float row[7];
        rgb_row_of(a, L, cur, last, sigma, row);
        add_products(row, acc);
        a = b;
    }
}

__device__ __forceinline__ void add_segment_rows_seq(const TrackLevel& L, const DevPose& cur, const DevPose& last,
                                                     float sigma, const int2* seg, int n, int lane, float acc[29]) {
    for (int i = lane; i < n; i += 32) {
        float row[7];
        rgb_row_of(rgb_fetch_entry(L, seg[i]), L, cur, last, sigma, row);
        add_products(row, acc);
    }
}

// ------------------------------------------------------------- reductions

// Block-wide sum of NV floats (deterministic).  Result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(float v[NV], float* smem /* [32][NV] */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    }
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) smem[wid * NV + k] = v[k];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] = lane < nw ? smem[lane * NV + k] : 0.f;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        }
    }
}

// Block-wide sum of the 29 per-thread values of the normal equations.  Each
// warp first reduces its 32 lanes by recursive halving (at every step a lane
// keeps one half of its values, sends the other half to its partner and adds
// what it receives: 31 shuffles in all), after which lane l holds the warp
// sum of value l; warp 0 then adds the warps' sums in warp order.  Result:
// value l in lane l (< 29) of warp 0.  Deterministic.
__device__ __forceinline__ float block_sum29(const float (&v)[29], float* smem /* [8][32] */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    float a[32];
#pragma unroll
    for (int k = 0; k < 29; ++k) a[k] = v[k];
    a[29] = a[30] = a[31] = 0.f;
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        const bool up = (lane & off) != 0;
#pragma unroll
        for (int k = 0; k < off; ++k) {
            const float send = up ? a[k] : a[k + off];
            const float keep = up ? a[k + off] : a[k];
            a[k] = keep + __shfl_xor_sync(0xffffffffu, send, off);
        }
    }
    smem[wid * 32 + lane] = a[0];
    __syncthreads();
    float r = 0.f;
    if (wid == 0)
        for (int w = 0; w < nw; ++w) r += smem[w * 32 + lane];
    return r;
}

__device__ __forceinline__ long long block_sum_ll(long long v, long long* smem) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) smem[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < nw ? smem[lane] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

// Last-block-done: returns true in every thread of the last block to finish.
__device__ __forceinline__ bool last_block(unsigned int* ticket) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

// Ticket increment with release (this block's prior writes, ordered before it
// by a block barrier) and acquire (the writes of the blocks that incremented
// before) semantics at GPU scope.
__device__ __forceinline__ unsigned int ticket_acq_rel(unsigned int* t) {
    unsigned int old;
    asm volatile("atom.add.acq_rel.gpu.u32 %0, [%1], 1;" : "=r"(old) : "l"(t) : "memory");
    return old;
}

// ----------------------------------------------------------- FP64 solver

// LDL^T of the 6x6 symmetric positive definite normal matrix and the solve
// (the effect of Eigen's ldlt().solve at Tracking.cc:388; for SPD systems the
// factorisation needs no pivoting).  Fully unrolled so that every array stays
// in registers.
__device__ __forceinline__ void ldlt6(const double* A, const double* b, double* x) {
    double L[6][6], D[6], Dinv[6], y[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        double d = A[k * 6 + k];
#pragma unroll
        for (int j = 0; j < k; ++j) d -= L[k][j] * L[k][j] * D[j];
        D[k] = d;
        const double inv = 1.0 / d;
        Dinv[k] = inv;
#pragma unroll
        for (int i = k + 1; i < 6; ++i) {
            double t = A[i * 6 + k];
#pragma unroll
            for (int j = 0; j < k; ++j) t -= L[i][j] * L[k][j] * D[j];
            L[i][k] = t * inv;
        }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double t = b[i];
#pragma unroll
        for (int j = 0; j < i; ++j) t -= L[i][j] * y[j];
        y[i] = t;
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) y[i] *= Dinv[i];
#pragma unroll
    for (int i = 5; i >= 0; --i) {
        double t = y[i];
#pragma unroll
        for (int j = i + 1; j < 6; ++j) t -= L[j][i] * x[j];
        x[i] = t;
    }
}

// exp of the se(3) tangent (upsilon, omega) -- the Sophus::SE3d::exp of
// Tracking.cc:389 restated from the mathematics (Rodrigues rotation, left
// Jacobian for the translation, Taylor series near zero).
__device__ __forceinline__ void se3_exp(const double* xi, double* T) {
    const double* u = xi;
    const double* w = xi + 3;
    double th2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    double th = sqrt(th2);
    double W[9] = {0, -w[2], w[1], w[2], 0, -w[0], -w[1], w[0], 0};
    double W2[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double s = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) s += W[i * 3 + k] * W[k * 3 + j];
            W2[i * 3 + j] = s;
        }
    double a, b, c;
    if (th < 1e-5) {
        a = 1 - th2 / 6 + th2 * th2 / 120;
        b = 0.5 - th2 / 24 + th2 * th2 / 720;
        c = 1.0 / 6 - th2 / 120 + th2 * th2 / 5040;
    } else {
        double s = sin(th), co = cos(th);
        a = s / th;
        b = (1 - co) / th2;
        c = (th - s) / (th2 * th);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double vi[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double I = (i == j) ? 1.0 : 0.0;
            T[i * 4 + j] = I + a * W[i * 3 + j] + b * W2[i * 3 + j];
            vi[j] = I + b * W[i * 3 + j] + c * W2[i * 3 + j];
        }
        T[i * 4 + 3] = vi[0] * u[0] + vi[1] * u[1] + vi[2] * u[2];
    }
    T[12] = T[13] = T[14] = 0;
    T[15] = 1;
}

__device__ __forceinline__ void mat4_mul(const double* A, const double* B, double* C) {
    double T[16];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double s = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) s += A[i * 4 + k] * B[k * 4 + j];
            T[i * 4 + j] = s;
        }
#pragma unroll
    for (int i = 0; i < 16; ++i) C[i] = T[i];
}

__device__ __forceinline__ void mat4_rigid_inv(const double* A, double* B) {
    double T[16];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) T[i * 4 + j] = A[j * 4 + i];
#pragma unroll
    for (int i = 0; i < 3; ++i)
        T[i * 4 + 3] = -(T[i * 4 + 0] * A[3] + T[i * 4 + 1] * A[7] + T[i * 4 + 2] * A[11]);
    T[12] = T[13] = T[14] = 0;
    T[15] = 1;
#pragma unroll
    for (int i = 0; i < 16; ++i) B[i] = T[i];
}

__device__ double euler_sin_norm(const double* T) {
    double a = atan2(-T[6], T[10]);
    double b = atan2(T[2], sqrt(T[0] * T[0] + T[1] * T[1]));
    double c = atan2(-T[1], T[0]);
    double sa = sin(a), sb = sin(b), sc = sin(c);
    return sqrt(sa * sa + sb * sb + sc * sc);
}

__device__ __forceinline__ void unpack29(const double* s, double* A, double* b) {
    int n = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = i; j < 7; ++j) {
            double v = s[n++];
            if (j == 6)
                b[i] = v;
            else
                A[j * 6 + i] = A[i * 6 + j] = v;
        }
}

// ------------------------------------------------------------------ kernels

// Frame start: the next pose starts from the last pose (TrackFrame's
// bootstrap fallback, Tracking.cc:156-159) and delta is the identity.
__device__ __forceinline__ void track_begin_body(const BlockCtx&, TrackState* st) {
    for (int i = 0; i < 16; ++i) {
        st->pose[i] = st->last_pose[i];
        st->init_pose[i] = st->last_pose[i];
        st->delta[i] = (i % 5 == 0) ? 1.0 : 0.0;
    }
    st->cur = make_dev_pose_d(st->pose);
    st->last = make_dev_pose_d(st->last_pose);
    st->failed = 0;
    st->icp_error = st->rgb_error = qnan();
    st->icp_count = st->rgb_count = 0;
}
__global__ void k_track_begin(TrackState* st) { track_begin_body(own_ctx(), st); }
FB_FUSED_KERNEL(k_track_begin, track_begin_body, 32)

// Fixed-order FP64 sum of nv values over nb block partials laid out as
// partials[b * stride + v], computed by the whole block: thread t sums value
// (t % 32) over the block chunk (t / 32), then the 8 chunk sums are added in
// order.  Deterministic for a given nb.  out: shared array of nv doubles.
__device__ void reduce_partials(const float* __restrict__ partials, int nb, int stride, int nv, double* out,
                                double* scratch /* [8][32] shared */) {
    const int v = threadIdx.x & 31, c = threadIdx.x >> 5, nc = blockDim.x >> 5;
    const int per = (nb + nc - 1) / nc;
    for (int v0 = 0; v0 < nv; v0 += 32) {
        double s = 0;
        if (v0 + v < nv) {
            const int b0 = c * per, b1 = min(nb, b0 + per);
#pragma unroll 8
            for (int b = b0; b < b1; ++b) s += (double)partials[(size_t)b * stride + v0 + v];
        }
        scratch[c * 32 + v] = s;
        __syncthreads();
        if (c == 0 && v0 + v < nv) {
            double t = 0;
            for (int q = 0; q < nc; ++q) t += scratch[q * 32 + v];
            out[v0 + v] = t;
        }
        __syncthreads();
    }
}

// Capacity of the per-warp correspondence segments for n pixels: every warp
// of the pass-A grid gets as many slots as the pixels it visits.
size_t track_list_capacity(int n) {
    const int g = track_cluster_grid(n);
    const int iters = (n + g * 256 - 1) / (g * 256);
    return (size_t)g * iters * 256;
}

// Sum of a cluster's block sums: rank 0's first `nv` threads add value t of
// every block of the cluster in rank order (FP64) through distributed shared
// memory.  Every block of the cluster must call it (it holds two cluster
// barriers: the block sums are complete before rank 0 reads, and stay alive
// until it has read them).  Returns the sum in rank 0's threads t < nv.
template <typename T>
__device__ __forceinline__ double cluster_sum(cg::cluster_group& cl, T* s_vals, int nv) {
    double v = 0;
    cl.sync();
    if (cl.block_rank() == 0 && (int)threadIdx.x < nv) {
#pragma unroll
        for (int r = 0; r < kTrackCluster; ++r) v += (double)cl.map_shared_rank(s_vals, r)[threadIdx.x];
    }
    cl.sync();
    return v;
}

// Compensated FP32 (the precision form's reduction).  two_sum is Knuth's
// error-free sum (s + e == a + b exactly); pair_add adds two (hi, lo) pairs
// with the rounding error of the high parts carried into the low part and
// the result renormalised (Dekker's fast two-sum), so a sum of many block
// sums keeps about twice the float precision.
__device__ __forceinline__ float2 two_sum(float a, float b) {
    const float s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    const float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
    return make_float2(s, e);
}

__device__ __forceinline__ float2 pair_add(float2 x, float2 y) {
    const float2 s = two_sum(x.x, y.x);
    const float lo = __fadd_rn(__fadd_rn(x.y, y.y), s.y);
    const float hi = __fadd_rn(s.x, lo);
    return make_float2(hi, __fsub_rn(lo, __fsub_rn(hi, s.x)));
}

// pass A (one cluster of kTrackCluster blocks per group): ICP rows reduced per
// block, then per cluster into the group sums; RGB correspondences appended by
// each warp to its own segment of `list` in pixel-visit order (ballot +
// popc: deterministic, no block barrier in the pixel loop), with the
// correspondence count and sum of squared differences reduced the same way
// (integers below 2^53, exact as doubles).  L.rgbok must be set.
template <int kMinBlocks, bool kComp>
__global__ void __cluster_dims__(kTrackCluster, 1, 1) __launch_bounds__(256, kMinBlocks)
    k_track_a(TrackLevel L, TrackState* st, int2* list, int* counts) {
    const int N = L.W * L.H;
    const int G = gridDim.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int p = blockIdx.x * 256 + threadIdx.x;
    if (st->failed) return;   // uniform over the grid: written by an earlier kernel
    // the pose loads are in flight while the first chunks are staged
    const DevPose cur = st->cur, last = st->last;
    cg::cluster_group cl = cg::this_cluster();
    __shared__ float sm[8 * 32];
    __shared__ long long smll[32];
    __shared__ double s_vals[32];
    __shared__ PixelStage stg;
    const int iters = (N + G * 256 - 1) / (G * 256);
    const int base = blockIdx.x * 256;
    if (threadIdx.x == 0) {
        mbar_init(&stg.bar[0], 1);
        mbar_init(&stg.bar[1], 1);
        for (int c = 0; c < 2 && c < iters && base + c * G * 256 < N; ++c) stage_chunk(stg, c, L, base + c * G * 256, N);
    }
    __syncthreads();
    float acc[29];
#pragma unroll
    for (int k = 0; k < 29; ++k) acc[k] = 0.f;
    long long rc = 0, rsq = 0;
    const int gw = blockIdx.x * kTrackWarps + wid;
    int2* seg = list + (size_t)gw * iters * 32;
    const unsigned lt = (1u << lane) - 1u;
    int run = 0;
    for (int k = 0; k < iters; ++k, p += G * 256) {
        if (base + k * G * 256 >= N) break;   // uniform: no pixel of this block's chunk k
        const int buf = k & 1;
        if (!take_chunk(stg, buf, (uint32_t)(k >> 1))) {
            if (threadIdx.x == 0) atomicOr((unsigned*)&st->failed, 2u);
            return;
        }
        PixelIn in;
        if (p < N) in = staged_pixel(stg, buf, threadIdx.x);
        __syncthreads();   // buffer `buf` is read: chunk k + 2 may overwrite it
        if (threadIdx.x == 0 && k + 2 < iters && base + (k + 2) * G * 256 < N)
            stage_chunk(stg, buf, L, base + (k + 2) * G * 256, N);
        int r = -1;
        if (p < N) {
            float row[7];
            if (pixel_pass_a(L, cur, last, in, row, &r)) add_products(row, acc);
            if (r != -1) {
                int d = (r & 511) - 255;
                rc += 1;
                rsq += d * d;
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, r != -1);
        if (r != -1) seg[run + __popc(m & lt)] = make_int2(in.dxy, r);
        run += __popc(m);
    }
    if (lane == 0) counts[gw] = run;
    const float bsum = block_sum29(acc, sm);
    // block_sum_ll leaves the total in lane 0 of warp 0
    const long long bc = __shfl_sync(0xffffffffu, block_sum_ll(rc, smll), 0);
    const long long bs = __shfl_sync(0xffffffffu, block_sum_ll(rsq, smll), 0);
    if constexpr (kComp) {
        // precision form: block sums as compensated FP32 pairs, counts as integers
        __shared__ float s_f[32];
        __shared__ long long s_c[2];
        if (wid == 0) s_f[lane] = lane < 29 ? bsum : 0.f;
        if (threadIdx.x == 0) {
            s_c[0] = bc;
            s_c[1] = bs;
        }
        cl.sync();
        if (cl.block_rank() == 0 && threadIdx.x < 31) {
            const int g = blockIdx.x / kTrackCluster;
            if (threadIdx.x < 29) {
                float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                for (int r = 0; r < kTrackCluster; ++r)
                    acc = pair_add(acc, make_float2(cl.map_shared_rank(s_f, r)[threadIdx.x], 0.f));
                st->grp_icp2[g][threadIdx.x] = acc;
            } else {
                long long t = 0;
#pragma unroll
                for (int r = 0; r < kTrackCluster; ++r) t += cl.map_shared_rank(s_c, r)[threadIdx.x - 29];
                if (threadIdx.x == 29)
                    st->grp_cnt[g] = t;
                else
                    st->grp_sq[g] = t;
            }
        }
        cl.sync();
        return;
    }
    if (wid == 0) s_vals[lane] = lane < 29 ? (double)bsum : lane == 29 ? (double)bc : lane == 30 ? (double)bs : 0.0;
    const double v = cluster_sum(cl, s_vals, 31);
    if (cl.block_rank() == 0 && threadIdx.x < 31) {
        const int g = blockIdx.x / kTrackCluster;
        if (threadIdx.x < 29)
            st->grp_icp[g][threadIdx.x] = v;
        else if (threadIdx.x == 29)
            st->grp_cnt[g] = (long long)v;
        else
            st->grp_sq[g] = (long long)v;
    }
}

// Staging of the tracker state for the solve of one iteration.
struct SolveIO {
    double delta[16], last_pose[16], init_pose[16], pose[16];
    DevPose cur;
    float icp_error, icp_count, rgb_error, rgb_count;
    int failed;    // this iteration failed: pose rolled back to last_pose
    int updated;   // delta, pose and cur hold a Gauss-Newton update
};

__device__ void solve_staged(SolveIO& io, const double* s, int min_count, int is_final);

// The end of an iteration, in the block that finished last: the group sums
// of both passes in group order (FP64, or compensated FP32 in the precision
// form) -- value t & 63 (0..28 ICP, 32..60 RGB) over four fixed ranges of
// groups, then the ranges in order -- the Gauss-Newton update with one
// thread, and the new state written back in parallel.
template <bool kComp>
__device__ __forceinline__ void finish_iteration(TrackState* st, unsigned int* ticket, int NG, long long c,
                                                 long long q, float sigma, int min_count, int is_final,
                                                 SolveIO& io, double (&s_part)[4][64], float2 (&s_partc)[4][64],
                                                 double (&sums)[64]) {
    {
        const int val = threadIdx.x & 63, part = threadIdx.x >> 6;
        const int per = (NG + 3) / 4, g0 = part * per, g1 = min(NG, g0 + per);
        // the range's values are loaded 16 at a time before any is added (one
        // L2 round trip for the usual ten groups), then added in group order
        if constexpr (kComp) {
            // compensated FP32 over the groups; to FP64 only for the solve
            float2 t = make_float2(0.f, 0.f);
            if ((val & 31) < 29) {
                const float2* src = val < 32 ? &st->grp_icp2[0][val] : &st->grp_rgb2[0][val - 32];
                for (int g = g0; g < g1; g += 16) {
                    float2 v[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (g + j < g1) v[j] = __ldcg(src + (size_t)(g + j) * 32);
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (g + j < g1) t = pair_add(t, v[j]);
                }
            }
            s_partc[part][val] = t;
        } else {
            double t = 0;
            if ((val & 31) < 29) {
                const double* src = val < 32 ? &st->grp_icp[0][val] : &st->grp_rgb[0][val - 32];
                for (int g = g0; g < g1; g += 16) {
                    double v[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (g + j < g1) v[j] = __ldcg(src + (size_t)(g + j) * 32);
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (g + j < g1) t += v[j];
                }
            }
            s_part[part][val] = t;
        }
    }
    __syncthreads();
    if (threadIdx.x < 64) {
        if constexpr (kComp) {
            const float2 t = pair_add(pair_add(pair_add(s_partc[0][threadIdx.x], s_partc[1][threadIdx.x]),
                                               s_partc[2][threadIdx.x]),
                                      s_partc[3][threadIdx.x]);
            sums[threadIdx.x] = (double)t.x + (double)t.y;
        } else {
            sums[threadIdx.x] = ((s_part[0][threadIdx.x] + s_part[1][threadIdx.x]) + s_part[2][threadIdx.x]) +
                                s_part[3][threadIdx.x];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *ticket = 0;
        solve_staged(io, sums, min_count, is_final);
    }
    __syncthreads();
    // write back in parallel
    if (threadIdx.x < 16) {
        st->pose[threadIdx.x] = io.pose[threadIdx.x];
        if (io.updated) st->delta[threadIdx.x] = io.delta[threadIdx.x];
    } else if (threadIdx.x >= 32 && threadIdx.x < 32 + (int)(sizeof(DevPose) / 4)) {
        if (io.updated) ((float*)&st->cur)[threadIdx.x - 32] = ((const float*)&io.cur)[threadIdx.x - 32];
    } else if (threadIdx.x >= 64 && threadIdx.x < 93) {
        st->icp_sums[threadIdx.x - 64] = sums[threadIdx.x - 64];
        st->rgb_sums[threadIdx.x - 64] = sums[32 + threadIdx.x - 64];
    } else if (threadIdx.x == 96) {
        st->icp_error = io.icp_error;
        st->icp_count = io.icp_count;
        st->rgb_error = io.rgb_error;
        st->rgb_count = io.rgb_count;
        st->rgb_cnt = c;
        st->rgb_sq = q;
        st->sigma = sigma;
        st->failed = io.failed;
    }
}

// pass B (clusters as in pass A): every block derives sigma from pass A's
// group counts (integers: the same value in every block) and builds the RGB
// rows of its warps' segments; each cluster reduces its rows into a group
// sum; the last cluster to finish adds the groups of both passes in group
// order (FP64) and performs the Gauss-Newton update with one warp.
template <int kMinBlocks, bool kComp>
__global__ void __cluster_dims__(kTrackCluster, 1, 1) __launch_bounds__(256, kMinBlocks)
    k_track_b(TrackLevel L, TrackState* st, unsigned int* ticket, const int2* list, const int* counts, int seg_size,
              int min_count, int is_final) {
    cg::cluster_group cl = cg::this_cluster();
    __shared__ float sm[32 * 29];
    __shared__ float s_rgb[32];
    __shared__ double s_part[4][64];
    __shared__ float2 s_partc[4][64];
    __shared__ double sums[64];
    __shared__ bool s_last;
    __shared__ SolveIO io;
    const int G = gridDim.x, NG = G / kTrackCluster, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // stage the solve's inputs early (used by the last cluster's first block)
    if (cl.block_rank() == 0) {
        if (threadIdx.x >= 64 && threadIdx.x < 80) {
            const int i = threadIdx.x - 64;
            io.delta[i] = st->delta[i];
            io.last_pose[i] = st->last_pose[i];
            io.init_pose[i] = st->init_pose[i];
        }
        if (threadIdx.x == 80) {
            io.icp_error = st->icp_error;
            io.icp_count = st->icp_count;
        }
    }
    if (st->failed) return;
    // the first row's inputs (list entry, then its gathers) are loaded while
    // the robust scale is reduced: neither needs the other
    const int gw = blockIdx.x * kTrackWarps + wid;
    const int2* seg = list + (size_t)gw * seg_size;
    const int nseg = counts[gw];
    RgbIn first{};
    if (lane < nseg) first = rgb_fetch_entry(L, seg[lane]);
    const DevPose cur = st->cur, last = st->last;
    // sigma = sqrt((float) sum / count) (Reduction.cu:606-608); every warp
    // adds the group counts itself (integers: exact in any order)
    long long c = 0, q = 0;
    for (int g = lane; g < NG; g += 32) {
        c += __ldcg(&st->grp_cnt[g]);
        q += __ldcg(&st->grp_sq[g]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_xor_sync(0xffffffffu, c, o);
        q += __shfl_xor_sync(0xffffffffu, q, o);
    }
    const float sigma = sqrtf((float)q / (float)(c == 0 ? 1 : c));
    float acc[29];
#pragma unroll
    for (int k = 0; k < 29; ++k) acc[k] = 0.f;
    add_segment_rows(L, cur, last, sigma, seg, nseg, lane, acc, first);
    const float bsum = block_sum29(acc, sm);
    if (wid == 0) s_rgb[lane] = lane < 29 ? bsum : 0.f;
    const int grp = blockIdx.x / kTrackCluster;
    if constexpr (kComp) {
        cl.sync();
        if (cl.block_rank() == 0 && threadIdx.x < 29) {
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int r = 0; r < kTrackCluster; ++r)
                acc = pair_add(acc, make_float2(cl.map_shared_rank(s_rgb, r)[threadIdx.x], 0.f));
            st->grp_rgb2[grp][threadIdx.x] = acc;
        }
        cl.sync();
        if (cl.block_rank() != 0) return;
    } else {
        const double v = cluster_sum(cl, s_rgb, 29);
        if (cl.block_rank() != 0) return;
        if (threadIdx.x < 29) st->grp_rgb[grp][threadIdx.x] = v;
    }
    // last cluster (its rank-0 block) to finish
    __syncthreads();
    if (threadIdx.x == 0) s_last = ticket_acq_rel(ticket) == (unsigned)(NG - 1);
    __syncthreads();
    if (!s_last) return;
    finish_iteration<kComp>(st, ticket, NG, c, q, sigma, min_count, is_final, io, s_part, s_partc, sums);
}

// Shape of the group forms below: groups per block and resident blocks per
// SM (4: half the registers, some spilled; 2: none spilled).
constexpr int kGroupsPerBlock = 1;
constexpr int kGrpMinBlocks = 4;

// Group forms of k_track_a / k_track_b for sessions sharing the GPU: one
// block per group does the work of the group's kTrackCluster clustered
// blocks -- logical blocks b = kTrackCluster * group + r, r in rank order,
// each with the pixels, warp segments and block sums the clustered block b
// has in a grid of G blocks -- and adds their sums in rank order as the
// cluster reduction does.  The results are therefore the clustered kernels'
// bit for bit, on a grid of G / kTrackCluster blocks: a session's pass holds
// a quarter of the block slots for longer, and other sessions' passes run
// beside it.
template <int kMinBlocks, bool kComp>
__device__ __forceinline__ void track_a_grp_body(const BlockCtx& ctx, TrackLevel L, TrackState* st, int2* list,
                                                 int* counts, int G, int gpc) {
    const int N = L.W * L.H, NG = G / kTrackCluster;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (st->failed) return;   // uniform over the grid: written by an earlier kernel
    __shared__ float sm[8 * 32];
    __shared__ long long smll[32];
    __shared__ double s_vals[kTrackCluster][32];
    __shared__ float s_f[kTrackCluster][32];
    __shared__ long long s_c[kTrackCluster][2];
    __shared__ PixelStage stg;
    const DevPose cur = st->cur, last = st->last;
    const int iters = (N + G * 256 - 1) / (G * 256);
    const unsigned lt = (1u << lane) - 1u;
    // thread 0 keeps the copies two chunks ahead of the block
    ChunkCursor prod{0, 0, 0, 0};
    uint32_t used = 0;
    if (threadIdx.x == 0) {
        mbar_init(&stg.bar[0], 1);
        mbar_init(&stg.bar[1], 1);
        prod.settle(ctx.bx, gpc, NG, iters, G * 256, N);
        for (int c = 0; c < 2 && prod.start >= 0; ++c) {
            stage_chunk(stg, c, L, prod.start, N);
            ++prod.k;
            prod.settle(ctx.bx, gpc, NG, iters, G * 256, N);
        }
    }
    __syncthreads();
    for (int j = 0; j < gpc; ++j) {
    const int g = ctx.bx * gpc + j;
    if (g >= NG) break;
    for (int r = 0; r < kTrackCluster; ++r) {
        const int b = g * kTrackCluster + r;
        int p = b * 256 + threadIdx.x;
        float acc[29];
#pragma unroll
        for (int k = 0; k < 29; ++k) acc[k] = 0.f;
        long long rc = 0, rsq = 0;
        const int gw = b * kTrackWarps + wid;
        int2* seg = list + (size_t)gw * iters * 32;
        int run = 0;
        for (int k = 0; k < iters; ++k, p += G * 256) {
            if (b * 256 + k * G * 256 >= N) break;   // uniform: no pixel of this chunk
            const int buf = (int)(used & 1u);
            if (!take_chunk(stg, buf, used >> 1)) {
                if (threadIdx.x == 0) atomicOr((unsigned*)&st->failed, 2u);
                return;
            }
            ++used;
            PixelIn in;
            if (p < N) in = staged_pixel(stg, buf, threadIdx.x);
            __syncthreads();   // buffer `buf` is read: the chunk two ahead may overwrite it
            if (threadIdx.x == 0 && prod.start >= 0) {
                stage_chunk(stg, buf, L, prod.start, N);
                ++prod.k;
                prod.settle(ctx.bx, gpc, NG, iters, G * 256, N);
            }
            int rr = -1;
            if (p < N) {
                float row[7];
                if (pixel_pass_a(L, cur, last, in, row, &rr)) add_products(row, acc);
                if (rr != -1) {
                    int d = (rr & 511) - 255;
                    rc += 1;
                    rsq += d * d;
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, rr != -1);
            if (rr != -1) seg[run + __popc(m & lt)] = make_int2(in.dxy, rr);
            run += __popc(m);
        }
        if (lane == 0) counts[gw] = run;
        const float bsum = block_sum29(acc, sm);
        const long long bc = __shfl_sync(0xffffffffu, block_sum_ll(rc, smll), 0);
        const long long bs = __shfl_sync(0xffffffffu, block_sum_ll(rsq, smll), 0);
        if constexpr (kComp) {
            if (wid == 0) s_f[r][lane] = lane < 29 ? bsum : 0.f;
            if (threadIdx.x == 0) {
                s_c[r][0] = bc;
                s_c[r][1] = bs;
            }
        } else {
            if (wid == 0)
                s_vals[r][lane] = lane < 29 ? (double)bsum : lane == 29 ? (double)bc : lane == 30 ? (double)bs : 0.0;
        }
        __syncthreads();   // sm / smll are reused by the next logical block
    }
    if (threadIdx.x < 31) {
        if constexpr (kComp) {
            if (threadIdx.x < 29) {
                float2 acc = make_float2(0.f, 0.f);
#pragma unroll
                for (int r = 0; r < kTrackCluster; ++r) acc = pair_add(acc, make_float2(s_f[r][threadIdx.x], 0.f));
                st->grp_icp2[g][threadIdx.x] = acc;
            } else {
                long long t = 0;
#pragma unroll
                for (int r = 0; r < kTrackCluster; ++r) t += s_c[r][threadIdx.x - 29];
                if (threadIdx.x == 29)
                    st->grp_cnt[g] = t;
                else
                    st->grp_sq[g] = t;
            }
        } else {
            double v = 0;
#pragma unroll
            for (int r = 0; r < kTrackCluster; ++r) v += s_vals[r][threadIdx.x];
            if (threadIdx.x < 29)
                st->grp_icp[g][threadIdx.x] = v;
            else if (threadIdx.x == 29)
                st->grp_cnt[g] = (long long)v;
            else
                st->grp_sq[g] = (long long)v;
        }
    }
    __syncthreads();   // s_vals / s_f / s_c are reused by the next group
    }
}

template <int kMinBlocks, bool kComp>
__device__ __forceinline__ void track_b_grp_body(const BlockCtx& ctx, TrackLevel L, TrackState* st,
                                                 unsigned int* ticket, const int2* list, const int* counts,
                                                 int seg_size, int min_count, int is_final, int NG, int gpc) {
    __shared__ float sm[32 * 29];
    __shared__ float s_rgb[kTrackCluster][32];
    __shared__ double s_part[4][64];
    __shared__ float2 s_partc[4][64];
    __shared__ double sums[64];
    __shared__ bool s_last;
    __shared__ SolveIO io;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // stage the solve's inputs early (used by the last block)
    if (threadIdx.x >= 64 && threadIdx.x < 80) {
        const int i = threadIdx.x - 64;
        io.delta[i] = st->delta[i];
        io.last_pose[i] = st->last_pose[i];
        io.init_pose[i] = st->init_pose[i];
    }
    if (threadIdx.x == 80) {
        io.icp_error = st->icp_error;
        io.icp_count = st->icp_count;
    }
    if (st->failed) return;
    const DevPose cur = st->cur, last = st->last;
    // sigma as in k_track_b
    long long c = 0, q = 0;
    for (int g = lane; g < NG; g += 32) {
        c += __ldcg(&st->grp_cnt[g]);
        q += __ldcg(&st->grp_sq[g]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_xor_sync(0xffffffffu, c, o);
        q += __shfl_xor_sync(0xffffffffu, q, o);
    }
    const float sigma = sqrtf((float)q / (float)(c == 0 ? 1 : c));
    for (int j = 0; j < gpc; ++j) {
    const int grp = ctx.bx * gpc + j;
    if (grp >= NG) break;
    for (int r = 0; r < kTrackCluster; ++r) {
        const int b = grp * kTrackCluster + r;
        float acc[29];
#pragma unroll
        for (int k = 0; k < 29; ++k) acc[k] = 0.f;
        const int gw = b * kTrackWarps + wid;
        add_segment_rows_seq(L, cur, last, sigma, list + (size_t)gw * seg_size, counts[gw], lane, acc);
        const float bsum = block_sum29(acc, sm);
        if (wid == 0) s_rgb[r][lane] = lane < 29 ? bsum : 0.f;
        __syncthreads();   // sm is reused by the next logical block
    }
    if constexpr (kComp) {
        if (threadIdx.x < 29) {
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int r = 0; r < kTrackCluster; ++r) acc = pair_add(acc, make_float2(s_rgb[r][threadIdx.x], 0.f));
            st->grp_rgb2[grp][threadIdx.x] = acc;
        }
    } else {
        if (threadIdx.x < 29) {
            double v = 0;
#pragma unroll
            for (int r = 0; r < kTrackCluster; ++r) v += (double)s_rgb[r][threadIdx.x];
            st->grp_rgb[grp][threadIdx.x] = v;
        }
    }
    __syncthreads();   // s_rgb is reused by the next group
    }
    // last block to finish
    __syncthreads();
    if (threadIdx.x == 0) s_last = ticket_acq_rel(ticket) == (unsigned)ctx.gx - 1u;
    __syncthreads();
    if (!s_last) return;
    finish_iteration<kComp>(st, ticket, NG, c, q, sigma, min_count, is_final, io, s_part, s_partc, sums);
}

template <int kMinBlocks, bool kComp>
__global__ void __launch_bounds__(256, kMinBlocks)
    k_track_a_grp(TrackLevel L, TrackState* st, int2* list, int* counts, int G, int gpc) {
    track_a_grp_body<kMinBlocks, kComp>(own_ctx(), L, st, list, counts, G, gpc);
}
template <int kMinBlocks, bool kComp>
__global__ void __launch_bounds__(256, kMinBlocks)
    k_track_a_grp_fused(const __grid_constant__ FusedParams<ArgsOf<decltype(&k_track_a_grp<kMinBlocks, kComp>)>> fp) {
    run_part(fp, [](const BlockCtx& c, const auto&... a) { track_a_grp_body<kMinBlocks, kComp>(c, a...); });
}

template <int kMinBlocks, bool kComp>
__global__ void __launch_bounds__(256, kMinBlocks)
    k_track_b_grp(TrackLevel L, TrackState* st, unsigned int* ticket, const int2* list, const int* counts,
                  int seg_size, int min_count, int is_final, int NG, int gpc) {
    track_b_grp_body<kMinBlocks, kComp>(own_ctx(), L, st, ticket, list, counts, seg_size, min_count, is_final, NG,
                                        gpc);
}
template <int kMinBlocks, bool kComp>
__global__ void __launch_bounds__(256, kMinBlocks)
    k_track_b_grp_fused(const __grid_constant__ FusedParams<ArgsOf<decltype(&k_track_b_grp<kMinBlocks, kComp>)>> fp) {
    run_part(fp, [](const BlockCtx& c, const auto&... a) { track_b_grp_body<kMinBlocks, kComp>(c, a...); });
}

// The Gauss-Newton update of one iteration (Tracking.cc:319-394) and, after
// the last one, the acceptance test (Tracking.cc:398-408), on staged state:
// io.delta / last_pose / init_pose / icp_error in; io.pose, delta, cur,
// errors, counts, failed and updated out (a failed count or error test
// leaves delta and cur as they were and sets pose = last_pose; a failed
// acceptance test does so after the update).  One thread; every array in
// registers.
__device__ void solve_staged(SolveIO& io, const double* s, int min_count, int is_final) {
    bool fail = false;
    {
        float r0 = (float)s[32 + 27], r1 = (float)s[32 + 28];
        float err = sqrtf(r0) / r1;
        io.rgb_error = err;
        io.rgb_count = r1;
        if (isnan(err) || (int)r1 < min_count) fail = true;
    }
    if (!fail) {
        float q0 = (float)s[27], q1 = (float)s[28];
        float icp_err = sqrtf(q0) / q1;
        io.icp_error = icp_err;
        io.icp_count = q1;
        if (isnan(icp_err) || (int)q1 < min_count) fail = true;
    }
    io.failed = 0;
    io.updated = 0;
    if (fail) {
        for (int i = 0; i < 16; ++i) io.pose[i] = io.last_pose[i];
        io.failed = 1;
        return;
    }
    double Ar[36], br[6], Ai[36], bi[6], A[36], b[6], x[6], dT[16], dinv[16], delta[16], lastp[16], pose[16];
    unpack29(s + 32, Ar, br);
    unpack29(s, Ai, bi);
    const float w = 1e-4f;
#pragma unroll
    for (int i = 0; i < 36; ++i) A[i] = Ar[i] * (double)w + Ai[i];
#pragma unroll
    for (int i = 0; i < 6; ++i) b[i] = br[i] * (double)w + bi[i];
    ldlt6(A, b, x);
    se3_exp(x, dT);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        delta[i] = io.delta[i];
        lastp[i] = io.last_pose[i];
    }
    mat4_mul(dT, delta, delta);
    mat4_rigid_inv(delta, dinv);
    mat4_mul(lastp, dinv, pose);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        io.delta[i] = delta[i];
        io.pose[i] = pose[i];
    }
    io.cur = make_dev_pose_d(pose);
    io.updated = 1;
    if (is_final) {
        double pinv[16], p[16], init[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) init[i] = io.init_pose[i];
        mat4_rigid_inv(init, pinv);
        mat4_mul(pinv, pose, p);
        double tn = sqrt(p[3] * p[3] + p[7] * p[7] + p[11] * p[11]);
        if (!(io.icp_error < 0.0001f && euler_sin_norm(p) <= 0.1 && tn <= 0.1)) {
            for (int i = 0; i < 16; ++i) io.pose[i] = io.last_pose[i];
            io.failed = 1;
        }
    }
}

// The Gauss-Newton update of one iteration (Tracking.cc:319-394) and, after
// the last one, the acceptance test (Tracking.cc:398-408).  One thread; the
// normal equations are in FP64, every array in registers.
// The Gauss-Newton update of one iteration (Tracking.cc:319-394) and, after
// the last one, the acceptance test (Tracking.cc:398-408), from the FP64 sums
// s (ICP in s[0..28], RGB in s[32..60]).  One thread; every array in
// registers.
__device__ __forceinline__ void solve_step(TrackState* st, const double* s, int min_count, int is_final) {
    bool fail = false;
    {
        float r0 = (float)s[32 + 27], r1 = (float)s[32 + 28];
        float err = sqrtf(r0) / r1;
        st->rgb_error = err;
        st->rgb_count = r1;
        if (isnan(err) || (int)r1 < min_count) fail = true;
    }
    float icp_err = st->icp_error;
    if (!fail) {
        float q0 = (float)s[27], q1 = (float)s[28];
        icp_err = sqrtf(q0) / q1;
        st->icp_error = icp_err;
        st->icp_count = q1;
        if (isnan(icp_err) || (int)q1 < min_count) fail = true;
    }
    if (fail) {
        for (int i = 0; i < 16; ++i) st->pose[i] = st->last_pose[i];
        __threadfence();
        st->failed = 1;
        return;
    }
    double Ar[36], br[6], Ai[36], bi[6], A[36], b[6], x[6], dT[16], dinv[16], delta[16], lastp[16], pose[16];
    unpack29(s + 32, Ar, br);
    unpack29(s, Ai, bi);
    const float w = 1e-4f;
#pragma unroll
    for (int i = 0; i < 36; ++i) A[i] = Ar[i] * (double)w + Ai[i];
#pragma unroll
    for (int i = 0; i < 6; ++i) b[i] = br[i] * (double)w + bi[i];
    ldlt6(A, b, x);
    se3_exp(x, dT);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        delta[i] = st->delta[i];
        lastp[i] = st->last_pose[i];
    }
    mat4_mul(dT, delta, delta);
    mat4_rigid_inv(delta, dinv);
    mat4_mul(lastp, dinv, pose);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        st->delta[i] = delta[i];
        st->pose[i] = pose[i];
    }
    st->cur = make_dev_pose_d(pose);
    if (is_final) {
        double pinv[16], p[16], init[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) init[i] = st->init_pose[i];
        mat4_rigid_inv(init, pinv);
        mat4_mul(pinv, pose, p);
        double tn = sqrt(p[3] * p[3] + p[7] * p[7] + p[11] * p[11]);
        if (!(icp_err < 0.0001f && euler_sin_norm(p) <= 0.1 && tn <= 0.1)) {
            for (int i = 0; i < 16; ++i) st->pose[i] = st->last_pose[i];
            __threadfence();
            st->failed = 1;
        }
    }
    __threadfence();
}

// Single-step entry points (the reference's ICPStep / RGBStep): reduce the
// sums of one pass into out[29] (+ rgb count / sum of squares) in FP64.
__global__ void __launch_bounds__(256) k_step_icp(TrackLevel L, DevPose cur, DevPose last, float* partials,
                                                  unsigned int* ticket, double* out) {
    __shared__ float sm[32 * 29];
    float acc[29];
#pragma unroll
    for (int k = 0; k < 29; ++k) acc[k] = 0.f;
    const int N = L.W * L.H;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x) {
        const int y = p / L.W, x = p - y * L.W;
        float row[7];
        if (icp_row(L, cur, last, x, y, row)) add_products(row, acc);
    }
    block_sum<29>(acc, sm);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < 29; ++k) partials[(size_t)blockIdx.x * 32 + k] = acc[k];
    if (!last_block(ticket)) return;
    __shared__ double scratch[8 * 32];
    __shared__ double sums[32];
    reduce_partials(partials, gridDim.x, 32, 29, sums, scratch);
    if (threadIdx.x < 29) out[threadIdx.x] = sums[threadIdx.x];
    if (threadIdx.x == 0) *ticket = 0;
}

__global__ void __launch_bounds__(256) k_step_rgb_a(TrackLevel L, DevPose cur, DevPose last, long long* partials,
                                                    unsigned int* ticket, int* residual, double* out) {
    __shared__ long long smll[32];
    long long rc = 0, rsq = 0;
    const int N = L.W * L.H;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x) {
        const int y = p / L.W, x = p - y * L.W;
        int r = rgb_corresp(L, cur, last, x, y);
        residual[p] = r;
        if (r != -1) {
            int d = (r & 511) - 255;
            rc += 1;
            rsq += d * d;
        }
    }
    long long bc = block_sum_ll(rc, smll);
    long long bs = block_sum_ll(rsq, smll);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = bc;
        partials[2 * blockIdx.x + 1] = bs;
    }
    if (!last_block(ticket)) return;
    if (threadIdx.x == 0) {
        long long c = 0, q = 0;
        for (int b = 0; b < gridDim.x; ++b) { c += partials[2 * b]; q += partials[2 * b + 1]; }
        out[29] = (double)c;
        out[30] = (double)q;
        out[31] = sqrtf((float)q / (float)(c == 0 ? 1 : c));
        *ticket = 0;
    }
}

__global__ void __launch_bounds__(256) k_step_rgb_b(TrackLevel L, DevPose cur, DevPose last, float* partials,
                                                    unsigned int* ticket, const int* residual, double* out) {
    __shared__ float sm[32 * 29];
    const float sigma = (float)out[31];
    float acc[29];
#pragma unroll
    for (int k = 0; k < 29; ++k) acc[k] = 0.f;
    const int N = L.W * L.H;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < N; p += gridDim.x * blockDim.x) {
        int r = residual[p];
        if (r == -1) continue;
        const int y = p / L.W, x = p - y * L.W;
        float row[7];
        rgb_row(L, cur, last, x, y, r, sigma, row);
        add_products(row, acc);
    }
    block_sum<29>(acc, sm);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < 29; ++k) partials[(size_t)blockIdx.x * 32 + k] = acc[k];
    if (!last_block(ticket)) return;
    __shared__ double scratch[8 * 32];
    __shared__ double sums[32];
    reduce_partials(partials, gridDim.x, 32, 29, sums, scratch);
    if (threadIdx.x < 29) out[threadIdx.x] = sums[threadIdx.x];
    if (threadIdx.x == 0) *ticket = 0;
}

// ---------------------------------------------------------------- launchers

// Two resident blocks of 256 threads per SM at most (the row kernels use
// ~110 registers per thread).
int track_grid(int n) {
    static int cap = 0;
    if (!cap) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cap = sms > 0 ? 2 * sms : 296;
        if (cap > kTrackMaxBlocks) cap = kTrackMaxBlocks;
    }
    int g = (n + 255) / 256;
    return g < cap ? g : cap;
}

int launch_track_begin(TrackState* st, cudaStream_t s) {
    fb_launch(k_track_begin, (const void*)k_track_begin_fused, 1, 1, 0, s, st);
    return 1;
}

// Grid of the clustered per-iteration kernels: track_grid rounded up to whole
// clusters, at most as many clusters as can be resident at once (a cluster
// needs all its blocks on one GPC, so fewer than 2 x SMs / kTrackCluster may
// fit), so that every launch runs in a single wave.
int track_cluster_grid(int n) {
    static int cap = 0;
    if (!cap) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        int c = sms > 0 ? 2 * sms / kTrackCluster : kTrackMaxGroups;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(c * kTrackCluster);
        cfg.blockDim = dim3(256);
        int ca = 0, cb = 0;
        // the register-rich instances (two blocks per SM) bound the grid of both
        if (cudaOccupancyMaxActiveClusters(&ca, (void*)k_track_a<2, false>, &cfg) == cudaSuccess && ca > 0 && ca < c)
            c = ca;
        if (cudaOccupancyMaxActiveClusters(&cb, (void*)k_track_b<2, false>, &cfg) == cudaSuccess && cb > 0 && cb < c)
            c = cb;
        cudaGetLastError();
        if (c > kTrackMaxGroups) c = kTrackMaxGroups;
        cap = c * kTrackCluster;
    }
    const int g = (n + 255) / 256;
    const int gc = (g + kTrackCluster - 1) / kTrackCluster * kTrackCluster;
    return gc < cap ? gc : cap;
}

int launch_track_iter(const TrackLevel& L, TrackState* st, unsigned int* tickets, int2* residual, int* counts,
                      int min_count, bool is_final, cudaStream_t s, bool shared_gpu, bool compensated) {
    const int n = L.W * L.H;
    const int g = track_cluster_grid(n);
    const int seg = (n + g * 256 - 1) / (g * 256) * 32;
    const int fin = is_final ? 1 : 0;
    // sessions sharing the GPU: the group forms, kGroupsPerBlock groups per
    // block, the same results; fused launches (a recorder) take the group
    // forms too, since clusters do not span the parts of a fused grid
    if (launch_recorder()) shared_gpu = true;
    const int ng = g / kTrackCluster, gpc = kGroupsPerBlock, gb = (ng + gpc - 1) / gpc;
    if (compensated) {
        if (shared_gpu) {
            fb_launch(k_track_a_grp<kGrpMinBlocks, true>, (const void*)k_track_a_grp_fused<kGrpMinBlocks, true>, gb,
                      256, 0, s, L, st, residual, counts, g, gpc);
            fb_launch(k_track_b_grp<kGrpMinBlocks, true>, (const void*)k_track_b_grp_fused<kGrpMinBlocks, true>, gb,
                      256, 0, s, L, st, tickets + 1, residual, counts, seg, min_count, fin, ng, gpc);
        } else {
            k_track_a<2, true><<<g, 256, 0, s>>>(L, st, residual, counts);
            k_track_b<2, true><<<g, 256, 0, s>>>(L, st, tickets + 1, residual, counts, seg, min_count, fin);
        }
    } else if (shared_gpu) {
        fb_launch(k_track_a_grp<kGrpMinBlocks, false>, (const void*)k_track_a_grp_fused<kGrpMinBlocks, false>, gb, 256,
                  0, s, L, st, residual, counts, g, gpc);
        fb_launch(k_track_b_grp<kGrpMinBlocks, false>, (const void*)k_track_b_grp_fused<kGrpMinBlocks, false>, gb, 256,
                  0, s, L, st, tickets + 1, residual, counts, seg, min_count, fin, ng, gpc);
    } else {
        k_track_a<2, false><<<g, 256, 0, s>>>(L, st, residual, counts);
        k_track_b<2, false><<<g, 256, 0, s>>>(L, st, tickets + 1, residual, counts, seg, min_count, fin);
    }
    return 2;
}

int launch_step_icp(const TrackLevel& L, const DevPose& cur, const DevPose& last, float* partials,
                     unsigned int* ticket, double* out, cudaStream_t s) {
    k_step_icp<<<track_grid(L.W * L.H), 256, 0, s>>>(L, cur, last, partials, ticket, out);
    return 1;
}

int launch_step_rgb(const TrackLevel& L, const DevPose& cur, const DevPose& last, float* partials,
                     unsigned int* tickets, int* residual, double* out, cudaStream_t s) {
    const int g = track_grid(L.W * L.H);
    k_step_rgb_a<<<g, 256, 0, s>>>(L, cur, last, (long long*)partials, tickets + 0, residual, out);
    k_step_rgb_b<<<g, 256, 0, s>>>(L, cur, last, partials, tickets + 1, residual, out);
    return 2;
}

}  // namespace fb
