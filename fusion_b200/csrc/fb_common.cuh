// Shared device definitions of the B200 dense-fusion path.
//
// Arithmetic convention.  Wherever the reference evaluates a float
// expression whose result becomes an integer, a pixel/voxel/block index or a
// threshold decision (projections truncated to pixels, voxel coordinates
// truncated to blocks, visibility and truncation tests, colour bytes), the
// kernels here evaluate it with the non-contracting intrinsics below, one
// IEEE binary32 operation at a time, in the order the reference writes it.
// The result is reproducible: the same inputs give the same indices on every
// run, in every batch mix and in the CPU oracle's reference-precision mode.
// Continuous quantities (normal-equation sums, TSDF averages, ray positions)
// use ordinary float arithmetic.
#ifndef FB_COMMON_CUH
#define FB_COMMON_CUH

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace fb {

// ---- non-contracting float ops (order-exact) ----
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }
// a / b given y, the correctly rounded reciprocal of b (__frcp_rn(b)), by
// Markstein's correction step (Markstein 1990): q = a y, r = a - q b (exact
// by FMA), q + r y rounded once.  This is the IEEE quotient fd(a, b) when a,
// b and a / b are normal floats or a is zero (the case r == 0 keeps q and its
// sign); b must not be zero.  Several quotients by one divisor then share
// one reciprocal.
__device__ __forceinline__ float fd_rcp(float a, float b, float y) {
    const float q = __fmul_rn(a, y);
    const float r = __fmaf_rn(-q, b, a);
    return r == 0.0f ? q : __fmaf_rn(r, y, q);
}
__device__ __forceinline__ float fsq(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }

struct f3 { float x, y, z; };
__device__ __forceinline__ f3 mk3(float x, float y, float z) { return {x, y, z}; }
// float3 * float3 (VectorMath.h:191-193): ((x*x') + (y*y')) + (z*z')
__device__ __forceinline__ float dot3(f3 a, f3 b) { return fa(fa(fm(a.x, b.x), fm(a.y, b.y)), fm(a.z, b.z)); }
__device__ __forceinline__ f3 add3(f3 a, f3 b) { return {fa(a.x, b.x), fa(a.y, b.y), fa(a.z, b.z)}; }
__device__ __forceinline__ f3 sub3(f3 a, f3 b) { return {fs(a.x, b.x), fs(a.y, b.y), fs(a.z, b.z)}; }
__device__ __forceinline__ f3 mul3(f3 a, float s) { return {fm(a.x, s), fm(a.y, s), fm(a.z, s)}; }
__device__ __forceinline__ f3 smul3(float s, f3 a) { return {fm(s, a.x), fm(s, a.y), fm(s, a.z)}; }
__device__ __forceinline__ f3 div3(f3 a, float s) { return {fd(a.x, s), fd(a.y, s), fd(a.z, s)}; }
__device__ __forceinline__ f3 neg3(f3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ f3 cross3(f3 a, f3 b) {
    return {fs(fm(a.y, b.z), fm(a.z, b.y)), fs(fm(a.z, b.x), fm(a.x, b.z)),
            fs(fm(a.x, b.y), fm(a.y, b.x))};
}
__device__ __forceinline__ float norm3(f3 a) { return fsq(dot3(a, a)); }
__device__ __forceinline__ f3 normalised3(f3 a) { return div3(a, norm3(a)); }
__device__ __forceinline__ f3 xyz(float4 a) { return {a.x, a.y, a.z}; }

// Row-major 3x3 rotation, Matrix3f (VectorMath.h:356-371)
struct M3 { f3 r0, r1, r2; };
__device__ __forceinline__ f3 mv(const M3& m, f3 a) { return {dot3(m.r0, a), dot3(m.r1, a), dot3(m.r2, a)}; }

// A camera pose as the kernels use it: rotation, its transpose and the
// translation, rounded from the double pose as Frame::GpuRotation /
// GpuInvRotation / GpuTranslation do (Core/Frame.cc:275-294).
struct DevPose {
    M3 R, Rinv;
    f3 t;
    float pad;
};

__host__ inline DevPose make_dev_pose(const double* T) {
    DevPose p;
    p.R.r0 = {(float)T[0], (float)T[1], (float)T[2]};
    p.R.r1 = {(float)T[4], (float)T[5], (float)T[6]};
    p.R.r2 = {(float)T[8], (float)T[9], (float)T[10]};
    p.Rinv.r0 = {(float)T[0], (float)T[4], (float)T[8]};
    p.Rinv.r1 = {(float)T[1], (float)T[5], (float)T[9]};
    p.Rinv.r2 = {(float)T[2], (float)T[6], (float)T[10]};
    p.t = {(float)T[3], (float)T[7], (float)T[11]};
    p.pad = 0;
    return p;
}

__device__ __forceinline__ DevPose make_dev_pose_d(const double* T) {
    DevPose p;
    p.R.r0 = {(float)T[0], (float)T[1], (float)T[2]};
    p.R.r1 = {(float)T[4], (float)T[5], (float)T[6]};
    p.R.r2 = {(float)T[8], (float)T[9], (float)T[10]};
    p.Rinv.r0 = {(float)T[0], (float)T[4], (float)T[8]};
    p.Rinv.r1 = {(float)T[1], (float)T[5], (float)T[9]};
    p.Rinv.r2 = {(float)T[2], (float)T[6], (float)T[10]};
    p.t = {(float)T[3], (float)T[7], (float)T[11]};
    p.pad = 0;
    return p;
}

// Intrinsics of one pyramid level (Utility/Intrinsics.h: K / 2^level in float)
struct Intr { float fx, fy, cx, cy, invfx, invfy; };

__host__ __device__ inline Intr make_intr(float fx, float fy, float cx, float cy, int level) {
    Intr k;
    int s = 1 << level;
    k.fx = fx / s;
    k.fy = fy / s;
    k.cx = cx / s;
    k.cy = cy / s;
    // reference hosts pass 1.0 / fx computed in double (Pyrdown.cu:87, FuseMap.cu:232)
    k.invfx = (float)(1.0 / (double)k.fx);
    k.invfy = (float)(1.0 / (double)k.fy);
    return k;
}

__device__ __forceinline__ float qnan() { return __int_as_float(0x7fffffff); }

// ---- voxel-block hash ----
// Hash entry, 16 bytes: block coordinates as int16 (the map spans +-32767
// blocks per axis around the first camera), the block index into the voxel
// pool (-1: slot empty) and the 1-based excess-list link (0: end of chain).
// The reference's HashEntry holds the same fields in 32 bytes
// (Mapping/DeviceMap.h:20-59) and stores ptr as a voxel index (block * 512).
struct __align__(16) HEntry {
    short x, y, z, pad;
    int ptr;
    int offset;
};

// Voxel, 8 bytes, as the reference's (Mapping/DeviceMap.h:61-93).
struct __align__(8) Voxel {
    float sdf;
    unsigned char weight;
    unsigned char r, g, b;
};

// Precision form: a voxel block is 3072 bytes -- TSDF as FP16 [512] (bytes
// 0-1023), then one 32-bit word per voxel [512] (1024-3071) holding red,
// green, blue and the weight in bytes 0-3.  6 bytes per voxel.
constexpr int kCBlockBytes = 3072;
constexpr int kCRgbw = 1024;
__host__ __device__ constexpr int c_red(int v) { return kCRgbw + 4 * v; }
__host__ __device__ constexpr int c_green(int v) { return kCRgbw + 4 * v + 1; }
__host__ __device__ constexpr int c_blue(int v) { return kCRgbw + 4 * v + 2; }
__host__ __device__ constexpr int c_weight(int v) { return kCRgbw + 4 * v + 3; }

// Per-pixel inputs of integration, made once per frame: {depth, n.x, n.y,
// n.z} with the depth NaN where integrateColor (FuseMap.cu:140-191) skips the
// pixel whatever the voxel -- depth NaN or outside [depth_min, depth_max], or
// a NaN normal -- and the colour as one word r | g << 8 | b << 16.  The
// floats are the raw depth and the normal unchanged, so both forms read them
// in place of the three images.
__device__ __forceinline__ void fuse_record(float dp, float4 n, const uint8_t* c3, float dmin, float dmax,
                                            float4* rec, uint32_t* col) {
    const bool ok = !(isnan(dp) || dp > dmax || dp < dmin) && !isnan(n.x);
    *rec = make_float4(ok ? dp : qnan(), n.x, n.y, n.z);
    *col = (uint32_t)c3[0] | (uint32_t)c3[1] << 8 | (uint32_t)c3[2] << 16;
}

// The precision form's fusion record: the same inputs in one 16-byte word,
// so integration gathers once per voxel -- x: the depth (NaN where skipped),
// y: n.x and n.y as FP16, z: n.z as FP16 | red << 16 | green << 24, w: blue.
__device__ __forceinline__ void fuse_record_packed(float dp, float4 n, const uint8_t* c3, float dmin, float dmax,
                                                   uint4* rec) {
    const bool ok = !(isnan(dp) || dp > dmax || dp < dmin) && !isnan(n.x);
    const __half2 nxy = __floats2half2_rn(n.x, n.y);
    const __half nz = __float2half_rn(n.z);
    *rec = make_uint4(__float_as_uint(ok ? dp : qnan()), *reinterpret_cast<const uint32_t*>(&nxy),
                      (uint32_t)__half_as_ushort(nz) | (uint32_t)c3[0] << 16 | (uint32_t)c3[1] << 24,
                      (uint32_t)c3[2]);
}

// Bucket of a block (Mapping/DeviceMap.cu:3-10): products wrap in 32 bits and
// the modulo is unsigned because NumBuckets is an unsigned constant.
__host__ __device__ __forceinline__ uint32_t bucket_of(int x, int y, int z, uint32_t nb) {
    uint32_t h = ((uint32_t)x * 73856093u) ^ ((uint32_t)y * 19349669u) ^ ((uint32_t)z * 83492791u);
    return h % nb;
}
// As bucket_of, with the modulo done as a mask when nb is a power of two
// (mask = nb - 1; 0 otherwise).  Same result.
__device__ __forceinline__ uint32_t bucket_of_m(int x, int y, int z, uint32_t nb, uint32_t mask) {
    uint32_t h = ((uint32_t)x * 73856093u) ^ ((uint32_t)y * 19349669u) ^ ((uint32_t)z * 83492791u);
    return mask ? (h & mask) : h % nb;
}
// voxelPosToBlockPos (DeviceMap.cu:150-161): floor division by 8, i.e. the
// arithmetic shift
__device__ __forceinline__ int block_of(int v) { return v >> 3; }
// voxelPosToLocalPos (DeviceMap.cu:167-178): the non-negative remainder
__device__ __forceinline__ int local_of(int v) { return v & 7; }

constexpr int kCoordLimit = 32767;

// Device-side error flags (OR-ed into a session word, reported per frame).
enum ErrFlag : uint32_t {
    kErrHeapExhausted = 1u << 0,      // voxel-block pool full: blocks not allocated
    kErrExcessFull = 1u << 1,         // excess list full: blocks not allocated
    kErrRequestSetFull = 1u << 2,     // per-frame request set overflowed
    kErrCoordRange = 1u << 3,         // block outside the +-32767 range skipped
    kErrNewListFull = 1u << 4,        // more new blocks in one frame than the pool
    kErrVisibleFull = 1u << 5,        // visible list capacity exceeded
    kErrSequentialInsert = 1u << 6,   // slow exact path taken (heap/excess edge cases)
    kErrTimeout = 1u << 7,            // a bounded device-side wait gave up (the kernel stopped early)
    kErrNormalW = 1u << 8,            // a valid normal given to integration had a w lane other than 1
};

}  // namespace fb

#endif
