// Model raycasting (the reference's Mapping/RenderScene.cu): per-pixel depth
// intervals from the visible blocks, then sphere tracing of the TSDF through
// the voxel-block hash with trilinear refinement and a central-difference
// normal.
//
// z ranges: each visible block is projected once (8 corners) and its
// rectangle at 1/8 resolution is min/max-ed into the z-range images with
// integer atomics on the float bits (all values are positive, so integer order
// is float order).  In the reference each block's rectangle is first split
// into 16x16 tiles appended to a list (Projection::createRenderingBlockList,
// RenderScene.cu:106-124) and filled by a second kernel; because every tile's
// lower-right corner is taken from the block's upper-left corner
// (RenderScene.cu:115-116), only the first tile of a block ever covers
// pixels: [ul, min(ul + 15, lr)].  That is the rectangle filled here.
#include <cuda_fp16.h>

#include <algorithm>

#include "fb_fused.cuh"
#include "fb_internal.h"

namespace fb {

__device__ __forceinline__ void zrange_init_body(const BlockCtx& ctx, MapView m, const int* __restrict__ skip) {
    if (skip && *skip) return;
    if (ctx.bx == 0 && threadIdx.x < 3) {
        m.ctr->bmin[threadIdx.x] = 0x7fffffff;
        m.ctr->bmax[threadIdx.x] = -0x7fffffff;
    }
    if (ctx.bx == 0 && threadIdx.x == 0) {
        m.ctr->ray_next = 0;
        m.ctr->n_tiles = 0;   // counted again by each z-range pass
    }
    const int n = m.zc * m.zr;
    for (int i = ctx.bx * blockDim.x + threadIdx.x; i < n; i += ctx.gx * blockDim.x) {
        m.zmin[i] = 100.f;   // CreateRenderingBlocks uploads 100 (RenderScene.cu:245-251)
        m.zmax[i] = 0.f;     // and clears zRangeY (RenderScene.cu:244)
    }
}

__global__ void __launch_bounds__(256) k_zrange_init(MapView m, const int* __restrict__ skip) {
    zrange_init_body(own_ctx(), m, skip);
}
FB_FUSED_KERNEL(k_zrange_init, zrange_init_body, 256)

// Histogram bucket of a raycast tile's cost: 16 buckets per octave (the
// exponent and the next four bits), 0..511.
__device__ __forceinline__ int cost_bucket(uint32_t c) {
    if (c == 0) return 0;
    const int msb = 31 - __clz(c);
    const uint32_t frac = msb >= 4 ? (c >> (msb - 4)) & 15u : (c << (4 - msb)) & 15u;
    return msb * 16 + (int)frac;
}

// The raycast's block order for its next launch of n tiles (one block of 256
// threads): the tiles sorted by the last raycast's costs, slowest first (to
// 1/16 octave; ties in any order), so that the longest rays start first and
// the launch does not end waiting for a slow tile that started last.  Clears
// the costs.  The order is a permutation of 0..n-1 whatever the costs hold.
__device__ __forceinline__ void order_tiles(const MapView& m, int n) {
    __shared__ int hist[512];
    __shared__ int wsum[8];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (n > m.rc_cap) {
        if (t == 0) m.rc_order[0] = 0;   // no order: blocks in grid order
        return;
    }
    hist[t] = 0;
    hist[t + 256] = 0;
    __syncthreads();
    for (int i = t; i < n; i += 256) atomicAdd(&hist[cost_bucket(m.rc_cost[i])], 1);
    __syncthreads();
    // bucket starts in descending bucket order: thread t owns buckets 511 - 2t
    // and 510 - 2t (a block-wide exclusive scan of their counts)
    const int h0 = hist[511 - 2 * t], h1 = hist[510 - 2 * t];
    int v = h0 + h1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) wsum[w] = v;
    __syncthreads();
    int base = 0;
    for (int q = 0; q < w; ++q) base += wsum[q];
    const int excl = base + v - (h0 + h1);
    hist[511 - 2 * t] = excl;   // every thread has read its two counts above
    hist[510 - 2 * t] = excl + h0;
    __syncthreads();
    for (int i = t; i < n; i += 256) {
        const int slot = atomicAdd(&hist[cost_bucket(m.rc_cost[i])], 1);
        m.rc_order[1 + slot] = i;
        m.rc_cost[i] = 0;
    }
    if (t == 0) m.rc_order[0] = n;
}

// Projection::projectBlock (RenderScene.cu:54-104) + the first tile's fill
// (fillBlocks, RenderScene.cu:156-179).  With ord_n > 0 the grid's last block
// prepares the next raycast's block order instead (order_tiles), beside the
// projection.
__device__ __forceinline__ void zrange_body(const BlockCtx& ctx, MapView m, Intr k, const DevPose* __restrict__ posep,
                                            const int* __restrict__ skip, int ord_n) {
    if (skip && *skip) return;
    if (ord_n > 0 && ctx.bx == ctx.gx - 1) {
        order_tiles(m, ord_n);
        return;
    }
    const int gx = ord_n > 0 ? ctx.gx - 1 : ctx.gx;
    const DevPose P = *posep;
    const int n = min(m.ctr->n_visible, m.NS);
    const int zc = m.zc, zr = m.zr;
    // box of the visible blocks (warp-reduced, then one atomic per warp)
    {
        int lo[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, hi[3] = {-0x7fffffff, -0x7fffffff, -0x7fffffff};
        for (int i = ctx.bx * blockDim.x + threadIdx.x; i < n; i += gx * blockDim.x) {
            const HEntry e = m.vis_blocks[i];
            lo[0] = min(lo[0], (int)e.x);
            lo[1] = min(lo[1], (int)e.y);
            lo[2] = min(lo[2], (int)e.z);
            hi[0] = max(hi[0], (int)e.x);
            hi[1] = max(hi[1], (int)e.y);
            hi[2] = max(hi[2], (int)e.z);
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lo[a] = __reduce_min_sync(0xffffffffu, lo[a]);
            hi[a] = __reduce_max_sync(0xffffffffu, hi[a]);
        }
        if ((threadIdx.x & 31) == 0 && lo[0] <= hi[0]) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                atomicMin(&m.ctr->bmin[a], lo[a]);
                atomicMax(&m.ctr->bmax[a], hi[a]);
            }
        }
    }
    for (int i = ctx.bx * blockDim.x + threadIdx.x; i < n; i += gx * blockDim.x) {
        const HEntry e = m.vis_blocks[i];
        int ulx = zc, uly = zr, lrx = -1, lry = -1;
        float zx = m.g.depth_max, zy = m.g.depth_min;
        for (int c = 0; c < 8; ++c) {
            const int tx = e.x + ((c & 1) ? 1 : 0), ty = e.y + ((c & 2) ? 1 : 0), tz = e.z + ((c & 4) ? 1 : 0);
            f3 p = mk3(fm((float)(tx * 8), m.g.voxel_size), fm((float)(ty * 8), m.g.voxel_size),
                       fm((float)(tz * 8), m.g.voxel_size));
            p = mv(P.Rinv, sub3(p, P.t));
            if ((double)p.z < 2e-1) continue;
            const float qx = fd(fa(fd(fm(k.fx, p.x), p.z), k.cx), 8.0f);
            const float qy = fd(fa(fd(fm(k.fy, p.y), p.z), k.cy), 8.0f);
            // upperLeft / lowerRight are short2 (DeviceMap.h:11-18)
            if ((float)ulx > floorf(qx)) ulx = (short)(int)floorf(qx);
            if ((float)lrx < ceilf(qx)) lrx = (short)(int)ceilf(qx);
            if ((float)uly > floorf(qy)) uly = (short)(int)floorf(qy);
            if ((float)lry < ceilf(qy)) lry = (short)(int)ceilf(qy);
            if (zx > p.z) zx = p.z;
            if (zy < p.z) zy = p.z;
        }
        if (ulx < 0) ulx = 0;
        if (uly < 0) uly = 0;
        if (lrx >= zc) lrx = zc - 1;
        if (lry >= zr) lry = zr - 1;
        if (ulx > lrx || uly > lry) continue;
        if (zx < m.g.depth_min) zx = m.g.depth_min;
        if (zy < m.g.depth_min) continue;
        atomicAdd(&m.ctr->n_tiles, 1);
        const int ex = min(ulx + 15, lrx), ey = min(uly + 15, lry);
        const int bzx = __float_as_int(zx), bzy = __float_as_int(zy);
        for (int y = uly; y <= ey; ++y)
            for (int x = ulx; x <= ex; ++x) {
                atomicMin((int*)&m.zmin[y * zc + x], bzx);
                atomicMax((int*)&m.zmax[y * zc + x], bzy);
            }
    }
}

__global__ void __launch_bounds__(256) k_zrange(MapView m, Intr k, const DevPose* __restrict__ posep,
                                  const int* __restrict__ skip, int ord_n) {
    zrange_body(own_ctx(), m, k, posep, skip, ord_n);
}
FB_FUSED_KERNEL(k_zrange, zrange_body, 256)

// Dense block index for the raycast: every allocated block inside the box of
// this frame's visible blocks (one block of margin) gets its pool index in
// grid[], -1 elsewhere; outside the box, or when the box exceeds the grid,
// lookups walk the hash table as before.  The index holds exactly what the
// hash table holds for those coordinates (one entry per block), so every
// lookup returns the same block: a ray's samples turn one indexed load instead
// of a bucket probe and chain walk, which also keeps a warp's lanes together.
//
// The box from the z-range pass's bounds (every block of the clearing kernel
// derives it; block 0 publishes it for the fill and the raycast).
struct GridBox {
    int o[3], n[3];
    bool on;
};

__device__ __forceinline__ GridBox grid_box(const MapView& m) {
    const MapCounters* c = m.ctr;
    GridBox b;
    long long vol = 1;
    for (int a = 0; a < 3; ++a) {
        b.o[a] = c->bmin[a] - 1;
        b.n[a] = c->bmax[a] - c->bmin[a] + 3;
        if (b.n[a] < 1) b.n[a] = 0;
        vol *= b.n[a];
    }
    b.on = c->bmin[0] <= c->bmax[0] && vol > 0 && vol <= m.grid_cap;
    return b;
}

__device__ __forceinline__ void grid_clear_body(const BlockCtx& ctx, MapView m, const int* __restrict__ skip) {
    if (skip && *skip) return;
    const GridBox gb = grid_box(m);
    if (ctx.bx == 0 && threadIdx.x < 3) {
        m.ctr->g_o[threadIdx.x] = gb.o[threadIdx.x];
        m.ctr->g_n[threadIdx.x] = gb.on ? gb.n[threadIdx.x] : 0;
        if (threadIdx.x == 0) m.ctr->g_on = gb.on ? 1 : 0;
    }
    if (!gb.on) return;
    const int vol = gb.n[0] * gb.n[1] * gb.n[2];
    int4* g4 = (int4*)m.grid;
    const int4 none = make_int4(-1, -1, -1, -1);
    for (int i = ctx.bx * blockDim.x + threadIdx.x; i < (vol + 3) / 4; i += ctx.gx * blockDim.x) g4[i] = none;
}

__global__ void __launch_bounds__(256) k_grid_clear(MapView m, const int* __restrict__ skip) {
    grid_clear_body(own_ctx(), m, skip);
}
FB_FUSED_KERNEL(k_grid_clear, grid_clear_body, 256)

// FindEntry's block (DeviceMap.cu:122-135): the first entry of the chain
// holding block (x, y, z), or -1.
__device__ __forceinline__ int first_ptr(const MapView& m, int x, int y, int z) {
    HEntry e = m.entries[bucket_of_m(x, y, z, (uint32_t)m.NB, m.nb_mask)];
    if (e.ptr != -1 && e.x == x && e.y == y && e.z == z) return e.ptr;
    for (int guard = 0; e.offset > 0 && e.offset <= m.NE && guard <= m.NE; ++guard) {
        e = m.entries[m.NB + e.offset - 1];
        if (e.x == x && e.y == y && e.z == z && e.ptr != -1) return e.ptr;
    }
    return -1;
}

__device__ __forceinline__ void grid_fill_body(const BlockCtx& ctx, MapView m, const int* __restrict__ skip) {
    if (skip && *skip) return;
    const MapCounters* c = m.ctr;
    if (!c->g_on) return;
    const int ox = c->g_o[0], oy = c->g_o[1], oz = c->g_o[2];
    const int nx = c->g_n[0], ny = c->g_n[1], nz = c->g_n[2];
    const int n = min(c->n_alloc, m.NS);
    for (int i = ctx.bx * blockDim.x + threadIdx.x; i < n; i += ctx.gx * blockDim.x) {
        const HEntry e = m.entries[m.alloc_list[i]];
        const int gx = e.x - ox, gy = e.y - oy, gz = e.z - oz;
        // a map with two entries for one block (the reference's racy
        // allocator makes them) gets the block the hash lookup finds
        if ((unsigned)gx < (unsigned)nx && (unsigned)gy < (unsigned)ny && (unsigned)gz < (unsigned)nz)
            m.grid[(gz * ny + gy) * nx + gx] = first_ptr(m, e.x, e.y, e.z);
    }
}

__global__ void __launch_bounds__(256) k_grid_fill(MapView m, const int* __restrict__ skip) {
    grid_fill_body(own_ctx(), m, skip);
}
FB_FUSED_KERNEL(k_grid_fill, grid_fill_body, 256)

// The raycast's view of the dense index (registers).
struct GridView {
    int ox, oy, oz, nx, ny, nz;
};

// ----------------------------------------------------------------- raycast

struct EntryCache {
    int x, y, z, ptr;
    bool set;
};

// Voxel access of the two forms.  Reference form: 8-byte voxels.
struct ExactVox {
    using ref = const Voxel*;
    static __device__ __forceinline__ ref at(const MapView& m, int ptr, int idx) {
        return m.voxels + (size_t)ptr * 512 + idx;
    }
    static __device__ __forceinline__ ref none() { return nullptr; }
    static __device__ __forceinline__ bool null(ref v) { return v == nullptr; }
    static __device__ __forceinline__ float sdf(ref v) { return v->sdf; }
    static __device__ __forceinline__ int weight(ref v) { return v->weight; }
    // TSDF and weight with one 8-byte load
    static __device__ __forceinline__ float sdf_w(ref v, int& w) {
        const uint2 raw = *reinterpret_cast<const uint2*>(v);
        w = (int)(raw.y & 0xffu);
        return __uint_as_float(raw.x);
    }
};

// Precision form: FP16 TSDF array, then one r, g, b, weight word per voxel.
struct CompactVox {
    struct ref {
        const uint8_t* blk;
        int idx;
    };
    static __device__ __forceinline__ ref at(const MapView& m, int ptr, int idx) {
        return ref{m.cvox + (size_t)ptr * kCBlockBytes, idx};
    }
    static __device__ __forceinline__ ref none() { return ref{nullptr, 0}; }
    static __device__ __forceinline__ bool null(ref v) { return v.blk == nullptr; }
    static __device__ __forceinline__ float sdf(ref v) {
        return __half2float(*(const __half*)(v.blk + 2 * v.idx));
    }
    static __device__ __forceinline__ int weight(ref v) { return v.blk[c_weight(v.idx)]; }
    static __device__ __forceinline__ float sdf_w(ref v, int& w) {
        w = weight(v);
        return sdf(v);
    }
};

// FindEntry's block (DeviceMap.cu:122-135) through the dense index where it
// covers (bx, by, bz), else the hash table: the pool index, or -1.
__device__ __forceinline__ int lookup_block(const MapView& m, const GridView& gv, int bx, int by, int bz) {
    const int gx = bx - gv.ox, gy = by - gv.oy, gz = bz - gv.oz;
    if ((unsigned)gx < (unsigned)gv.nx && (unsigned)gy < (unsigned)gv.ny && (unsigned)gz < (unsigned)gv.nz)
        return max(__ldg(m.grid + (gz * gv.ny + gy) * gv.nx + gx), -1);
    int b = (int)bucket_of_m(bx, by, bz, (uint32_t)m.NB, m.nb_mask);
    HEntry e = m.entries[b];
    bool found = e.ptr != -1 && e.x == bx && e.y == by && e.z == bz;
    for (int guard = 0; !found && e.offset > 0 && e.offset <= m.NE && guard <= m.NE; ++guard) {
        e = m.entries[m.NB + e.offset - 1];
        found = e.x == bx && e.y == by && e.z == bz && e.ptr != -1;
    }
    return found ? e.ptr : -1;
}

// FindEntry with the cache of FindVoxel(float3, cache, valid)
// (DeviceMap.cu:97-114): the pool index of block (bx, by, bz), or -1.  The
// reference's cache starts as HashEntry() -- position (0,0,0), ptr -1 -- and
// a first probe inside block (0,0,0) then reads voxel index -1 + local
// index; here the cache starts empty.  The cache holds what the lookup
// returns, so it changes no result.
__device__ __forceinline__ int find_block(const MapView& m, const GridView& gv, int bx, int by, int bz,
                                          EntryCache& c) {
    if (c.set && bx == c.x && by == c.y && bz == c.z) return c.ptr;
    const int ptr = lookup_block(m, gv, bx, by, bz);
    if (ptr < 0) return -1;
    c.x = bx;
    c.y = by;
    c.z = bz;
    c.ptr = ptr;
    c.set = true;
    return ptr;
}

// FindVoxel of integer voxel coordinates: the voxel, or none for a missing
// block (valid = whether the block exists).
template <class VR>
__device__ __forceinline__ typename VR::ref find_voxel_i(const MapView& m, const GridView& gv, int vx, int vy, int vz,
                                                         EntryCache& c, bool& valid) {
    const int ptr = find_block(m, gv, block_of(vx), block_of(vy), block_of(vz), c);
    valid = ptr >= 0;
    if (ptr < 0) return VR::none();
    return VR::at(m, ptr, local_of(vz) * 64 + local_of(vy) * 8 + local_of(vx));
}

// FindVoxel(float3, cache, valid) (DeviceMap.cu:97-114): voxel coordinates
// truncated toward zero (make_int3 of the float position).
template <class VR>
__device__ __forceinline__ typename VR::ref find_voxel(const MapView& m, const GridView& gv, f3 p, EntryCache& c,
                                                       bool& valid) {
    return find_voxel_i<VR>(m, gv, __float2int_rz(p.x), __float2int_rz(p.y), __float2int_rz(p.z), c, valid);
}

// Rendering::readSdf (RenderScene.cu:290-295)
template <class VR>
__device__ __forceinline__ float read_sdf(const MapView& m, const GridView& gv, f3 p, EntryCache& c, bool& valid) {
    const typename VR::ref v = find_voxel<VR>(m, gv, p, c, valid);
    if (VR::null(v)) return qnan();
    int w;
    const float sdf = VR::sdf_w(v, w);
    if (w == 0) valid = false;
    return sdf;
}

// One corner of a trilinear read: the voxel's TSDF in block q, NaN for a
// missing block (q < 0).  The load always reads a voxel of the pool (block
// 0 for a missing block) so that the eight loads issue without branches.
template <class VR>
__device__ __forceinline__ float corner_sdf(const MapView& m, int q, int idx) {
    const float v = VR::sdf(VR::at(m, max(q, 0), idx));
    return q < 0 ? qnan() : v;
}

// Rendering::readSdfInterped (RenderScene.cu:297-319).  The eight corners are
// the voxels at the truncated coordinates of pt and of pt + 1 per axis (each
// sum rounded as the reference rounds it), read in the reference's order and
// blended by its lerp sequence; `valid` ends as the last corner's (x+1, y+1,
// z+1) lookup leaves it.  The corners lie in at most eight blocks, one per
// axis combination whose coordinates cross a block boundary: each distinct
// block is looked up once (the first through the entry cache), then the
// eight TSDF loads issue together.  Every lane of a warp runs the same code
// whether or not its corners straddle blocks (only the extra lookups are
// conditional), where a per-corner lookup through the one-entry cache made
// straddling lanes run a second, eight-lookup path.
template <class VR>
__device__ float read_sdf_interp(const MapView& m, const GridView& gv, f3 pt, EntryCache& c, bool& valid) {
    const f3 f = mk3(fs(pt.x, floorf(pt.x)), fs(pt.y, floorf(pt.y)), fs(pt.z, floorf(pt.z)));
    auto lerp = [](float a, float b, float t) { return fa(fm(fs(1.0f, t), a), fm(t, b)); };
    const int x0 = __float2int_rz(pt.x), x1 = __float2int_rz(fa(pt.x, 1.f));
    const int y0 = __float2int_rz(pt.y), y1 = __float2int_rz(fa(pt.y, 1.f));
    const int z0 = __float2int_rz(pt.z), z1 = __float2int_rz(fa(pt.z, 1.f));
    const int bx0 = block_of(x0), bx1 = block_of(x1);
    const int by0 = block_of(y0), by1 = block_of(y1);
    const int bz0 = block_of(z0), bz1 = block_of(z1);
    const bool sx = bx1 != bx0, sy = by1 != by0, sz = bz1 != bz0;
    const int q000 = find_block(m, gv, bx0, by0, bz0, c);
    const int q100 = sx ? lookup_block(m, gv, bx1, by0, bz0) : q000;
    const int q010 = sy ? lookup_block(m, gv, bx0, by1, bz0) : q000;
    const int q110 = sy ? (sx ? lookup_block(m, gv, bx1, by1, bz0) : q010) : q100;
    int q001 = q000, q101 = q100, q011 = q010, q111 = q110;
    if (sz) {
        q001 = lookup_block(m, gv, bx0, by0, bz1);
        q101 = sx ? lookup_block(m, gv, bx1, by0, bz1) : q001;
        q011 = sy ? lookup_block(m, gv, bx0, by1, bz1) : q001;
        q111 = sy ? (sx ? lookup_block(m, gv, bx1, by1, bz1) : q011) : q101;
    }
    valid = q111 >= 0;
    const int ax = local_of(x0), bxl = local_of(x1);
    const int ay = local_of(y0) * 8, byl = local_of(y1) * 8;
    const int az = local_of(z0) * 64, bzl = local_of(z1) * 64;
    const float s000 = corner_sdf<VR>(m, q000, az + ay + ax);
    const float s100 = corner_sdf<VR>(m, q100, az + ay + bxl);
    const float s010 = corner_sdf<VR>(m, q010, az + byl + ax);
    const float s110 = corner_sdf<VR>(m, q110, az + byl + bxl);
    const float s001 = corner_sdf<VR>(m, q001, bzl + ay + ax);
    const float s101 = corner_sdf<VR>(m, q101, bzl + ay + bxl);
    const float s011 = corner_sdf<VR>(m, q011, bzl + byl + ax);
    const float s111 = corner_sdf<VR>(m, q111, bzl + byl + bxl);
    const float r0 = lerp(s000, s100, f.x), r1 = lerp(s010, s110, f.x);
    const float r2 = lerp(r0, r1, f.y);
    const float r0b = lerp(s001, s101, f.x), r1b = lerp(s011, s111, f.x);
    const float r3 = lerp(r0b, r1b, f.y);
    return lerp(r2, r3, f.z);
}

// Rendering::readNormal (RenderScene.cu:321-352): the six samples at
// pt +- 1 per axis, in the reference's order, and the normal from their three
// differences.  Offsets and differences stay in registers (a dynamically
// indexed table of samples would live in local memory).
template <class VR>
__device__ bool read_normal(const MapView& m, const GridView& gv, f3 pt, EntryCache& c, const M3& Rinv, f3& n) {
    bool valid;
    float prev = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
    for (int q = 0; q < 6; ++q) {
        const float d = (q & 1) ? -1.0f : 1.0f;
        const int a = q >> 1;
        const f3 ps = mk3(fa(pt.x, a == 0 ? d : 0.0f), fa(pt.y, a == 1 ? d : 0.0f), fa(pt.z, a == 2 ? d : 0.0f));
        const float sq = read_sdf_interp<VR>(m, gv, ps, c, valid);
        if (isnan(sq) || sq == 1.0f || !valid) return false;
        if (q & 1) {
            const float g = fs(prev, sq);
            gx = a == 0 ? g : gx;
            gy = a == 1 ? g : gy;
            gz = a == 2 ? g : gz;
        }
        prev = sq;
    }
    n = normalised3(mv(Rinv, mk3(gx, gy, gz)));
    return true;
}

// The dense index's extent from this frame's counters (all zero when the
// index is off: every lookup then walks the table).
__device__ __forceinline__ GridView grid_view(const MapView& m) {
    GridView gv;
    gv.ox = m.ctr->g_o[0];
    gv.oy = m.ctr->g_o[1];
    gv.oz = m.ctr->g_o[2];
    gv.nx = m.ctr->g_n[0];
    gv.ny = m.ctr->g_n[1];
    gv.nz = m.ctr->g_n[2];
    return gv;
}

// One ray of Rendering::operator() (RenderScene.cu:354-440), in three parts
// that every raycast kernel runs in this order: ray_begin, ray_step until it
// reports the end of the march loop, ray_finish.
struct Ray {
    f3 result, dir;
    float dist_s, dist_e, sdf;
};

// The ray of pixel (x, y) from its depth interval; false when the pixel has
// none (its vertex and normal are NaN).
__device__ __forceinline__ bool ray_begin(const MapView& m, const DevPose& P, const Intr& k, int x, int y, Ray& r) {
    // floor(x / 8) of a pixel coordinate (>= 0) is x >> 3; (double)z < 1e-3
    // holds exactly when z < 0.001f (the float identities' test checks it)
    const int lx = x >> 3, ly = y >> 3;
    const float zrx = m.zmin[ly * m.zc + lx], zry = m.zmax[ly * m.zc + lx];
    if (zry < 0.001f || zrx < 0.001f || isnan(zrx) || isnan(zry)) return false;
    const float vinv = m.g.voxel_size_inv;
    f3 p;
    p.z = zrx;
    p.x = fm(fm(p.z, fs((float)x, k.cx)), k.invfx);
    p.y = fm(fm(p.z, fs((float)y, k.cy)), k.invfy);
    r.dist_s = fm(norm3(p), vinv);
    const f3 block_s = mul3(add3(mv(P.R, p), P.t), vinv);
    p.z = zry;
    p.x = fm(fm(p.z, fs((float)x, k.cx)), k.invfx);
    p.y = fm(fm(p.z, fs((float)y, k.cy)), k.invfy);
    r.dist_e = fm(norm3(p), vinv);
    const f3 block_e = mul3(add3(mv(P.R, p), P.t), vinv);
    r.dir = normalised3(sub3(block_e, block_s));
    r.result = block_s;
    r.sdf = 1.0f;
    return true;
}

// One turn of the march loop; true when the loop has ended (its condition
// failed, or a sample at or behind the surface).
template <class VR>
__device__ __forceinline__ bool ray_step(const MapView& m, const GridView& gv, float stepScale, Ray& r,
                                         EntryCache& c) {
    if (!(r.dist_s < r.dist_e)) return true;
    bool valid;
    float step;
    r.sdf = read_sdf<VR>(m, gv, r.result, c, valid);
    if (!valid) {
        step = 8.0f;
    } else {
        if (r.sdf <= 0.1f && r.sdf >= -0.5f) r.sdf = read_sdf_interp<VR>(m, gv, r.result, c, valid);
        if (r.sdf <= 0.0f) return true;
        step = !isnan(r.sdf) ? fmaxf(fm(r.sdf, stepScale), 1.0f) : 8.0f;
    }
    r.result = add3(r.result, smul3(step, r.dir));
    r.dist_s = fa(r.dist_s, step);
    return false;
}

// After the loop: a ray whose last sample is at or behind the surface (sdf
// <= 0) is refined by two steps and gets its vertex and normal; every other
// ray gives NaN.
template <class VR>
__device__ __forceinline__ void ray_finish(const MapView& m, const GridView& gv, const DevPose& P, float stepScale,
                                           Ray r, EntryCache& c, float4& vout, float4& nout) {
    const float4 nan4 = make_float4(qnan(), qnan(), qnan(), qnan());
    vout = nan4;
    nout = nan4;
    if (!(r.sdf <= 0.0f)) return;
    bool valid;
    float step = fm(r.sdf, stepScale);
    r.result = add3(r.result, smul3(step, r.dir));
    r.sdf = read_sdf_interp<VR>(m, gv, r.result, c, valid);
    step = fm(r.sdf, stepScale);
    r.result = add3(r.result, smul3(step, r.dir));
    f3 n;
    if (read_normal<VR>(m, gv, r.result, c, P.Rinv, n)) {
        const f3 q = mv(P.Rinv, sub3(mul3(r.result, m.g.voxel_size), P.t));
        vout = make_float4(q.x, q.y, q.z, 1.0f);
        nout = make_float4(n.x, n.y, n.z, 1.0f);
    }
}

// The whole ray of pixel (x, y): writes its vertex and normal.
template <class VR>
__device__ __forceinline__ void raycast_pixel(const MapView& m, const GridView& gv, const DevPose& P, const Intr& k,
                                              int x, int y, float4* __restrict__ vout_p,
                                              float4* __restrict__ nout_p) {
    float4 vout = make_float4(qnan(), qnan(), qnan(), qnan()), nout = vout;
    Ray r;
    if (ray_begin(m, P, k, x, y, r)) {
        const float stepScale = m.g.step_scale;
        EntryCache c;
        c.set = false;
        while (!ray_step<VR>(m, gv, stepScale, r, c)) {
        }
        ray_finish<VR>(m, gv, P, stepScale, r, c, vout, nout);
    }
    *vout_p = vout;
    *nout_p = nout;
}

// One thread per pixel in CUDA blocks of the session's tile shape.  Block b
// of the grid traces tile rc_order[1 + b] when the z-range pass ordered this
// launch's tiles (rc_order[0] == the tile count), else tile b; each warp
// records its duration as its tile's cost for the next order.
template <class VR>
__device__ __forceinline__ void raycast_body(const BlockCtx& ctx, MapView m, float4* __restrict__ vmap,
                                             float4* __restrict__ nmap, int vp, int W, int H, Intr k,
                                             const DevPose* __restrict__ posep, const int* __restrict__ skip) {
    if (skip && *skip) return;
    if (m.ctr->n_tiles == 0) return;   // CreateRenderingBlocks returned false: maps untouched
    // the warp's start time and tile wait in shared memory (not in registers
    // across the ray)
    __shared__ long long s_t0[4];
    __shared__ int s_tile[4];
    const int lt = threadIdx.y * blockDim.x + threadIdx.x, wq = lt >> 5;   // blockDim <= 128
    const int nt = ctx.gx * ctx.gy, b = ctx.by * ctx.gx + ctx.bx;
    int tile = b;
    if (m.rc_order && nt <= m.rc_cap && m.rc_order[0] == nt) tile = m.rc_order[1 + b];
    if ((lt & 31) == 0) {
        s_t0[wq] = clock64();
        s_tile[wq] = tile;
    }
    const int ty = tile / ctx.gx, tx = tile - ty * ctx.gx;
    const int x = tx * blockDim.x + threadIdx.x;
    const int y = ty * blockDim.y + threadIdx.y;
    if (x < W && y < H) {
        const size_t o = (size_t)y * vp + x;
        raycast_pixel<VR>(m, grid_view(m), *posep, k, x, y, vmap + o, nmap + o);
    }
    if ((lt & 31) == 0 && m.rc_cost && s_tile[wq] < m.rc_cap)
        atomicMax(&m.rc_cost[s_tile[wq]], (uint32_t)min(clock64() - s_t0[wq], 0xffffffffLL));
}

// Nine CTAs of 128 threads per SM (56 registers; the compiler's own choice
// of 72 leaves seven, and the tail of the launch is longer).
template <class VR>
__global__ void __launch_bounds__(128, 9) k_raycast(MapView m, float4* __restrict__ vmap, float4* __restrict__ nmap,
                                                 int vp, int W, int H, Intr k, const DevPose* __restrict__ posep,
                                                 const int* __restrict__ skip) {
    raycast_body<VR>(own_ctx(), m, vmap, nmap, vp, W, H, k, posep, skip);
}
// (the fused form keeps the compiler's register count: its spills at nine
// CTAs per SM cost more in batched steps than the occupancy gains)
template <class VR>
__global__ void __launch_bounds__(128)
    k_raycast_fused(const __grid_constant__ FusedParams<ArgsOf<decltype(&k_raycast<VR>)>> fp) {
    run_part(fp, [](const BlockCtx& c, const auto&... a) { raycast_body<VR>(c, a...); });
}

// The same rays from a work queue: a grid of resident CTAs whose warps take
// 8 x 4 pixel tiles (row-major tile order) from a counter, one atomic per
// warp and tile, until every tile is taken, so a warp that drew cheap rays
// takes more tiles instead of leaving its slot idle until the grid's last
// CTAs end.  Every pixel runs raycast_pixel as in k_raycast: the same bits.
// (Refilling each lane whose ray has ended with a new pixel, the finished
// rays queued so that the whole warp computes their normals together, was
// measured 1.7x slower than k_raycast at 640x480: a warp's lanes then march
// unrelated rays, and their voxel reads no longer fall on shared lines.)
template <class VR>
__device__ __forceinline__ void raycast_queue_body(const BlockCtx&, MapView m, float4* __restrict__ vmap,
                                                   float4* __restrict__ nmap, int vp, int W, int H, Intr k,
                                                   const DevPose* __restrict__ posep,
                                                   const int* __restrict__ skip) {
    if (skip && *skip) return;
    if (m.ctr->n_tiles == 0) return;   // CreateRenderingBlocks returned false: maps untouched
    const GridView gv = grid_view(m);
    const int tiles_x = (W + 7) >> 3;
    const unsigned total = (unsigned)tiles_x * (unsigned)((H + 3) >> 2);
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned t = 0;
        if (lane == 0) t = atomicAdd(&m.ctr->ray_next, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= total) break;
        const int x = (int)(t % (unsigned)tiles_x) * 8 + (lane & 7);
        const int y = (int)(t / (unsigned)tiles_x) * 4 + (lane >> 3);
        if (x < W && y < H) {
            const size_t o = (size_t)y * vp + x;
            raycast_pixel<VR>(m, gv, *posep, k, x, y, vmap + o, nmap + o);
        }
    }
}

template <class VR>
__global__ void __launch_bounds__(128) k_raycast_queue(MapView m, float4* __restrict__ vmap,
                                                       float4* __restrict__ nmap, int vp, int W, int H, Intr k,
                                                       const DevPose* __restrict__ posep,
                                                       const int* __restrict__ skip) {
    raycast_queue_body<VR>(own_ctx(), m, vmap, nmap, vp, W, H, k, posep, skip);
}
template <class VR>
__global__ void __launch_bounds__(128)
    k_raycast_queue_fused(const __grid_constant__ FusedParams<ArgsOf<decltype(&k_raycast_queue<VR>)>> fp) {
    run_part(fp, [](const BlockCtx& c, const auto&... a) { raycast_queue_body<VR>(c, a...); });
}

static int sm_count_rc() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

// CTAs of the queued raycast resident on one SM (its register count decides).
static int queue_ctas_per_sm(bool compact) {
    static int n[2] = {0, 0};
    int& v = n[compact ? 1 : 0];
    if (!v) {
        if (compact)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_raycast_queue<CompactVox>, 128, 0);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_raycast_queue<ExactVox>, 128, 0);
        if (v <= 0) v = 8;
    }
    return v;
}

int launch_zrange(const MapView& m, const Intr& k, const DevPose* pose, const int* skip, cudaStream_t s,
                  int rc_tiles) {
    fb_launch(k_zrange_init, (const void*)k_zrange_init_fused, (m.zc * m.zr + 255) / 256, 256, 0, s, m, skip);
    // one more block prepares the raycast's block order when there is one to prepare
    const int ord_n = m.rc_order ? rc_tiles : 0;
    fb_launch(k_zrange, (const void*)k_zrange_fused, sm_count_rc() * 2 + (ord_n > 0 ? 1 : 0), 256, 0, s, m, k, pose,
              skip, ord_n);
    fb_launch(k_grid_clear, (const void*)k_grid_clear_fused, sm_count_rc() * 4, 256, 0, s, m, skip);
    fb_launch(k_grid_fill, (const void*)k_grid_fill_fused, sm_count_rc() * 4, 256, 0, s, m, skip);
    return 4;
}

int launch_raycast(const MapView& m, float4* vmap, float4* nmap, int p, int W, int H, const Intr& k,
                    const DevPose* pose, const int* skip, cudaStream_t s, int bx, int by) {
    if (bx == 0 && by == 0) {
        // resident CTAs only (4 warps each), no more than the tiles need
        const int tiles = ((W + 7) >> 3) * ((H + 3) >> 2);
        const int blocks = std::min(sm_count_rc() * queue_ctas_per_sm(m.cvox != nullptr), (tiles + 3) / 4);
        if (m.cvox)
            fb_launch(k_raycast_queue<CompactVox>, (const void*)k_raycast_queue_fused<CompactVox>, blocks, 128, 0, s,
                      m, vmap, nmap, p, W, H, k, pose, skip);
        else
            fb_launch(k_raycast_queue<ExactVox>, (const void*)k_raycast_queue_fused<ExactVox>, blocks, 128, 0, s, m,
                      vmap, nmap, p, W, H, k, pose, skip);
        return 1;
    }
    dim3 b(bx, by), g((W + bx - 1) / bx, (H + by - 1) / by);
    if (m.cvox)
        fb_launch(k_raycast<CompactVox>, (const void*)k_raycast_fused<CompactVox>, g, b, 0, s, m, vmap, nmap, p, W, H,
                  k, pose, skip);
    else
        fb_launch(k_raycast<ExactVox>, (const void*)k_raycast_fused<ExactVox>, g, b, 0, s, m, vmap, nmap, p, W, H, k,
                  pose, skip);
    return 1;
}

}  // namespace fb
