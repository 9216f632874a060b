// Voxel-block hash map: block allocation, visibility and TSDF/colour
// integration (the reference's Mapping/DeviceMap.cu, Mapping/FuseMap.cu).
//
// Allocation is deterministic.  The reference lets every pixel's probes race
// for a per-bucket try-lock (DeviceMap.cu:23-62): requests that lose the lock
// are dropped and entries can be duplicated.  Here one frame's requests are
// collected first and then inserted as if one at a time, without contention,
// in canonical order -- ascending (bucket, x, y, z) -- so the resulting hash
// state (slot, voxel block and chain link of every entry) depends only on the
// inputs.  The kernels:
//   requests : per pixel, the reference's probe walk along the truncation band
//              (Fusion::CreateBlocks, FuseMap.cu:80-111); blocks that are not in
//              the map go into a per-frame open-addressing request set (CAS on
//              64-bit keys); the first insert of a key appends it to the list
//              of new blocks.
//   scan / place / rank : a counting sort of the new blocks by bucket
//              (per-bucket counters taken by the requests, a two-level scan
//              over all buckets whose top level runs in the last chunk block
//              to finish), then the rank of each block inside its bucket by
//              coordinates.
//   insert   : (also the counters after the frame and the clearing of the
//              per-bucket counters) each new block computes from its rank alone where the
//              sequential insertion would put it: free-stack position, head
//              slot or excess slot, and its chain link; the one block per
//              bucket that extends an existing chain links the old tail.  If
//              the pool or the excess list would run out, or an earlier
//              exhaustion left empty entries inside chains, a single thread
//              performs the same insertions one by one with the reference's
//              exact CreateBlock rules instead.
// Visibility walks the list of allocated entries rather than every slot of
// the table (CheckVisibleBlockKernel, FuseMap.cu:113-138, scans all of them).
// Integration processes one visible block per CTA iteration: 256 threads, two
// voxels each, one 16-byte load (issued one block ahead) and at most one
// 16-byte store per thread; the per-pixel inputs come from the frame's fusion
// records (one 16-byte gather of depth and normal, one word of colour).
#include <cuda_fp16.h>

#include "fb_fused.cuh"
#include "fb_internal.h"

namespace fb {

// FindEntry (DeviceMap.cu:122-135): slot of the live entry for a block, or -1.
__device__ __forceinline__ int find_slot(const MapView& m, int x, int y, int z) {
    int b = (int)bucket_of_m(x, y, z, (uint32_t)m.NB, m.nb_mask);
    HEntry e = m.entries[b];
    if (e.ptr != -1 && e.x == x && e.y == y && e.z == z) return b;
    for (int guard = 0; e.offset > 0 && e.offset <= m.NE && guard <= m.NE; ++guard) {
        int s = m.NB + e.offset - 1;
        e = m.entries[s];
        if (e.x == x && e.y == y && e.z == z && e.ptr != -1) return s;
    }
    return -1;
}

__device__ __forceinline__ unsigned long long block_key(int x, int y, int z) {
    return (1ull << 63) | ((unsigned long long)(x & 0xFFFF) << 32) | ((unsigned long long)(y & 0xFFFF) << 16) |
           (unsigned long long)(z & 0xFFFF);
}

__device__ __forceinline__ uint32_t mix64(unsigned long long k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return (uint32_t)k;
}

__device__ __forceinline__ void request_block(const MapView& m, int x, int y, int z) {
    if (x < -kCoordLimit || x > kCoordLimit || y < -kCoordLimit || y > kCoordLimit || z < -kCoordLimit ||
        z > kCoordLimit) {
        atomicOr(&m.ctr->err, kErrCoordRange);
        return;
    }
    if (find_slot(m, x, y, z) >= 0) return;
    const unsigned long long key = block_key(x, y, z);
    uint32_t h = mix64(key) & (uint32_t)(m.reqcap - 1);
    for (int probe = 0; probe < 64; ++probe) {
        unsigned long long old = atomicCAS(&m.reqset[h], 0ull, key);
        if (old == 0ull) {
            int idx = atomicAdd(&m.ctr->n_req, 1);
            if (idx < m.newcap) {
                NewBlock nb;
                nb.x = (short)x;
                nb.y = (short)y;
                nb.z = (short)z;
                nb.pad = 0;
                nb.bucket = bucket_of_m(x, y, z, (uint32_t)m.NB, m.nb_mask);
                nb.setslot = (int)h;
                // arrival order inside the bucket (any order: the rank
                // below orders the bucket by coordinates)
                nb.j = atomicAdd(&m.bucket_cnt[nb.bucket], 1);
                nb.rank = 0;
                nb.pad2 = 0;
                m.newblk[idx] = nb;
            } else {
                atomicOr(&m.ctr->err, kErrNewListFull);
                atomicExch(&m.reqset[h], 0ull);
            }
            return;
        }
        if (old == key) return;
        h = (h + 1) & (uint32_t)(m.reqcap - 1);
    }
    atomicOr(&m.ctr->err, kErrRequestSetFull);
}

// Fusion::CreateBlocks (FuseMap.cu:80-111) for one pixel of the raw depth map.
__device__ __forceinline__ void alloc_requests_body(const BlockCtx& ctx, MapView m, const float* __restrict__ raw,
                                                    int rp, int W, int H, Intr k, const DevPose* __restrict__ posep,
                                                    const int* __restrict__ skip) {
    if (skip && *skip) return;
    const int x = ctx.bx * blockDim.x + threadIdx.x;
    const int y = ctx.by * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const float z = raw[(size_t)y * rp + x];
    const float dmin = m.g.depth_min, dmax = m.g.depth_max;
    if (isnan(z) || z < dmin || z > dmax) return;
    const DevPose P = *posep;
    const float thresh = m.g.trunc_dist / 2;
    const float zn = fminf(dmax, fs(z, thresh));
    const float zf = fminf(dmax, fa(z, thresh));
    if (zn >= zf) return;
    const float vinv = m.g.voxel_size_inv;
    const float ux = fs((float)x, k.cx), uy = fs((float)y, k.cy);
    f3 pn = mul3(add3(mv(P.R, mk3(fm(fm(zn, ux), k.invfx), fm(fm(zn, uy), k.invfy), zn)), P.t), vinv);
    f3 pf = mul3(add3(mv(P.R, mk3(fm(fm(zf, ux), k.invfx), fm(fm(zf, uy), k.invfy), zf)), P.t), vinv);
    f3 dir = sub3(pf, pn);
    const float len = norm3(dir);
    const int nSteps = (int)ceil(2.0 * (double)len);
    dir = div3(dir, (float)(nSteps - 1));
    int px = 0, py = 0, pz = 0;
    bool have = false;
    for (int i = 0; i < nSteps; ++i) {
        // make_int3(float3) truncates toward zero (VectorMath.h:36-38)
        int bx = block_of(__float2int_rz(pn.x)), by = block_of(__float2int_rz(pn.y)),
            bz = block_of(__float2int_rz(pn.z));
        if (!have || bx != px || by != py || bz != pz) {
            request_block(m, bx, by, bz);
            px = bx;
            py = by;
            pz = bz;
            have = true;
        }
        pn = add3(pn, dir);
    }
}

__global__ void __launch_bounds__(256) k_alloc_requests(MapView m, const float* __restrict__ raw, int rp, int W,
                                  int H, Intr k, const DevPose* __restrict__ posep, const int* __restrict__ skip) {
    alloc_requests_body(own_ctx(), m, raw, rp, W, H, k, posep, skip);
}
FB_FUSED_KERNEL(k_alloc_requests, alloc_requests_body, 256)

__device__ __forceinline__ void scan_top_body(MapView m);

// Per chunk of kScanChunk buckets: number of new blocks, and of those that go
// to the excess list (all but the first when the bucket's head slot is empty).
// The last block to finish then scans the chunk sums (scan_top_body).
__device__ __forceinline__ void scan_chunks_body(const BlockCtx& ctx, MapView m) {
    __shared__ int s_c[256], s_x[256];
    __shared__ bool s_last;
    const int base = ctx.bx * kScanChunk;
    const bool any = m.ctr->n_req > 0;
    int c = 0, xs = 0;
    for (int q = threadIdx.x; any && q < kScanChunk; q += 256) {
        int b = base + q;
        if (b >= m.NB) break;
        int n = m.bucket_cnt[b];
        if (n) {
            int he = m.entries[b].ptr == -1 ? 1 : 0;
            c += n;
            xs += n - he;
        }
    }
    s_c[threadIdx.x] = c;
    s_x[threadIdx.x] = xs;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s_c[threadIdx.x] += s_c[threadIdx.x + o];
            s_x[threadIdx.x] += s_x[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        m.chunk_sums[2 * ctx.bx] = s_c[0];
        m.chunk_sums[2 * ctx.bx + 1] = s_x[0];
        __threadfence();
        s_last = atomicAdd(&m.ctr->scan_ticket, 1u) == (unsigned)ctx.gx - 1u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) m.ctr->scan_ticket = 0;
    scan_top_body(m);
}

__global__ void __launch_bounds__(256) k_scan_chunks(MapView m) {
    scan_chunks_body(own_ctx(), m);
}
FB_FUSED_KERNEL(k_scan_chunks, scan_chunks_body, 256)

// Exclusive scan over the chunk sums (the 256 threads of the last chunk
// block, chunks in order); snapshot of the counters and choice of the
// parallel or sequential insertion path.
__device__ __forceinline__ void scan_top_body(MapView m) {
    MapCounters* c = m.ctr;
    const int M = min(c->n_req, m.newcap);
    __shared__ int s_a[256], s_e[256];
    __shared__ int s_base_a, s_base_e;
    if (threadIdx.x == 0) {
        s_base_a = 0;
        s_base_e = 0;
    }
    __syncthreads();
    if (M > 0) {
        for (int c0 = 0; c0 < m.nchunks; c0 += 256) {
            const int i = c0 + threadIdx.x;
            const int a = i < m.nchunks ? __ldcg(&m.chunk_sums[2 * i]) : 0;
            const int e = i < m.nchunks ? __ldcg(&m.chunk_sums[2 * i + 1]) : 0;
            s_a[threadIdx.x] = a;
            s_e[threadIdx.x] = e;
            __syncthreads();
            for (int o = 1; o < 256; o <<= 1) {   // inclusive Hillis-Steele scan
                int ta = threadIdx.x >= o ? s_a[threadIdx.x - o] : 0;
                int te = threadIdx.x >= o ? s_e[threadIdx.x - o] : 0;
                __syncthreads();
                s_a[threadIdx.x] += ta;
                s_e[threadIdx.x] += te;
                __syncthreads();
            }
            if (i < m.nchunks) {
                m.chunk_sums[2 * i] = s_base_a + s_a[threadIdx.x] - a;
                m.chunk_sums[2 * i + 1] = s_base_e + s_e[threadIdx.x] - e;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                s_base_a += s_a[255];
                s_base_e += s_e[255];
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        const int total_x = s_base_e;
        c->excess_total = total_x;
        c->snap_M = M;
        c->snap_hc = c->heap_counter;
        c->snap_ep = c->entry_ptr;
        c->snap_na = c->n_alloc;
        // the parallel path reproduces sequential insertion only while the
        // free stack and the excess list suffice and no chain holds an empty
        // entry left by an earlier exhaustion
        c->fast = (M <= c->heap_counter + 1) && (c->entry_ptr - 1 + total_x <= m.NE) && !c->holes;
    }
}


// Per chunk: exclusive scan of the per-bucket counts into segment starts and
// excess starts.
__device__ __forceinline__ void scan_apply_body(const BlockCtx& ctx, MapView m) {
    if (m.ctr->snap_M == 0) return;
    __shared__ int s_c[256], s_x[256];
    constexpr int per = kScanChunk / 256;
    const int base = ctx.bx * kScanChunk + threadIdx.x * per;
    int cnt[per], he[per];
    int c = 0, xs = 0;
#pragma unroll
    for (int q = 0; q < per; ++q) {
        int b = base + q;
        cnt[q] = 0;
        he[q] = 0;
        if (b < m.NB) {
            cnt[q] = m.bucket_cnt[b];
            if (cnt[q]) he[q] = m.entries[b].ptr == -1 ? 1 : 0;
        }
        c += cnt[q];
        xs += cnt[q] - he[q];
    }
    s_c[threadIdx.x] = c;
    s_x[threadIdx.x] = xs;
    __syncthreads();
    // Hillis-Steele inclusive scan over 256 thread totals
    for (int o = 1; o < 256; o <<= 1) {
        int ac = threadIdx.x >= o ? s_c[threadIdx.x - o] : 0;
        int ax = threadIdx.x >= o ? s_x[threadIdx.x - o] : 0;
        __syncthreads();
        s_c[threadIdx.x] += ac;
        s_x[threadIdx.x] += ax;
        __syncthreads();
    }
    int run_c = m.chunk_sums[2 * ctx.bx] + s_c[threadIdx.x] - c;
    int run_x = m.chunk_sums[2 * ctx.bx + 1] + s_x[threadIdx.x] - xs;
#pragma unroll
    for (int q = 0; q < per; ++q) {
        int b = base + q;
        if (cnt[q]) {
            m.bucket_start[b] = run_c;
            m.bucket_x[b] = (run_x << 1) | he[q];
        }
        run_c += cnt[q];
        run_x += cnt[q] - he[q];
    }
}

__global__ void __launch_bounds__(256) k_scan_apply(MapView m) {
    scan_apply_body(own_ctx(), m);
}
FB_FUSED_KERNEL(k_scan_apply, scan_apply_body, 256)

__device__ __forceinline__ void alloc_place_body(const BlockCtx& ctx, MapView m) {
    const int M = m.ctr->snap_M;
    for (int i = ctx.bx * blockDim.x + threadIdx.x; i < M; i += ctx.gx * blockDim.x) {
        const NewBlock& nb = m.newblk[i];
        m.arrival[m.bucket_start[nb.bucket] + nb.j] = i;
    }
}

__global__ void __launch_bounds__(256) k_alloc_place(MapView m) {
    alloc_place_body(own_ctx(), m);
}
FB_FUSED_KERNEL(k_alloc_place, alloc_place_body, 256)

__device__ __forceinline__ bool coord_less(const NewBlock& a, const NewBlock& b) {
    if (a.x != b.x) return a.x < b.x;
    if (a.y != b.y) return a.y < b.y;
    return a.z < b.z;
}

__device__ __forceinline__ void alloc_rank_body(const BlockCtx& ctx, MapView m) {
    const int M = m.ctr->snap_M;
    for (int p = ctx.bx * blockDim.x + threadIdx.x; p < M; p += ctx.gx * blockDim.x) {
        const int i = m.arrival[p];
        const NewBlock me = m.newblk[i];
        const int s = m.bucket_start[me.bucket], n = m.bucket_cnt[me.bucket];
        int r = 0;
        for (int q = s; q < s + n; ++q)
            if (coord_less(m.newblk[m.arrival[q]], me)) ++r;
        m.newblk[i].rank = s + r;
        m.order[s + r] = i;
    }
}

__global__ void __launch_bounds__(256) k_alloc_rank(MapView m) {
    alloc_rank_body(own_ctx(), m);
}
FB_FUSED_KERNEL(k_alloc_rank, alloc_rank_body, 256)

// CreateBlock (DeviceMap.cu:23-62) without lock contention, one block at a
// time, for the sequential path.  Returns the slot written or -1.
__device__ int create_block_seq(const MapView& m, int x, int y, int z, int& hc, int& ep, int& holes) {
    const int b = (int)bucket_of_m(x, y, z, (uint32_t)m.NB, m.nb_mask);
    HEntry* e = &m.entries[b];
    HEntry* eEmpty = nullptr;
    if (e->x == x && e->y == y && e->z == z && e->ptr != -1) return -1;
    if (e->ptr == -1) eEmpty = e;
    for (int guard = 0; e->offset > 0 && e->offset <= m.NE && guard <= m.NE; ++guard) {
        e = &m.entries[m.NB + e->offset - 1];
        if (e->x == x && e->y == y && e->z == z && e->ptr != -1) return -1;
        if (e->ptr == -1 && !eEmpty) eEmpty = e;
    }
    // CreateEntry (DeviceMap.cu:12-21)
    auto create_entry = [&](int offset) {
        HEntry n;
        n.x = (short)x;
        n.y = (short)y;
        n.z = (short)z;
        n.pad = 0;
        int old = hc--;
        int ptr = old >= 0 ? m.heap[old] : -1;
        if (ptr != -1) {
            n.ptr = ptr;
            n.offset = offset;
        } else {
            n.ptr = -1;
            n.offset = 0;
        }
        return n;
    };
    if (eEmpty) {
        *eEmpty = create_entry(e->offset);
        if (eEmpty->ptr == -1) holes = 1;
        return (int)(eEmpty - m.entries);
    }
    int offset = ep++;
    if (offset <= m.NE) {
        HEntry* n = &m.entries[m.NB + offset - 1];
        *n = create_entry(0);
        e->offset = offset;
        if (n->ptr == -1) holes = 1;
        return (int)(n - m.entries);
    }
    return -1;
}

// The insertion (parallel or sequential path), the clearing of the per-bucket
// counters for the next frame, and the map counters after this frame: every
// thread reads only the snapshot, so the first thread can write the counters
// at once.
__device__ __forceinline__ void alloc_insert_body(const BlockCtx& ctx, MapView m) {
    MapCounters* c = m.ctr;
    const int M = c->snap_M;
    const bool fast = c->fast;
    const int gtid = ctx.bx * blockDim.x + threadIdx.x, gstride = ctx.gx * blockDim.x;
    if (gtid == 0) {
        if (M > 0 && fast) {
            c->heap_counter = c->snap_hc - M;
            c->entry_ptr = c->snap_ep + c->excess_total;
            c->n_alloc = c->snap_na + M;
            c->seq_path = 0;
        }
        c->n_new = M;
        c->n_req = 0;
        c->n_visible = 0;
        c->n_tiles = 0;
    }
    if (M == 0) return;
    const int hc0 = c->snap_hc, ep0 = c->snap_ep, na0 = c->snap_na;
    if (!fast) {
        if (gtid == 0) {
            int hc = hc0, ep = ep0, holes = c->holes, na = na0;
            for (int R = 0; R < M; ++R) {
                const NewBlock nb = m.newblk[m.order[R]];
                int slot = create_block_seq(m, nb.x, nb.y, nb.z, hc, ep, holes);
                if (slot >= 0 && m.entries[slot].ptr != -1) m.alloc_list[na++] = slot;
            }
            unsigned err = kErrSequentialInsert;
            if (hc < -1) err |= kErrHeapExhausted;
            if (ep - 1 > m.NE) err |= kErrExcessFull;
            atomicOr(&c->err, err);
            c->heap_counter = hc;
            c->entry_ptr = ep;
            c->holes = holes;
            c->n_alloc = na;
            c->seq_path = 1;
        }
        for (int R = gtid; R < M; R += gstride) {
            const NewBlock& nb = m.newblk[m.order[R]];
            m.reqset[nb.setslot] = 0ull;
            m.bucket_cnt[nb.bucket] = 0;
        }
        return;
    }
    for (int R = gtid; R < M; R += gstride) {
        const int i = m.order[R];
        const NewBlock nb = m.newblk[i];
        const int b = (int)nb.bucket;
        const int s = m.bucket_start[b], bx = m.bucket_x[b];
        const int he = bx & 1, xs = bx >> 1;
        const int r = R - s;
        // the bucket's blocks are consecutive in canonical order: another
        // follows this one exactly when the next block has the same bucket
        const bool more = R + 1 < M && (int)m.newblk[m.order[R + 1]].bucket == b;
        HEntry e;
        e.x = nb.x;
        e.y = nb.y;
        e.z = nb.z;
        e.pad = 0;
        e.ptr = m.heap[hc0 - R];
        int slot;
        if (he && r == 0) {
            slot = b;
            e.offset = more ? ep0 + xs : 0;
        } else {
            const int q = r - he;                 // rank among this bucket's excess blocks
            const int off = ep0 + xs + q;
            slot = m.NB + off - 1;
            e.offset = more ? off + 1 : 0;
            if (q == 0 && !he) {
                // link the tail of the existing chain (CreateBlock's e->offset = offset)
                int t = b;
                for (int guard = 0; m.entries[t].offset > 0 && m.entries[t].offset <= m.NE && guard <= m.NE;
                     ++guard)
                    t = m.NB + m.entries[t].offset - 1;
                m.entries[t].offset = off;
            }
        }
        m.entries[slot] = e;
        m.alloc_list[na0 + R] = slot;
        m.reqset[nb.setslot] = 0ull;
        m.bucket_cnt[b] = 0;
    }
}

__global__ void __launch_bounds__(256) k_alloc_insert(MapView m) {
    alloc_insert_body(own_ctx(), m);
}
FB_FUSED_KERNEL(k_alloc_insert, alloc_insert_body, 256)


// ---------------------------------------------------------------- visibility

// Fusion::CheckVertexVisibility / CheckBlockVisibility (FuseMap.cu:36-78);
// the eight corners are reached by the reference's sequence of float adds.
__device__ __forceinline__ bool vertex_visible(f3 p, const DevPose& P, const Intr& k, int W, int H,
                                               const MapGeom& g) {
    p = mv(P.Rinv, sub3(p, P.t));
    if (p.z < 1e-3f) return false;
    float u = fa(fd(fm(k.fx, p.x), p.z), k.cx), v = fa(fd(fm(k.fy, p.y), p.z), k.cy);
    return u >= 0 && v >= 0 && u < (float)W && v < (float)H && p.z >= g.depth_min && p.z <= g.depth_max;
}

__device__ bool block_visible(int bx, int by, int bz, const DevPose& P, const Intr& k, int W, int H,
                              const MapGeom& g) {
    const float s = g.block_width;
    f3 c = mk3(fm((float)bx, s), fm((float)by, s), fm((float)bz, s));
    if (vertex_visible(c, P, k, W, H, g)) return true;
    c.z = fa(c.z, s);
    if (vertex_visible(c, P, k, W, H, g)) return true;
    c.y = fa(c.y, s);
    if (vertex_visible(c, P, k, W, H, g)) return true;
    c.x = fa(c.x, s);
    if (vertex_visible(c, P, k, W, H, g)) return true;
    c.z = fs(c.z, s);
    if (vertex_visible(c, P, k, W, H, g)) return true;
    c.y = fs(c.y, s);
    if (vertex_visible(c, P, k, W, H, g)) return true;
    c.x = fs(c.x, s);
    c.y = fa(c.y, s);
    if (vertex_visible(c, P, k, W, H, g)) return true;
    c.x = fa(c.x, s);
    c.y = fs(c.y, s);
    c.z = fa(c.z, s);
    if (vertex_visible(c, P, k, W, H, g)) return true;
    return false;
}

__device__ __forceinline__ void reset_visible_body(const BlockCtx& ctx, MapCounters* c) {
    c->n_visible = 0;
    c->n_tiles = 0;
}

__global__ void __launch_bounds__(32) k_reset_visible(MapCounters* c) {
    reset_visible_body(own_ctx(), c);
}
FB_FUSED_KERNEL(k_reset_visible, reset_visible_body, 32)

__device__ __forceinline__ void visibility_body(const BlockCtx& ctx, MapView m, int W, int H, Intr k,
                                                const DevPose* __restrict__ posep, const int* __restrict__ skip) {
    if (skip && *skip) return;
    const DevPose P = *posep;
    const int n = m.ctr->n_alloc;
    const int lane = threadIdx.x & 31;
    const int nIter = (n + ctx.gx * blockDim.x - 1) / (ctx.gx * blockDim.x);
    for (int it = 0; it < nIter; ++it) {
        const int i = (it * ctx.gx + ctx.bx) * blockDim.x + threadIdx.x;
        bool vis = false;
        int slot = -1;
        HEntry e;
        if (i < n) {
            slot = m.alloc_list[i];
            e = m.entries[slot];
            vis = block_visible(e.x, e.y, e.z, P, k, W, H, m.g);
        }
        // warp-aggregated append
        unsigned mask = __ballot_sync(0xffffffffu, vis);
        if (mask) {
            int base = 0;
            if (lane == 0) base = atomicAdd(&m.ctr->n_visible, __popc(mask));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (vis) {
                int o = base + __popc(mask & ((1u << lane) - 1));
                if (o < m.NS) {
                    m.visible[o] = slot;
                    m.vis_blocks[o] = e;   // read by integration and z ranges without a second gather
                } else {
                    atomicOr(&m.ctr->err, kErrVisibleFull);
                }
            }
        }
    }
}

__global__ void __launch_bounds__(256) k_visibility(MapView m, int W, int H, Intr k,
                                  const DevPose* __restrict__ posep, const int* __restrict__ skip) {
    visibility_body(own_ctx(), m, W, H, k, posep, skip);
}
FB_FUSED_KERNEL(k_visibility, visibility_body, 256)

// --------------------------------------------------------------- integration

// Fusion records of caller images (fb_fuse_map_color; the frame path makes
// them in the level-0 map kernel): see fuse_record.  The integration kernels
// use 1 for the normal's w lane, which ComputeNMap sets on every valid normal
// (Pyrdown.cu:93-125); a valid normal with another w lane is flagged.
__global__ void k_fuse_records(MapView m, const float* __restrict__ raw, int rp, const uint8_t* __restrict__ rgb,
                               int cp, const float4* __restrict__ nmap, int np, int W, int H) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const float4 n = nmap[(size_t)y * np + x];
    if (!isnan(n.x) && n.w != 1.0f) atomicOr(&m.ctr->err, kErrNormalW);
    if (m.cvox)
        fuse_record_packed(raw[(size_t)y * rp + x], n, rgb + (size_t)y * cp + 3 * x, m.g.depth_min, m.g.depth_max,
                           (uint4*)m.frec + (size_t)y * W + x);
    else
        fuse_record(raw[(size_t)y * rp + x], n, rgb + (size_t)y * cp + 3 * x, m.g.depth_min, m.g.depth_max,
                    m.frec + (size_t)y * W + x, m.fcol + (size_t)y * W + x);
}

// Fusion::integrateColor (FuseMap.cu:140-191) for one voxel, every operation
// rounded as the reference's float expression.  rec / col: the frame's fusion
// records (W wide).  Returns true when the voxel changed.
__device__ __forceinline__ bool integrate_voxel(Voxel& vox, int vx, int vy, int vz, const float4* __restrict__ rec,
                                                const uint32_t* __restrict__ col, int W, int H, const Intr& k,
                                                const DevPose& P, const MapGeom& g,
                                                const float* __restrict__ div255) {
    f3 pos = mk3(fm((float)vx, g.voxel_size), fm((float)vy, g.voxel_size), fm((float)vz, g.voxel_size));
    pos = mv(P.Rinv, sub3(pos, P.t));
    // the two quotients by pos.z share one reciprocal (fd_rcp); positions are
    // sums of products of voxel-scale values, normal floats or exactly zero
    float pu, pv;
    if (pos.z != 0.0f) {
        const float rz = __frcp_rn(pos.z);
        pu = fa(fd_rcp(fm(k.fx, pos.x), pos.z, rz), k.cx);
        pv = fa(fd_rcp(fm(k.fy, pos.y), pos.z, rz), k.cy);
    } else {
        pu = fa(fd(fm(k.fx, pos.x), pos.z), k.cx);
        pv = fa(fd(fm(k.fy, pos.y), pos.z), k.cy);
    }
    const int u = __float2int_rz(pu), v = __float2int_rz(pv);  // make_int2(float2)
    if (u < 0 || v < 0 || u >= W || v >= H) return false;
    const int pix = v * W + u;
    const float4 r = __ldg(rec + pix);   // r.x: the raw depth, NaN where the pixel is skipped
    const float thresh = g.trunc_dist;
    float sdf = fs(r.x, pos.z);
    if (!(sdf >= -thresh)) return false;
    sdf = fminf(1.0f, fd_rcp(sdf, thresh, __frcp_rn(thresh)));
    // w = nl * normalised(float4(pos, 1)): the dot runs over all four lanes
    // (the normal's w lane is 1, so its term is 1 / nrm)
    const float nrm = fsq(fa(fa(fa(fm(pos.x, pos.x), fm(pos.y, pos.y)), fm(pos.z, pos.z)), 1.0f));
    // nrm >= 1: the four quotients share its reciprocal (1 / nrm is that
    // reciprocal itself)
    const float rn = __frcp_rn(nrm);
    const float w = fa(fa(fa(fm(r.y, fd_rcp(pos.x, nrm, rn)), fm(r.z, fd_rcp(pos.y, nrm, rn))),
                          fm(r.w, fd_rcp(pos.z, nrm, rn))),
                       rn);
    const uint32_t c = __ldg(col + pix);
    const uint32_t cr = c & 255u, cg = (c >> 8) & 255u, cb = c >> 16;
    if (vox.weight == 0) {
        vox.sdf = sdf;
        vox.weight = 1;
        vox.r = (unsigned char)cr;
        vox.g = (unsigned char)cg;
        vox.b = (unsigned char)cb;
        return true;
    }
    const float a = fm(w, 0.2f), oa = fs(1.0f, a);
    const float W0 = (float)vox.weight;
    // (float)c / 255 of a byte c: the table holds those 256 IEEE quotients
    float rr = fm(fa(fm(a, div255[cr]), fm(oa, div255[vox.r])), 255.f);
    float gg = fm(fa(fm(a, div255[cg]), fm(oa, div255[vox.g])), 255.f);
    float bb = fm(fa(fm(a, div255[cb]), fm(oa, div255[vox.b])), 255.f);
    vox.sdf = fd(fa(fm(vox.sdf, W0), fm(w, sdf)), fa(W0, w));
    vox.weight = (unsigned char)min(255, (int)vox.weight + 1);
    // make_uchar3(float3): truncate to int, then to the low byte
    vox.r = (unsigned char)__float2int_rz(rr);
    vox.g = (unsigned char)__float2int_rz(gg);
    vox.b = (unsigned char)__float2int_rz(bb);
    return true;
}

__device__ __forceinline__ void integrate_body(const BlockCtx& ctx, MapView m, int W, int H, Intr k,
                                               const DevPose* __restrict__ posep, const int* __restrict__ skip) {
    if (skip && *skip) return;
    __shared__ float s_div255[256];
    s_div255[threadIdx.x] = fd((float)threadIdx.x, 255.f);   // blockDim.x == 256
    __syncthreads();
    const DevPose P = *posep;
    const int n = min(m.ctr->n_visible, m.NS);
    const int t = threadIdx.x;
    const int lx = (2 * t) & 7, ly = (t >> 2) & 7, lz = t >> 5;
    const float4* __restrict__ rec = m.frec;
    const uint32_t* __restrict__ col = m.fcol;
    // the next block's entry and voxels are loaded while this block's voxels
    // are integrated (the blocks of one CTA are distinct)
    HEntry e_nx;
    uint4 raw_nx;
    if (ctx.bx < n) {
        e_nx = m.vis_blocks[ctx.bx];
        raw_nx = *((const uint4*)(m.voxels + (size_t)e_nx.ptr * 512) + t);
    }
    for (int b = ctx.bx; b < n; b += ctx.gx) {
        const HEntry e = e_nx;
        const int vx = e.x * 8 + lx, vy = e.y * 8 + ly, vz = e.z * 8 + lz;
        uint4* base = (uint4*)(m.voxels + (size_t)e.ptr * 512) + t;
        const uint4 raw2 = raw_nx;
        if (b + ctx.gx < n) {
            e_nx = m.vis_blocks[b + ctx.gx];
            raw_nx = *((const uint4*)(m.voxels + (size_t)e_nx.ptr * 512) + t);
        }
        Voxel v0 = *(const Voxel*)&raw2.x, v1 = *(const Voxel*)&raw2.z;
        bool c0 = integrate_voxel(v0, vx, vy, vz, rec, col, W, H, k, P, m.g, s_div255);
        bool c1 = integrate_voxel(v1, vx + 1, vy, vz, rec, col, W, H, k, P, m.g, s_div255);
        if (c0 || c1) {
            uint4 o;
            *(Voxel*)&o.x = v0;
            *(Voxel*)&o.z = v1;
            *base = o;
        }
    }
}

__global__ void __launch_bounds__(256) k_integrate(MapView m, int W, int H, Intr k, const DevPose* __restrict__ posep,
                                  const int* __restrict__ skip) {
    integrate_body(own_ctx(), m, W, H, k, posep, skip);
}
FB_FUSED_KERNEL(k_integrate, integrate_body, 256)

// Precision form of k_integrate: 6-byte voxels (FP16 TSDF and one r, g, b,
// weight word), contracted FP32.  One wave of CTAs of 128 threads; each CTA
// takes every gridDim.x-th visible block.  The block's voxel loads are issued
// before the projections, so they overlap the record gathers.  Thread t owns
// four x-consecutive voxels, so its TSDF (8 B) and words (16 B) are two
// coalesced vector loads and stores; which (y, z) it owns is chosen per frame
// so that a warp's 32 voxels of one gather lie along the viewing direction.
// The per-pixel inputs are one packed 16-byte record (fuse_record_packed):
// the gathers, not the voxel traffic, bound this kernel (L1 wavefronts of
// scattered loads), so one gather per voxel instead of two matters most.
// Camera-space positions come from a per-block origin and the columns of
// Rinv scaled by the voxel size (voxel q of the four at origin + q x-column).
//
// The update is integrateColor's (FuseMap.cu:140-191): project (truncated
// pixel), record depth valid, sdf >= -T, sdf = min(1, sdf / T),
// w = n . normalised(p, 1) over four lanes, first observation or weighted
// running average, weight + 1 capped at 255, colour c0 + 0.2 w (c - c0).
// The colour is blended on floats 1.5 * 2^23 + byte, whose low mantissa bits
// are the byte: one exact subtraction and one fused multiply-add rounded
// toward zero give floor(c0 + 0.2 w (c - c0)) modulo 256 (the reference
// truncates toward zero; the two differ only where the sum is negative and
// wraps).
__device__ __forceinline__ float byte_as_magic(uint32_t word, uint32_t sel) {
    // byte `sel` of `word` into the low byte of 0x4b400000 = 1.5 * 2^23
    return __uint_as_float(__byte_perm(word, 0x4b400000u, sel | 0x7650u));
}

__device__ __forceinline__ void integrate_compact_body(const BlockCtx& ctx, MapView m, int W, int H, Intr k,
                                                       const DevPose* __restrict__ posep,
                                                       const int* __restrict__ skip) {
    if (skip && *skip) return;
    const DevPose P = *posep;
    const int n = min(m.ctr->n_visible, m.NS);
    const int t = threadIdx.x, l = t & 31, wq = t >> 5;
    // voxels of a warp's gather lie along the world axis closest to the
    // viewing direction (the camera's z axis in world coordinates is row 2 of
    // Rinv), where they project onto few pixels: lane bits 1-4 and the warp
    // index split the block's y and z coordinates accordingly; each thread
    // keeps four x-consecutive voxels (vector loads and stores)
    const float ax = fabsf(P.Rinv.r2.x), ay = fabsf(P.Rinv.r2.y), az = fabsf(P.Rinv.r2.z);
    int ly, lz;
    if (az >= ax && az >= ay) {          // view along z: 8 z x 2 y per warp
        ly = ((l >> 1) & 1) | (wq << 1);
        lz = (l >> 2) & 7;
    } else if (ay >= ax) {               // view along y: 8 y x 2 z per warp
        ly = (l >> 1) & 7;
        lz = ((l >> 4) & 1) | (wq << 1);
    } else {                             // view along x: 4 y x 4 z per warp
        ly = ((l >> 1) & 3) | ((wq & 1) << 2);
        lz = ((l >> 3) & 3) | ((wq >> 1) << 2);
    }
    const int lx = 4 * (l & 1);
    const int idx = lz * 64 + ly * 8 + lx;
    const float vs = m.g.voxel_size, T = m.g.trunc_dist, invT = 1.0f / T;
    // camera = Rinv (world - t): basis columns Rinv e_i * vs and offset -Rinv t
    const f3 bx = mk3(P.Rinv.r0.x * vs, P.Rinv.r1.x * vs, P.Rinv.r2.x * vs);
    const f3 by = mk3(P.Rinv.r0.y * vs, P.Rinv.r1.y * vs, P.Rinv.r2.y * vs);
    const f3 bz = mk3(P.Rinv.r0.z * vs, P.Rinv.r1.z * vs, P.Rinv.r2.z * vs);
    const f3 c0 = mk3(-(P.Rinv.r0.x * P.t.x + P.Rinv.r0.y * P.t.y + P.Rinv.r0.z * P.t.z),
                      -(P.Rinv.r1.x * P.t.x + P.Rinv.r1.y * P.t.y + P.Rinv.r1.z * P.t.z),
                      -(P.Rinv.r2.x * P.t.x + P.Rinv.r2.y * P.t.y + P.Rinv.r2.z * P.t.z));
    const uint4* __restrict__ rec = (const uint4*)m.frec;   // packed records (fuse_record_packed)
    for (int b = ctx.bx; b < n; b += ctx.gx) {
        const HEntry e4 = m.vis_blocks[b];
        const int4 e = make_int4(e4.x, e4.y, e4.z, e4.ptr);
        uint8_t* blk = m.cvox + (size_t)e.w * kCBlockBytes;
        uint2 sd = *(const uint2*)(blk + 2 * idx);
        const uint4 cw = *(const uint4*)(blk + kCRgbw + 4 * idx);
        const float ox = (float)(e.x * 8 + lx), oy = (float)(e.y * 8 + ly), oz = (float)(e.z * 8 + lz);
        f3 p;
        p.x = fmaf(bx.x, ox, fmaf(by.x, oy, fmaf(bz.x, oz, c0.x)));
        p.y = fmaf(bx.y, ox, fmaf(by.y, oy, fmaf(bz.y, oz, c0.y)));
        p.z = fmaf(bx.z, ox, fmaf(by.z, oy, fmaf(bz.z, oz, c0.z)));
        // the four projections, then their record gathers issued together;
        // voxel q sits at p + q bx (recomputed where needed: fewer live
        // registers than keeping the four positions)
        int pix[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const f3 pq = mk3(fmaf((float)q, bx.x, p.x), fmaf((float)q, bx.y, p.y), fmaf((float)q, bx.z, p.z));
            const float rz = __fdividef(1.0f, pq.z);
            const int u = __float2int_rz(fmaf(k.fx * pq.x, rz, k.cx));
            const int v = __float2int_rz(fmaf(k.fy * pq.y, rz, k.cy));
            pix[q] = ((unsigned)u < (unsigned)W && (unsigned)v < (unsigned)H) ? v * W + u : -1;
        }
        uint4 r[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) r[q] = pix[q] >= 0 ? __ldg(rec + pix[q]) : make_uint4(0x7fffffffu, 0u, 0u, 0u);
        const __half2 s01 = *(const __half2*)&sd.x, s23 = *(const __half2*)&sd.y;
        float sdf[4] = {__low2float(s01), __high2float(s01), __low2float(s23), __high2float(s23)};
        uint32_t word[4] = {cw.x, cw.y, cw.z, cw.w};
        bool changed = false;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const f3 pq = mk3(fmaf((float)q, bx.x, p.x), fmaf((float)q, bx.y, p.y), fmaf((float)q, bx.z, p.z));
            const float so = __uint_as_float(r[q].x) - pq.z;
            if (!(so >= -T)) continue;   // NaN depth (skipped pixel or outside the image) fails too
            const float ts = fminf(1.0f, so * invT);
            const float2 nxy = __half22float2(*reinterpret_cast<const __half2*>(&r[q].y));
            const float nz = __half2float(__ushort_as_half((unsigned short)(r[q].z & 0xffffu)));
            const uint32_t cq = (r[q].z >> 16) | (r[q].w << 16);   // r | g << 8 | b << 16
            const float w = fmaf(nxy.x, pq.x, fmaf(nxy.y, pq.y, fmaf(nz, pq.z, 1.0f))) *
                            rsqrtf(fmaf(pq.x, pq.x, fmaf(pq.y, pq.y, fmaf(pq.z, pq.z, 1.0f))));
            const uint32_t W0 = word[q] >> 24;
            if (W0 == 0) {
                sdf[q] = ts;
                word[q] = cq | (1u << 24);
            } else {
                const float Wf = (float)W0, a = 0.2f * w;
                sdf[q] = __fdividef(fmaf(sdf[q], Wf, w * ts), Wf + w);
                const float r0 = byte_as_magic(word[q], 0), g0 = byte_as_magic(word[q], 1),
                            b0 = byte_as_magic(word[q], 2);
                const float rn = __fmaf_rz(a, byte_as_magic(cq, 0) - r0, r0);
                const float gn = __fmaf_rz(a, byte_as_magic(cq, 1) - g0, g0);
                const float bn = __fmaf_rz(a, byte_as_magic(cq, 2) - b0, b0);
                const uint32_t rg = __byte_perm(__float_as_uint(rn), __float_as_uint(gn), 0x0040u);
                const uint32_t bw = __byte_perm(__float_as_uint(bn), (W0 < 255u ? W0 + 1u : 255u), 0x0040u);
                word[q] = __byte_perm(rg, bw, 0x5410u);
            }
            changed = true;
        }
        if (changed) {
            const __half2 n01 = __floats2half2_rn(sdf[0], sdf[1]), n23 = __floats2half2_rn(sdf[2], sdf[3]);
            sd.x = *(const uint32_t*)&n01;
            sd.y = *(const uint32_t*)&n23;
            *(uint2*)(blk + 2 * idx) = sd;
            *(uint4*)(blk + kCRgbw + 4 * idx) = make_uint4(word[0], word[1], word[2], word[3]);
        }
    }
}

__global__ void __launch_bounds__(128, 7) k_integrate_compact(MapView m, int W, int H, Intr k,
                                  const DevPose* __restrict__ posep, const int* __restrict__ skip) {
    integrate_compact_body(own_ctx(), m, W, H, k, posep, skip);
}
FB_FUSED_KERNEL(k_integrate_compact, integrate_compact_body, 128, 7)

// ------------------------------------------------- the reference's layouts

// The reference's HashEntry (Mapping/DeviceMap.h:17-59, __align__(16): 32
// bytes): block position, voxel index of the block (block * 512) or -1, and
// the chain offset.
struct RefHashEntry {
    int x, y, z, ptr, offset, pad[3];
};
static_assert(sizeof(RefHashEntry) == 32, "the reference's HashEntry");

__device__ __forceinline__ RefHashEntry to_ref_entry(const HEntry& e) {
    RefHashEntry r;
    r.x = e.x;
    r.y = e.y;
    r.z = e.z;
    r.ptr = e.ptr >= 0 ? e.ptr * 512 : -1;
    r.offset = e.offset;
    r.pad[0] = r.pad[1] = r.pad[2] = 0;
    return r;
}

// n entries (from a table or the visible list) in the reference's layout.
__global__ void k_export_ref_entries(const HEntry* __restrict__ src, const int* __restrict__ count, int n,
                                     RefHashEntry* __restrict__ dst) {
    const int lim = count ? min(*count, n) : n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < lim; i += gridDim.x * blockDim.x)
        dst[i] = to_ref_entry(src[i]);
}

// Precision-form voxels in the reference's 8-byte Voxel layout (FP16 TSDF
// widened to float).
__global__ void k_export_ref_voxels(MapView m, Voxel* __restrict__ dst) {
    const size_t n = (size_t)m.NS * 512;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint8_t* blk = m.cvox + (i / 512) * kCBlockBytes;
        const int v = (int)(i % 512);
        Voxel o;
        o.sdf = __half2float(reinterpret_cast<const __half*>(blk)[v]);
        const uint32_t w = *reinterpret_cast<const uint32_t*>(blk + kCRgbw + 4 * v);
        o.weight = (uint8_t)(w >> 24);
        o.r = (uint8_t)w;
        o.g = (uint8_t)(w >> 8);
        o.b = (uint8_t)(w >> 16);
        dst[i] = o;
    }
}

__global__ void k_export_ref_counters(const MapCounters* __restrict__ c, int* heap_counter, int* entry_ptr) {
    if (heap_counter) *heap_counter = c->heap_counter;
    if (entry_ptr) *entry_ptr = c->entry_ptr;
}

// ---------------------------------------------------------------------- reset

// ResetHashKernel / ResetSdfBlockKernel (FuseMap.cu:321-350) on all of the
// table (the reference leaves pos and offset of released entries in place).
__global__ void k_map_reset(MapView m) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t ne = (size_t)m.NB + m.NE;
    for (size_t i = tid; i < ne; i += stride) {
        HEntry e;
        e.x = e.y = e.z = e.pad = 0;
        e.ptr = -1;
        e.offset = 0;
        m.entries[i] = e;
    }
    for (size_t i = tid; i < (size_t)m.NS; i += stride) m.heap[i] = m.NS - (int)i - 1;
    if (m.cvox) {
        // precision form: FP16 NaN TSDF, weight 0, colour 0 (64 + 128 uint4 per block)
        const uint4 nan8 = make_uint4(0x7e007e00u, 0x7e007e00u, 0x7e007e00u, 0x7e007e00u);
        const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
        uint4* vv = (uint4*)m.cvox;
        for (size_t i = tid; i < (size_t)m.NS * (kCBlockBytes / 16); i += stride)
            vv[i] = (i % (kCBlockBytes / 16)) < 64 ? nan8 : zero;
    } else {
        const uint4 released = make_uint4(0x7fffffffu, 0u, 0x7fffffffu, 0u);  // {NaN, w 0, rgb 0} x 2
        uint4* vv = (uint4*)m.voxels;
        for (size_t i = tid; i < (size_t)m.NS * 256; i += stride) vv[i] = released;
    }
    for (size_t i = tid; i < (size_t)m.NB; i += stride) m.bucket_cnt[i] = 0;
    for (size_t i = tid; i < (size_t)m.reqcap; i += stride) m.reqset[i] = 0ull;
    if (tid == 0) {
        MapCounters* c = m.ctr;
        c->heap_counter = m.NS - 1;
        c->entry_ptr = 1;
        c->holes = 0;
        c->n_alloc = 0;
        c->n_req = 0;
        c->n_new = 0;
        c->n_visible = 0;
        c->n_tiles = 0;
        c->excess_total = 0;
        c->err = 0;
        c->seq_path = 0;
        c->snap_M = 0;
        c->ray_next = 0;
        c->scan_ticket = 0;
    }
}

// ------------------------------------------------------------------ launchers

static int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

int launch_map_reset(const MapView& m, cudaStream_t s) { k_map_reset<<<sm_count() * 8, 256, 0, s>>>(m);
    return 1;
}

int launch_allocate(const MapView& m, const float* raw, int rp, int W, int H, const Intr& k, const DevPose* pose,
                     const int* skip, cudaStream_t s) {
    dim3 b(32, 8), g((W + 31) / 32, (H + 7) / 8);
    fb_launch(k_alloc_requests, (const void*)k_alloc_requests_fused, g, b, 0, s, m, raw, rp, W, H, k, pose, skip);
    const int gs = sm_count() * 4;
    fb_launch(k_scan_chunks, (const void*)k_scan_chunks_fused, m.nchunks, 256, 0, s, m);
    fb_launch(k_scan_apply, (const void*)k_scan_apply_fused, m.nchunks, 256, 0, s, m);
    fb_launch(k_alloc_place, (const void*)k_alloc_place_fused, gs, 256, 0, s, m);
    fb_launch(k_alloc_rank, (const void*)k_alloc_rank_fused, gs, 256, 0, s, m);
    fb_launch(k_alloc_insert, (const void*)k_alloc_insert_fused, gs, 256, 0, s, m);
    return 6;
}

int launch_visibility(const MapView& m, int W, int H, const Intr& k, const DevPose* pose, const int* skip,
                       cudaStream_t s, bool after_allocate) {
    // the allocation's last kernel (k_alloc_insert) zeroes the same counters
    if (!after_allocate) fb_launch(k_reset_visible, (const void*)k_reset_visible_fused, 1, 1, 0, s, m.ctr);
    fb_launch(k_visibility, (const void*)k_visibility_fused, sm_count() * 4, 256, 0, s, m, W, H, k, pose, skip);
    return after_allocate ? 1 : 2;
}

int launch_export_visible(const MapView& m, void* dst, int capacity, cudaStream_t s) {
    k_export_ref_entries<<<sm_count() * 2, 256, 0, s>>>(m.vis_blocks, &m.ctr->n_visible, min(capacity, m.NS),
                                                          (RefHashEntry*)dst);
    return 1;
}

int launch_export_reference(const MapView& m, void* entries, void* voxels, int* heap_counter, int* entry_ptr,
                            cudaStream_t s) {
    k_export_ref_entries<<<sm_count() * 8, 256, 0, s>>>(m.entries, nullptr, m.NB + m.NE, (RefHashEntry*)entries);
    if (m.cvox) k_export_ref_voxels<<<sm_count() * 8, 256, 0, s>>>(m, (Voxel*)voxels);
    k_export_ref_counters<<<1, 1, 0, s>>>(m.ctr, heap_counter, entry_ptr);
    return m.cvox ? 3 : 2;
}

int launch_fuse_records(const MapView& m, const float* raw, int rp, const uint8_t* rgb, int cp, const float4* nmap,
                        int np, int W, int H, cudaStream_t s) {
    dim3 b(32, 8), g((W + 31) / 32, (H + 7) / 8);
    k_fuse_records<<<g, b, 0, s>>>(m, raw, rp, rgb, cp, nmap, np, W, H);
    return 1;
}

int launch_integrate(const MapView& m, int W, int H, const Intr& k, const DevPose* pose, const int* skip,
                     cudaStream_t s, int ctas_per_sm) {
    const int ctas = sm_count() * (ctas_per_sm ? ctas_per_sm : m.cvox ? 7 : 8);
    if (m.cvox)
        fb_launch(k_integrate_compact, (const void*)k_integrate_compact_fused, ctas, 128, 0, s, m, W, H, k, pose, skip);
    else
        fb_launch(k_integrate, (const void*)k_integrate_fused, ctas, 256, 0, s, m, W, H, k, pose, skip);
    return 1;
}

}  // namespace fb
