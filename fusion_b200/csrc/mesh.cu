// Marching-cubes mesh extraction of the map (MeshScene, Mapping/MeshScene.cu:
// 20-355, called by Mapping::CreateModel, Mapping.cc:131-140) and the ASCII
// PLY writer of System::WriteMeshToDisk (Core/System.cc:140-193).
//
// Per voxel of every allocated block, as the reference: the cube of the voxel
// and its +x/+y/+z neighbours (any corner missing, NaN or exactly 1.0 -> no
// cube), central-difference gradients at the corners from the 24 voxels
// around the cube (any NaN -> no cube), the case index from sdf < 0, and on
// every cut edge the reference's vertex: interpolation parameter, position
// (voxel + offset) * voxel size, normal = normalised gradient interpolated
// along the edge, colour by the reference's uchar3 arithmetic.
//
// The case table is this library's own construction (build_case): on each
// cube face the cut edges are paired -- a face whose two negative corners sit
// on a diagonal keeps them apart -- and oriented so that the negative side
// lies to the left seen from outside the cube; the pairs close into loops
// across the faces and each loop is triangulated without chords lying in a
// cube face.  Every cut edge
// carries a vertex and two cubes sharing a face pair that face's edges the
// same way, so the mesh is closed wherever the field is defined.  The
// reference's vertices are reproduced exactly; the triangulation of a cube's
// polygon may differ from the reference's table (and the reference's
// classic table leaves holes on some ambiguous faces).  Triangles wind so
// that their right-hand normal points to the negative side.
//
// GPU layout: one CTA of 512 threads per allocated block, one thread per
// voxel.  The CTA finds the 27 blocks around its own once and stages the
// 11^3 voxel region the block's cubes and gradients read (local coordinates
// -1 .. 9) in shared memory, so each voxel costs shared-memory reads instead
// of the reference's 32 hash lookups.  Two passes make the output
// deterministic: triangle counts per block, an exclusive scan, then every
// block writes its triangles at its offset in voxel order.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda_fp16.h>

#include "../../include/fusion_b200.h"
#include "fb_internal.h"

namespace fb {

// ---------------------------------------------------------------- tables

// Corners (MeshScene.cu:105-140) and the twelve edges of buildVertexList
// (MeshScene.cu:185-256), as corner pairs in the reference's direction.
__host__ __device__ constexpr int corner_dx(int i) { return i == 1 || i == 2 || i == 5 || i == 6; }
__host__ __device__ constexpr int corner_dy(int i) { return i == 2 || i == 3 || i == 6 || i == 7; }
__host__ __device__ constexpr int corner_dz(int i) { return i >= 4; }
__host__ __device__ constexpr int edge_a(int e) { return e < 8 ? e : e - 8; }
__host__ __device__ constexpr int edge_b(int e) { return e < 8 ? ((e & 3) == 3 ? e - 3 : e + 1) : e - 4; }

static int edge_of(int a, int b) {
    for (int e = 0; e < 12; ++e)
        if ((edge_a(e) == a && edge_b(e) == b) || (edge_a(e) == b && edge_b(e) == a)) return e;
    return -1;
}

// Edges e and f lie on a common face of the cube.
static bool share_face(int e, int f) {
    const int a = edge_a(e), b = edge_b(e), c = edge_a(f), d = edge_b(f);
    const int ca[3] = {corner_dx(a), corner_dy(a), corner_dz(a)}, cb[3] = {corner_dx(b), corner_dy(b), corner_dz(b)};
    const int cc[3] = {corner_dx(c), corner_dy(c), corner_dz(c)}, cd[3] = {corner_dx(d), corner_dy(d), corner_dz(d)};
    for (int k = 0; k < 3; ++k)
        if (ca[k] == cb[k] && cc[k] == cd[k] && ca[k] == cc[k]) return true;
    return false;
}

// Triangulates the loop's sub-polygon loop[i .. j] (a polygon side or
// diagonal joins i and j) with diagonals that never join two vertices on
// one cube face: such a chord would lie in the face and, when the
// neighbouring cube draws the same chord, give an edge with four triangles.
// Triangles keep the loop's orientation.  Returns false if impossible.
static bool triangulate(const int* loop, int m, int i, int j, int8_t* tri, int* n) {
    if (j - i < 2) return true;
    auto allowed = [&](int p, int q) { return q == p + 1 || (p == 0 && q == m - 1) || !share_face(loop[p], loop[q]); };
    for (int k = i + 1; k < j; ++k) {
        if (!allowed(i, k) || !allowed(k, j)) continue;
        const int saved = *n;
        if (*n == 5) return false;
        tri[3 * *n + 0] = (int8_t)loop[i];
        tri[3 * *n + 1] = (int8_t)loop[k];
        tri[3 * *n + 2] = (int8_t)loop[j];
        ++*n;
        if (triangulate(loop, m, i, k, tri, n) && triangulate(loop, m, k, j, tri, n)) return true;
        *n = saved;
    }
    return false;
}

// The triangles of cube case `ci` (bit i set: corner i has sdf < 0) as edge
// triples; returns their number (at most 5) or -1 if the construction fails
// (it does not for any case; the tests check all 256).
int build_case(int ci, int8_t tri[16]) {
    // faces as corner quadruples, counter-clockwise seen from outside the cube
    int faces[6][4] = {{0, 3, 2, 1}, {4, 5, 6, 7}, {0, 1, 5, 4}, {3, 7, 6, 2}, {0, 4, 7, 3}, {1, 2, 6, 5}};
    const int outward[6][3] = {{0, 0, -1}, {0, 0, 1}, {0, -1, 0}, {0, 1, 0}, {-1, 0, 0}, {1, 0, 0}};
    for (int f = 0; f < 6; ++f) {   // orientation check of the list above
        const int* q = faces[f];
        int u[3], v[3];
        for (int k = 0; k < 3; ++k) {
            const int c0[3] = {corner_dx(q[0]), corner_dy(q[0]), corner_dz(q[0])};
            const int c1[3] = {corner_dx(q[1]), corner_dy(q[1]), corner_dz(q[1])};
            const int c2[3] = {corner_dx(q[2]), corner_dy(q[2]), corner_dz(q[2])};
            u[k] = c1[k] - c0[k];
            v[k] = c2[k] - c1[k];
        }
        const int c[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
        if (c[0] * outward[f][0] + c[1] * outward[f][1] + c[2] * outward[f][2] <= 0) return -1;
    }
    auto neg = [ci](int corner) { return (ci >> corner) & 1; };
    // next[e]: the cut edge that follows e along the polygon boundary
    int next[12];
    for (int e = 0; e < 12; ++e) next[e] = -1;
    for (int f = 0; f < 6; ++f) {
        const int* q = faces[f];
        int n_neg = 0;
        for (int k = 0; k < 4; ++k) n_neg += neg(q[k]);
        if (n_neg == 0 || n_neg == 4) continue;
        const bool diagonal = n_neg == 2 && neg(q[0]) == neg(q[2]);
        for (int k = 0; k < 4; ++k) {
            const int a = q[k], b = q[(k + 1) & 3];
            if (!(neg(a) && !neg(b))) continue;
            // leaving the negative region at edge (a, b): walk on around the
            // face (counter-clockwise) to where it is entered again, or, on a
            // diagonal face, close off corner a alone
            int en;
            if (diagonal) {
                en = edge_of(q[(k + 3) & 3], a);
            } else {
                int j = (k + 1) & 3;
                while (!(!neg(q[j]) && neg(q[(j + 1) & 3]))) j = (j + 1) & 3;
                en = edge_of(q[j], q[(j + 1) & 3]);
            }
            const int ex = edge_of(a, b);
            if (next[ex] != -1) return -1;
            next[ex] = en;
        }
    }
    int n = 0;
    bool used[12] = {};
    for (int s = 0; s < 12; ++s) {
        if (next[s] < 0 || used[s]) continue;
        int loop[12], m = 0;
        int e = s;
        while (!used[e]) {
            used[e] = true;
            loop[m++] = e;
            e = next[e];
            if (e < 0) return -1;
        }
        if (e != s || m < 3) return -1;
        if (!triangulate(loop, m, 0, m - 1, tri, &n)) return -1;
    }
    for (int e = 0; e < 12; ++e)   // every cut edge is on a loop
        if (neg(edge_a(e)) != neg(edge_b(e)) && !used[e]) return -1;
    for (int i = 3 * n; i < 16; ++i) tri[i] = -1;
    return n;
}

__constant__ int8_t c_tri[256][16];
__constant__ int c_ntri[256];

static int build_tables(int8_t tri[256][16], int ntri[256]) {
    for (int ci = 0; ci < 256; ++ci) {
        ntri[ci] = build_case(ci, tri[ci]);
        if (ntri[ci] < 0) return FB_EINVAL;
    }
    return FB_OK;
}

// Uploads the tables to the current device once.
static int ensure_tables() {
    static std::mutex lock;
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return FB_ECUDA;
    std::lock_guard<std::mutex> guard(lock);
    if (done[dev]) return FB_OK;
    int8_t tri[256][16];
    int ntri[256];
    if (build_tables(tri, ntri) != FB_OK) return FB_EINVAL;
    if (cudaMemcpyToSymbol(c_tri, tri, sizeof tri) != cudaSuccess) return FB_ECUDA;
    if (cudaMemcpyToSymbol(c_ntri, ntri, sizeof ntri) != cudaSuccess) return FB_ECUDA;
    done[dev] = true;
    return FB_OK;
}

// ---------------------------------------------------------------- kernels

constexpr int kMeshThreads = 512;
constexpr int kHalo = 11;                          // local coordinates -1 .. 9
constexpr int kRegion = kHalo * kHalo * kHalo;     // 1331
constexpr int kColSide = 9;                        // colours of local 0 .. 8

struct MeshSmem {
    int ptr[27];                 // blocks around this one, (dx + 1) + 3 (dy + 1) + 9 (dz + 1)
    float sdf[kRegion];          // NaN where no block (Voxel(), DeviceMap.h:63-65)
    uint32_t rgb[kColSide * kColSide * kColSide];
    int warp_sum[kMeshThreads / 32];
};

// FindEntry (DeviceMap.cu:122-135): block index of block (x, y, z), or -1.
__device__ int find_block(const MapView& m, int x, int y, int z) {
    const int b = (int)bucket_of_m(x, y, z, (uint32_t)m.NB, m.nb_mask);
    HEntry e = m.entries[b];
    if (e.ptr != -1 && e.x == x && e.y == y && e.z == z) return e.ptr;
    for (int guard = 0; e.offset > 0 && e.offset <= m.NE && guard <= m.NE; ++guard) {
        e = m.entries[m.NB + e.offset - 1];
        if (e.x == x && e.y == y && e.z == z && e.ptr != -1) return e.ptr;
    }
    return -1;
}

__device__ void stage_block(const MapView& m, const HEntry& self, MeshSmem& s) {
    const int t = threadIdx.x;
    if (t < 27) {
        const int dx = t % 3 - 1, dy = (t / 3) % 3 - 1, dz = t / 9 - 1;
        // the block itself is looked up too: a map with duplicate entries
        // for one block (the reference's racy allocator makes them) reads the
        // first one, as FindVoxel does
        s.ptr[t] = find_block(m, self.x + dx, self.y + dy, self.z + dz);
    }
    __syncthreads();
    for (int r = t; r < kRegion; r += kMeshThreads) {
        const int u = r % kHalo, v = (r / kHalo) % kHalo, w = r / (kHalo * kHalo);
        const int lx = u - 1, ly = v - 1, lz = w - 1;
        const int ox = lx < 0 ? -1 : (lx > 7 ? 1 : 0);
        const int oy = ly < 0 ? -1 : (ly > 7 ? 1 : 0);
        const int oz = lz < 0 ? -1 : (lz > 7 ? 1 : 0);
        const int p = s.ptr[(ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)];
        const int idx = (lz - 8 * oz) * 64 + (ly - 8 * oy) * 8 + (lx - 8 * ox);
        float sdf = qnan();
        uint32_t col = 0;
        if (p >= 0) {
            if (m.cvox) {
                const uint8_t* blk = m.cvox + (size_t)p * kCBlockBytes;
                sdf = __half2float(reinterpret_cast<const __half*>(blk)[idx]);
                col = *reinterpret_cast<const uint32_t*>(blk + kCRgbw + 4 * idx) & 0xffffffu;
            } else {
                const Voxel vx = m.voxels[(size_t)p * 512 + idx];
                sdf = vx.sdf;
                col = (uint32_t)vx.r | (uint32_t)vx.g << 8 | (uint32_t)vx.b << 16;
            }
        }
        s.sdf[r] = sdf;
        if (u >= 1 && u <= kColSide && v >= 1 && v <= kColSide && w >= 1 && w <= kColSide)
            s.rgb[(u - 1) + kColSide * (v - 1) + kColSide * kColSide * (w - 1)] = col;
    }
    __syncthreads();
}

// Region index of local voxel (x, y, z), each in -1 .. 9.
__device__ __forceinline__ int rix(int x, int y, int z) { return (x + 1) + kHalo * (y + 1) + kHalo * kHalo * (z + 1); }

// readVertexAndColor + readNormal's NaN tests + the case index
// (MeshScene.cu:43-183).  -1: no cube or no surface in it.
__device__ int classify(const MeshSmem& s, int x, int y, int z, float sd[8]) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        sd[i] = s.sdf[rix(x + corner_dx(i), y + corner_dy(i), z + corner_dz(i))];
        if (sd[i] == 1.0f || isnan(sd[i])) return -1;
    }
    // the 24 gradient neighbours outside the cube
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int cx = x + corner_dx(i), cy = y + corner_dy(i), cz = z + corner_dz(i);
        const float a = s.sdf[rix(corner_dx(i) ? cx + 1 : cx - 1, cy, cz)];
        const float b = s.sdf[rix(cx, corner_dy(i) ? cy + 1 : cy - 1, cz)];
        const float c = s.sdf[rix(cx, cy, corner_dz(i) ? cz + 1 : cz - 1)];
        if (isnan(a) || isnan(b) || isnan(c)) return -1;
    }
    int ci = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i)
        if (sd[i] < 0) ci |= 1 << i;
    return (ci == 0 || ci == 255) ? -1 : ci;
}

// interp (MeshScene.cu:142-150); the thresholds compare in double, as the
// reference's float-vs-double-literal comparisons do.
__device__ __forceinline__ float interp(float v1, float v2) {
    if ((double)fabsf(fs(0.f, v1)) < 1e-6) return 0.f;
    if ((double)fabsf(fs(0.f, v2)) < 1e-6) return 1.f;
    if ((double)fabsf(fs(v1, v2)) < 1e-6) return 0.f;
    return fd(fs(0.f, v1), fs(v2, v1));
}

// Central-difference gradient at corner i (readNormal, MeshScene.cu:43-103).
__device__ __forceinline__ f3 corner_gradient(const MeshSmem& s, int x, int y, int z, int i) {
    const int cx = x + corner_dx(i), cy = y + corner_dy(i), cz = z + corner_dz(i);
    return mk3(fs(s.sdf[rix(cx + 1, cy, cz)], s.sdf[rix(cx - 1, cy, cz)]),
               fs(s.sdf[rix(cx, cy + 1, cz)], s.sdf[rix(cx, cy - 1, cz)]),
               fs(s.sdf[rix(cx, cy, cz + 1)], s.sdf[rix(cx, cy, cz - 1)]));
}

// One vertex of edge e (buildVertexList, MeshScene.cu:185-256, and the
// scaling / normalisation of MarchingCube, MeshScene.cu:284-292).
// normal: n_a + val (n_b - n_a) as one fused multiply-add per component,
// then n / sqrt(n . n) with n . n = fma(z, z, fma(y, y, x x)).
// colour: c_a + (int)val * (c_b - c_a) in bytes (operator*(int, uchar3)).
__device__ void edge_vertex(const MeshSmem& s, int x, int y, int z, int3 g, const float sd[8], int e, float vs,
                            float* V, float* N, uint8_t* C) {
    const int a = edge_a(e), b = edge_b(e);
    const float val = interp(sd[a], sd[b]);
    // position: the corner a coordinates, the moving axis a's coordinate +/- val
    const int ax = corner_dx(a), ay = corner_dy(a), az = corner_dz(a);
    const int dx = corner_dx(b) - ax, dy = corner_dy(b) - ay, dz = corner_dz(b) - az;
    const float mv = (dx + dy + dz) > 0 ? val : fs(1.f, val);
    const float px = dx ? mv : (float)ax, py = dy ? mv : (float)ay, pz = dz ? mv : (float)az;
    V[0] = fm(fa((float)(g.x + x), px), vs);
    V[1] = fm(fa((float)(g.y + y), py), vs);
    V[2] = fm(fa((float)(g.z + z), pz), vs);
    const f3 na = corner_gradient(s, x, y, z, a), nb = corner_gradient(s, x, y, z, b);
    const f3 n = mk3(__fmaf_rn(val, fs(nb.x, na.x), na.x), __fmaf_rn(val, fs(nb.y, na.y), na.y),
                     __fmaf_rn(val, fs(nb.z, na.z), na.z));
    const float len = fsq(__fmaf_rn(n.z, n.z, __fmaf_rn(n.y, n.y, fm(n.x, n.x))));
    N[0] = fd(n.x, len);
    N[1] = fd(n.y, len);
    N[2] = fd(n.z, len);
    const uint32_t ca = s.rgb[(x + ax) + kColSide * (y + ay) + kColSide * kColSide * (z + az)];
    const uint32_t cb =
        s.rgb[(x + corner_dx(b)) + kColSide * (y + corner_dy(b)) + kColSide * kColSide * (z + corner_dz(b))];
    const int k = (int)val;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const uint8_t ua = (uint8_t)(ca >> (8 * c)), ub = (uint8_t)(cb >> (8 * c));
        C[c] = (uint8_t)(ua + (uint8_t)((uint8_t)(ub - ua) * k));
    }
}

// Block-wide exclusive scan of one int per thread (512 threads).
__device__ int block_exclusive_scan(int v, MeshSmem& s, int* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s.warp_sum[w] = incl;
    __syncthreads();
    if (w == 0) {
        int ws = lane < kMeshThreads / 32 ? s.warp_sum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, ws, o);
            if (lane >= o) ws += y;
        }
        if (lane < kMeshThreads / 32) s.warp_sum[lane] = ws;   // inclusive warp prefix
    }
    __syncthreads();
    const int before = w ? s.warp_sum[w - 1] : 0;
    *total = s.warp_sum[kMeshThreads / 32 - 1];
    return before + incl - v;
}

__global__ void __launch_bounds__(kMeshThreads) k_mesh_count(MapView m, int n_blocks, uint32_t* counts) {
    __shared__ MeshSmem s;
    const int blk = blockIdx.x;
    if (blk >= n_blocks) return;
    const HEntry self = m.entries[m.alloc_list[blk]];
    stage_block(m, self, s);
    const int t = threadIdx.x, x = t & 7, y = (t >> 3) & 7, z = t >> 6;
    float sd[8];
    const int ci = classify(s, x, y, z, sd);
    int total = 0;
    block_exclusive_scan(ci >= 0 ? c_ntri[ci] : 0, s, &total);
    if (t == 0) counts[blk] = (uint32_t)total;
}

// Exclusive scan of n counts into offsets[0 .. n] (offsets[n] = total), one
// CTA of 1024 threads walking tiles of 4096 in order.
__global__ void __launch_bounds__(1024) k_mesh_scan(const uint32_t* counts, int n, unsigned long long* offsets) {
    __shared__ unsigned long long warp_sum[32];
    __shared__ unsigned long long carry;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (t == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += 4096) {
        unsigned long long v[4], sum = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = base + 4 * t + k;
            v[k] = i < n ? counts[i] : 0;
            sum += v[k];
        }
        unsigned long long incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_sum[w] = incl;
        __syncthreads();
        if (w == 0) {
            unsigned long long ws = warp_sum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, ws, o);
                if (lane >= o) ws += y;
            }
            warp_sum[lane] = ws;
        }
        __syncthreads();
        unsigned long long run = carry + (w ? warp_sum[w - 1] : 0) + incl - sum;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = base + 4 * t + k;
            if (i < n) offsets[i] = run;
            run += v[k];
        }
        __syncthreads();
        if (t == 0) carry += warp_sum[31];
        __syncthreads();
    }
    if (t == 0) offsets[n] = carry;
}

__global__ void __launch_bounds__(kMeshThreads) k_mesh_emit(MapView m, int n_blocks,
                                                             const unsigned long long* offsets,
                                                             unsigned long long cap, float* V, float* N,
                                                             uint8_t* C) {
    __shared__ MeshSmem s;
    const int blk = blockIdx.x;
    if (blk >= n_blocks) return;
    const HEntry self = m.entries[m.alloc_list[blk]];
    stage_block(m, self, s);
    const int t = threadIdx.x, x = t & 7, y = (t >> 3) & 7, z = t >> 6;
    float sd[8];
    const int ci = classify(s, x, y, z, sd);
    const int nt = ci >= 0 ? c_ntri[ci] : 0;
    int total = 0;
    const int local = block_exclusive_scan(nt, s, &total);
    const unsigned long long first = offsets[blk] + (unsigned long long)local;
    const int3 g = make_int3(self.x * 8, self.y * 8, self.z * 8);
    for (int j = 0; j < nt; ++j) {
        const unsigned long long id = first + j;
        if (id >= cap) break;
#pragma unroll 1
        for (int k = 0; k < 3; ++k) {
            const size_t o = (size_t)(id * 3 + k);
            edge_vertex(s, x, y, z, g, sd, c_tri[ci][3 * j + k], m.g.voxel_size, V + 3 * o, N + 3 * o, C + 3 * o);
        }
    }
}

// Mesh of the map: *total = triangles found (all of them, also beyond `cap`);
// the first min(total, cap) are written when V, N and C are given.
// n_blocks: the allocated-list length.  Synchronous on `st`.
int launch_mesh(const MapView& m, int n_blocks, float* V, float* N, uint8_t* C, unsigned long long cap,
                unsigned long long* total, cudaStream_t st) {
    *total = 0;
    if (n_blocks <= 0) return FB_OK;
    const int rc = ensure_tables();
    if (rc != FB_OK) return rc;
    uint32_t* counts = nullptr;
    unsigned long long* offsets = nullptr;
    if (cudaMallocAsync((void**)&counts, sizeof(uint32_t) * n_blocks, st) != cudaSuccess) return FB_ENOMEM;
    if (cudaMallocAsync((void**)&offsets, sizeof(unsigned long long) * (n_blocks + 1), st) != cudaSuccess) {
        cudaFreeAsync(counts, st);
        return FB_ENOMEM;
    }
    k_mesh_count<<<n_blocks, kMeshThreads, 0, st>>>(m, n_blocks, counts);
    k_mesh_scan<<<1, 1024, 0, st>>>(counts, n_blocks, offsets);
    if (V && N && C && cap > 0) k_mesh_emit<<<n_blocks, kMeshThreads, 0, st>>>(m, n_blocks, offsets, cap, V, N, C);
    const cudaError_t le = cudaGetLastError();
    unsigned long long tot = 0;
    const cudaError_t ce = cudaMemcpyAsync(&tot, offsets + n_blocks, sizeof tot, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(counts, st);
    cudaFreeAsync(offsets, st);
    const cudaError_t se = cudaStreamSynchronize(st);
    if (le != cudaSuccess || ce != cudaSuccess || se != cudaSuccess) {
        fb_set_error_text(cudaGetErrorString(le != cudaSuccess ? le : (ce != cudaSuccess ? ce : se)));
        return FB_ECUDA;
    }
    *total = tot;
    return FB_OK;
}

}  // namespace fb

extern "C" {

int fb_mesh_case_table(int8_t* tri, int32_t* counts) {
    if (!tri || !counts) return FB_EINVAL;
    int8_t t[256][16];
    int n[256];
    if (fb::build_tables(t, n) != FB_OK) return FB_EINVAL;
    std::memcpy(tri, t, sizeof t);
    for (int i = 0; i < 256; ++i) counts[i] = n[i];
    return FB_OK;
}

int fb_write_ply(const char* path, const float* vertex, const float* normal, const uint8_t* color,
                 uint64_t no_triangles) {
    if (!path || (no_triangles && (!vertex || !normal || !color))) return FB_EINVAL;
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        fb_set_error_text("fb_write_ply: cannot open the file");
        return FB_EINVAL;
    }
    std::vector<char> buf(1 << 22);
    setvbuf(f, buf.data(), _IOFBF, buf.size());
    const unsigned long long nv = (unsigned long long)no_triangles * 3;
    std::fprintf(f,
                 "ply\nformat ascii 1.0\nelement vertex %llu\nproperty float x\nproperty float y\n"
                 "property float z\nproperty float nx\nproperty float ny\nproperty float nz\n"
                 "property uchar red\nproperty uchar green\nproperty uchar blue\nelement face %llu\n"
                 "property list uchar uint vertex_indices\nend_header\n",
                 nv, (unsigned long long)no_triangles);
    for (unsigned long long i = 0; i < nv; ++i)
        std::fprintf(f, "%g %g %g %g %g %g %d %d %d\n", vertex[3 * i], vertex[3 * i + 1], vertex[3 * i + 2],
                     normal[3 * i], normal[3 * i + 1], normal[3 * i + 2], (int)color[3 * i], (int)color[3 * i + 1],
                     (int)color[3 * i + 2]);
    for (unsigned long long i = 0; i < (unsigned long long)no_triangles; ++i)
        std::fprintf(f, "3 %llu %llu %llu\n", 3 * i, 3 * i + 1, 3 * i + 2);
    const bool ok = std::ferror(f) == 0;
    if (std::fclose(f) != 0 || !ok) {
        fb_set_error_text("fb_write_ply: write failed");
        return FB_EINVAL;
    }
    return FB_OK;
}

}  // extern "C"
