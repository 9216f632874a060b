// Session persistence: snapshots of a session's whole state (fb_snapshot /
// fb_restore) and the reference's map file (System::WriteMapToDisk /
// ReadMapFromDisk, Core/System.cc:195-271).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include <cuda_fp16.h>

#include "session_internal.h"

// ---------------------------------------------------------------- snapshots
//
// A snapshot holds everything a session needs to continue exactly where it
// was: the tracker's host state, the device tracker state, both frames, and
// the map -- counters, the whole hash table, the free-block stack, the
// allocated and visible lists and the used prefix of the voxel pool.  Blocks
// are taken from the free stack in order and never given back, so the used
// blocks are exactly the pool prefix [0, NumBlocks - 1 - heap_counter); the
// rest of the pool is in its reset state and is not stored.  The reference
// dumps its whole device map (System::WriteMapToDisk, Core/System.cc:195-236);
// this is the same idea with the unused pool left out and the tracker added.

namespace {

constexpr char kSnapMagic[8] = {'F', 'B', 'S', 'N', 'A', 'P', '0', '1'};

struct SnapHeader {
    char magic[8];
    fb_config cfg;
    int next, state, last_state, no_missed, frames_after_reloc, used_blocks;
    uint64_t frame_id;
    double pose[16];
    MapCounters ctr;
    uint64_t total_bytes;
};

int clamp_count(int v, int hi) { return v < 0 ? 0 : v > hi ? hi : v; }

// The byte ranges of a session's state in snapshot order (device pointer,
// size), after the header.
std::vector<std::pair<void*, size_t>> snapshot_ranges(fb_session* s, const MapCounters& c) {
    std::vector<std::pair<void*, size_t>> r;
    const MapView& m = s->map;
    const int used = clamp_count(m.NS - 1 - c.heap_counter, m.NS);
    const int na = clamp_count(c.n_alloc, m.NS);
    const int nv = clamp_count(c.n_visible, m.NS);
    r.push_back({m.entries, ((size_t)m.NB + m.NE) * sizeof(HEntry)});
    r.push_back({m.heap, (size_t)m.NS * sizeof(int)});
    r.push_back({m.alloc_list, (size_t)na * sizeof(int)});
    r.push_back({m.visible, (size_t)nv * sizeof(int)});
    r.push_back({m.vis_blocks, (size_t)nv * sizeof(HEntry)});
    if (m.cvox)
        r.push_back({m.cvox, (size_t)used * kCBlockBytes});
    else
        r.push_back({m.voxels, (size_t)used * 512 * sizeof(Voxel)});
    r.push_back({s->st, sizeof(TrackState)});
    for (int f = 0; f < 2; ++f) {
        FrameBuf& F = s->fr[f];
        const size_t n0 = (size_t)s->W[0] * s->H[0];
        r.push_back({F.depth_in, n0 * 2});
        r.push_back({F.rgb, n0 * 3});
        r.push_back({F.raw, n0 * 4});
        for (int l = 0; l < 3; ++l) {
            const size_t n = (size_t)s->W[l] * s->H[l];
            r.push_back({F.depth[l], n * 4});
            r.push_back({F.vmap[l], n * 16});
            r.push_back({F.nmap[l], n * 16});
            r.push_back({F.gray[l], n});
            r.push_back({F.dx[l], n * 2});
            r.push_back({F.dy[l], n * 2});
            r.push_back({F.rgbok[l], n});
        }
    }
    return r;
}


}  // namespace

extern "C" {

int fb_snapshot_bytes(fb_session* s, size_t* bytes) {
    if (!s || !bytes) return FB_EINVAL;
    MapCounters c;
    int rc = read_counters(s, &c);
    if (rc) return rc;
    size_t n = sizeof(SnapHeader);
    for (auto& r : snapshot_ranges(s, c)) n += r.second;
    *bytes = n;
    return FB_OK;
}

int fb_snapshot(fb_session* s, void* buf, size_t capacity, size_t* written) {
    if (!s || !buf) return FB_EINVAL;
    SnapHeader h;
    std::memset(&h, 0, sizeof h);
    int rc = read_counters(s, &h.ctr);
    if (rc) return rc;
    const auto ranges = snapshot_ranges(s, h.ctr);
    size_t total = sizeof h;
    for (auto& r : ranges) total += r.second;
    if (capacity < total) {
        fb_set_error_text("fb_snapshot: buffer smaller than fb_snapshot_bytes");
        return FB_EINVAL;
    }
    std::memcpy(h.magic, kSnapMagic, 8);
    h.cfg = s->cfg;
    h.next = s->next;
    h.state = s->state;
    h.last_state = s->last_state;
    h.no_missed = s->no_missed;
    h.frames_after_reloc = s->frames_after_reloc;
    h.frame_id = s->frame_id;
    std::memcpy(h.pose, s->pose, sizeof h.pose);
    h.used_blocks = clamp_count(s->map.NS - 1 - h.ctr.heap_counter, s->map.NS);
    h.total_bytes = total;
    char* out = (char*)buf;
    std::memcpy(out, &h, sizeof h);
    size_t o = sizeof h;
    for (auto& r : ranges) {
        if (r.second) FB_CUDA(cudaMemcpyAsync(out + o, r.first, r.second, cudaMemcpyDeviceToHost, s->stream));
        o += r.second;
    }
    FB_CUDA(cudaStreamSynchronize(s->stream));
    if (written) *written = total;
    return FB_OK;
}

int fb_restore(fb_session* s, const void* buf, size_t size) {
    if (!s || !buf || size < sizeof(SnapHeader)) return FB_EINVAL;
    SnapHeader h;
    std::memcpy(&h, buf, sizeof h);
    if (std::memcmp(h.magic, kSnapMagic, 8) != 0 || h.total_bytes != size) {
        fb_set_error_text("fb_restore: not a snapshot of this format");
        return FB_EINVAL;
    }
    if (std::memcmp(&h.cfg, &s->cfg, sizeof h.cfg) != 0) {
        fb_set_error_text("fb_restore: the snapshot was taken with another configuration");
        return FB_EINVAL;
    }
    // the unused pool and the per-frame scratch in their reset state first
    launch_map_reset(s->map, s->stream);
    if (check_launch()) return FB_ECUDA;
    const auto ranges = snapshot_ranges(s, h.ctr);
    size_t o = sizeof h;
    for (auto& r : ranges) {
        if (o + r.second > size) return FB_EINVAL;
        if (r.second)
            FB_CUDA(cudaMemcpyAsync(r.first, (const char*)buf + o, r.second, cudaMemcpyHostToDevice, s->stream));
        o += r.second;
    }
    FB_CUDA(cudaMemcpyAsync(s->ctr, &h.ctr, sizeof h.ctr, cudaMemcpyHostToDevice, s->stream));
    FB_CUDA(cudaStreamSynchronize(s->stream));
    s->next = h.next;
    s->state = h.state;
    s->last_state = h.last_state;
    s->no_missed = h.no_missed;
    s->frames_after_reloc = h.frames_after_reloc;
    s->frame_id = h.frame_id;
    std::memcpy(s->pose, h.pose, sizeof s->pose);
    return FB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- map files
//
// System::WriteMapToDisk / ReadMapFromDisk (Core/System.cc:195-271, through
// Mapping::DownloadToRAM / UploadFromRAM, Mapping/Mapping.cc:153-213): the
// reference's dump of its device map, in its byte layout -- four int sizes
// (NumSdfBlocks, NumBuckets, NumVoxels, NumEntries), the heap counter, the
// excess-list counter and the visible count, the free-block stack, the
// bucket locks, every voxel (8 bytes: sdf, weight, rgb), every hash entry,
// the visible-entry list (32-byte HashEntry: int3 pos, ptr as a voxel index,
// offset, padding), then the key-point map (an int lock per key and a
// 288-byte SURF per entry).  This library keeps no key points: it writes
// them unlocked (-1) and zero, and skips them when reading.  A file loads
// into a session whose sizes match the file's.

namespace {

struct RefEntry {
    int32_t x, y, z, ptr, offset, pad[3];
};
static_assert(sizeof(RefEntry) == 32, "the reference's __align__(16) HashEntry");
static_assert(sizeof(Voxel) == 8, "the reference's Voxel");
constexpr size_t kKeyLocks = 100000;    // KeyMap::MaxKeys (Mapping/DeviceMap.h)
constexpr size_t kKeyEntries = 500000;  // KeyMap::maxEntries = MaxKeys * nBuckets
constexpr size_t kSurfBytes = 288;      // sizeof(SURF): bool, float3, float4 (16-aligned), float[64]
constexpr int kFileChunkBlocks = 4096;  // voxel blocks per host staging chunk

struct FileCloser {
    FILE* f;
    ~FileCloser() {
        if (f) std::fclose(f);
    }
};

bool put(FILE* f, const void* p, size_t n) { return std::fwrite(p, 1, n, f) == n; }
bool get(FILE* f, void* p, size_t n) { return std::fread(p, 1, n, f) == n; }

bool put_fill(FILE* f, int32_t value, size_t count) {
    std::vector<int32_t> buf(std::min(count, (size_t)1 << 18), value);
    for (size_t done = 0; done < count;) {
        const size_t k = std::min(buf.size(), count - done);
        if (!put(f, buf.data(), k * 4)) return false;
        done += k;
    }
    return true;
}

bool skip(FILE* f, size_t bytes) {
    std::vector<char> buf(std::min(bytes, (size_t)1 << 22));
    for (size_t done = 0; done < bytes;) {
        const size_t k = std::min(buf.size(), bytes - done);
        if (!get(f, buf.data(), k)) return false;
        done += k;
    }
    return true;
}

RefEntry to_ref(const HEntry& e) {
    RefEntry r{};
    r.x = e.x;
    r.y = e.y;
    r.z = e.z;
    r.ptr = e.ptr >= 0 ? e.ptr * 512 : -1;
    r.offset = e.offset;
    return r;
}

int file_error(const char* what) {
    fb_set_error_text(what);
    return FB_EINVAL;
}

}  // namespace

extern "C" {

int fb_write_map_file(fb_session* s, const char* path) {
    if (!s || !path) return FB_EINVAL;
    const MapView& m = s->map;
    const size_t NE_all = (size_t)m.NB + m.NE;
    if ((size_t)m.NS * 512 > (size_t)INT32_MAX || NE_all > (size_t)INT32_MAX)
        return file_error("fb_write_map_file: the map is too large for the file's int sizes");
    FB_CUDA(cudaStreamSynchronize(s->stream));
    MapCounters c;
    FB_CUDA(cudaMemcpy(&c, s->ctr, sizeof c, cudaMemcpyDeviceToHost));
    FileCloser fc{std::fopen(path, "wb")};
    if (!fc.f) return file_error("fb_write_map_file: cannot open the file");
    FILE* f = fc.f;
    const int32_t head[4] = {m.NS, m.NB, m.NS * 512, (int32_t)NE_all};
    const uint32_t nvis = (uint32_t)std::max(c.n_visible, 0);
    bool ok = put(f, head, sizeof head) && put(f, &c.heap_counter, 4) && put(f, &c.entry_ptr, 4) && put(f, &nvis, 4);
    std::vector<int32_t> heap(m.NS);
    FB_CUDA(cudaMemcpy(heap.data(), m.heap, 4 * heap.size(), cudaMemcpyDeviceToHost));
    ok = ok && put(f, heap.data(), 4 * heap.size()) && put_fill(f, -1, m.NB);   // locks: EntryAvailable
    std::vector<Voxel> vox((size_t)kFileChunkBlocks * 512);
    std::vector<uint8_t> cb(m.cvox ? (size_t)kFileChunkBlocks * kCBlockBytes : 0);
    for (int b0 = 0; ok && b0 < m.NS; b0 += kFileChunkBlocks) {
        const int nb = std::min(kFileChunkBlocks, m.NS - b0);
        if (m.cvox) {
            FB_CUDA(cudaMemcpy(cb.data(), m.cvox + (size_t)b0 * kCBlockBytes, (size_t)nb * kCBlockBytes,
                               cudaMemcpyDeviceToHost));
            for (int b = 0; b < nb; ++b) {
                const uint8_t* blk = cb.data() + (size_t)b * kCBlockBytes;
                for (int v = 0; v < 512; ++v) {
                    uint16_t h;
                    std::memcpy(&h, blk + 2 * v, 2);
                    Voxel& o = vox[(size_t)b * 512 + v];
                    o.sdf = half_bits_to_float(h);
                    o.weight = blk[c_weight(v)];
                    o.r = blk[c_red(v)];
                    o.g = blk[c_green(v)];
                    o.b = blk[c_blue(v)];
                }
            }
        } else {
            FB_CUDA(cudaMemcpy(vox.data(), m.voxels + (size_t)b0 * 512, (size_t)nb * 512 * sizeof(Voxel),
                               cudaMemcpyDeviceToHost));
        }
        ok = put(f, vox.data(), (size_t)nb * 512 * sizeof(Voxel));
    }
    std::vector<HEntry> ent(NE_all);
    FB_CUDA(cudaMemcpy(ent.data(), m.entries, sizeof(HEntry) * NE_all, cudaMemcpyDeviceToHost));
    std::vector<RefEntry> ref(NE_all);
    for (size_t i = 0; i < NE_all; ++i) ref[i] = to_ref(ent[i]);
    ok = ok && put(f, ref.data(), sizeof(RefEntry) * NE_all);
    // the visible-entry list, the rest of its array zero
    const size_t nv = std::min<size_t>(nvis, (size_t)m.NS);
    std::vector<HEntry> vis(nv);
    if (nv) FB_CUDA(cudaMemcpy(vis.data(), m.vis_blocks, sizeof(HEntry) * nv, cudaMemcpyDeviceToHost));
    std::fill(ref.begin(), ref.end(), RefEntry{});
    for (size_t i = 0; i < nv; ++i) ref[i] = to_ref(vis[i]);
    ok = ok && put(f, ref.data(), sizeof(RefEntry) * NE_all);
    ok = ok && put_fill(f, -1, kKeyLocks) && put_fill(f, 0, kKeyEntries * kSurfBytes / 4);
    if (!ok || std::fflush(f) != 0) return file_error("fb_write_map_file: write failed");
    return FB_OK;
}

int fb_read_map_file(fb_session* s, const char* path) {
    if (!s || !path) return FB_EINVAL;
    const MapView& m = s->map;
    const size_t NE_all = (size_t)m.NB + m.NE;
    FileCloser fc{std::fopen(path, "rb")};
    if (!fc.f) return file_error("fb_read_map_file: cannot open the file");
    FILE* f = fc.f;
    int32_t head[4], hc, ep;
    uint32_t nvis;
    if (!get(f, head, sizeof head) || !get(f, &hc, 4) || !get(f, &ep, 4) || !get(f, &nvis, 4))
        return file_error("fb_read_map_file: truncated header");
    if (head[0] != m.NS || head[1] != m.NB || (int64_t)head[2] != (int64_t)m.NS * 512 || (size_t)head[3] != NE_all)
        return file_error("fb_read_map_file: the file's map sizes differ from the session's");
    std::vector<int32_t> heap(m.NS);
    if (!get(f, heap.data(), 4 * heap.size()) || !skip(f, 4 * (size_t)m.NB))
        return file_error("fb_read_map_file: truncated file");
    for (int32_t v : heap)
        if (v < -1 || v >= m.NS) return file_error("fb_read_map_file: free-block stack out of range");
    // reset first: the per-frame scratch and anything not in the file
    FB_CUDA(cudaStreamSynchronize(s->stream));
    launch_map_reset(s->map, s->stream);
    if (check_launch()) return FB_ECUDA;
    FB_CUDA(cudaStreamSynchronize(s->stream));
    FB_CUDA(cudaMemcpy(m.heap, heap.data(), 4 * heap.size(), cudaMemcpyHostToDevice));
    std::vector<Voxel> vox((size_t)kFileChunkBlocks * 512);
    std::vector<uint8_t> cb(m.cvox ? (size_t)kFileChunkBlocks * kCBlockBytes : 0);
    for (int b0 = 0; b0 < m.NS; b0 += kFileChunkBlocks) {
        const int nb = std::min(kFileChunkBlocks, m.NS - b0);
        if (!get(f, vox.data(), (size_t)nb * 512 * sizeof(Voxel))) return file_error("fb_read_map_file: truncated voxels");
        if (m.cvox) {
            // precision form: TSDF rounded to FP16, weight and colour as stored
            for (int b = 0; b < nb; ++b) {
                uint8_t* blk = cb.data() + (size_t)b * kCBlockBytes;
                for (int v = 0; v < 512; ++v) {
                    const Voxel& x = vox[(size_t)b * 512 + v];
                    const __half h = __float2half_rn(x.sdf);
                    std::memcpy(blk + 2 * v, &h, 2);
                    blk[c_weight(v)] = x.weight;
                    blk[c_red(v)] = x.r;
                    blk[c_green(v)] = x.g;
                    blk[c_blue(v)] = x.b;
                }
            }
            FB_CUDA(cudaMemcpy(m.cvox + (size_t)b0 * kCBlockBytes, cb.data(), (size_t)nb * kCBlockBytes,
                               cudaMemcpyHostToDevice));
        } else {
            FB_CUDA(cudaMemcpy(m.voxels + (size_t)b0 * 512, vox.data(), (size_t)nb * 512 * sizeof(Voxel),
                               cudaMemcpyHostToDevice));
        }
    }
    std::vector<RefEntry> ref(NE_all);
    if (!get(f, ref.data(), sizeof(RefEntry) * NE_all)) return file_error("fb_read_map_file: truncated hash table");
    std::vector<HEntry> ent(NE_all);
    std::vector<std::pair<int, int>> alloc;   // (block, slot)
    int holes = 0;
    for (size_t i = 0; i < NE_all; ++i) {
        const RefEntry& r = ref[i];
        if (r.ptr != -1 && (r.ptr < 0 || r.ptr % 512 || r.ptr / 512 >= m.NS))
            return file_error("fb_read_map_file: hash entry with a bad voxel pointer");
        if (r.offset > m.NE) return file_error("fb_read_map_file: hash entry with a bad link");
        HEntry& e = ent[i];
        if (r.ptr >= 0) {
            if (r.x < -32767 || r.x > 32767 || r.y < -32767 || r.y > 32767 || r.z < -32767 || r.z > 32767)
                return file_error("fb_read_map_file: block coordinates beyond +-32767");
            e.x = (short)r.x;
            e.y = (short)r.y;
            e.z = (short)r.z;
            alloc.push_back({r.ptr / 512, (int)i});
        } else {
            const bool fits = r.x >= -32767 && r.x <= 32767 && r.y >= -32767 && r.y <= 32767 && r.z >= -32767 &&
                              r.z <= 32767;
            e.x = fits ? (short)r.x : 0;
            e.y = fits ? (short)r.y : 0;
            e.z = fits ? (short)r.z : 0;
            // an empty slot a chain passes through -- a bucket head with a
            // link or a used excess slot -- means the pool ran out once
            const bool linked_head = i < (size_t)m.NB && r.offset > 0;
            const bool used_excess = i >= (size_t)m.NB && i < (size_t)m.NB + (size_t)std::max(0, ep - 1);
            if (linked_head || used_excess) holes = 1;
        }
        e.pad = 0;
        e.ptr = r.ptr >= 0 ? r.ptr / 512 : -1;
        e.offset = std::max(r.offset, 0);   // the reference ends a chain at any offset <= 0
    }
    if (alloc.size() > (size_t)m.NS) return file_error("fb_read_map_file: more allocated entries than blocks");
    FB_CUDA(cudaMemcpy(m.entries, ent.data(), sizeof(HEntry) * NE_all, cudaMemcpyHostToDevice));
    // the allocated list in block order (this library allocates blocks in
    // list order, so its own maps come back in their original order)
    std::sort(alloc.begin(), alloc.end());
    std::vector<int> alloc_slots(alloc.size());
    for (size_t i = 0; i < alloc.size(); ++i) alloc_slots[i] = alloc[i].second;
    if (!alloc_slots.empty())
        FB_CUDA(cudaMemcpy(m.alloc_list, alloc_slots.data(), 4 * alloc_slots.size(), cudaMemcpyHostToDevice));
    // the visible list: the entries' slots found through the hash chains
    if (nvis > NE_all) return file_error("fb_read_map_file: visible count out of range");
    if (!get(f, ref.data(), sizeof(RefEntry) * NE_all)) return file_error("fb_read_map_file: truncated visible list");
    std::vector<int> vis_slots;
    std::vector<HEntry> vis_entries;
    for (uint32_t i = 0; i < nvis && vis_slots.size() < (size_t)m.NS; ++i) {
        const RefEntry& r = ref[i];
        size_t b = bucket_of(r.x, r.y, r.z, (uint32_t)m.NB);
        for (int guard = 0; guard <= m.NE; ++guard) {
            const HEntry& e = ent[b];
            if (e.ptr >= 0 && e.x == r.x && e.y == r.y && e.z == r.z) {
                vis_slots.push_back((int)b);
                vis_entries.push_back(e);
                break;
            }
            if (e.offset <= 0) break;
            b = (size_t)m.NB + e.offset - 1;
        }
    }
    if (!vis_slots.empty()) {
        FB_CUDA(cudaMemcpy(m.visible, vis_slots.data(), 4 * vis_slots.size(), cudaMemcpyHostToDevice));
        FB_CUDA(cudaMemcpy(m.vis_blocks, vis_entries.data(), sizeof(HEntry) * vis_entries.size(),
                           cudaMemcpyHostToDevice));
    }
    if (!skip(f, 4 * kKeyLocks + kKeyEntries * kSurfBytes)) return file_error("fb_read_map_file: truncated key map");
    MapCounters c;
    FB_CUDA(cudaMemcpy(&c, s->ctr, sizeof c, cudaMemcpyDeviceToHost));
    c.heap_counter = hc;
    c.entry_ptr = ep;
    c.holes = holes;
    c.n_alloc = (int)alloc_slots.size();
    c.n_visible = (int)vis_slots.size();
    c.err = 0;
    FB_CUDA(cudaMemcpy(s->ctr, &c, sizeof c, cudaMemcpyHostToDevice));
    // System::ReadMapFromDisk: the tracker restarts and the map is no longer fused
    s->state = s->last_state = 1;
    if (!s->mapping_disabled) drop_graphs(s);
    s->mapping_disabled = true;
    return FB_OK;
}

}  // extern "C"
