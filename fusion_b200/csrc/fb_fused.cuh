// Fused launches: one kernel launch that runs the same stage kernel for many
// sessions at once (the batch step of fb_batch_set_mode(b, 2)).
//
// Every frame-path kernel is written as a body that takes its block
// coordinates as an argument (BlockCtx) instead of reading blockIdx and
// gridDim.  Two kernels wrap each body:
//   - the ordinary kernel (one session), which passes its own coordinates;
//   - the fused kernel, whose 1-D grid is the concatenation of up to
//     kFusedMaxParts sessions' grids ("parts"): each block finds its part,
//     takes that part's argument tuple and runs the body with the
//     coordinates it has in that part's own grid.
// The parts and their argument tuples are the fused kernel's parameter (a
// __grid_constant__ block of at most a few KB), so a body reads its
// arguments from the constant bank as the ordinary kernel does, instead of
// holding them in registers.
// A body therefore sees exactly what it sees in a launch of its own -- the
// same arguments, blocks and grid size -- and computes the same bits.
//
// Host side: the launch helpers start kernels through fb_launch().  While a
// LaunchRecorder is installed on the calling thread, fb_launch records the
// launch (fused kernel, grid, block, argument tuple) instead of starting it;
// the batch step records every session's frame this way, merges the
// sessions' launches of the same stage, and starts each merged launch once.
#ifndef FB_FUSED_CUH
#define FB_FUSED_CUH

#include <cuda/std/tuple>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <type_traits>
#include <utility>
#include <vector>

namespace fb {

// The block coordinates a kernel body sees (x and y of blockIdx / gridDim).
struct BlockCtx {
    int bx, by, gx, gy;
};

__device__ __forceinline__ BlockCtx own_ctx() {
    return BlockCtx{(int)blockIdx.x, (int)blockIdx.y, (int)gridDim.x, (int)gridDim.y};
}

// One part of a fused launch: the blocks [start, start + gx * gy) of the
// fused 1-D grid run the part's kernel as a gx x gy grid.
struct FusedPart {
    int start, gx, gy, pad;
};

constexpr int kFusedMaxParts = 32;

// Parameter of a fused kernel: n parts (ascending start) and their argument
// tuples (type Tup, stored as bytes: kFusedMaxParts slots of sizeof(Tup)).
// Layout (host and device): parts at 0, n at 16 * kFusedMaxParts, the
// tuples from 16 * kFusedMaxParts + 16.
template <class Tup>
struct alignas(16) FusedParams {
    FusedPart parts[kFusedMaxParts];
    int n, pad[3];
    alignas(16) unsigned char args[kFusedMaxParts * sizeof(Tup)];
};

// The byte layout of FusedParams for a tuple of `tup_size` bytes.
constexpr size_t kFusedNOffset = sizeof(FusedPart) * kFusedMaxParts;
constexpr size_t kFusedArgsOffset = kFusedNOffset + 16;
constexpr size_t fused_param_bytes(size_t tup_size) {
    return (kFusedArgsOffset + kFusedMaxParts * tup_size + 15) & ~(size_t)15;
}

// The argument tuple of a kernel: its parameter types, in order.
template <class F>
struct KernelArgs;
template <class... P>
struct KernelArgs<void (*)(P...)> {
    using type = cuda::std::tuple<std::decay_t<P>...>;
};
template <class F>
using ArgsOf = typename KernelArgs<F>::type;

// Runs body(ctx, args...) for this block's part of a fused launch: the
// last part whose start is <= blockIdx.x.
template <class Tup, class Body>
__device__ __forceinline__ void run_part(const FusedParams<Tup>& fp, Body body) {
    static_assert(alignof(Tup) <= 16 && sizeof(FusedParams<Tup>) <= 32764, "fused kernel parameter");
    const int b = (int)blockIdx.x;
    int lo = 0, hi = fp.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (fp.parts[mid].start <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    const FusedPart& p = fp.parts[lo];
    const int local = b - p.start;
    const BlockCtx c{local % p.gx, local / p.gx, p.gx, p.gy};
    const Tup& t = reinterpret_cast<const Tup*>(fp.args)[lo];
    cuda::std::apply([&](const auto&... a) { body(c, a...); }, t);
}

// The fused form of kernel `single` (whose body is `body`), with the given
// launch bounds: named single##_fused.
#define FB_FUSED_KERNEL(single, body, ...)                                                                     \
    __global__ void __launch_bounds__(__VA_ARGS__)                                                             \
        single##_fused(const __grid_constant__ fb::FusedParams<fb::ArgsOf<decltype(&single)>> fp) {           \
        fb::run_part(fp, [](const fb::BlockCtx& c, const auto&... a) { body(c, a...); });                      \
    }

// ------------------------------------------------------------------ host side

// One recorded launch.
struct LaunchRec {
    uint64_t slot;          // position in the frame's canonical launch order
    const void* fused;      // the fused kernel
    dim3 grid, block;
    size_t smem;
    size_t off, size;       // the argument tuple in the recorder's bytes
};

// Records the launches of one session's frame.  slot(): the stage, pyramid
// level and iteration of the launches that follow; each launch inside one
// (stage, level, iteration) gets the next sub-slot.
struct LaunchRecorder {
    std::vector<LaunchRec> recs;
    std::vector<unsigned char> bytes;
    uint64_t base = 0;
    int sub = 0;
    void slot(int stage, int level, int iter) {
        base = (uint64_t)stage << 48 | (uint64_t)level << 40 | (uint64_t)iter << 16;
        sub = 0;
    }
    void add(const void* fused, dim3 g, dim3 b, size_t smem, const void* args, size_t size) {
        const size_t off = (bytes.size() + 15) & ~(size_t)15;
        bytes.resize(off + size);
        std::memcpy(bytes.data() + off, args, size);
        recs.push_back(LaunchRec{base | (uint64_t)sub++, fused, g, b, smem, off, size});
    }
    void clear() {
        recs.clear();
        bytes.clear();
        base = 0;
        sub = 0;
    }
};

// The recorder of the calling thread (null: launches start at once).
LaunchRecorder*& launch_recorder();

// Canonical stages of a frame, in issue order (the slot's stage field).
enum FusedStage : int {
    kSlotResize = 1,
    kSlotPyramid,
    kSlotTrackInit,
    kSlotTrack,
    kSlotAllocate,
    kSlotVisibility,
    kSlotIntegrate,
    kSlotRenderVisibility,
    kSlotZRange,
    kSlotRaycast,
    kSlotCommit,
    kSlotOut,
};

// Tags the launches that follow (no-op without a recorder).
inline void launch_slot(int stage, int level = 0, int iter = 0) {
    if (LaunchRecorder* r = launch_recorder()) r->slot(stage, level, iter);
}

// Starts kernel k on st, or records it (with its fused form) when the
// calling thread has a recorder.
template <class... P, class... A>
void fb_launch(void (*k)(P...), const void* fused, dim3 grid, dim3 block, size_t smem, cudaStream_t st,
               A&&... a) {
    if (LaunchRecorder* r = launch_recorder()) {
        const ArgsOf<void (*)(P...)> t(static_cast<std::decay_t<P>>(a)...);
        r->add(fused, grid, block, smem, &t, sizeof t);
        return;
    }
    k<<<grid, block, smem, st>>>(std::forward<A>(a)...);
}

}  // namespace fb

#endif
