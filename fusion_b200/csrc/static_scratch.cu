// fb_rgb_step_static: the photometric normal equations of fb_rgb_step with the
// scratch memory taken from a fixed device array inside this library instead
// of a buffer the caller allocates.
//
// Who needs it: callers that cannot allocate device memory at the point where
// they track a frame.  A frame loop with a latency budget cannot afford
// cudaFree, which waits for the whole device; and some host applications hand
// all device memory to their own allocator and give plug-ins none.  Such
// callers pass only their images and get the same sums.
//
// The array is g_rgb_scratch below: kStaticScratchBytes (1.25 MiB), enough
// for images of up to kStaticMaxPixels pixels (640 x 480).  Every GPU that
// loads the library reserves it until the process exits.  Host code cannot use
// the array's name as a device address, so the first call on each device looks
// the address up with cudaGetSymbolAddress while that device is current and
// keeps it; that first call should come before any stream capture.  All calls
// on a device share the one array, and it keeps the contents of the last call:
// the completion counters the kernels need at zero are cleared at every call,
// and two calls whose work overlaps on the GPU (different streams, or host
// threads without ordering) corrupt each other's sums.  The call is
// synchronous: it returns once the sums have reached the host.
#include <mutex>

#include "session_internal.h"

using namespace fb;

namespace {

constexpr size_t kStaticMaxPixels = 640 * 480;
// partials (kTrackMaxBlocks x 32 floats) | completion counters (256 B) |
// output sums (32 doubles) | one correspondence per pixel
constexpr size_t kOffTickets = (size_t)kTrackMaxBlocks * 32 * 4;
constexpr size_t kOffOut = kOffTickets + 256;
constexpr size_t kOffResidual = kOffOut + 32 * 8;
constexpr size_t kStaticScratchBytes = kOffResidual + kStaticMaxPixels * 4;

static __device__ __align__(256) unsigned char g_rgb_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_lock;
void* g_addr[kMaxDevices] = {};

// Device address of g_rgb_scratch on the current device (looked up once).
int scratch_address(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        fb_set_error_text("fb_rgb_step_static: no current device, or a device index of 64 or more");
        return FB_ECUDA;
    }
    std::lock_guard<std::mutex> guard(g_lock);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_rgb_scratch);
        if (e != cudaSuccess || !p) {
            fb_set_error_text(e != cudaSuccess ? cudaGetErrorString(e) : "no address for the static scratch");
            return FB_ECUDA;
        }
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return FB_OK;
}

}  // namespace

extern "C" {

size_t fb_rgb_step_static_max_pixels(void) { return kStaticMaxPixels; }

int fb_rgb_step_static(const fb_image* gcurr, const fb_image* glast, const fb_image* vcurr, const fb_image* vlast,
                       const fb_image* dx, const fb_image* dy, const float Rcurr[9], const float RcurrInv[9],
                       const float Rlast[9], const float RlastInv[9], const float tcurr[3], const float tlast[3],
                       const float K[4], float residual[2], double A[36], double b[6], void* stream) {
    int rc = rgb_step_check(gcurr, glast, vcurr, vlast, dx, dy, Rcurr, RcurrInv, Rlast, RlastInv, tcurr, tlast, K,
                            residual, A, b);
    if (rc) return rc;
    if ((size_t)gcurr->cols * gcurr->rows > kStaticMaxPixels) {
        fb_set_error_text("fb_rgb_step_static: image larger than the static scratch (at most 307200 pixels)");
        return FB_EINVAL;
    }
    void* base = nullptr;
    rc = scratch_address(&base);
    if (rc) return rc;
    unsigned char* p = (unsigned char*)base;
    StepScratch sc;
    sc.partials = (float*)p;
    sc.tickets = (unsigned int*)(p + kOffTickets);
    sc.out = (double*)(p + kOffOut);
    sc.residual = (int*)(p + kOffResidual);
    return rgb_step_run(gcurr, glast, vcurr, vlast, dx, dy, Rcurr, RcurrInv, Rlast, RlastInv, tcurr, tlast, K, sc,
                        residual, A, b, (cudaStream_t)stream);
}

}  // extern "C"
