// fb_rgb_step_static: the photometric normal equations of fb_rgb_step with the
// scratch memory taken from a fixed device array inside this library instead
// of a buffer the caller allocates.
//
// Who needs it: callers that cannot allocate device memory at the point where
// they track a frame.  Code that records into a CUDA graph may not call
// cudaMalloc while its stream is being captured; a frame loop with a latency
// budget cannot afford cudaFree, which waits for the whole device; and some
// host applications hand all device memory to their own allocator and give
// plug-ins none.  Such callers pass only their images and get the same sums.
//
// The array is g_rgb_scratch below: kStaticScratchBytes (1.25 MiB), enough
// for images of up to kStaticMaxPixels pixels (640 x 480).  Every GPU that
// loads the library reserves it until the process exits.  Host code cannot use
// the array's name as a device address, so the first call on each device looks
// the address up with cudaGetSymbolAddress while that device is current and
// keeps it; make that first call outside any stream capture.  All calls on a
// device share the one array, and it keeps the contents of the last call: the
// completion counters the kernels need at zero are cleared at every call, and
// two calls whose work overlaps on the GPU (different streams, or host threads
// without ordering) corrupt each other's sums.
#include <mutex>

#include "../../include/fusion_b200.h"
#include "fb_internal.h"

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
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FB_ECUDA;
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

int image_ok(const fb_image* im, size_t elem) {
    return im && im->data && im->cols > 0 && im->rows > 0 && im->pitch >= elem * (size_t)im->cols &&
           im->pitch % elem == 0;
}

DevPose pose_of(const float R[9], const float Rinv[9], const float t[3]) {
    DevPose p;
    p.R.r0 = {R[0], R[1], R[2]};
    p.R.r1 = {R[3], R[4], R[5]};
    p.R.r2 = {R[6], R[7], R[8]};
    p.Rinv.r0 = {Rinv[0], Rinv[1], Rinv[2]};
    p.Rinv.r1 = {Rinv[3], Rinv[4], Rinv[5]};
    p.Rinv.r2 = {Rinv[6], Rinv[7], Rinv[8]};
    p.t = {t[0], t[1], t[2]};
    p.pad = 0;
    return p;
}

}  // namespace

extern "C" {

size_t fb_rgb_step_static_max_pixels(void) { return kStaticMaxPixels; }

int fb_rgb_step_static(const fb_image* gcurr, const fb_image* glast, const fb_image* vcurr, const fb_image* vlast,
                       const fb_image* dx, const fb_image* dy, const float Rcurr[9], const float RcurrInv[9],
                       const float Rlast[9], const float RlastInv[9], const float tcurr[3], const float tlast[3],
                       const float K[4], float residual[2], double A[36], double b[6], void* stream) {
    if (!image_ok(gcurr, 1) || !image_ok(glast, 1) || !image_ok(vcurr, 16) || !image_ok(vlast, 16) ||
        !image_ok(dx, 2) || !image_ok(dy, 2))
        return FB_EINVAL;
    if (!Rcurr || !RcurrInv || !Rlast || !RlastInv || !tcurr || !tlast || !K || !residual || !A || !b)
        return FB_EINVAL;
    const int W = gcurr->cols, H = gcurr->rows;
    if (glast->cols != W || glast->rows != H || vcurr->cols != W || vcurr->rows != H || vlast->cols != W ||
        vlast->rows != H || dx->cols != W || dy->cols != W || dx->rows != H || dy->rows != H ||
        gcurr->pitch != glast->pitch || vcurr->pitch != vlast->pitch || dx->pitch != dy->pitch)
        return FB_EINVAL;
    if ((size_t)W * H > kStaticMaxPixels) {
        fb_set_error_text("fb_rgb_step_static: image larger than the static scratch (at most 307200 pixels)");
        return FB_EINVAL;
    }
    void* base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    unsigned char* p = (unsigned char*)base;
    float* partials = (float*)p;
    unsigned int* tickets = (unsigned int*)(p + kOffTickets);
    double* out = (double*)(p + kOffOut);
    int* res = (int*)(p + kOffResidual);
    cudaStream_t st = (cudaStream_t)stream;
    TrackLevel L{};
    L.W = W;
    L.H = H;
    L.vp = (int)(vcurr->pitch / 16);
    L.gp = (int)gcurr->pitch;
    L.sp = (int)(dx->pitch / 2);
    L.k.fx = K[0];
    L.k.fy = K[1];
    L.k.cx = K[2];
    L.k.cy = K[3];
    L.k.invfx = (float)(1.0 / (double)K[0]);
    L.k.invfy = (float)(1.0 / (double)K[1]);
    L.vcurr = (const float4*)vcurr->data;
    L.vlast = (const float4*)vlast->data;
    L.gcurr = (const uint8_t*)gcurr->data;
    L.glast = (const uint8_t*)glast->data;
    L.dx = (const int16_t*)dx->data;
    L.dy = (const int16_t*)dy->data;
    // the completion counters must start at zero; everything else in the
    // array is overwritten by the kernels before it is read
    cudaError_t e = cudaMemsetAsync(tickets, 0, 16, st);
    if (e != cudaSuccess) {
        fb_set_error_text(cudaGetErrorString(e));
        return FB_ECUDA;
    }
    launch_step_rgb(L, pose_of(Rcurr, RcurrInv, tcurr), pose_of(Rlast, RlastInv, tlast), partials, tickets, res,
                    out, st);
    e = cudaGetLastError();
    double host[32];
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, out, sizeof host, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        fb_set_error_text(cudaGetErrorString(e));
        return FB_ECUDA;
    }
    int n = 0;
    for (int i = 0; i < 6; ++i)
        for (int j = i; j < 7; ++j) {
            double v = (double)(float)host[n++];   // the reference's sums are floats
            if (j == 6)
                b[i] = v;
            else
                A[j * 6 + i] = A[i * 6 + j] = v;
        }
    residual[0] = (float)host[27];
    residual[1] = (float)host[28];
    return FB_OK;
}

}  // extern "C"
