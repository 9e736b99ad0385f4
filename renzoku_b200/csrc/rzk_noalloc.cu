// rzk_noalloc.cu - the gather for callers that must not allocate device memory.
//
// Some callers cannot let a library call cudaMalloc: a host application whose device
// memory is owned by another framework's allocator or held to a fixed budget, or a frame
// loop where an allocation (which can synchronise the device and can fail mid-frame) is
// not acceptable.  rzk_gather_noalloc serves them: its only scratch - the work counter of
// the persistent kernel, the spatially ordered VPL copy with its sort scratch (when it
// fits) and the per-chunk partial sums of one band of receivers at a time - lives in the
// fixed array below, which every GPU that loads the library holds until the process exits.
// The caller still passes the scene, the inputs and the output buffer.
#include "rzk_internal.cuh"

#include <algorithm>
#include <mutex>

namespace rzk {
rzk_status launch_gather_scratch(const DevScene &s, const rzk_receiver *recv, int n_recv, int img_w,
                                 const rzk_vpl *vpls, int n_vpl, int mode, float tau, float scale,
                                 float *out, int n_chunks, float *partial, int *work, cudaStream_t st);
}  // namespace rzk

using namespace rzk;

// Scratch of rzk_gather_noalloc: [work counter (256 B) | ordered VPLs | sort scratch |
// partial sums of one band].
static __device__ __align__(256) unsigned char g_noalloc_scratch[RZK_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;

// Device address of g_noalloc_scratch per device.  In host code the array's name is only a
// host-side stand-in, so its device address is looked up once per device, with that device
// current, by the first call there (std::call_once: concurrent first calls from several
// host threads wait for the one lookup).
struct ScratchAddr {
    std::once_flag once;
    void *ptr = nullptr;
    cudaError_t err = cudaSuccess;
};
ScratchAddr g_scratch[kMaxDevices];

size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

extern "C" rzk_status rzk_gather_noalloc(rzk_scene *scene, const rzk_receiver *d_recv, int n_recv,
                                         int image_width, const rzk_vpl *d_vpls, int n_vpl, int clamp_mode,
                                         float tau, float scale, float *d_rgb, void *stream) {
    if (!scene || !scene->ctx || n_recv < 0 || n_vpl < 0 || image_width < 0) return RZK_ERR_INVALID;
    if (n_recv > 0 && (!d_recv || !d_rgb || ((uintptr_t)d_recv & 15u))) return RZK_ERR_INVALID;
    if (n_vpl > 0 && (!d_vpls || ((uintptr_t)d_vpls & 15u))) return RZK_ERR_INVALID;
    if (clamp_mode < RZK_CLAMP_NONE || clamp_mode > RZK_CLAMP_RADIANCE) return RZK_ERR_INVALID;
    // The receivers are gathered in bands of whole warp-tile rows (4 image rows, or 32
    // receivers without an image width), one band after another on the stream, so that
    // the partial sums of one band - not of the whole image - must fit.  The smallest band
    // must fit with one chunk.
    const size_t room = (size_t)RZK_NOALLOC_SCRATCH_BYTES - 256;
    const long long unit = image_width > 0 ? 4LL * image_width : 32LL;
    const long long min_band = std::min<long long>(unit, n_recv);
    const size_t plane = sizeof(float) * 3;   // bytes of one receiver in one chunk's partial sums
    if (plane * (size_t)min_band > room) return RZK_ERR_CAPACITY;
    if (n_recv == 0) return RZK_OK;
    int dev = 0;
    RZK_CUDA_TRY(cudaGetDevice(&dev));
    // the scene's arrays live on its context's device; kernels launched on another device
    // would read them through peer mappings or fault
    if (dev != scene->ctx->device) return RZK_ERR_INVALID;
    if (dev < 0 || dev >= kMaxDevices) return RZK_ERR_UNSUPPORTED;
    ScratchAddr &sa = g_scratch[dev];
    std::call_once(sa.once, [&sa] { sa.err = cudaGetSymbolAddress(&sa.ptr, g_noalloc_scratch); });
    if (sa.err != cudaSuccess || !sa.ptr) {
        set_last_cuda_error(sa.err, "cudaGetSymbolAddress", __FILE__, __LINE__);
        return RZK_ERR_CUDA;
    }
    char *base = (char *)sa.ptr;
    int *work = (int *)base;
    // rzk_gather's chunking (at most 32 chunks of at least 128 VPLs).  With more than one
    // chunk the VPLs are first put in rzk_gather's spatial order (Hilbert-curve index of
    // their cells, stable) when the ordered copy and its sort scratch fit beside the
    // smallest band's partial sums: the image is then rzk_gather's bit for bit, since a
    // receiver's sum depends only on the chunking and the VPL order, never on the band.
    // Otherwise the caller's VPL order (and, for image rows too wide for 32 chunks, fewer
    // chunks) change only the float summation order.
    const int want_chunks = std::max(1, std::min(32, (n_vpl + 127) / 128));
    const size_t order_bytes = up256(sizeof(rzk_vpl) * (size_t)n_vpl) + order_scratch_bytes(n_vpl);
    int n_chunks = want_chunks;
    bool ordered = false;
    size_t avail = room;
    if (want_chunks > 1) {
        if (order_bytes + plane * (size_t)want_chunks * (size_t)min_band <= room) {
            ordered = true;
            avail = room - order_bytes;
        } else {
            n_chunks = (int)std::max<size_t>(1, std::min<size_t>(want_chunks, room / (plane * (size_t)min_band)));
        }
    }
    // the most whole units whose n_chunks partial planes fit (at least the smallest band,
    // which fits by the choices above)
    long long band = (long long)(avail / (plane * (size_t)n_chunks * (size_t)unit)) * unit;
    band = std::max(band, min_band);
    cudaStream_t st = (cudaStream_t)stream;
    // layout: [work counter | ordered VPLs + sort scratch | partial sums of one band]
    float *partial = (float *)(base + 256 + (ordered ? order_bytes : 0));
    const rzk_vpl *vpls = d_vpls;
    if (ordered) {
        char *ob = base + 256;
        OrderTable t;
        order_table_init(t);
        order_table_add(t, d_vpls, n_vpl, scene->box);
        RZK_TRY(order_vpls(t, ob + up256(sizeof(rzk_vpl) * (size_t)n_vpl), (rzk_vpl *)ob, st));
        vpls = (const rzk_vpl *)ob;
    }
    for (long long r0 = 0; r0 < n_recv; r0 += band) {
        const int nb = (int)std::min<long long>(band, n_recv - r0);
        // the array keeps the previous band's and call's contents: the work counter must
        // start at zero, and the partial sums are cleared so that no earlier values can
        // reach the image even if a work item gives up (a bounded wait timing out, reported
        // in the context's error word)
        RZK_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int), st));
        RZK_CUDA_TRY(cudaMemsetAsync(partial, 0, plane * (size_t)nb * (size_t)n_chunks, st));
        // a band starts on a warp-tile row, so its tiles are the whole image's tiles; the
        // kernel packs chunk c's partial sums at c * nb * 12 bytes
        RZK_TRY(launch_gather_scratch(scene->dev(), d_recv + r0, nb, image_width, vpls, n_vpl, clamp_mode, tau,
                                      scale, d_rgb + 3 * r0, n_chunks, partial, work, st));
    }
    return RZK_OK;
}
