// rzk_noalloc.cu - the gather for callers that must not allocate device memory.
//
// Some callers cannot let a library call cudaMalloc: a host application whose device
// memory is owned by another framework's allocator or held to a fixed budget, or a frame
// loop where an allocation (which can synchronise the device and can fail mid-frame) is
// not acceptable.  rzk_gather_noalloc serves them: its only scratch - the per-chunk
// partial sums of the gather, the work counter of the persistent kernel and, when they fit
// beside the partial sums, the spatially ordered VPL copy and its sort scratch - lives in
// the fixed array below, which every GPU that loads the library holds until the process
// exits.  The caller still passes the scene, the inputs and the output buffer.
#include "rzk_internal.cuh"

#include <algorithm>
#include <mutex>

namespace rzk {
rzk_status launch_gather_scratch(const DevScene &s, const rzk_receiver *recv, int n_recv, int img_w,
                                 const rzk_vpl *vpls, int n_vpl, int mode, float tau, float scale,
                                 float *out, int n_chunks, float *partial, int *work, cudaStream_t st);
}  // namespace rzk

using namespace rzk;

// Scratch of rzk_gather_noalloc: [work counter (256 B) | partial sums | ordered VPLs | sort
// scratch].
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
    // the partial sums of one VPL chunk must fit: n_recv x 3 floats
    const size_t room = (size_t)RZK_NOALLOC_SCRATCH_BYTES - 256;
    const size_t per_chunk = up256(sizeof(float) * 3 * (size_t)n_recv);
    if (per_chunk > room) return RZK_ERR_CAPACITY;
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
    float *partial = (float *)(base + 256);
    // rzk_gather's chunking (at most 32 chunks of at least 128 VPLs) where its partial sums
    // fit; with more than one chunk the VPLs are first put in rzk_gather's spatial order
    // (Hilbert-curve index of their cells, stable) when the ordered copy and its sort
    // scratch fit beside two chunks' partial sums, so that the result is rzk_gather's bit
    // for bit whenever rzk_gather's chunk count fits.  Otherwise fewer chunks (or the
    // caller's VPL order) change only the float summation order.
    const int want_chunks = std::max(1, std::min(32, (n_vpl + 127) / 128));
    const size_t order_bytes = up256(sizeof(rzk_vpl) * (size_t)n_vpl) + order_scratch_bytes(n_vpl);
    bool ordered = want_chunks > 1 && order_bytes + 2 * per_chunk <= room;
    int n_chunks = (int)std::min<size_t>((size_t)want_chunks, (room - (ordered ? order_bytes : 0)) / per_chunk);
    if (n_chunks <= 1) {
        n_chunks = 1;
        ordered = false;
    }
    cudaStream_t st = (cudaStream_t)stream;
    // the array keeps the previous call's contents: the work counter must start at zero,
    // and the partial sums are cleared so that no earlier call's values can reach the image
    // even if a work item gives up (a bounded wait timing out, reported in the context's
    // error word)
    RZK_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int), st));
    RZK_CUDA_TRY(cudaMemsetAsync(partial, 0, per_chunk * (size_t)n_chunks, st));
    const rzk_vpl *vpls = d_vpls;
    if (ordered) {
        char *ob = base + 256 + per_chunk * (size_t)n_chunks;
        OrderTable t;
        order_table_init(t);
        order_table_add(t, d_vpls, n_vpl, scene->box);
        RZK_TRY(order_vpls(t, ob + up256(sizeof(rzk_vpl) * (size_t)n_vpl), (rzk_vpl *)ob, st));
        vpls = (const rzk_vpl *)ob;
    }
    // the kernel packs chunk c's partial sums at c * n_recv * 12 bytes, inside the
    // per_chunk * n_chunks bytes reserved (and cleared) before the ordered copy
    return launch_gather_scratch(scene->dev(), d_recv, n_recv, image_width, vpls, n_vpl, clamp_mode, tau,
                                 scale, d_rgb, n_chunks, partial, work, st);
}
