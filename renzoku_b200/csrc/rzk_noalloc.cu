// rzk_noalloc.cu - the gather for callers that must not allocate device memory.
//
// Some callers cannot let a library call cudaMalloc: a host application whose device
// memory is owned by another framework's allocator or held to a fixed budget, or a frame
// loop where an allocation (which can synchronise the device and can fail mid-frame) is
// not acceptable.  rzk_gather_noalloc serves them: its only scratch - the work counter of
// the persistent kernel, the spatially ordered VPL copy with its sort scratch (when it
// fits) and the chunk ring in which the kernel sums each tile's chunks - lives in the fixed
// array below, which every GPU that loads the library holds until the process exits.  The
// caller still passes the scene, the inputs and the output buffer.
#include "rzk_internal.cuh"

#include <algorithm>
#include <mutex>

namespace rzk {
rzk_status launch_gather_scratch(const DevScene &s, const rzk_receiver *recv, int n_recv, int img_w,
                                 const rzk_vpl *vpls, int n_vpl, int mode, float tau, float scale,
                                 float *out, int n_chunks, void *ring_mem, size_t ring_mem_bytes, int *work,
                                 cudaStream_t st);
}  // namespace rzk

using namespace rzk;

// Scratch of rzk_gather_noalloc: [work counter (256 B) | ordered VPLs | sort scratch |
// chunk ring].
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
    const size_t room = (size_t)RZK_NOALLOC_SCRATCH_BYTES - 256;
    // rzk_gather's chunking (at most 32 chunks of at least 128 VPLs) and chunk ring: the
    // persistent kernel sums each 8 x 4 tile's chunks in chunk order as soon as the tile's
    // last chunk is written, so the scratch holds the chunk sums of a window of tiles (a
    // ring of slots), not of the image.  With more than one chunk the VPLs are first put in
    // rzk_gather's spatial order (Hilbert-curve index of their cells, stable) when the
    // ordered copy and its sort scratch leave room for a ring of at least 512 tiles (or all
    // of the image's): the image is then rzk_gather's bit for bit, since a receiver's sum
    // depends only on the chunking and the VPL order, never on the ring.  Otherwise the
    // caller's VPL order changes only the float summation order.
    const int n_chunks = std::max(1, std::min(32, (n_vpl + 127) / 128));
    const long long wtiles = image_width > 0
                                 ? (long long)((image_width + 7) / 8) *
                                       ((((long long)n_recv + image_width - 1) / image_width + 3) / 4)
                                 : ((long long)n_recv + 31) / 32;
    const size_t order_bytes = up256(sizeof(rzk_vpl) * (size_t)n_vpl) + order_scratch_bytes(n_vpl);
    const bool ordered = n_chunks > 1 && order_bytes < room &&
                         ring_slots_fitting(room - order_bytes, n_chunks) >= std::min<long long>(wtiles, 512);
    const size_t ring_room = room - (ordered ? order_bytes : 0);
    if (ring_slots_fitting(ring_room, n_chunks) < 1) return RZK_ERR_CAPACITY;
    cudaStream_t st = (cudaStream_t)stream;
    // layout: [work counter | ordered VPLs + sort scratch | chunk ring]
    const rzk_vpl *vpls = d_vpls;
    if (ordered) {
        char *ob = base + 256;
        OrderTable t;
        order_table_init(t);
        order_table_add(t, d_vpls, n_vpl, scene->box);
        RZK_TRY(order_vpls(t, ob + up256(sizeof(rzk_vpl) * (size_t)n_vpl), (rzk_vpl *)ob, st));
        vpls = (const rzk_vpl *)ob;
    }
    // the array keeps the previous call's contents: the launcher zeroes the work counter and
    // the ring's counters; every chunk sum is written before the tile's sum reads it
    return launch_gather_scratch(scene->dev(), d_recv, n_recv, image_width, vpls, n_vpl, clamp_mode, tau, scale,
                                 d_rgb, n_chunks, base + 256 + (ordered ? order_bytes : 0), ring_room, work, st);
}
