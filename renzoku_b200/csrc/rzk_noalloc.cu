// rzk_noalloc.cu - the gather for callers that must not allocate device memory.
//
// Some callers cannot let a library call cudaMalloc: a host application whose device
// memory is owned by another framework's allocator or held to a fixed budget, or a frame
// loop where an allocation (which can synchronise the device and can fail mid-frame) is
// not acceptable.  rzk_gather_noalloc serves them: its only scratch - the per-chunk
// partial sums of the gather and the work counter of the persistent kernel - lives in
// the fixed array below, which every GPU that loads the library holds until the process
// exits.  The caller still passes the scene, the inputs and the output buffer.
#include "rzk_internal.cuh"

#include <algorithm>

namespace rzk {
rzk_status launch_gather_scratch(const DevScene &s, const rzk_receiver *recv, int n_recv, int img_w,
                                 const rzk_vpl *vpls, int n_vpl, int mode, float tau, float scale,
                                 float *out, int n_chunks, float *partial, int *work, cudaStream_t st);
}  // namespace rzk

using namespace rzk;

// Scratch of rzk_gather_noalloc: 256 bytes for the work counter, then the partial sums.
static __device__ __align__(256) unsigned char g_noalloc_scratch[RZK_NOALLOC_SCRATCH_BYTES];

namespace {
// Device address of g_noalloc_scratch per device.  In host code the array's name is only
// a host-side stand-in, so its device address is looked up once per device, with that
// device current, on the first call there.
void *g_scratch_addr[64] = {nullptr};
}  // namespace

extern "C" rzk_status rzk_gather_noalloc(rzk_scene *scene, const rzk_receiver *d_recv, int n_recv,
                                         int image_width, const rzk_vpl *d_vpls, int n_vpl, int clamp_mode,
                                         float tau, float scale, float *d_rgb, void *stream) {
    if (!scene || n_recv < 0 || n_vpl < 0 || image_width < 0) return RZK_ERR_INVALID;
    if (n_recv > 0 && (!d_recv || !d_rgb || ((uintptr_t)d_recv & 15u))) return RZK_ERR_INVALID;
    if (n_vpl > 0 && (!d_vpls || ((uintptr_t)d_vpls & 15u))) return RZK_ERR_INVALID;
    if (clamp_mode < RZK_CLAMP_NONE || clamp_mode > RZK_CLAMP_RADIANCE) return RZK_ERR_INVALID;
    // the partial sums of one VPL chunk must fit: n_recv x 3 floats
    const size_t room = (size_t)RZK_NOALLOC_SCRATCH_BYTES - 256;
    const size_t per_chunk = sizeof(float) * 3 * (size_t)n_recv;
    if (per_chunk > room) return RZK_ERR_CAPACITY;
    if (n_recv == 0) return RZK_OK;
    int dev = 0;
    RZK_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return RZK_ERR_UNSUPPORTED;
    if (!g_scratch_addr[dev]) {
        void *ptr = nullptr;
        RZK_CUDA_TRY(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        g_scratch_addr[dev] = ptr;
    }
    char *base = (char *)g_scratch_addr[dev];
    int *work = (int *)base;
    float *partial = (float *)(base + 256);
    // as many VPL chunks as fit (at most 32, at least 128 VPLs each): more chunks balance
    // the persistent kernel better; the chunk count only changes the summation order
    int max_chunks = (int)std::min<size_t>(32, room / per_chunk);
    int n_chunks = std::max(1, std::min(max_chunks, (n_vpl + 127) / 128));
    cudaStream_t st = (cudaStream_t)stream;
    // the array keeps the previous call's contents: the work counter must start at zero;
    // every partial sum is overwritten by the kernel
    RZK_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int), st));
    return launch_gather_scratch(scene->dev(), d_recv, n_recv, image_width, d_vpls, n_vpl, clamp_mode, tau,
                                 scale, d_rgb, n_chunks, partial, work, st);
}
