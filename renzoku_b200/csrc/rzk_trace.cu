// rzk_trace.cu - batched visibility and closest-hit queries (the Aggregate interface).
#include "rzk_traverse.cuh"

namespace rzk {

namespace {

constexpr int kTraceBlock = 128;

// Aggregate::hit(p, q, tmin, time) (aggregate.cc:84-90): Ray(p, q - p) over
// [tmin, |q - p| - tmin].
__global__ void __launch_bounds__(kTraceBlock) occluded_kernel(DevScene s, const float *p,
                                                               const float *q, int n,
                                                               uint8_t *out) {
    __shared__ int stack_mem[STACK_CAP * kTraceBlock];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Stack<kTraceBlock> stk;
    stk.init(stack_mem + threadIdx.x);
    V3 a = ld3(p + 3 * i), b = ld3(q + 3 * i);
    Ray r = make_ray(a, sub(b, a));
    float tmax = len(sub(b, a)) - s.tmin;
    out[i] = any_hit<kTraceBlock, false, true>(s, r, s.tmin, tmax, stk) ? 1 : 0;
}

__global__ void __launch_bounds__(kTraceBlock) closest_kernel(DevScene s, const float *o,
                                                              const float *d, int n, float *t_out,
                                                              rzk_receiver *recv) {
    __shared__ int stack_mem[STACK_CAP * kTraceBlock];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Stack<kTraceBlock> stk;
    stk.init(stack_mem + threadIdx.x);
    Ray r = make_ray(ld3(o + 3 * i), ld3(d + 3 * i));
    float t, b, g;
    int slot = closest_hit<kTraceBlock>(s, r, s.tmin, RAY_TMAX, stk, &t, &b, &g);
    if (slot < 0) {
        if (t_out) t_out[i] = -1.0f;
        if (recv) write_miss(recv + i);
        return;
    }
    if (t_out) t_out[i] = t;
    if (recv) {
        HitGeo h;
        fill_hit(s, r, slot, t, b, g, h);
        write_receiver(h, r, recv + i);
    }
}

// One thread per pixel; a block covers an 16 x 8 pixel tile so that a warp's primary
// rays are spatially coherent.
__global__ void __launch_bounds__(kTraceBlock) primary_kernel(DevScene s, rzk_camera cam,
                                                              rzk_receiver *out) {
    __shared__ int stack_mem[STACK_CAP * kTraceBlock];
    int j = blockIdx.x * 16 + (threadIdx.x & 15);
    int i = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (i >= cam.height || j >= cam.width) return;
    Stack<kTraceBlock> stk;
    stk.init(stack_mem + threadIdx.x);
    Ray r = camera_ray(cam, i, j);
    float t, b, g;
    rzk_receiver *o = out + (size_t)i * cam.width + j;
    int slot = closest_hit<kTraceBlock>(s, r, s.tmin, RAY_TMAX, stk, &t, &b, &g);
    if (slot < 0) { write_miss(o); return; }
    HitGeo h;
    fill_hit(s, r, slot, t, b, g, h);
    write_receiver(h, r, o);
}

}  // namespace

rzk_status launch_occluded(const DevScene &s, const float *p, const float *q, int n, uint8_t *out,
                           cudaStream_t st) {
    if (n <= 0) return RZK_OK;
    occluded_kernel<<<(n + kTraceBlock - 1) / kTraceBlock, kTraceBlock, 0, st>>>(s, p, q, n, out);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

rzk_status launch_closest(const DevScene &s, const float *o, const float *d, int n, float *t,
                          rzk_receiver *recv, cudaStream_t st) {
    if (n <= 0) return RZK_OK;
    closest_kernel<<<(n + kTraceBlock - 1) / kTraceBlock, kTraceBlock, 0, st>>>(s, o, d, n, t, recv);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

rzk_status launch_primary(const DevScene &s, const rzk_camera &cam, rzk_receiver *out,
                          cudaStream_t st) {
    if (cam.width <= 0 || cam.height <= 0) return RZK_OK;
    dim3 grid((cam.width + 15) / 16, (cam.height + 7) / 8);
    primary_kernel<<<grid, kTraceBlock, 0, st>>>(s, cam, out);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

}  // namespace rzk
