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

// Queries on rays the caller constructed (the reference's Ray fields, its own interval):
// the caller's ray is used as stored.  Any-hit walks the any-hit tree (same answer, see
// rzk_sah.cu); closest-hit walks the reference tree in the reference's visit order, which
// decides ties.
__global__ void __launch_bounds__(kTraceBlock) ray_query_kernel(DevScene s, const int *perm, const rzk_ray *rays,
                                                                int n, int closest, rzk_ray_hit *out) {
    __shared__ int stack_mem[STACK_CAP * kTraceBlock];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Stack<kTraceBlock> stk;
    stk.init(stack_mem + threadIdx.x);
    const rzk_ray &q = rays[i];
    Ray r;
    r.o = ld3(q.o);
    r.d = ld3(q.d);
    r.inv_d = ld3(q.inv_d);
    r.org_inv_d = ld3(q.org_inv_d);
    rzk_ray_hit h{0, 0.0f, 0.0f, 0.0f, -1, {0, 0, 0}};
    if (closest) {
        float t, b, g;
        const int slot = closest_hit<kTraceBlock>(s, r, q.tmin, q.tmax, stk, &t, &b, &g);
        if (slot >= 0) {
            h.hit = 1;
            h.t = t;
            h.beta = b;
            h.gamma = g;
            h.tri = perm[slot];
        }
    } else {
        h.hit = any_hit<kTraceBlock, false, true>(s, r, q.tmin, q.tmax, stk) ? 1 : 0;
    }
    out[i] = h;
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

rzk_status launch_ray_query(const DevScene &s, const int *perm, const rzk_ray *rays, int n, int closest,
                            rzk_ray_hit *out, cudaStream_t st) {
    if (n <= 0) return RZK_OK;
    ray_query_kernel<<<(n + kTraceBlock - 1) / kTraceBlock, kTraceBlock, 0, st>>>(s, perm, rays, n, closest, out);
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
