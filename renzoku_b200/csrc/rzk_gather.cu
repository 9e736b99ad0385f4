// rzk_gather.cu - the VPL gather: per (shading point, VPL) pair, shadow-ray visibility
// through the LBVH, geometry term, both BRDFs and the clamp
// (VirtualPointLight::gather_point, vpl.cc:661-688), summed per shading point.
//
// Layout: a CTA owns BLOCK consecutive receivers (one per thread, loaded once into
// registers) and one contiguous chunk of VPLs.  The chunk streams through shared memory
// in TILE-VPL tiles, double-buffered, each tile one bulk copy (cp.async.bulk, no
// multicast) completing on an mbarrier.  Every thread walks the tile in VPL order; the
// shading term is evaluated first and the shadow ray is traced only when it is non-zero
// (a zero term contributes zero whatever the visibility, so the sum is unchanged).
// Per-thread sums are written per chunk and a second kernel adds the chunks in chunk
// order, so the image does not depend on scheduling; with one chunk the summation order
// is exactly the reference's (VPL order, single precision).
#include "rzk_traverse.cuh"

#include <algorithm>

namespace rzk {

namespace {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Bounded wait on a bulk-copy barrier: gives up after ~2^24 polls and reports it.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t *err) {
    for (uint32_t it = 0; it < (1u << 24); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicOr(err, ERR_TIMEOUT);
    return false;
}

struct RecvRegs {
    V3 p, ng, ns, wo;
    Onb uvn;
    int mat;
};

__device__ __forceinline__ RecvRegs load_receiver(const rzk_receiver *r) {
    const float4 *q = reinterpret_cast<const float4 *>(r);
    float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3), e = __ldg(q + 4),
           f = __ldg(q + 5);
    RecvRegs o;
    o.p = mk(a.x, a.y, a.z);
    o.ng = mk(a.w, b.x, b.y);
    o.ns = mk(b.z, b.w, c.x);
    o.wo = mk(c.y, c.z, c.w);
    o.uvn.u = mk(d.x, d.y, d.z);
    o.uvn.v = mk(d.w, e.x, e.y);
    o.uvn.n = mk(e.z, e.w, f.x);
    o.mat = __float_as_int(f.y);
    return o;
}

__device__ __forceinline__ rzk_material load_material(const rzk_material *m) {
    const float4 *q = reinterpret_cast<const float4 *>(m);
    float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
    rzk_material o;
    o.type = __float_as_int(a.x);
    o.kd[0] = a.y; o.kd[1] = a.z; o.kd[2] = a.w;
    o.ks[0] = b.x; o.ks[1] = b.y; o.ks[2] = b.z;
    o.p0 = b.w; o.p1 = c.x;
    o.pad[0] = o.pad[1] = o.pad[2] = 0.0f;
    return o;
}

// The shading part of gather_point after its visibility test (vpl.cc:676-687);
// pn is the receiver's shading normal (LocalGeometry::n, local_geometry.h:52-56).
__device__ __forceinline__ Rgb shade(const DevScene &s, const RecvRegs &r, const rzk_material &rm,
                                     const rzk_vpl &l, int mode, float tau, V3 &q) {
    q = ld3(l.p);
    float G = form_factor_abs(r.p, r.ns, q, ld3(l.n));
    V3 wi = unit(sub(q, r.p));
    Rgb sb = brdf_eval(rm, r.uvn, r.wo, wi);
    Rgb lb;
    if (l.mat >= 0) {
        rzk_material lm = load_material(s.mats + l.mat);
        Onb lu{ld3(l.u), ld3(l.v), ld3(l.nn)};
        lb = brdf_eval(lm, lu, ld3(l.wi), neg(wi));
    } else {
        lb = crgb(1.0f, 1.0f, 1.0f);
    }
    return radiance_terms(crgb(l.contrib[0], l.contrib[1], l.contrib[2]), sb, lb, G, mode, tau);
}

template <int BLOCK, int TILE>
__global__ void __launch_bounds__(BLOCK) gather_kernel(DevScene s, const rzk_receiver *recv, int n_recv,
                                                       const rzk_vpl *vpls, int n_vpl, int chunk_len,
                                                       int mode, float tau, float *partial) {
    __shared__ __align__(128) rzk_vpl tile[2][TILE];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int stack_mem[STACK_CAP * BLOCK];
    __shared__ int abort_flag;

    const int t = threadIdx.x;
    const int ri = blockIdx.x * BLOCK + t;
    const int chunk = blockIdx.y;
    const int j0 = chunk * chunk_len;
    const int j1 = min(n_vpl, j0 + chunk_len);
    const int n_tiles = j1 > j0 ? (j1 - j0 + TILE - 1) / TILE : 0;

    RecvRegs r;
    bool active = false;
    rzk_material rm;
    if (ri < n_recv) {
        r = load_receiver(recv + ri);
        active = r.mat >= 0;
        if (active) rm = load_material(s.mats + r.mat);
    }
    Stack<BLOCK> stk;
    stk.init(stack_mem + t);

    if (t == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        abort_flag = 0;
        fence_barrier_init();
    }
    __syncthreads();
    if (t == 0 && n_tiles > 0) {
        int cnt = min(TILE, j1 - j0);
        mbar_expect_tx(&bar[0], cnt * (uint32_t)sizeof(rzk_vpl));
        bulk_g2s(&tile[0][0], vpls + j0, cnt * (uint32_t)sizeof(rzk_vpl), &bar[0]);
    }

    Rgb sum = crgb(0.0f, 0.0f, 0.0f);
    for (int k = 0; k < n_tiles; ++k) {
        const int buf = k & 1;
        if (t == 0 && k + 1 < n_tiles) {
            int jn = j0 + (k + 1) * TILE;
            int cnt = min(TILE, j1 - jn);
            fence_proxy_async();
            mbar_expect_tx(&bar[buf ^ 1], cnt * (uint32_t)sizeof(rzk_vpl));
            bulk_g2s(&tile[buf ^ 1][0], vpls + jn, cnt * (uint32_t)sizeof(rzk_vpl), &bar[buf ^ 1]);
        }
        if (!mbar_wait_bounded(&bar[buf], (k >> 1) & 1, s.err)) abort_flag = 1;
        const int cnt = min(TILE, j1 - (j0 + k * TILE));
        if (active && !abort_flag) {
            for (int v = 0; v < cnt; ++v) {
                const rzk_vpl &l = tile[buf][v];
                V3 q;
                Rgb L = shade(s, r, rm, l, mode, tau, q);
                if (cblack(L)) continue;
                Ray ray = make_ray(r.p, sub(q, r.p));
                float tmax = len(sub(q, r.p)) - s.tmin;
                if (any_hit<BLOCK, false>(s, ray, s.tmin, tmax, stk)) continue;
                sum = cadd(sum, L);
            }
        }
        __syncthreads();
        if (abort_flag) break;
    }
    if (ri < n_recv) {
        float *o = partial + 3 * ((size_t)chunk * n_recv + ri);
        o[0] = sum.r; o[1] = sum.g; o[2] = sum.b;
    }
}

__global__ void reduce_chunks_kernel(const float *partial, int n_recv, int n_chunks, float scale,
                                     float *out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * n_recv) return;
    float acc = partial[i];
    for (int c = 1; c < n_chunks; ++c) acc += partial[(size_t)c * 3 * n_recv + i];
    out[i] = acc * scale;
}

// LightTransportMatrix::fill: every pair, visibility always traced.
constexpr int kMatBlock = 128;
__global__ void __launch_bounds__(kMatBlock) matrix_kernel(DevScene s, const rzk_receiver *recv,
                                                           int n_recv, const rzk_vpl *vpls, int n_vpl,
                                                           int mode, float tau, float *mat,
                                                           uint8_t *vis, int incident) {
    __shared__ int stack_mem[STACK_CAP * kMatBlock];
    const int ri = blockIdx.x * kMatBlock + threadIdx.x;
    if (ri >= n_recv) return;
    Stack<kMatBlock> stk;
    stk.init(stack_mem + threadIdx.x);
    RecvRegs r = load_receiver(recv + ri);
    for (int j = blockIdx.y; j < n_vpl; j += gridDim.y) {
    rzk_vpl l = vpls[j];
    Rgb L = crgb(0.0f, 0.0f, 0.0f);
    bool visible = false;
    if (incident) {
        // VirtualPointLight::incident_radiance (vpl.cc:411-440): geometric normal, no
        // visibility, surface BRDF white.
        V3 q = ld3(l.p);
        float G = form_factor_abs(r.p, r.ng, q, ld3(l.n));
        V3 wi = unit(sub(q, r.p));
        Rgb lb = crgb(1.0f, 1.0f, 1.0f);
        if (l.mat >= 0) {
            rzk_material lm = load_material(s.mats + l.mat);
            Onb lu{ld3(l.u), ld3(l.v), ld3(l.nn)};
            lb = brdf_eval(lm, lu, ld3(l.wi), neg(wi));
        }
        L = radiance_terms(crgb(l.contrib[0], l.contrib[1], l.contrib[2]), crgb(1.0f, 1.0f, 1.0f),
                           lb, G, mode, tau);
    } else if (r.mat >= 0) {
        V3 q = ld3(l.p);
        Ray ray = make_ray(r.p, sub(q, r.p));
        float tmax = len(sub(q, r.p)) - s.tmin;
        if (!any_hit<kMatBlock, false>(s, ray, s.tmin, tmax, stk)) {
            visible = true;
            rzk_material rm = load_material(s.mats + r.mat);
            L = shade(s, r, rm, l, mode, tau, q);
        }
    }
    size_t k = (size_t)j * n_recv + ri;
    mat[3 * k] = L.r; mat[3 * k + 1] = L.g; mat[3 * k + 2] = L.b;
    if (vis) vis[k] = visible ? 1 : 0;
    }
}

// Seeded pairs for the "0.1 x mean contribution" clamp base; block partials in double.
constexpr int kMeanBlock = 128;
__global__ void __launch_bounds__(kMeanBlock) mean_kernel(DevScene s, const rzk_receiver *recv,
                                                          int n_recv, const rzk_vpl *vpls, int n_vpl,
                                                          uint32_t seed, int n_pairs, double *block_sums) {
    __shared__ int stack_mem[STACK_CAP * kMeanBlock];
    __shared__ double red[kMeanBlock];
    const int k = blockIdx.x * kMeanBlock + threadIdx.x;
    double val = 0.0;
    if (k < n_pairs) {
        uint4 blk = philox4x32_10(make_uint4(0u, (uint32_t)k, 3u, 0x52454e5au), seed, 0x4b5a4f52u);
        int ri = (int)(blk.x % (uint32_t)n_recv);
        int vi = (int)(blk.y % (uint32_t)n_vpl);
        RecvRegs r = load_receiver(recv + ri);
        if (r.mat >= 0) {
            Stack<kMeanBlock> stk;
            stk.init(stack_mem + threadIdx.x);
            rzk_vpl l = vpls[vi];
            V3 q = ld3(l.p);
            Ray ray = make_ray(r.p, sub(q, r.p));
            float tmax = len(sub(q, r.p)) - s.tmin;
            if (!any_hit<kMeanBlock, false>(s, ray, s.tmin, tmax, stk)) {
                rzk_material rm = load_material(s.mats + r.mat);
                Rgb L = shade(s, r, rm, l, RZK_CLAMP_NONE, 0.0f, q);
                val = (double)cval(L);
            }
        }
    }
    red[threadIdx.x] = val;
    __syncthreads();
    for (int w = kMeanBlock / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) block_sums[blockIdx.x] = red[0];
}

__global__ void mean_final_kernel(const double *block_sums, int nb, int n_pairs, double *out) {
    if (threadIdx.x != 0) return;
    double acc = 0.0;
    for (int b = 0; b < nb; ++b) acc += block_sums[b];
    *out = n_pairs > 0 ? acc / n_pairs : 0.0;
}

}  // namespace

// Tile configurations compiled in; the autotuner picks one per workload.
struct GatherVariant {
    int block, tile;
};
static const GatherVariant kVariants[] = {{128, 64}, {128, 32}, {64, 64}, {64, 128}};

int gather_variant_count() { return (int)(sizeof(kVariants) / sizeof(kVariants[0])); }

rzk_status launch_gather(rzk_context *ctx, const DevScene &s, const rzk_receiver *recv, int n_recv,
                         const rzk_vpl *vpls, int n_vpl, int mode, float tau, float scale,
                         float *out, int variant, int n_chunks, cudaStream_t st) {
    if (n_recv <= 0) return RZK_OK;
    if (variant < 0 || variant >= gather_variant_count()) variant = 0;
    const GatherVariant gv = kVariants[variant];
    const int rb = (n_recv + gv.block - 1) / gv.block;
    const int max_chunks = std::max(1, (n_vpl + gv.tile - 1) / gv.tile);
    if (n_chunks <= 0) {
        int sms = 148;
        int target = 8 * sms;
        n_chunks = std::max(1, std::min(max_chunks, (target + rb - 1) / rb));
    }
    n_chunks = std::min(std::min(n_chunks, max_chunks), 65535);
    if (n_vpl <= 0) n_chunks = 1;
    // chunk boundaries are multiples of 128 VPLs whatever the variant's tile, so every
    // variant sums the same VPLs in the same order for a given n_chunks
    int chunk_len = n_vpl > 0 ? (n_vpl + n_chunks - 1) / n_chunks : 0;
    chunk_len = (chunk_len + 127) / 128 * 128;
    if (chunk_len > 0) n_chunks = (n_vpl + chunk_len - 1) / chunk_len;
    size_t need = sizeof(float) * 3 * (size_t)n_recv * n_chunks;
    if (need > ctx->partial_bytes) {
        if (ctx->d_partial) cudaFree(ctx->d_partial);
        ctx->d_partial = nullptr;
        ctx->partial_bytes = 0;
        RZK_CUDA_TRY(cudaMalloc((void **)&ctx->d_partial, need));
        ctx->partial_bytes = need;
    }
    dim3 grid(rb, n_chunks);
    switch (variant) {
        case 0: gather_kernel<128, 64><<<grid, 128, 0, st>>>(s, recv, n_recv, vpls, n_vpl, chunk_len, mode, tau, ctx->d_partial); break;
        case 1: gather_kernel<128, 32><<<grid, 128, 0, st>>>(s, recv, n_recv, vpls, n_vpl, chunk_len, mode, tau, ctx->d_partial); break;
        case 2: gather_kernel<64, 64><<<grid, 64, 0, st>>>(s, recv, n_recv, vpls, n_vpl, chunk_len, mode, tau, ctx->d_partial); break;
        default: gather_kernel<64, 128><<<grid, 64, 0, st>>>(s, recv, n_recv, vpls, n_vpl, chunk_len, mode, tau, ctx->d_partial); break;
    }
    RZK_CUDA_TRY(cudaGetLastError());
    reduce_chunks_kernel<<<(3 * n_recv + 255) / 256, 256, 0, st>>>(ctx->d_partial, n_recv, n_chunks,
                                                                   scale, out);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

rzk_status launch_matrix(const DevScene &s, const rzk_receiver *recv, int n_recv, const rzk_vpl *vpls,
                         int n_vpl, int mode, float tau, float *mat, uint8_t *vis, bool incident,
                         cudaStream_t st) {
    if (n_recv <= 0 || n_vpl <= 0) return RZK_OK;
    dim3 grid((n_recv + kMatBlock - 1) / kMatBlock, std::min(n_vpl, 65535));
    matrix_kernel<<<grid, kMatBlock, 0, st>>>(s, recv, n_recv, vpls, n_vpl, mode, tau, mat, vis,
                                              incident ? 1 : 0);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

rzk_status launch_mean(rzk_context *ctx, const DevScene &s, const rzk_receiver *recv, int n_recv,
                       const rzk_vpl *vpls, int n_vpl, uint32_t seed, int n_pairs, double *h_mean,
                       cudaStream_t st) {
    if (n_pairs <= 0 || n_recv <= 0 || n_vpl <= 0) { *h_mean = 0.0; return RZK_OK; }
    int nb = (n_pairs + kMeanBlock - 1) / kMeanBlock;
    double *buf = nullptr;
    RZK_CUDA_TRY(cudaMalloc((void **)&buf, sizeof(double) * (nb + 1)));
    mean_kernel<<<nb, kMeanBlock, 0, st>>>(s, recv, n_recv, vpls, n_vpl, seed, n_pairs, buf + 1);
    mean_final_kernel<<<1, 32, 0, st>>>(buf + 1, nb, n_pairs, buf);
    cudaError_t e = cudaMemcpyAsync(h_mean, buf, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(buf);
    if (e != cudaSuccess) { set_last_cuda_error(e, "mean", __FILE__, __LINE__); return RZK_ERR_CUDA; }
    (void)ctx;
    return RZK_OK;
}

}  // namespace rzk
