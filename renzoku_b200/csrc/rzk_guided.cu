// rzk_guided.cu - LightSlice-guided path tracing (VirtualPointLight::guided_path_trace /
// trace_wellington with METRO_RANDOM, vpl.cc:907-1040): at every surface vertex, direct
// light from FirstBounce::radiance (first_bounce.h:54-71, AreaLight::first_bounce,
// area_light.cc:48-142: one light sample and one BRDF sample, balance heuristic), then one
// continuation direction drawn with probability 1/2 from the BRDF or from LightSlice's
// sampler at the nearest valid slice - its Jensen map, or its Metropolis chain over the
// slice's incoming-radiance density (the reference's default, LocalSampler::METROPOLIS,
// lightslice.cc:80) - weighted by the balance heuristic against the other technique and by
// 2 for the one-sample choice.
//
// The Metropolis chains: the reference runs one chain per slice, sequentially as pixels ask
// for samples, warming up with 1,024 states and handing out 1,024-state caches in shuffled
// order (metropolis_fetch_cached_sample, lightslice.cc:1709-1761).  Here eight chains per
// slice, one warp each, run before the paths - each with the same start (a cluster drawn from
// the slice's cluster distribution), the same 1,024-state warm-up, the same mutations
// (uniform over the hemisphere or a 9-degree cone around the current direction, each with
// probability 1/2), the same density and acceptance (lightslice.cc:1763-1911) - from the
// streams (seed, 8, slice * 8 + chain), keep their states after the warm-up in the slice's
// pool, and each path draws a state uniformly from its slice's pool.  The chains share one
// stationary distribution, so samples follow it in both; they are the same only in
// distribution.
//
// Extension beyond the reference (whose recursion runs to max_bounce): Russian roulette at
// vertices deeper than rr_depth, surviving with probability rr_prob and dividing the
// continuation by it; rr_depth = 0 turns it off.
//
// One thread per path (sample s of pixel k is path k * spp + s) drawing from the
// counter-based stream (seed, 6, path); a second kernel sums each pixel's samples in sample
// order.  The recursion is unrolled into a
// chain of vertices whose continuation terms are folded back from the deepest vertex, so
// every sum is formed in the reference's order.
#include "rzk_guide.cuh"

#include <algorithm>

namespace rzk {
namespace {

constexpr int kPtBlock = 128;
constexpr int kMaxBounce = 16;
constexpr int kChainWarmup = 1024;         // metropolis_fetch_cached_sample's num_samples
constexpr int kChainDefault = 4096;        // pool states per slice when the caller gives 0
constexpr int kChainsPerSlice = 8;         // independent chains per slice, each its own warm-up
constexpr unsigned kFull = 0xffffffffu;

struct PtParams {
    rzk_camera cam;
    int spp, max_bounce, rr_depth, direct;
    float rr_prob;
    uint32_t seed;
};

__device__ __forceinline__ float balance(float a, float b) { return a / (a + b); }   // Mis::balance

__device__ __forceinline__ GuideRecv to_recv(const HitGeo &h, const Ray &ray) {
    GuideRecv r;
    r.p = h.p;
    r.ns = h.ns;
    r.wo = neg(ray.d);
    r.uvn = h.uvn;
    r.mat = h.mat;
    return r;
}

// FirstBounce::radiance with AreaLight::first_bounce and no direction sampler
template <int STRIDE>
__device__ Rgb first_bounce(const DevScene &s, const GuideRecv &r, const rzk_material &m, Rng &g,
                            Stack<STRIDE> &stk) {
    const float u = g.uniform();
    int k = -1;
    float light_pdf = 0.0f;
    for (int i = 0; i < s.n_lights; ++i)
        if (u < s.light_cdf[i]) { k = i; light_pdf = s.light_pdf[i]; break; }
    if (k < 0) return crgb(0.0f, 0.0f, 0.0f);
    const DevLight &L = s.lights[k];
    float rho_d = 0.0f, rho_s = 0.0f;
    if (m.type != RZK_BSDF_LAMBERTIAN) rho_terms(m, rho_d, rho_s);
    Rgb Lo = crgb(0.0f, 0.0f, 0.0f);
    const V3 p = r.p, pn = r.ns;
    // a point on the light
    V3 q, qn;
    float pdf;
    light_sample_point(L, g, q, qn, pdf);
    if (pdf > 0.0f) {
        Ray sr = make_ray(p, sub(q, p));
        const float tmax = len(sub(q, p)) - s.tmin;
        if (!any_hit<STRIDE, false, true>(s, sr, s.tmin, tmax, stk)) {
            const V3 wi = unit(sub(q, p));
            const Rgb Le = light_query(L, q, qn, neg(wi));
            const float G = form_factor_abs(p, pn, q, qn);
            if (G > 0.0f) {
                const Rgb brdf = brdf_eval(m, r.uvn, r.wo, wi);
                const float dsp = brdf_pdf(m, r.uvn, r.wo, wi, rho_d, rho_s);
                const V3 pq = sub(q, p);
                const float sq = pq.x * pq.x + pq.y * pq.y + pq.z * pq.z;
                const float w1 = balance(pdf * sq / fabsf(dot(unit(sub(p, q)), qn)), dsp);
                Lo = cadd(Lo, cmul(cscl(Le, w1 * G / pdf), brdf));
            }
        }
    }
    // a direction from the BRDF that reaches this light
    V3 wi;
    float dsp;
    (void)brdf_sample(m, r.uvn, r.wo, g, wi, dsp);
    if (dsp > 0.0f) {
        Ray ray = make_ray(p, wi);
        HitGeo h;
        if (trace_closest(s, ray, stk, h) && h.light == k) {
            const V3 q2 = add(p, scl(wi, h.t));
            const V3 qn2 = h.ns;
            const Rgb Le = light_query(L, q2, qn2, neg(wi));
            const V3 pq = sub(q2, p);
            const float sq = pq.x * pq.x + pq.y * pq.y + pq.z * pq.z;
            const float lpdf = light_area_pdf(L, q2) * sq / fabsf(dot(unit(sub(p, q2)), qn2));
            const float w2 = balance(dsp, lpdf);
            const Rgb brdf = brdf_eval(m, r.uvn, r.wo, wi);
            const float cs = fabsf(dot(wi, r.ns));
            Lo = cadd(Lo, cmul(cscl(Le, w2 * cs / dsp), brdf));
        }
    }
    return cdiv(Lo, light_pdf);
}

struct Vertex {
    Rgb radiance;   // direct part
    Rgb brdf;
    float weight, cos, pdf;
    int rr;
};

template <int STRIDE, bool METRO>
__device__ Rgb trace_path(const DevScene &s, const GuideDev &G, const PtParams &P, const GuideRecv &r0,
                          int light0, Rng &g, Stack<STRIDE> &stk) {
    Vertex vx[kMaxBounce];
    GuideRecv r = r0;
    int light = light0;
    int depth = 0;     // vertices with a pending continuation
    Rgb value = crgb(0.0f, 0.0f, 0.0f);
    for (int bounce = 1;; ++bounce) {
        if (bounce > P.max_bounce) { value = crgb(0.0f, 0.0f, 0.0f); break; }
        if (light >= 0) {   // only reachable at the first vertex
            value = crgb(0.0f, 0.0f, 0.0f);
            if (bounce == 1 && P.direct) value = light_query(s.lights[light], r.p, r.ns, r.wo);
            break;
        }
        if (r.mat < 0) { value = crgb(0.0f, 0.0f, 0.0f); break; }   // a surface without a material
        const rzk_material m = *(s.mats + r.mat);
        const bool is_brdf = g.uniform() < 0.5f;
        Rgb radiance = crgb(0.0f, 0.0f, 0.0f);
        if (bounce > 1 || P.direct) radiance = first_bounce(s, r, m, g, stk);
        if (bounce >= P.max_bounce) { value = radiance; break; }
        int rr = 0;
        if (P.rr_depth > 0 && bounce > P.rr_depth) {
            if (g.uniform() >= P.rr_prob) { value = radiance; break; }
            rr = 1;
        }
        float p6[6];
        map6(r, m, G.diag, p6);
        const int slice = guide_slice(G, r, p6);   // the vertex's sampling record, found once
        V3 wi;
        float pdf;
        Rgb brdf;
        if (is_brdf) brdf = brdf_sample(m, r.uvn, r.wo, g, wi, pdf);
        else if (METRO) brdf = guide_metro_sample_at(G, r, m, slice, g, wi, pdf);
        else brdf = guide_sample_at(G, r, m, slice, g, wi, pdf);
        if (!(pdf > 0.0f)) { value = radiance; break; }
        // the vertex's MIS weight and cosine are formed before the closest-hit query (pure
        // functions of values already known, so the same numbers), which leaves the vertex's
        // receiver and material dead, not held in registers, through the traversal
        float other;
        if (is_brdf) {
            other = METRO ? guide_metro_pdf_at(G, r, slice, wi) : guide_pdf_at(G, r, slice, wi);
        } else {
            float rho_d = 0.0f, rho_s = 0.0f;
            if (m.type != RZK_BSDF_LAMBERTIAN) rho_terms(m, rho_d, rho_s);
            other = brdf_pdf(m, r.uvn, r.wo, wi, rho_d, rho_s);
        }
        const float weight = pdf / (pdf + other);
        const float cosv = fabsf(dot(wi, r.ns));
        Ray ray = make_ray(r.p, wi);
        HitGeo h;
        if (!trace_closest(s, ray, stk, h)) { value = radiance; break; }
        if (h.light >= 0) { value = radiance; break; }   // no double count of direct light
        Vertex &v = vx[depth++];
        v.radiance = radiance;
        v.brdf = brdf;
        v.weight = weight;
        v.cos = cosv;
        v.pdf = pdf;
        v.rr = rr;
        r = to_recv(h, ray);
        light = h.light;
    }
    // radiance += weight * Li * brdf * cos / pdf * 2, from the deepest vertex back
    for (int i = depth - 1; i >= 0; --i) {
        const Vertex &v = vx[i];
        Rgb t = cscl(cdiv(cscl(cmul(cscl(value, v.weight), v.brdf), v.cos), v.pdf), 2.0f);
        if (v.rr) t = cdiv(t, P.rr_prob);
        value = cadd(v.radiance, t);
    }
    return value;
}

// one thread per path: sample s of pixel k is path k * spp + s, so neighbouring threads
// share a pixel (and their first hit)
template <bool METRO>
__global__ void __launch_bounds__(kPtBlock) guided_kernel(DevScene s, GuideDev G, PtParams P, float *paths) {
    __shared__ int stack_mem[STACK_CAP * kPtBlock];
    const long long path = (long long)blockIdx.x * kPtBlock + threadIdx.x;
    const int W = P.cam.width, H = P.cam.height;
    if (path >= (long long)W * H * P.spp) return;
    Stack<kPtBlock> stk;
    stk.init(stack_mem + threadIdx.x);
    const int k = (int)(path / P.spp);
    const int i = k / W, j = k - i * W;
    Rng g;
    g.init(P.seed, 6u, (uint32_t)path);
    Ray ray = camera_ray(P.cam, i, j);
    HitGeo h;
    Rgb L = crgb(0.0f, 0.0f, 0.0f);
    if (trace_closest(s, ray, stk, h)) L = trace_path<kPtBlock, METRO>(s, G, P, to_recv(h, ray), h.light, g, stk);
    paths[3 * path] = L.r;
    paths[3 * path + 1] = L.g;
    paths[3 * path + 2] = L.b;
}

// eval_incoming_radiance of slice s at (x, y), the slice's points split over the warp's lanes
// (every lane returns the sum)
__device__ __forceinline__ float chain_density(const GuideDev &G, int s, float x, float y, int lane) {
    const float r2 = G.density_radius * G.density_radius;
    float sr = 0.0f, sg = 0.0f, sb = 0.0f;
    int x0, x1, y0, y1;
    guide_cells(G, x, y, x0, x1, y0, y1);
    const int *cell = G.m_cell + (size_t)s * (G.m_grid * G.m_grid + 1);
    for (int cy = y0; cy <= y1; ++cy) {
        for (int i = cell[cy * G.m_grid + x0] + lane, e = cell[cy * G.m_grid + x1 + 1]; i < e; i += 32) {
            const float2 q = G.m_pt[i];
            const float dx = q.x - x, dy = q.y - y;
            if (dx * dx + dy * dy < r2) {
                const float4 c = G.m_rad[i];
                sr += c.x;
                sg += c.y;
                sb += c.z;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(kFull, sr, o);
        sg += __shfl_xor_sync(kFull, sg, o);
        sb += __shfl_xor_sync(kFull, sb, o);
    }
    return 1e-2f * G.sum_f[s] + sqrtf(sr * sr + sg * sg + sb * sb);
}

// One warp per chain runs a Metropolis chain of slice blockIdx.x (LightSlice::metropolis_sample,
// lightslice.cc:1763-1911, with the constructor's settings, lightslice.cc:42-55); the slice's
// kChainsPerSlice chains (blockIdx.y) each warm up for 1,024 states and then fill their share
// of out[slice][n] in order.  Every lane draws the same numbers from the stream
// (seed, 8, slice * kChainsPerSlice + chain) and so takes the same decisions; the density is
// summed over the lanes; lane 0 stores each state: (direction, density), or with SQUARE (point
// on the record's unit square, density, 0).  A slice without a valid sampling record gets
// zeros (paths never choose it).
template <bool SQUARE>
__global__ void __launch_bounds__(32) metro_chain_kernel(GuideDev G, uint32_t seed, int n, float4 *out) {
    const int s = blockIdx.x, chain = blockIdx.y, lane = threadIdx.x;
    const int per = (n + kChainsPerSlice - 1) / kChainsPerSlice;
    const int first = min(n, chain * per), last = min(n, first + per);
    float4 *dst = out + (size_t)s * n + first;
    const int count = last - first;
    if (!G.rec_valid[s]) {
        for (int i = lane; i < count; i += 32) dst[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    const Onb rec = guide_rec_onb(G, s);
    // mutation_pdf over {UNIFORM 0.33, VPL 0, CONE_PERTURB 0.33} (DiscretePdf, pdf.cc:18-57)
    const float m_total = 0.33f + 0.0f + 0.33f;
    const float p_uniform = 0.33f / m_total, p_perturb = 0.33f / m_total;
    const float cos_max = cosf(A_PI * 0.05f);                       // perturb_cos_theta_max
    const float cone_pdf = 1.0f / (TWO_PI * (1.0f - cos_max));       // perturb_cone_pdf
    // the VPL mutation has probability 0, so both transition densities are these
    const float t_new = p_uniform * INV_2PI + p_perturb * cone_pdf;
    const float t_old = p_uniform * INV_2PI + p_perturb * cone_pdf;
    Rng g;
    g.init(seed, 8u, (uint32_t)(s * kChainsPerSlice + chain));
    // start: a cluster drawn from the slice's cluster distribution, its direction
    V3 w = mk(0.0f, 0.0f, 0.0f);
    float f = 0.0f, wx = 0.0f, wy = 0.0f;   // wx, wy: the state on the unit square
    {
        const float u = g.uniform();
        int k = -1;
        for (int i = G.c_off[s], e = G.c_off[s + 1]; i < e; ++i)
            if (u < G.c_cdf[i]) { k = i; break; }
        if (k >= 0) {
            w = mk(G.c_wi[3 * (size_t)k], G.c_wi[3 * (size_t)k + 1], G.c_wi[3 * (size_t)k + 2]);
            guide_direction_to_square(w2l(rec, w), wx, wy);
            f = chain_density(G, s, wx, wy, lane);
        }
    }
    for (int step = 1; step < kChainWarmup + count; ++step) {
        const float v = g.uniform();                  // mutation_pdf.sample: cdf {1/2, 1/2, 1}
        const float a = g.uniform(), b = g.uniform(); // Vec2::random: x then y
        V3 wi;
        if (v < p_uniform) {
            const float phi = TWO_PI * a;
            const float theta = acosf(b);
            wi = unit(guide_spherical(rec, theta, phi));
        } else {
            const float cos_theta = 1.0f - a * (1.0f - cos_max);
            const float phi = TWO_PI * b;
            const float theta = acosf(cos_theta);
            wi = guide_spherical(onb_from_n(w), theta, phi);
        }
        const V3 lw = w2l(rec, wi);
        if (lw.z > 0.0f) {   // no jump to the lower half of the hemisphere
            float sx, sy;
            guide_direction_to_square(lw, sx, sy);
            const float fn = chain_density(G, s, sx, sy, lane);
            const float acceptance = fminf(1.0f, (fn * t_old) / (f * t_new));
            const float t = g.uniform();
            if (t < acceptance) {
                w = wi;
                f = fn;
                wx = sx;
                wy = sy;
            }
        }
        if (step >= kChainWarmup && lane == 0)
            dst[step - kChainWarmup] = SQUARE ? make_float4(wx, wy, f, 0.0f) : make_float4(w.x, w.y, w.z, f);
    }
}

// eval_incoming_radiance for listed (slice, point) pairs: one thread each
__global__ void density_kernel(GuideDev G, const int32_t *slice, const float *xy, int n, float *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = slice[i];
    out[i] = (s >= 0 && s < G.n_slices) ? guide_density(G, s, xy[2 * i], xy[2 * i + 1]) : 0.0f;
}

// the pixel's mean: its samples summed in sample order, divided by spp
__global__ void guided_mean_kernel(const float *paths, int n_pix, int spp, float *out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_pix) return;
    Rgb sum = crgb(0.0f, 0.0f, 0.0f);
    for (int smp = 0; smp < spp; ++smp) {
        const float *q = paths + 3 * ((size_t)k * spp + smp);
        sum = cadd(sum, crgb(q[0], q[1], q[2]));
    }
    const Rgb avg = cdiv(sum, (float)spp);
    out[3 * (size_t)k] = avg.r;
    out[3 * (size_t)k + 1] = avg.g;
    out[3 * (size_t)k + 2] = avg.b;
}

}  // namespace
}  // namespace rzk

using namespace rzk;

extern "C" {

rzk_status rzk_guided_render(rzk_context *ctx, rzk_scene *scene, rzk_lightslice *ls, const rzk_camera *cam,
                             const rzk_guided_params *params, float *d_rgb, float *d_paths, void *stream) {
    if (!ctx || !scene || !ls || !cam || !params || !d_rgb) return RZK_ERR_INVALID;
    const rzk_guided_params &q = *params;
    if (q.spp <= 0 || q.max_bounce < 1 || q.max_bounce > kMaxBounce || q.rr_depth < 0 ||
        (q.rr_depth > 0 && !(q.rr_prob > 0.0f && q.rr_prob <= 1.0f)) || cam->width <= 0 || cam->height <= 0 ||
        (q.sampler != RZK_GUIDE_JENSEN && q.sampler != RZK_GUIDE_METROPOLIS) || q.chain_samples < 0 ||
        q.chain_samples > (1 << 24))
        return RZK_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    GuideDev G;
    rzk_status r = guide_tables(ls, &G, st);
    if (r != RZK_OK) return r;
    PtParams P;
    P.cam = *cam;
    P.spp = q.spp;
    P.max_bounce = q.max_bounce;
    P.rr_depth = q.rr_depth;
    P.rr_prob = q.rr_prob;
    P.direct = q.direct_lighting ? 1 : 0;
    P.seed = q.seed;
    const long long n = (long long)cam->width * cam->height;
    const long long n_paths = n * q.spp;
    if (n_paths > (1LL << 31)) return RZK_ERR_CAPACITY;
    // context scratch: the chains' pools (METROPOLIS), then the per-path radiance (without d_paths)
    const bool metro = q.sampler == RZK_GUIDE_METROPOLIS;
    const int pool_n = q.chain_samples > 0 ? q.chain_samples : kChainDefault;
    const size_t pool_bytes = metro ? sizeof(float4) * (size_t)G.n_slices * pool_n : 0;
    r = ensure_scratch(ctx, pool_bytes + (d_paths ? 0 : sizeof(float) * 3 * (size_t)n_paths));
    if (r != RZK_OK) return r;
    float *paths = d_paths ? d_paths : (float *)((char *)ctx->d_partial + pool_bytes);
    const unsigned blocks = (unsigned)((n_paths + kPtBlock - 1) / kPtBlock);
    if (metro) {
        G.pool = (const float4 *)ctx->d_partial;
        G.pool_n = pool_n;
        if (G.n_slices > 0)
            metro_chain_kernel<false><<<dim3(G.n_slices, kChainsPerSlice), 32, 0, st>>>(G, q.seed, pool_n,
                                                                                      (float4 *)ctx->d_partial);
        RZK_CUDA_TRY(cudaGetLastError());
        guided_kernel<true><<<blocks, kPtBlock, 0, st>>>(scene->dev(), G, P, paths);
    } else {
        guided_kernel<false><<<blocks, kPtBlock, 0, st>>>(scene->dev(), G, P, paths);
    }
    RZK_CUDA_TRY(cudaGetLastError());
    guided_mean_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(paths, (int)n, q.spp, d_rgb);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

rzk_status rzk_lightslice_density(rzk_lightslice *ls, const int32_t *d_slice, const float *d_xy, int n, float *d_out,
                                  void *stream) {
    if (!ls || n < 0 || (n > 0 && (!d_slice || !d_xy || !d_out))) return RZK_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    GuideDev G;
    rzk_status r = guide_tables(ls, &G, st);
    if (r != RZK_OK) return r;
    if (n == 0) return RZK_OK;
    density_kernel<<<(n + 255) / 256, 256, 0, st>>>(G, d_slice, d_xy, n, d_out);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

rzk_status rzk_lightslice_chains(rzk_lightslice *ls, uint32_t seed, int n_samples, float *d_out, void *stream) {
    if (!ls || n_samples <= 0 || n_samples > (1 << 24) || !d_out) return RZK_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    GuideDev G;
    rzk_status r = guide_tables(ls, &G, st);
    if (r != RZK_OK) return r;
    if (G.n_slices == 0) return RZK_OK;
    metro_chain_kernel<true><<<dim3(G.n_slices, kChainsPerSlice), 32, 0, st>>>(G, seed, n_samples, (float4 *)d_out);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

}  // extern "C"
