// rzk_guided.cu - LightSlice-guided path tracing (VirtualPointLight::guided_path_trace /
// trace_wellington with METRO_RANDOM, vpl.cc:907-1040): at every surface vertex, direct
// light from FirstBounce::radiance (first_bounce.h:54-71, AreaLight::first_bounce,
// area_light.cc:48-142: one light sample and one BRDF sample, balance heuristic), then one
// continuation direction drawn with probability 1/2 from the BRDF or from LightSlice's
// Jensen map of the nearest valid slice, weighted by the balance heuristic against the
// other technique and by 2 for the one-sample choice.
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

template <int STRIDE>
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
        else brdf = guide_sample_at(G, r, m, slice, g, wi, pdf);
        if (!(pdf > 0.0f)) { value = radiance; break; }
        Ray ray = make_ray(r.p, wi);
        HitGeo h;
        if (!trace_closest(s, ray, stk, h)) { value = radiance; break; }
        if (h.light >= 0) { value = radiance; break; }   // no double count of direct light
        float other;
        if (is_brdf) {
            other = guide_pdf_at(G, r, slice, wi);
        } else {
            float rho_d = 0.0f, rho_s = 0.0f;
            if (m.type != RZK_BSDF_LAMBERTIAN) rho_terms(m, rho_d, rho_s);
            other = brdf_pdf(m, r.uvn, r.wo, wi, rho_d, rho_s);
        }
        Vertex &v = vx[depth++];
        v.radiance = radiance;
        v.brdf = brdf;
        v.weight = pdf / (pdf + other);
        v.cos = fabsf(dot(wi, r.ns));
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
    if (trace_closest(s, ray, stk, h)) L = trace_path(s, G, P, to_recv(h, ray), h.light, g, stk);
    paths[3 * path] = L.r;
    paths[3 * path + 1] = L.g;
    paths[3 * path + 2] = L.b;
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
        (q.rr_depth > 0 && !(q.rr_prob > 0.0f && q.rr_prob <= 1.0f)) || cam->width <= 0 || cam->height <= 0)
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
    float *paths = d_paths;
    if (!paths) {   // per-path radiance in the context's scratch
        r = ensure_scratch(ctx, sizeof(float) * 3 * (size_t)n_paths);
        if (r != RZK_OK) return r;
        paths = (float *)ctx->d_partial;
    }
    guided_kernel<<<(unsigned)((n_paths + kPtBlock - 1) / kPtBlock), kPtBlock, 0, st>>>(scene->dev(), G, P, paths);
    RZK_CUDA_TRY(cudaGetLastError());
    guided_mean_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(paths, (int)n, q.spp, d_rgb);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

}  // extern "C"
