// rzk_vplgen.cu - VPL generation, one thread per light particle
// (VplGenerator::generate_vpl / trace_vpl, vpl_generator.cc:43-181;
// SubpathGenerator::sample_direct_vertex, path.cc:171-334; AreaLight::sample,
// area_light.cc:27-46; Material::sample, lambertian.cc:5-26, phong.cc:21-72,
// ward.cc:26-99).
//
// Particle k draws from the counter-based stream (seed, 0, k), so its path does not
// depend on how many particles run or in which order.  Each particle writes up to
// max_bounce - 1 VPLs into its own slots; an exclusive scan of the per-particle counts
// then compacts them into the reference's push order (particle-major, bounce-minor).
#include "rzk_sample.cuh"

namespace rzk {

namespace {

constexpr int kGenBlock = 128;

__device__ __forceinline__ void store_vpl(rzk_vpl *o, const HitGeo &h, V3 wi, Rgb c, int bounce, int path) {
    float w[24];
    st3(w + 0, h.p); st3(w + 3, h.ns); st3(w + 6, h.uvn.u); st3(w + 9, h.uvn.v);
    st3(w + 12, h.uvn.n); st3(w + 15, wi);
    w[18] = c.r; w[19] = c.g; w[20] = c.b;
    w[21] = __int_as_float(h.mat); w[22] = __int_as_float(bounce); w[23] = __int_as_float(path);
    float4 *dst = reinterpret_cast<float4 *>(o);
#pragma unroll
    for (int k = 0; k < 6; ++k) dst[k] = make_float4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
}

__global__ void __launch_bounds__(kGenBlock) vplgen_kernel(DevScene s, uint32_t seed, int n_particles,
                                                           int max_bounce, int per, rzk_vpl *slots,
                                                           int *counts) {
    __shared__ int stack_mem[STACK_CAP * kGenBlock];
    const int k = blockIdx.x * kGenBlock + threadIdx.x;
    if (k >= n_particles) return;
    Stack<kGenBlock> stk;
    stk.init(stack_mem + threadIdx.x);
    rzk_vpl *out = slots + (size_t)k * per;
    int n = 0;
    counts[k] = 0;
    if (s.n_lights == 0) return;
    Rng g;
    g.init(seed, 0u, (uint32_t)k);
    // sample_direct_vertex: Vec2 sample.random(rd) -> light choice on x (scene.cc:205-209)
    float sx = g.uniform();
    (void)g.uniform();
    int li = -1;
    float light_pdf = 0.0f;
    for (int i = 0; i < s.n_lights; ++i)
        if (sx < s.light_cdf[i]) { li = i; light_pdf = s.light_pdf[i]; break; }
    if (li < 0) return;
    const DevLight &L = s.lights[li];
    // AreaLight::sample -> Surface::sample -> Quad::sample / Triangle::sample
    int which = 0;
    float pdf_sel = 1.0f;
    if (L.kind == RZK_PRIM_QUAD) {
        float t = g.uniform();
        if (t <= L.t0_ratio) { which = 0; pdf_sel = L.t0_ratio; }
        else { which = 1; pdf_sel = 1.0f - L.t0_ratio; }
    }
    V3 tp0 = mk(L.p0[which].x, L.p0[which].y, L.p0[which].z);
    V3 tp1 = mk(L.p1[which].x, L.p1[which].y, L.p1[which].z);
    V3 tp2 = mk(L.p2[which].x, L.p2[which].y, L.p2[which].z);
    float u0 = g.uniform(), u1 = g.uniform();
    float tmp = sqrtf(1.0f - u0);
    float b = 1.0f - tmp;
    float c = u1 * tmp;
    float a = 1.0f - b - c;
    V3 q = add(add(scl(tp0, a), scl(tp1, b)), scl(tp2, c));
    V3 qn = mk(L.n[which].x, L.n[which].y, L.n[which].z);
    float pdf_t = 1.0f / L.n[which].w;
    float pdf_q = L.kind == RZK_PRIM_QUAD ? pdf_sel * pdf_t : pdf_t;
    if (L.flags & RZK_SURF_FLIPPED) qn = neg(qn);
    float cx = g.uniform(), cy = g.uniform();
    float phi = TWO_PI * cx;
    float sin_theta = sqrtf(cy);
    float x = sin_theta * cosf(phi);
    float y = sin_theta * sinf(phi);
    float z = sqrtf(1.f - sin_theta * sin_theta);
    Onb luvn = onb_from_nu(mk(L.basis_n.x, L.basis_n.y, L.basis_n.z), mk(L.basis_u.x, L.basis_u.y, L.basis_u.z));
    V3 wo_q = unit(l2w(luvn, mk(x, y, z)));
    Rgb Le = crgb(L.emit.x, L.emit.y, L.emit.z);
    float pdf_wo = z * INV_PI;
    if (pdf_q <= 0.0f || pdf_wo <= 0.0f) return;
    float acc_pdf = light_pdf;
    acc_pdf *= pdf_q * pdf_wo;
    Rgb contrib = cdiv(cscl(Le, fabsf(dot(qn, wo_q))), acc_pdf);
    Ray r = make_ray(q, wo_q);
    HitGeo h;
    if (!trace_closest(s, r, stk, h)) return;
    if (h.light >= 0) return;
    float cosr = fabsf(dot(h.ns, r.d)) / (h.t * h.t);
    acc_pdf *= cosr;
    V3 actual_wi = neg(r.d);
    if (acc_pdf == 0.0f) return;
    if (max_bounce <= 1) return;
    if (n < per) store_vpl(out + n, h, actual_wi, contrib, 1, k);
    n++;
    rzk_material m = ld_mat(s.mats + h.mat);
    V3 wi;
    float pdf_wi;
    Rgb brdf = brdf_sample(m, h.uvn, actual_wi, g, wi, pdf_wi);
    if (!(pdf_wi <= 0.0f || cblack(brdf))) {
        float cs = fabsf(dot(wi, h.ns));
        Rgb T = cdiv(cscl(cmul(contrib, brdf), cs), pdf_wi);
        Ray rr = make_ray(h.p, wi);
        for (int bounce = 2; bounce < max_bounce; ++bounce) {
            HitGeo hh;
            if (!trace_closest(s, rr, stk, hh)) break;
            if (hh.light >= 0) break;
            V3 wi2 = unit(neg(rr.d));
            if (n < per) store_vpl(out + n, hh, wi2, T, bounce, k);
            n++;
            float continuation = 1.0f;
            if (bounce >= 4) {
                continuation = smin(1.0f, 0.99f);   // white.avg() vs 0.99 (vpl_generator.cc:84-90)
                if (g.uniform() > continuation) break;
            }
            V3 wo;
            float pdf;
            rzk_material m2 = ld_mat(s.mats + hh.mat);
            Rgb b2 = brdf_sample(m2, hh.uvn, wi2, g, wo, pdf);
            if (pdf <= 0.0f || cblack(b2)) break;
            pdf *= continuation;
            Rgb f = cdiv(cscl(b2, fabsf(dot(hh.ns, wo))), pdf);
            T = cmul(T, f);
            rr = make_ray(hh.p, wo);
        }
    }
    counts[k] = n < per ? n : per;
}

__global__ void compact_kernel(const rzk_vpl *slots, const int *counts, const int *offsets,
                               int n_particles, int per, rzk_vpl *out, int cap) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_particles) return;
    int c = counts[k], o = offsets[k];
    for (int i = 0; i < c; ++i) {
        if (o + i >= cap) break;
        const float4 *src = reinterpret_cast<const float4 *>(slots + (size_t)k * per + i);
        float4 *dst = reinterpret_cast<float4 *>(out + o + i);
#pragma unroll
        for (int w = 0; w < 6; ++w) dst[w] = src[w];
    }
}

// Light table: areas, quad split ratio and larger-triangle basis (quad.cc:9-19,
// quad.h:114-120), and the luminance of radiance * area * pi for POWER selection
// (scene.cc:185-203, area_light.h:93-95).
struct LightSrc { int first_tri, n_tris, kind, flags; float emit[3]; };

__global__ void light_setup_kernel(const LightSrc *src, int n_lights, const float *v, const float *tri_n,
                                   const float *tri_u, const float *tri_area, DevLight *out, float *lum) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_lights) return;
    LightSrc ls = src[i];
    DevLight d;
    float area[2] = {0.0f, 0.0f};
    for (int k = 0; k < 2; ++k) {
        int t = ls.first_tri + (k < ls.n_tris ? k : 0);
        d.p0[k] = make_float4(v[9 * t], v[9 * t + 1], v[9 * t + 2], 0.0f);
        d.p1[k] = make_float4(v[9 * t + 3], v[9 * t + 4], v[9 * t + 5], 0.0f);
        d.p2[k] = make_float4(v[9 * t + 6], v[9 * t + 7], v[9 * t + 8], 0.0f);
        area[k] = tri_area[t];
        d.n[k] = make_float4(tri_n[3 * t], tri_n[3 * t + 1], tri_n[3 * t + 2], area[k]);
    }
    float total;
    int first = 0;
    if (ls.kind == RZK_PRIM_QUAD) {
        total = area[0] + area[1];
        d.t0_ratio = area[0] / total;
        first = d.t0_ratio >= 0.5f ? 0 : 1;
    } else {
        total = area[0];
        d.t0_ratio = 1.0f;
    }
    int bt = ls.first_tri + first;
    d.basis_n = make_float4(tri_n[3 * bt], tri_n[3 * bt + 1], tri_n[3 * bt + 2], 0.0f);
    d.basis_u = make_float4(tri_u[3 * bt], tri_u[3 * bt + 1], tri_u[3 * bt + 2], 0.0f);
    d.emit = make_float4(ls.emit[0], ls.emit[1], ls.emit[2], 0.0f);
    d.kind = ls.kind;
    d.flags = ls.flags;
    d.n_tris = ls.n_tris;
    out[i] = d;
    Rgb pw = cscl(cscl(crgb(ls.emit[0], ls.emit[1], ls.emit[2]), total), A_PI);
    lum[i] = cval(pw);
}

}  // namespace

rzk_status setup_lights(rzk_scene *s, const std::vector<int> &first_tri, const std::vector<int> &n_tris,
                        const std::vector<int> &kind, const std::vector<int> &flags,
                        const std::vector<float> &emit, cudaStream_t st) {
    const int nl = (int)first_tri.size();
    s->n_lights = nl;
    if (nl == 0) return RZK_OK;
    std::vector<LightSrc> src(nl);
    for (int i = 0; i < nl; ++i) {
        src[i].first_tri = first_tri[i]; src[i].n_tris = n_tris[i];
        src[i].kind = kind[i]; src[i].flags = flags[i];
        for (int c = 0; c < 3; ++c) src[i].emit[c] = emit[3 * i + c];
    }
    LightSrc *d_src = nullptr;
    float *d_lum = nullptr;
    RZK_CUDA_TRY(cudaMalloc((void **)&d_src, sizeof(LightSrc) * nl));
    RZK_CUDA_TRY(cudaMalloc((void **)&d_lum, sizeof(float) * nl));
    RZK_CUDA_TRY(cudaMalloc((void **)&s->d_lights, sizeof(DevLight) * nl));
    RZK_CUDA_TRY(cudaMalloc((void **)&s->d_light_pdf, sizeof(float) * nl));
    RZK_CUDA_TRY(cudaMalloc((void **)&s->d_light_cdf, sizeof(float) * nl));
    s->device_bytes += sizeof(DevLight) * nl + 2 * sizeof(float) * nl;
    RZK_CUDA_TRY(cudaMemcpyAsync(d_src, src.data(), sizeof(LightSrc) * nl, cudaMemcpyHostToDevice, st));
    light_setup_kernel<<<(nl + 127) / 128, 128, 0, st>>>(d_src, nl, s->d_v, s->d_tri_n, s->d_tri_u,
                                                         s->d_tri_area, s->d_lights, d_lum);
    RZK_CUDA_TRY(cudaGetLastError());
    std::vector<float> lum(nl), pdf(nl), cdf(nl);
    RZK_CUDA_TRY(cudaMemcpyAsync(lum.data(), d_lum, sizeof(float) * nl, cudaMemcpyDeviceToHost, st));
    RZK_CUDA_TRY(cudaStreamSynchronize(st));
    cudaFree(d_src);
    cudaFree(d_lum);
    // DiscretePdf::set_distribution (pdf.cc:18-57)
    float sum = 0.0f;
    for (int i = 0; i < nl; ++i) sum += lum[i];
    if (sum == 0.0f) {
        for (int i = 0; i < nl; ++i) pdf[i] = cdf[i] = 0.0f;
    } else {
        for (int i = 0; i < nl; ++i) pdf[i] = lum[i] / sum;
        cdf[0] = pdf[0];
        for (int i = 1; i < nl; ++i) cdf[i] = cdf[i - 1] + pdf[i];
        cdf[nl - 1] = 1.0f;
    }
    RZK_CUDA_TRY(cudaMemcpyAsync(s->d_light_pdf, pdf.data(), sizeof(float) * nl, cudaMemcpyHostToDevice, st));
    RZK_CUDA_TRY(cudaMemcpyAsync(s->d_light_cdf, cdf.data(), sizeof(float) * nl, cudaMemcpyHostToDevice, st));
    RZK_CUDA_TRY(cudaStreamSynchronize(st));
    return RZK_OK;
}

rzk_status launch_vplgen(rzk_scene *sc, uint32_t seed, int n_particles, int max_bounce, rzk_vpl *out,
                         int cap, int *d_count, cudaStream_t st) {
    if (n_particles <= 0) {
        if (d_count) RZK_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(int), st));
        return RZK_OK;
    }
    const int per = max_bounce > 1 ? max_bounce - 1 : 1;
    size_t slots_bytes = sizeof(rzk_vpl) * (size_t)n_particles * per;
    size_t scan_bytes = exclusive_scan_tmp_bytes(n_particles);
    size_t bytes = slots_bytes + 2 * sizeof(int) * (size_t)n_particles + scan_bytes + 1024;
    char *buf = nullptr;
    RZK_CUDA_TRY(cudaMalloc((void **)&buf, bytes));
    struct Free { char *p; ~Free() { if (p) cudaFree(p); } } guard{buf};
    rzk_vpl *slots = (rzk_vpl *)buf;
    int *counts = (int *)(buf + slots_bytes);
    int *offs = counts + n_particles;
    char *scan_tmp = (char *)(offs + n_particles);
    scan_tmp = (char *)(((uintptr_t)scan_tmp + 255) & ~(uintptr_t)255);
    DevScene s = sc->dev();
    vplgen_kernel<<<(n_particles + kGenBlock - 1) / kGenBlock, kGenBlock, 0, st>>>(
        s, seed, n_particles, max_bounce, per, slots, counts);
    RZK_CUDA_TRY(cudaGetLastError());
    rzk_status e = exclusive_scan_i32(counts, offs, n_particles, d_count, scan_tmp, scan_bytes, st);
    if (e != RZK_OK) return e;
    compact_kernel<<<(n_particles + 127) / 128, 128, 0, st>>>(slots, counts, offs, n_particles, per, out, cap);
    RZK_CUDA_TRY(cudaGetLastError());
    RZK_CUDA_TRY(cudaStreamSynchronize(st));
    return RZK_OK;
}

}  // namespace rzk
