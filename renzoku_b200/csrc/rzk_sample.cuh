// rzk_sample.cuh - BRDF sampling and pdfs, closest-hit tracing and area-light sampling
// shared by the VPL generator and the guided path tracer.
#ifndef RZK_SAMPLE_CUH_
#define RZK_SAMPLE_CUH_

#include "rzk_traverse.cuh"

namespace rzk {

// Phong / Ward sampling weights (phong.cc:6-16, ward.cc:15-24): Rgb::max of kd and ks,
// normalised by their sum.
__device__ __forceinline__ void rho_terms(const rzk_material &m, float &rho_d, float &rho_s) {
    float rd = m.kd[0]; if (m.kd[1] > rd) rd = m.kd[1]; if (m.kd[2] > rd) rd = m.kd[2];
    float rs = m.ks[0]; if (m.ks[1] > rs) rs = m.ks[1]; if (m.ks[2] > rs) rs = m.ks[2];
    float total = rd + rs;
    if (total > 0.0f) { rd /= total; rs /= total; }
    rho_d = rd; rho_s = rs;
}

// Phong / Ward / Lambertian pdf (lambertian.cc:70-75, phong.cc:89-103, ward.cc:118-134)
__device__ inline float brdf_pdf(const rzk_material &m, const Onb &uvn, V3 wo, V3 wi, float rho_d, float rho_s) {
    if (dot(wi, uvn.n) <= ZERO_EPSILON || dot(wo, uvn.n) <= ZERO_EPSILON) return 0.0f;
    if (m.type == RZK_BSDF_LAMBERTIAN) return dot(uvn.n, wi) * INV_PI;
    if (m.type == RZK_BSDF_PHONG) {
        float n = m.p0;
        V3 nn = uvn.n;
        float pdf = rho_d * (dot(nn, wi) * INV_PI);
        V3 wr = sub(scl(nn, 2 * dot(wi, nn)), wi);
        float ca = dot(wo, wr);
        if (ca > 0.0f) pdf += rho_s * (n + 1) * INV_2PI * powf(ca, n);
        return pdf;
    }
    float ax = m.p0, ay = m.p1;
    float ax2 = ax * ax, ay2 = ay * ay;
    float inv4 = 1.0f / (4 * A_PI * ax * ay);
    float z = dot(uvn.n, wi);
    V3 wh = unit(w2l(uvn, add(wi, wo)));
    float expo = expf(-(wh.x * wh.x / ax2 + wh.y * wh.y / ay2) / (wh.z * wh.z));
    float ct = wh.z;
    V3 lwo = unit(w2l(uvn, wo));
    float ct3 = ct * ct * ct;
    return rho_d * (z * INV_PI) + rho_s * (inv4 / (dot(wh, lwo) * ct3) * expo);
}

__device__ inline Rgb brdf_sample(const rzk_material &m, const Onb &uvn, V3 wo, Rng &g, V3 &wi, float &pdf) {
    if (dot(wo, uvn.n) <= ZERO_EPSILON) { wi = mk(0, 0, 0); pdf = 0.0f; return crgb(0, 0, 0); }
    if (m.type == RZK_BSDF_LAMBERTIAN) {
        float sx = g.uniform(), sy = g.uniform();
        float phi = TWO_PI * sx;
        float sin_theta = sqrtf(sy);
        float x = sin_theta * cosf(phi);
        float y = sin_theta * sinf(phi);
        float z = sqrtf(1 - sin_theta * sin_theta);
        wi = unit(l2w(uvn, mk(x, y, z)));
        pdf = z * INV_PI;
        return cscl(crgb(m.kd[0], m.kd[1], m.kd[2]), INV_PI);
    }
    float rho_d, rho_s;
    rho_terms(m, rho_d, rho_s);
    float eps = g.uniform();
    if (eps < rho_d) {
        float sx = g.uniform(), sy = g.uniform();
        float phi = TWO_PI * sx;
        float sin_theta = sqrtf(sy);
        float x = sin_theta * cosf(phi);
        float y = sin_theta * sinf(phi);
        float z = sqrtf(1.0f - sin_theta * sin_theta);
        wi = unit(l2w(uvn, mk(x, y, z)));
    } else if (m.type == RZK_BSDF_PHONG) {
        float sx = g.uniform(), sy = g.uniform();
        Onb o = onb_from_nu(wo, uvn.n);
        float phi = TWO_PI * sx;
        float alpha = acosf(powf(sy, 1.0f / (m.p0 + 1)));
        float st_ = sinf(alpha), ct_ = cosf(alpha), sp = sinf(phi), cp = cosf(phi);
        V3 wr = l2w(o, mk(st_ * cp, st_ * sp, ct_));
        V3 nn = uvn.n;
        float d = dot(wr, nn);
        if (d < 0.0f) { wi = mk(0, 0, 0); pdf = 0.0f; return crgb(0, 0, 0); }
        wi = sub(scl(nn, 2 * d), wr);
    } else {
        // Vec2 sampler(rd.rand_exclude_01(), rd.rand_exclude_01()) (ward.cc:58) as the
        // reference's compiler evaluates it: right to left, the second coordinate first.
        float sy = g.uniform_ex01();
        float sx = g.uniform_ex01();
        float ax = m.p0, ay = m.p1;
        float ax2 = ax * ax, ay2 = ay * ay, ay_ax = ay / ax;
        V3 lwo = unit(w2l(uvn, wo));
        float angle = TWO_PI * sx;
        float phi = atanf(ay_ax * tanf(angle));
        if (sinf(phi) * sinf(angle) < 0 || cosf(phi) * cosf(angle) < 0) phi += A_PI;
        float cp = cosf(phi), sp = sinf(phi);
        float theta = atanf(sqrtf(-logf(sy) / (cp * cp / ax2 + sp * sp / ay2)));
        float st_ = sinf(theta), ct_ = cosf(theta);
        V3 wh = mk(st_ * cp, st_ * sp, ct_);
        V3 lwi = sub(scl(wh, 2 * dot(lwo, wh)), lwo);
        wi = l2w(uvn, lwi);
    }
    pdf = brdf_pdf(m, uvn, wo, wi, rho_d, rho_s);
    return brdf_eval(m, uvn, wo, wi);
}

__device__ __forceinline__ rzk_material ld_mat(const rzk_material *m) { return *m; }

template <int STRIDE>
__device__ __forceinline__ bool trace_closest(const DevScene &s, const Ray &r, Stack<STRIDE> &stk, HitGeo &h) {
    float t, b, g;
    int slot = closest_hit<STRIDE>(s, r, s.tmin, RAY_TMAX, stk, &t, &b, &g);
    if (slot < 0) return false;
    fill_hit(s, r, slot, t, b, g, h);
    return true;
}


// Linear::solve33 / det (linear.h:23-47): Cramer's rule as the reference writes it.
__device__ __forceinline__ float det33(float a, float b, float c, float d, float e, float f, float g, float h,
                                       float i) {
    return (a * e * i + b * f * g + c * d * h) - (c * e * g + b * d * i + a * f * h);
}

// Triangle::pdf (triangle.cc:310-327): 1 / area where the barycentric solution lies in [0,1]^3.
__device__ __forceinline__ float light_tri_pdf(const DevLight &L, int k, V3 p) {
    const float4 a = L.p0[k], b = L.p1[k], c = L.p2[k];
    const float inv = 1.0f / det33(a.x, b.x, c.x, a.y, b.y, c.y, a.z, b.z, c.z);
    const float x = inv * det33(p.x, b.x, c.x, p.y, b.y, c.y, p.z, b.z, c.z);
    const float y = inv * det33(a.x, p.x, c.x, a.y, p.y, c.y, a.z, p.z, c.z);
    const float z = inv * det33(a.x, b.x, p.x, a.y, b.y, p.y, a.z, b.z, p.z);
    if (x >= 0.0f && x <= 1.0f && y >= 0.0f && y <= 1.0f && z >= 0.0f && z <= 1.0f) return 1.0f / L.n[k].w;
    return 0.0f;
}

// Surface::pdf(p) -> Quad::pdf (quad.cc:89-91) or Triangle::pdf
__device__ __forceinline__ float light_area_pdf(const DevLight &L, V3 p) {
    if (L.kind == RZK_PRIM_QUAD)
        return L.t0_ratio * light_tri_pdf(L, 0, p) + (1.0f - L.t0_ratio) * light_tri_pdf(L, 1, p);
    return light_tri_pdf(L, 0, p);
}

// AreaLight::query (area_light.cc:19-25) with AreaLight::pdf(p, n, wo) (area_light.h:114-123)
__device__ __forceinline__ Rgb light_query(const DevLight &L, V3 p, V3 n, V3 wo) {
    if (dot(wo, n) < ZERO_EPSILON) return crgb(0.0f, 0.0f, 0.0f);
    const float pdf_p = light_area_pdf(L, p);
    const float pdf_wo = pdf_p <= 0.0f ? 0.0f : dot(wo, n) * INV_PI;
    if (pdf_p * pdf_wo <= 0.0f) return crgb(0.0f, 0.0f, 0.0f);
    return crgb(L.emit.x, L.emit.y, L.emit.z);
}

// Surface::sample -> Quad::sample (quad.cc:75-87) / Triangle::sample (triangle.cc:298-308),
// the normal flipped on a flipped surface (surface.cc:98-102)
__device__ __forceinline__ void light_sample_point(const DevLight &L, Rng &g, V3 &q, V3 &qn, float &pdf) {
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
    q = add(add(scl(tp0, a), scl(tp1, b)), scl(tp2, c));
    qn = mk(L.n[which].x, L.n[which].y, L.n[which].z);
    float pdf_t = 1.0f / L.n[which].w;
    pdf = L.kind == RZK_PRIM_QUAD ? pdf_sel * pdf_t : pdf_t;
    if (L.flags & RZK_SURF_FLIPPED) qn = neg(qn);
}

}  // namespace rzk

#endif  // RZK_SAMPLE_CUH_
