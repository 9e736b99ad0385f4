// rzk_math.cuh - device-side vector math, predicates and BRDFs of the VPL gather path.
//
// Every expression follows the reference's operation order (vec3_cpu.h, ray.h,
// boundingbox.h, triangle.cc, onb.cc, lambertian.cc, phong.cc, ward.cc, form_factor.h,
// vpl_interface.h).  The library is compiled with -fmad=false and IEEE division and
// square root, so each operation rounds exactly like the reference built with
// -ffp-contract=off: Morton codes, the BVH, ray/box/triangle predicates, primary hits and
// the receivers are bit-identical to the reference's.  Transcendentals (powf, expf, ...)
// are CUDA's own and agree to a few ulps.
#pragma once

#include <cstdint>
#include "../../include/rzk_types.h"

namespace rzk {

constexpr float A_PI = 3.14159265358979f;
constexpr float INV_PI = 0.31830988618379f;
constexpr float TWO_PI = 6.28318530717959f;
constexpr float INV_2PI = 0.15915494309190f;
constexpr float RAY_TMAX = 1e6f;
constexpr float ZERO_EPSILON = 1e-6f;
constexpr float ONB_EPSILON = 0.01f;
constexpr int STACK_CAP = 64;  // Stack::capacity (aggregate_bvh.cc:243-281)

struct V3 { float x, y, z; };
__host__ __device__ __forceinline__ V3 mk(float x, float y, float z) { return V3{x, y, z}; }
__host__ __device__ __forceinline__ V3 ld3(const float *f) { return V3{f[0], f[1], f[2]}; }
__host__ __device__ __forceinline__ void st3(float *f, V3 v) { f[0] = v.x; f[1] = v.y; f[2] = v.z; }
__host__ __device__ __forceinline__ V3 add(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ V3 sub(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ V3 mul(V3 a, V3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ __forceinline__ V3 dvv(V3 a, V3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
__host__ __device__ __forceinline__ V3 scl(V3 a, float t) { return mk(a.x * t, a.y * t, a.z * t); }
__host__ __device__ __forceinline__ V3 neg(V3 a) { return mk(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ float len(V3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
// unit_vector: one reciprocal, three multiplies (vec3_cpu.h:406-413)
__host__ __device__ __forceinline__ V3 unit(V3 a) {
    float inv = 1.0f / len(a);
    return mk(a.x * inv, a.y * inv, a.z * inv);
}
__host__ __device__ __forceinline__ bool isnan3(V3 a) { return a.x != a.x || a.y != a.y || a.z != a.z; }
// std::min / std::max select rules, also Vec3 min / max (vec3_cpu.h:415-429)
__host__ __device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__host__ __device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }
__host__ __device__ __forceinline__ V3 vmin(V3 a, V3 b) { return mk(smin(a.x, b.x), smin(a.y, b.y), smin(a.z, b.z)); }
__host__ __device__ __forceinline__ V3 vmax(V3 a, V3 b) { return mk(smax(a.x, b.x), smax(a.y, b.y), smax(a.z, b.z)); }

struct Onb { V3 u, v, n; };
// Onb::init_from_n (onb.cc:42-56)
__host__ __device__ inline Onb onb_from_n(V3 n_) {
    Onb o;
    V3 i = mk(1.0f, 0.0f, 0.0f), j = mk(0.0f, 1.0f, 0.0f);
    o.n = unit(n_);
    o.u = cross(o.n, i);
    if (len(o.u) < ONB_EPSILON) o.u = cross(o.n, j);
    o.v = cross(o.n, o.u);
    o.u = unit(o.u);   // make_unit_vector: same reciprocal-multiply sequence
    o.v = unit(o.v);
    return o;
}
// Onb::init_from_nu (onb.cc:93-103)
__host__ __device__ inline Onb onb_from_nu(V3 n_, V3 u_) {
    V3 c = unit(cross(n_, u_));
    if (isnan3(c)) return onb_from_n(n_);
    Onb o;
    o.n = unit(n_);
    o.v = c;
    o.u = cross(o.v, o.n);
    return o;
}
__host__ __device__ __forceinline__ V3 l2w(const Onb &o, V3 a) {   // onb.cc:138-140
    return add(add(scl(o.u, a.x), scl(o.v, a.y)), scl(o.n, a.z));
}
__host__ __device__ __forceinline__ V3 w2l(const Onb &o, V3 w) {   // onb.cc:134-136
    return mk(dot(o.u, w), dot(o.v, w), dot(o.n, w));
}

struct Rgb { float r, g, b; };
__host__ __device__ __forceinline__ Rgb crgb(float r, float g, float b) { return Rgb{r, g, b}; }
__host__ __device__ __forceinline__ Rgb cmul(Rgb a, Rgb b) { return crgb(a.r * b.r, a.g * b.g, a.b * b.b); }
__host__ __device__ __forceinline__ Rgb cscl(Rgb a, float t) { return crgb(a.r * t, a.g * t, a.b * t); }
__host__ __device__ __forceinline__ Rgb cdiv(Rgb a, float t) { return crgb(a.r / t, a.g / t, a.b / t); }
__host__ __device__ __forceinline__ Rgb cadd(Rgb a, Rgb b) { return crgb(a.r + b.r, a.g + b.g, a.b + b.b); }
__host__ __device__ __forceinline__ float cval(Rgb a) { return sqrtf(a.r * a.r + a.g * a.g + a.b * a.b); }
__host__ __device__ __forceinline__ bool cblack(Rgb a) { return a.r == 0.0f && a.g == 0.0f && a.b == 0.0f; }

// ---------------------------------------------------------------------------------
// Rays and predicates
// ---------------------------------------------------------------------------------
struct Ray { V3 o, d, inv_d, org_inv_d; };

// Ray::Ray (ray.h:17-36)
__host__ __device__ __forceinline__ Ray make_ray(V3 o, V3 d_) {
    Ray r;
    r.o = o;
    r.d = unit(d_);
    if (isnan3(r.d)) r.d = mk(0.0f, 0.0f, 0.0f);
    V3 dd = mk(fabsf(r.d.x) < ZERO_EPSILON ? ZERO_EPSILON : r.d.x,
               fabsf(r.d.y) < ZERO_EPSILON ? ZERO_EPSILON : r.d.y,
               fabsf(r.d.z) < ZERO_EPSILON ? ZERO_EPSILON : r.d.z);
    r.inv_d = dvv(mk(1.0f, 1.0f, 1.0f), dd);
    r.org_inv_d = mul(neg(o), r.inv_d);
    return r;
}

// BoundingBox::hit (boundingbox.h:238-280); bmin / bmax as the two xyz triples of a
// packed node record.
__device__ __forceinline__ bool box_hit(float4 lo, float4 hi, const Ray &r, float tmin, float tmax) {
    float x0 = lo.x * r.inv_d.x + r.org_inv_d.x;
    float y0 = lo.y * r.inv_d.y + r.org_inv_d.y;
    float z0 = lo.z * r.inv_d.z + r.org_inv_d.z;
    float x1 = hi.x * r.inv_d.x + r.org_inv_d.x;
    float y1 = hi.y * r.inv_d.y + r.org_inv_d.y;
    float z1 = hi.z * r.inv_d.z + r.org_inv_d.z;
    float tminbox = smax(tmin, smax(smin(x0, x1), smax(smin(y0, y1), smin(z0, z1))));
    float tmaxbox = smin(tmax, smin(smax(x0, x1), smin(smax(y0, y1), smax(z0, z1))));
    return (tminbox <= tmaxbox) && (tmax >= tminbox && tmaxbox >= tmin);
}

// The same test also returning the entry distance tminbox (for visit ordering only).
__device__ __forceinline__ bool box_hit_t(float4 lo, float4 hi, const Ray &r, float tmin, float tmax,
                                          float &tnear) {
    float x0 = lo.x * r.inv_d.x + r.org_inv_d.x;
    float y0 = lo.y * r.inv_d.y + r.org_inv_d.y;
    float z0 = lo.z * r.inv_d.z + r.org_inv_d.z;
    float x1 = hi.x * r.inv_d.x + r.org_inv_d.x;
    float y1 = hi.y * r.inv_d.y + r.org_inv_d.y;
    float z1 = hi.z * r.inv_d.z + r.org_inv_d.z;
    float tminbox = smax(tmin, smax(smin(x0, x1), smax(smin(y0, y1), smin(z0, z1))));
    float tmaxbox = smin(tmax, smin(smax(x0, x1), smin(smax(y0, y1), smax(z0, z1))));
    tnear = tminbox;
    return (tminbox <= tmaxbox) && (tmax >= tminbox && tmaxbox >= tmin);
}

// The slab test of box_hit with single-instruction min / max and one final compare, for
// the gather's packet traversal.  With finite box bounds, ray origin and tmin / tmax
// (receivers and VPLs are finite; |inv_d| <= 1e6 by the ZERO_EPSILON substitution of
// ray.h:23-27) no slab value is NaN, so fminf / fmaxf select the same value as the
// reference's (b < a) ? b : a up to the sign of a zero, which no comparison below can
// see; and since tminbox >= tmin and tmaxbox <= tmax by construction, the reference's
// "tmax >= tminbox && tmaxbox >= tmin" follows from tminbox <= tmaxbox.  The answer is
// therefore the reference's answer bit for bit.
__device__ __forceinline__ bool box_hit_fast(float4 lo, float4 hi, const Ray &r, float tmin, float tmax,
                                             float &tnear) {
    float x0 = lo.x * r.inv_d.x + r.org_inv_d.x;
    float y0 = lo.y * r.inv_d.y + r.org_inv_d.y;
    float z0 = lo.z * r.inv_d.z + r.org_inv_d.z;
    float x1 = hi.x * r.inv_d.x + r.org_inv_d.x;
    float y1 = hi.y * r.inv_d.y + r.org_inv_d.y;
    float z1 = hi.z * r.inv_d.z + r.org_inv_d.z;
    float tminbox = fmaxf(fmaxf(tmin, fminf(x0, x1)), fmaxf(fminf(y0, y1), fminf(z0, z1)));
    float tmaxbox = fminf(fminf(tmax, fmaxf(x0, x1)), fminf(fmaxf(y0, y1), fmaxf(z0, z1)));
    tnear = tminbox;
    return tminbox <= tmaxbox;
}

// Triangle::hit (triangle.cc:158-275) on a packed record:
//   a = {p0.x, p0.y, p0.z, A}, b = {B, C, D, E}, c = {F, -, -, -}
// with (A,B,C) = p0 - p1 and (D,E,F) = p0 - p2, exactly the reference's p01 / p02.
template <bool WANT_T>
__device__ __forceinline__ bool tri_hit(float4 a, float4 b, float4 c, const Ray &r, float tmin,
                                        float tmax, float *t_out, float *beta_out,
                                        float *gamma_out) {
    const float A = a.w, B = b.x, C = b.y, D = b.z, E = b.w, F = c.x;
    const float G = r.d.x, H = r.d.y, I = r.d.z;
    const float J = a.x - r.o.x, K = a.y - r.o.y, L = a.z - r.o.z;
    float EIHF = E * I - H * F;
    float GFDI = G * F - D * I;
    float DHEG = D * H - E * G;
    float denom = (A * EIHF + B * GFDI + C * DHEG);
    if (-ZERO_EPSILON < denom && denom < ZERO_EPSILON) return false;
    float beta = (J * EIHF + K * GFDI + L * DHEG) / denom;
    if (beta < 0.0f || beta > 1.0f) return false;
    float AKJB = A * K - J * B;
    float JCAL = J * C - A * L;
    float BLKC = B * L - K * C;
    float gamma = (I * AKJB + H * JCAL + G * BLKC) / denom;
    if (gamma < 0.0f || beta + gamma > 1.0f) return false;
    float t = -(F * AKJB + E * JCAL + D * BLKC) / denom;
    if (t >= tmin && t <= tmax) {
        if (WANT_T) { *t_out = t; *beta_out = beta; *gamma_out = gamma; }
        return true;
    }
    return false;
}

// ---------------------------------------------------------------------------------
// BRDFs (lambertian.cc:63-68, phong.cc:74-87, ward.cc:104-116)
// ---------------------------------------------------------------------------------
__device__ inline Rgb brdf_eval(const rzk_material &m, const Onb &uvn, V3 wo, V3 wi) {
    Rgb kd = crgb(m.kd[0], m.kd[1], m.kd[2]);
    if (m.type == RZK_BSDF_WARD) {
        float ax = m.p0, ay = m.p1;
        float ax2 = ax * ax, ay2 = ay * ay;
        float inv4 = 1.0f / (4 * A_PI * ax * ay);   // Ward::Ward (ward.cc:5-9)
        V3 lwi = w2l(uvn, wi), lwo = w2l(uvn, wo);
        if (lwi.z <= ZERO_EPSILON || lwo.z <= ZERO_EPSILON) return crgb(0.0f, 0.0f, 0.0f);
        V3 wh = add(lwi, lwo);
        float expo = expf(-(wh.x * wh.x / ax2 + wh.y * wh.y / ay2) / (wh.z * wh.z));
        Rgb ks = crgb(m.ks[0], m.ks[1], m.ks[2]);
        Rgb spec = cscl(cdiv(cscl(ks, inv4), sqrtf(lwi.z * lwo.z)), expo);
        return cadd(cscl(kd, INV_PI), spec);
    }
    if (dot(wi, uvn.n) <= ZERO_EPSILON || dot(wo, uvn.n) <= ZERO_EPSILON) return crgb(0.0f, 0.0f, 0.0f);
    Rgb b = cscl(kd, INV_PI);
    if (m.type == RZK_BSDF_PHONG) {
        float n = m.p0;
        V3 nn = uvn.n;
        V3 wr = sub(scl(nn, 2 * dot(wi, nn)), wi);
        float ca = dot(wo, wr);
        if (ca > 0.0f) {
            Rgb ks = crgb(m.ks[0], m.ks[1], m.ks[2]);
            b = cadd(b, cscl(cscl(cscl(ks, (n + 2)), INV_2PI), powf(ca, n)));
        }
    }
    return b;
}

// FormFactor::form_factor_abs (form_factor.h:11-21)
__device__ __forceinline__ float form_factor_abs(V3 p, V3 pn, V3 q, V3 qn) {
    V3 pq = sub(q, p);
    float d1 = dot(pn, pq);
    float d2 = -dot(qn, pq);
    float dpq = dot(pq, pq);
    return fabsf((d1 * d2) / (dpq * dpq));
}

// RadianceTerms + clamp_term (vpl_interface.h:50-123, vpl.cc:214-230)
__device__ __forceinline__ Rgb radiance_terms(Rgb power, Rgb sb, Rgb lb, float G, int mode,
                                              float tau, Rgb *no_clamp = nullptr) {
    Rgb r, nc;
    if (mode == RZK_CLAMP_REFLECTIVITY) {
        Rgb refl = cmul(cscl(sb, G), lb);
        float lum = cval(refl);
        r = lum > tau ? cmul(cscl(refl, tau / lum), power) : cmul(refl, power);
        nc = cmul(cmul(cscl(power, G), sb), lb);
    } else if (mode == RZK_CLAMP_RADIANCE) {
        nc = cmul(cmul(cscl(power, G), sb), lb);
        float br = cval(nc);
        r = br > tau ? cscl(nc, tau / br) : nc;
    } else if (mode == RZK_CLAMP_FORM_FACTOR) {
        r = G > tau ? cmul(cscl(cmul(lb, sb), tau), power) : cmul(cscl(cmul(lb, sb), G), power);
        nc = cmul(cmul(cscl(power, G), sb), lb);
    } else {
        nc = cmul(cmul(cscl(power, G), sb), lb);
        r = nc;
    }
    if (no_clamp) *no_clamp = nc;
    return r;
}

// ---------------------------------------------------------------------------------
// Counter-based random stream: Philox4x32-10 (Salmon et al., SC'11).
// Draw d of (seed, stream, path) = word d&3 of the block at counter
// {d>>2, path, stream, 0x52454e5a} under key {seed, 0x4b5a4f52}.
// ---------------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c.y ^ k0;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c.w ^ k1;
        c = make_uint4(n0, (uint32_t)p1, n2, (uint32_t)p0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

struct Rng {
    uint32_t seed, stream, path, d;
    uint4 block;
    uint32_t block_idx;
    __device__ __forceinline__ void init(uint32_t s, uint32_t st, uint32_t p) {
        seed = s; stream = st; path = p; d = 0; block_idx = 0xffffffffu;
    }
    __device__ __forceinline__ uint32_t next_u32() {
        uint32_t bi = d >> 2;
        if (bi != block_idx) {
            block = philox4x32_10(make_uint4(bi, path, stream, 0x52454e5au), seed, 0x4b5a4f52u);
            block_idx = bi;
        }
        uint32_t w = d & 3;
        d++;
        return w == 0 ? block.x : (w == 1 ? block.y : (w == 2 ? block.z : block.w));
    }
    // Random::operator() and rand_exclude_01 (random.h:60-71)
    __device__ __forceinline__ float uniform() {
        return (next_u32() & 0x00ffffffu) * (1.0f / 16777216.0f);
    }
    __device__ __forceinline__ float uniform_ex01() {
        return (next_u32() & 0x00ffffffu) * (1.0f / 16777216.0f) + (1.0f / 33554432.0f);
    }
};

}  // namespace rzk
