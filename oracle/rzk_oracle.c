/*
 * rzk_oracle.c - TEST INFRASTRUCTURE ONLY: CPU restatement of the reference's VPL
 * gather path (see rzk_oracle.h).  The product never links this file; tests/, the
 * smoke check and the CPU-baseline leg of bench.py load it as the checker.
 *
 * Reference files cited are from the reference project's flat source directory.
 */
#define _GNU_SOURCE
#include "rzk_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------ */
/* Constants (common.h:36-55, random.h:33-37).                                     */
/* ------------------------------------------------------------------------------ */
#define A_PI 3.14159265358979f
#define INV_PI 0.31830988618379f
#define TWO_PI 6.28318530717959f
#define INV_2PI 0.15915494309190f
#define RAY_TMAX 1e6f
#define ZERO_EPSILON 1e-6f
#define ONB_EPSILON 0.01f
#define STACK_CAP 64
static const float DEGREE_TO_RADIAN = A_PI / 180.0f;
static const float INV_TWO_POW_24 = 1.0f / 16777216.0f;
static const float INV_TWO_POW_25 = 1.0f / 33554432.0f;

/* ------------------------------------------------------------------------------ */
/* Vec3 in the reference's operation order (vec3_cpu.h:140-430).                   */
/* ------------------------------------------------------------------------------ */
typedef struct { float x, y, z; } v3;
static inline v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 ld(const float *f) { return mk(f[0], f[1], f[2]); }
static inline void st(float *f, v3 v) { f[0] = v.x; f[1] = v.y; f[2] = v.z; }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 dvv(v3 a, v3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline v3 scl(v3 a, float t) { return mk(a.x * t, a.y * t, a.z * t); }
static inline v3 neg(v3 a) { return mk(-a.x, -a.y, -a.z); }
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float len(v3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
/* unit_vector: one reciprocal then three multiplies (vec3_cpu.h:406-413). */
static inline v3 unit(v3 a) { float inv = 1.0f / len(a); return mk(a.x * inv, a.y * inv, a.z * inv); }
static inline int isnan3(v3 a) { return a.x != a.x || a.y != a.y || a.z != a.z; }
/* std::min / std::max and Vec3 min / max select rules (vec3_cpu.h:415-429). */
static inline float smin(float a, float b) { return (b < a) ? b : a; }
static inline float smax(float a, float b) { return (a < b) ? b : a; }
static inline v3 vmin(v3 a, v3 b) { return mk(smin(a.x, b.x), smin(a.y, b.y), smin(a.z, b.z)); }
static inline v3 vmax(v3 a, v3 b) { return mk(smax(a.x, b.x), smax(a.y, b.y), smax(a.z, b.z)); }

/* Onb (onb.cc:42-140). */
typedef struct { v3 u, v, n; } onb;
static onb onb_from_n(v3 n_) {
    onb o;
    v3 i = mk(1.0f, 0.0f, 0.0f), j = mk(0.0f, 1.0f, 0.0f);
    o.n = unit(n_);
    o.u = cross(o.n, i);
    if (len(o.u) < ONB_EPSILON) o.u = cross(o.n, j);
    o.v = cross(o.n, o.u);
    { float inv = 1.0f / len(o.u); o.u = mk(o.u.x * inv, o.u.y * inv, o.u.z * inv); }
    { float inv = 1.0f / len(o.v); o.v = mk(o.v.x * inv, o.v.y * inv, o.v.z * inv); }
    return o;
}
static onb onb_from_nu(v3 n_, v3 u_) {   /* onb.cc:93-103 */
    v3 c = unit(cross(n_, u_));
    if (isnan3(c)) return onb_from_n(n_);
    onb o;
    o.n = unit(n_);
    o.v = c;
    o.u = cross(o.v, o.n);
    return o;
}
static onb onb_from_nv(v3 n_, v3 v_) {   /* onb.cc:117-127 */
    v3 c = unit(cross(v_, n_));
    if (isnan3(c)) return onb_from_n(n_);
    onb o;
    o.n = unit(n_);
    o.u = c;
    o.v = cross(o.n, o.u);
    return o;
}
static inline v3 l2w(const onb *o, v3 a) {   /* onb.cc:138-140 */
    return add(add(scl(o->u, a.x), scl(o->v, a.y)), scl(o->n, a.z));
}
static inline v3 w2l(const onb *o, v3 w) {   /* onb.cc:134-136 */
    return mk(dot(o->u, w), dot(o->v, w), dot(o->n, w));
}

/* Rgb (rgb.h). */
typedef struct { float r, g, b; } rgb;
static inline rgb crgb(float r, float g, float b) { rgb c = {r, g, b}; return c; }
static inline rgb cmul(rgb a, rgb b) { return crgb(a.r * b.r, a.g * b.g, a.b * b.b); }
static inline rgb cscl(rgb a, float t) { return crgb(a.r * t, a.g * t, a.b * t); }
static inline rgb cdiv(rgb a, float t) { return crgb(a.r / t, a.g / t, a.b / t); }
static inline rgb cadd(rgb a, rgb b) { return crgb(a.r + b.r, a.g + b.g, a.b + b.b); }
static inline float cval(rgb a) { return sqrtf(a.r * a.r + a.g * a.g + a.b * a.b); }
static inline int cblack(rgb a) { return a.r == 0.0f && a.g == 0.0f && a.b == 0.0f; }
static const rgb BLACK = {0.0f, 0.0f, 0.0f};
static const rgb WHITE = {1.0f, 1.0f, 1.0f};

/* ------------------------------------------------------------------------------ */
/* Scene.                                                                          */
/* ------------------------------------------------------------------------------ */
typedef struct {        /* one flattened triangle (triangle.cc:7-22) */
    v3 p0, p1, p2;
    v3 n;               /* facet normal unit(cross(p0 - p1, p0 - p2)) */
    v3 u;               /* tangent (quad.cc:20-22 overrides for both halves) */
    float area;         /* cross(p01, p02).length() * 0.5 */
    v3 bmin, bmax;      /* BoundingBox(p0, p1, p2) (boundingbox.h:27-30) */
    int surf;
} ro_tri;

typedef struct {
    int kind, mat, flags, light;
    int first_tri, n_tris;
    rgb emit;
    float area;          /* Shape::area(): quad_area or tri_area */
    float t0_ratio;      /* Quad: t0.area / quad_area (quad.cc:9-10) */
    int first;           /* Quad::first: 0 -> t0, 1 -> t1 (quad.cc:13-19) */
} ro_surf;

struct ro_scene {
    int n_tris, n_surfs, n_mats, n_lights;
    ro_tri *tris;            /* input order */
    ro_surf *surfs;
    rzk_material *mats;
    int *lights;             /* surface index of each area light */
    float *light_pdf, *light_cdf;
    float tmin;
    /* BVH */
    uint32_t *codes;         /* input order */
    uint32_t *sorted_codes;
    int32_t *perm;           /* sorted slot -> input triangle */
    rzk_bvh_node *nodes;
    int n_nodes;
};

int ro_num_triangles(const ro_scene *s) { return s->n_tris; }
int ro_num_nodes(const ro_scene *s) { return s->n_nodes; }
int ro_num_lights(const ro_scene *s) { return s->n_lights; }

static void tri_init(ro_tri *t, v3 p0, v3 p1, v3 p2) {   /* triangle.cc:7-22 */
    t->p0 = p0; t->p1 = p1; t->p2 = p2;
    v3 p01 = sub(p0, p1), p02 = sub(p0, p2);
    t->area = len(cross(p01, p02)) * 0.5f;
    t->u = unit(p01);
    t->n = unit(cross(p01, p02));
    t->bmin = vmin(vmin(p0, p1), p2);
    t->bmax = vmax(vmax(p0, p1), p2);
}

/* morton.h:28-46 */
static uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
static uint32_t morton3(float x, float y, float z) {
    x = smin(smax(x * 1024.0f, 0.0f), 1023.0f);
    y = smin(smax(y * 1024.0f, 0.0f), 1023.0f);
    z = smin(smax(z * 1024.0f, 0.0f), 1023.0f);
    return expand_bits((uint32_t)x) * 4 + expand_bits((uint32_t)y) * 2 + expand_bits((uint32_t)z);
}

/* morton.h:16-26 */
static int clz32(uint32_t v) { return v == 0 ? 32 : __builtin_clz(v); }

/* morton.h:48-88 */
static int find_split(const uint32_t *c, int first, int last) {
    uint32_t fc = c[first], lc = c[last];
    if (fc == lc) return (first + last) >> 1;
    int common = clz32(fc ^ lc);
    int split = first, step = last - first;
    do {
        step = (step + 1) >> 1;
        int ns = split + step;
        if (ns < last) {
            if (clz32(fc ^ c[ns]) > common) split = ns;
        }
    } while (step > 1);
    return split;
}

static void bvh_build(ro_scene *s) {
    int n = s->n_tris;
    s->codes = (uint32_t *)calloc(n > 0 ? n : 1, 4);
    s->sorted_codes = (uint32_t *)calloc(n > 0 ? n : 1, 4);
    s->perm = (int32_t *)calloc(n > 0 ? n : 1, 4);
    s->n_nodes = 0;
    s->nodes = NULL;
    if (n <= 0) return;
    /* scene box: reset() to the origin, then merge every triangle box
       (aggregate_bvh.cc:59,73; boundingbox.h:100-103) */
    v3 bmin = mk(0.0f, 0.0f, 0.0f), bmax = mk(0.0f, 0.0f, 0.0f);
    for (int i = 0; i < n; ++i) {
        bmin = vmin(bmin, s->tris[i].bmin);
        bmax = vmax(bmax, s->tris[i].bmax);
    }
    /* morton_box (morton.h:98-102) */
    v3 ext = sub(bmax, bmin);
    for (int i = 0; i < n; ++i) {
        v3 c = scl(add(s->tris[i].bmin, s->tris[i].bmax), 0.5f);
        c = dvv(sub(c, bmin), ext);
        s->codes[i] = morton3(c.x, c.y, c.z);
    }
    /* stable sort of (code, index) (morton.h:109-120; qsort is a stable merge sort on
       this glibc, so equal codes keep input order): LSD radix, 4 x 8 bits */
    int32_t *tmp = (int32_t *)malloc((size_t)n * 4);
    for (int i = 0; i < n; ++i) s->perm[i] = i;
    for (int pass = 0; pass < 4; ++pass) {
        int cnt[257];
        memset(cnt, 0, sizeof(cnt));
        int sh = 8 * pass;
        for (int i = 0; i < n; ++i) cnt[((s->codes[s->perm[i]] >> sh) & 255) + 1]++;
        for (int b = 0; b < 256; ++b) cnt[b + 1] += cnt[b];
        for (int i = 0; i < n; ++i) tmp[cnt[(s->codes[s->perm[i]] >> sh) & 255]++] = s->perm[i];
        memcpy(s->perm, tmp, (size_t)n * 4);
    }
    free(tmp);
    for (int i = 0; i < n; ++i) s->sorted_codes[i] = s->codes[s->perm[i]];
    /* BFS split loop (aggregate_bvh.cc:116-181) */
    int cap = 2 * n;   /* 2n - 1 nodes are produced */
    rzk_bvh_node *nodes = (rzk_bvh_node *)calloc((size_t)cap, sizeof(rzk_bvh_node));
    int *level_first = (int *)malloc(sizeof(int) * 130);
    int *level_last = (int *)malloc(sizeof(int) * 130);
    int n_levels = 0;
    int first = 0, last = 1, next_last = 1, num = 1, level = 0;
    nodes[0].start = 0;
    nodes[0].end = n - 1;
    level_first[0] = 0; level_last[0] = 1; n_levels = 1;
    for (;;) {
        rzk_bvh_node *nd = &nodes[first];
        nd->level = level;
        if (nd->start == nd->end) {
            nd->left = -1;
            nd->right = -1;
        } else {
            int split = find_split(s->sorted_codes, nd->start, nd->end);
            nd->left = next_last;
            nd->right = next_last + 1;
            next_last += 2;
            num += 2;
            nodes[nd->left].start = nd->start;
            nodes[nd->left].end = split;
            nodes[nd->right].start = split + 1;
            nodes[nd->right].end = nd->end;
        }
        first++;
        if (first == last) {
            if (next_last == last) break;
            last = next_last;
            level_first[n_levels] = first;
            level_last[n_levels] = last;
            n_levels++;
            level++;
        }
    }
    /* bottom-up box link (aggregate_bvh.cc:183-209) */
    for (int l = n_levels - 1; l >= 0; --l) {
        for (int j = level_first[l]; j < level_last[l]; ++j) {
            rzk_bvh_node *nd = &nodes[j];
            v3 mn, mx;
            if (nd->left < 0) {
                if (nd->right < 0) {
                    const ro_tri *t = &s->tris[s->perm[nd->start]];
                    mn = t->bmin; mx = t->bmax;
                } else {
                    mn = ld(nodes[nd->right].bmin); mx = ld(nodes[nd->right].bmax);
                }
            } else {
                mn = ld(nodes[nd->left].bmin); mx = ld(nodes[nd->left].bmax);
                if (nd->right >= 0) {
                    mn = vmin(mn, ld(nodes[nd->right].bmin));
                    mx = vmax(mx, ld(nodes[nd->right].bmax));
                }
            }
            st(nd->bmin, mn);
            st(nd->bmax, mx);
        }
    }
    free(level_first);
    free(level_last);
    s->nodes = nodes;
    s->n_nodes = num;
}

ro_scene *ro_scene_create(const rzk_scene_desc *d) {
    ro_scene *s = (ro_scene *)calloc(1, sizeof(ro_scene));
    s->n_surfs = d->n_prims;
    s->n_mats = d->n_mats;
    s->tmin = d->tmin > 0.0f ? d->tmin : 1e-3f;
    s->mats = (rzk_material *)malloc(sizeof(rzk_material) * (d->n_mats > 0 ? d->n_mats : 1));
    if (d->n_mats > 0) memcpy(s->mats, d->mats, sizeof(rzk_material) * d->n_mats);
    s->surfs = (ro_surf *)calloc(d->n_prims > 0 ? d->n_prims : 1, sizeof(ro_surf));
    int nt = 0;
    for (int i = 0; i < d->n_prims; ++i) nt += d->prim_kind[i] == RZK_PRIM_QUAD ? 2 : 1;
    s->n_tris = nt;
    s->tris = (ro_tri *)calloc(nt > 0 ? nt : 1, sizeof(ro_tri));
    s->lights = (int *)calloc(d->n_prims > 0 ? d->n_prims : 1, sizeof(int));
    int k = 0;
    for (int i = 0; i < d->n_prims; ++i) {
        const float *v = d->prim_v + 12 * i;
        ro_surf *sf = &s->surfs[i];
        sf->kind = d->prim_kind[i];
        sf->mat = d->prim_mat[i];
        sf->flags = d->prim_flags ? d->prim_flags[i] : 0;
        sf->first_tri = k;
        sf->light = -1;
        if (sf->mat < 0) {
            sf->emit = crgb(d->prim_emit[3 * i], d->prim_emit[3 * i + 1], d->prim_emit[3 * i + 2]);
            sf->light = s->n_lights;
            s->lights[s->n_lights++] = i;
        }
        if (sf->kind == RZK_PRIM_QUAD) {   /* quad.cc:5-28 */
            v3 p0 = ld(v), p1 = ld(v + 3), p2 = ld(v + 6), p3 = ld(v + 9);
            tri_init(&s->tris[k], p0, p1, p2);
            tri_init(&s->tris[k + 1], p0, p2, p3);
            sf->area = s->tris[k].area + s->tris[k + 1].area;
            sf->t0_ratio = s->tris[k].area / sf->area;
            sf->first = sf->t0_ratio >= 0.5f ? 0 : 1;
            v3 tg = unit(sub(p0, p1));
            s->tris[k].u = tg;
            s->tris[k + 1].u = tg;
            s->tris[k].surf = i;
            s->tris[k + 1].surf = i;
            sf->n_tris = 2;
            k += 2;
        } else {
            tri_init(&s->tris[k], ld(v), ld(v + 3), ld(v + 6));
            s->tris[k].surf = i;
            sf->area = s->tris[k].area;
            sf->t0_ratio = 1.0f;
            sf->first = 0;
            sf->n_tris = 1;
            k += 1;
        }
    }
    /* POWER light selection (scene.cc:185-203, pdf.cc:18-57): luminance of
       radiance * area * pi (area_light.h:93-95). */
    s->light_pdf = (float *)calloc(s->n_lights > 0 ? s->n_lights : 1, sizeof(float));
    s->light_cdf = (float *)calloc(s->n_lights > 0 ? s->n_lights : 1, sizeof(float));
    if (s->n_lights > 0) {
        float sum = 0.0f;
        for (int i = 0; i < s->n_lights; ++i) {
            const ro_surf *sf = &s->surfs[s->lights[i]];
            rgb pw = cscl(cscl(sf->emit, sf->area), A_PI);
            s->light_pdf[i] = cval(pw);
            sum += s->light_pdf[i];
        }
        if (sum == 0.0f) {
            for (int i = 0; i < s->n_lights; ++i) s->light_pdf[i] = s->light_cdf[i] = 0.0f;
        } else {
            for (int i = 0; i < s->n_lights; ++i) s->light_pdf[i] = s->light_pdf[i] / sum;
            s->light_cdf[0] = s->light_pdf[0];
            for (int i = 1; i < s->n_lights; ++i) s->light_cdf[i] = s->light_cdf[i - 1] + s->light_pdf[i];
            s->light_cdf[s->n_lights - 1] = 1.0f;
        }
    }
    bvh_build(s);
    return s;
}

void ro_scene_destroy(ro_scene *s) {
    if (!s) return;
    free(s->tris); free(s->surfs); free(s->mats); free(s->lights);
    free(s->light_pdf); free(s->light_cdf);
    free(s->codes); free(s->sorted_codes); free(s->perm); free(s->nodes);
    free(s);
}

void ro_morton_codes(const ro_scene *s, uint32_t *codes) {
    memcpy(codes, s->codes, sizeof(uint32_t) * (size_t)s->n_tris);
}

void ro_bvh_dump(const ro_scene *s, uint32_t *morton_sorted, int32_t *perm, rzk_bvh_node *nodes) {
    memcpy(morton_sorted, s->sorted_codes, sizeof(uint32_t) * (size_t)s->n_tris);
    memcpy(perm, s->perm, sizeof(int32_t) * (size_t)s->n_tris);
    memcpy(nodes, s->nodes, sizeof(rzk_bvh_node) * (size_t)s->n_nodes);
}

/* ------------------------------------------------------------------------------ */
/* Rays and predicates.                                                            */
/* ------------------------------------------------------------------------------ */
typedef struct { v3 o, d, inv_d, org_inv_d; } ray;

static ray make_ray(v3 o, v3 d_) {   /* ray.h:17-36 */
    ray r;
    r.o = o;
    r.d = unit(d_);
    if (isnan3(r.d)) r.d = mk(0.0f, 0.0f, 0.0f);
    v3 dd = mk(fabsf(r.d.x) < ZERO_EPSILON ? ZERO_EPSILON : r.d.x,
               fabsf(r.d.y) < ZERO_EPSILON ? ZERO_EPSILON : r.d.y,
               fabsf(r.d.z) < ZERO_EPSILON ? ZERO_EPSILON : r.d.z);
    r.inv_d = dvv(mk(1.0f, 1.0f, 1.0f), dd);
    r.org_inv_d = mul(neg(o), r.inv_d);
    return r;
}

/* BoundingBox::hit (boundingbox.h:238-280) */
static inline int box_hit(const float *bmin, const float *bmax, const ray *r, float tmin, float tmax) {
    float x0 = bmin[0] * r->inv_d.x + r->org_inv_d.x;
    float y0 = bmin[1] * r->inv_d.y + r->org_inv_d.y;
    float z0 = bmin[2] * r->inv_d.z + r->org_inv_d.z;
    float x1 = bmax[0] * r->inv_d.x + r->org_inv_d.x;
    float y1 = bmax[1] * r->inv_d.y + r->org_inv_d.y;
    float z1 = bmax[2] * r->inv_d.z + r->org_inv_d.z;
    float tminbox = smax(tmin, smax(smin(x0, x1), smax(smin(y0, y1), smin(z0, z1))));
    float tmaxbox = smin(tmax, smin(smax(x0, x1), smin(smax(y0, y1), smax(z0, z1))));
    return (tminbox <= tmaxbox) && (tmax >= tminbox && tmaxbox >= tmin);
}

/* Triangle::hit (triangle.cc:158-275): returns 1 on a hit with t in [tmin, tmax]. */
static inline int tri_hit(const ro_tri *tr, const ray *r, float tmin, float tmax,
                          float *t_out, float *beta_out, float *gamma_out) {
    v3 p01 = sub(tr->p0, tr->p1);
    float A = p01.x, B = p01.y, C = p01.z;
    v3 p02 = sub(tr->p0, tr->p2);
    float D = p02.x, E = p02.y, F = p02.z;
    float G = r->d.x, H = r->d.y, I = r->d.z;
    v3 p0o = sub(tr->p0, r->o);
    float J = p0o.x, K = p0o.y, L = p0o.z;
    float EIHF = E * I - H * F;
    float GFDI = G * F - D * I;
    float DHEG = D * H - E * G;
    float denom = (A * EIHF + B * GFDI + C * DHEG);
    if (-ZERO_EPSILON < denom && denom < ZERO_EPSILON) return 0;
    float beta = (J * EIHF + K * GFDI + L * DHEG) / denom;
    if (beta < 0.0f || beta > 1.0f) return 0;
    float AKJB = A * K - J * B;
    float JCAL = J * C - A * L;
    float BLKC = B * L - K * C;
    float gamma = (I * AKJB + H * JCAL + G * BLKC) / denom;
    if (gamma < 0.0f || beta + gamma > 1.0f) return 0;
    float t = -(F * AKJB + E * JCAL + D * BLKC) / denom;
    if (t >= tmin && t <= tmax) {
        if (t_out) { *t_out = t; *beta_out = beta; *gamma_out = gamma; }
        return 1;
    }
    return 0;
}

/* AggregateBvh::hit any-hit (aggregate_bvh.cc:452-478), 64-entry stack that drops
   pushes when full (aggregate_bvh.cc:243-281). */
static int any_hit(const ro_scene *s, const ray *r, float tmin, float tmax, ro_counters *c) {
    if (s->n_nodes == 0) return 0;
    const rzk_bvh_node *nodes = s->nodes;
    if (c) { c->rays++; c->root_tests++; }
    if (!box_hit(nodes[0].bmin, nodes[0].bmax, r, tmin, tmax)) return 0;
    int stack[STACK_CAP];
    int top = -1;
    stack[++top] = 0;
    while (top >= 0) {
        const rzk_bvh_node *nd = &nodes[stack[top--]];
        if (nd->left < 0 && nd->right < 0) {
            if (c) c->leaf_tests++;
            if (tri_hit(&s->tris[s->perm[nd->start]], r, tmin, tmax, NULL, NULL, NULL)) return 1;
        } else {
            if (c) c->inner_pops++;
            if (nd->left >= 0 && box_hit(nodes[nd->left].bmin, nodes[nd->left].bmax, r, tmin, tmax)) {
                if (top < STACK_CAP - 1) stack[++top] = nd->left; else if (c) c->overflows++;
            }
            if (nd->right >= 0 && box_hit(nodes[nd->right].bmin, nodes[nd->right].bmax, r, tmin, tmax)) {
                if (top < STACK_CAP - 1) stack[++top] = nd->right; else if (c) c->overflows++;
            }
        }
    }
    return 0;
}

/* Closest hit (aggregate_bvh.cc:402-448): returns sorted slot or -1. */
static int closest_hit(const ro_scene *s, const ray *r, float tmin, float tmax, float *t_out,
                       float *beta_out, float *gamma_out, ro_counters *c) {
    if (s->n_nodes == 0) return -1;
    const rzk_bvh_node *nodes = s->nodes;
    if (c) { c->rays++; c->root_tests++; }
    if (!box_hit(nodes[0].bmin, nodes[0].bmax, r, tmin, tmax)) return -1;
    int stack[STACK_CAP];
    int top = -1;
    stack[++top] = 0;
    int best = -1;
    float bt = RAY_TMAX, bb = 0.0f, bg = 0.0f;
    while (top >= 0) {
        const rzk_bvh_node *nd = &nodes[stack[top--]];
        if (nd->left < 0 && nd->right < 0) {
            if (c) c->leaf_tests++;
            float t, b, g;
            if (tri_hit(&s->tris[s->perm[nd->start]], r, tmin, tmax, &t, &b, &g)) {
                tmax = t;
                bt = t; bb = b; bg = g;
                best = nd->start;
            }
        } else {
            if (c) c->inner_pops++;
            if (nd->left >= 0 && box_hit(nodes[nd->left].bmin, nodes[nd->left].bmax, r, tmin, tmax)) {
                if (top < STACK_CAP - 1) stack[++top] = nd->left; else if (c) c->overflows++;
            }
            if (nd->right >= 0 && box_hit(nodes[nd->right].bmin, nodes[nd->right].bmax, r, tmin, tmax)) {
                if (top < STACK_CAP - 1) stack[++top] = nd->right; else if (c) c->overflows++;
            }
        }
    }
    if (best >= 0) { *t_out = bt; *beta_out = bb; *gamma_out = bg; }
    return best;
}

/* Local geometry of a closest hit: Triangle::fill_hit_record (triangle.cc:277-296) then
   Surface::fill_hit_record (surface.cc:62-96). */
typedef struct {
    v3 p, ng, ns;
    onb uvn;
    int mat, light, surf;
    float t;
} hitgeo;

static void fill_hit(const ro_scene *s, const ray *r, int slot, float t, float beta,
                     float gamma, hitgeo *h) {
    const ro_tri *tr = &s->tris[s->perm[slot]];
    const ro_surf *sf = &s->surfs[tr->surf];
    v3 normal = tr->n;
    /* unit_vector(n0 + beta (n1 - n0) + gamma (n2 - n0)) with n0 = n1 = n2 = n */
    v3 dn = sub(tr->n, tr->n);
    v3 shading = unit(add(add(tr->n, scl(dn, beta)), scl(dn, gamma)));
    if (sf->flags & RZK_SURF_FLIPPED) { normal = neg(normal); shading = neg(shading); }
    if ((sf->flags & RZK_SURF_TWO_SIDED) && dot(shading, r->d) > 0.0f) {
        if (sf->mat >= 0) { shading = neg(shading); normal = neg(normal); }
    }
    h->uvn = onb_from_nu(shading, tr->u);
    h->p = add(r->o, scl(r->d, t));   /* r.org() + t * r.dir() */
    h->ng = normal;
    h->ns = shading;
    h->mat = sf->mat;
    h->light = sf->light;
    h->surf = tr->surf;
    h->t = t;
}

static void hit_to_receiver(const hitgeo *h, const ray *r, rzk_receiver *o) {
    memset(o, 0, sizeof(*o));
    st(o->p, h->p);
    st(o->ng, h->ng);
    st(o->ns, h->ns);
    st(o->wo, neg(r->d));
    st(o->u, h->uvn.u);
    st(o->v, h->uvn.v);
    st(o->n, h->uvn.n);
    o->mat = h->mat;
    o->light = h->light;
    o->flags = 1;
}

static void miss_receiver(rzk_receiver *o) {
    memset(o, 0, sizeof(*o));
    o->mat = -1;
    o->light = -1;
}

void ro_occluded(const ro_scene *s, const float *p, const float *q, int n, uint8_t *out,
                 ro_counters *cnt) {
    for (int i = 0; i < n; ++i) {   /* aggregate.cc:84-90 */
        v3 a = ld(p + 3 * i), b = ld(q + 3 * i);
        ray r = make_ray(a, sub(b, a));
        float tmax = len(sub(b, a)) - s->tmin;
        out[i] = (uint8_t)any_hit(s, &r, s->tmin, tmax, cnt);
    }
}

void ro_closest(const ro_scene *s, const float *o, const float *d, int n, float *t_out,
                rzk_receiver *recv, ro_counters *cnt) {
    for (int i = 0; i < n; ++i) {
        ray r = make_ray(ld(o + 3 * i), ld(d + 3 * i));
        float t, b, g;
        int slot = closest_hit(s, &r, s->tmin, RAY_TMAX, &t, &b, &g, cnt);
        if (slot < 0) { t_out[i] = -1.0f; miss_receiver(&recv[i]); continue; }
        hitgeo h;
        fill_hit(s, &r, slot, t, b, g, &h);
        t_out[i] = t;
        hit_to_receiver(&h, &r, &recv[i]);
    }
}

/* ------------------------------------------------------------------------------ */
/* Camera.                                                                         */
/* ------------------------------------------------------------------------------ */
void ro_camera_setup(const float eye[3], const float lookat[3], const float up[3],
                     float fov_deg, int width, int height, float film_w, float film_h,
                     rzk_camera *out) {
    memset(out, 0, sizeof(*out));
    /* Camera::focal_length_from_fov (camera.h:228-230) */
    float focal = film_h / (2.0f * tanf(fov_deg / 2 * DEGREE_TO_RADIAN));
    v3 e = ld(eye), l = ld(lookat), u = ld(up);
    onb o = onb_from_nv(sub(e, l), u);   /* camera.cc:25 */
    st(out->eye, e);
    st(out->u, o.u);
    st(out->v, o.v);
    st(out->n, o.n);
    out->focal = focal;
    float W = (float)width, H = (float)height;
    float inv2 = 1.0f / 2.0f;            /* Size2::operator/(Float) (size.h:26-29) */
    out->cop[0] = W * inv2;
    out->cop[1] = H * inv2;
    out->scale[0] = W / film_w;          /* Size2::operator/(Size2) */
    out->scale[1] = H / film_h;
    out->width = width;
    out->height = height;
}

static ray camera_ray(const rzk_camera *c, int i, int j) {   /* camera.cc:52-65 */
    float H = (float)c->height;
    float px = (float)j + 0.5f;
    float py = H - 1 - (float)i + 0.5f;
    float fx = (px - c->cop[0]) / c->scale[0];
    float fy = (py - c->cop[1]) / c->scale[1];
    onb o = {ld(c->u), ld(c->v), ld(c->n)};
    v3 dir = unit(l2w(&o, mk(fx, fy, -c->focal)));
    return make_ray(ld(c->eye), dir);
}

void ro_primary_rays(const rzk_camera *cam, float *o, float *d) {
    for (int i = 0; i < cam->height; ++i)
        for (int j = 0; j < cam->width; ++j) {
            ray r = camera_ray(cam, i, j);
            st(o + 3 * (i * cam->width + j), r.o);
            st(d + 3 * (i * cam->width + j), r.d);
        }
}

typedef struct {
    const ro_scene *s;
    const rzk_camera *cam;
    rzk_receiver *out;
    int row0, row1;
} prim_job;

static void *primary_worker(void *arg) {
    prim_job *jb = (prim_job *)arg;
    for (int i = jb->row0; i < jb->row1; ++i)
        for (int j = 0; j < jb->cam->width; ++j) {
            ray r = camera_ray(jb->cam, i, j);
            float t, b, g;
            rzk_receiver *o = &jb->out[i * jb->cam->width + j];
            int slot = closest_hit(jb->s, &r, jb->s->tmin, RAY_TMAX, &t, &b, &g, NULL);
            if (slot < 0) { miss_receiver(o); continue; }
            hitgeo h;
            fill_hit(jb->s, &r, slot, t, b, g, &h);
            hit_to_receiver(&h, &r, o);
        }
    return NULL;
}

void ro_primary(const ro_scene *s, const rzk_camera *cam, rzk_receiver *out, int n_threads) {
    if (n_threads < 1) n_threads = 1;
    pthread_t th[256];
    prim_job jobs[256];
    if (n_threads > 256) n_threads = 256;
    int H = cam->height;
    for (int t = 0; t < n_threads; ++t) {
        jobs[t].s = s; jobs[t].cam = cam; jobs[t].out = out;
        jobs[t].row0 = (int)((int64_t)H * t / n_threads);
        jobs[t].row1 = (int)((int64_t)H * (t + 1) / n_threads);
        if (n_threads == 1) primary_worker(&jobs[t]);
        else pthread_create(&th[t], NULL, primary_worker, &jobs[t]);
    }
    if (n_threads > 1) for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------------------ */
/* BRDFs, float (lambertian.cc:63-68, phong.cc:74-87, ward.cc:104-116).             */
/* ------------------------------------------------------------------------------ */
static rgb brdf_eval(const rzk_material *m, const onb *uvn, v3 wo, v3 wi) {
    rgb kd = crgb(m->kd[0], m->kd[1], m->kd[2]);
    rgb ks = crgb(m->ks[0], m->ks[1], m->ks[2]);
    if (m->type == RZK_BSDF_WARD) {
        float ax = m->p0, ay = m->p1;
        float ax2 = ax * ax, ay2 = ay * ay;
        float inv4 = 1.0f / (4 * A_PI * ax * ay);   /* ward.cc:5-9 */
        v3 lwi = w2l(uvn, wi), lwo = w2l(uvn, wo);
        if (lwi.z <= ZERO_EPSILON || lwo.z <= ZERO_EPSILON) return BLACK;
        v3 wh = add(lwi, lwo);
        float expo = expf(-(wh.x * wh.x / ax2 + wh.y * wh.y / ay2) / (wh.z * wh.z));
        rgb spec = cscl(cdiv(cscl(ks, inv4), sqrtf(lwi.z * lwo.z)), expo);
        return cadd(cscl(kd, INV_PI), spec);
    }
    if (dot(wi, uvn->n) <= ZERO_EPSILON || dot(wo, uvn->n) <= ZERO_EPSILON) return BLACK;
    rgb b = cscl(kd, INV_PI);
    if (m->type == RZK_BSDF_PHONG) {
        float n = m->p0;
        v3 nn = uvn->n;
        v3 wr = sub(scl(nn, 2 * dot(wi, nn)), wi);
        float ca = dot(wo, wr);
        if (ca > 0.0f) b = cadd(b, cscl(cscl(cscl(ks, (n + 2)), INV_2PI), powf(ca, n)));
    }
    return b;
}

/* FormFactor::form_factor_abs (form_factor.h:11-21) */
static inline float form_factor_abs(v3 p, v3 pn, v3 q, v3 qn) {
    v3 pq = sub(q, p);
    float d1 = dot(pn, pq);
    float d2 = -dot(qn, pq);
    float dpq = dot(pq, pq);
    return fabsf((d1 * d2) / (dpq * dpq));
}

/* RadianceTerms + clamp_term (vpl_interface.h:50-123, vpl.cc:214-230) */
static rgb radiance_terms(rgb power, rgb sb, rgb lb, float G, int mode, float tau, rgb *no_clamp) {
    rgb r, nc;
    switch (mode) {
        case RZK_CLAMP_REFLECTIVITY: {
            rgb refl = cmul(cscl(sb, G), lb);
            float lum = cval(refl);
            if (lum > tau) r = cmul(cscl(refl, tau / lum), power);
            else r = cmul(refl, power);
            nc = cmul(cmul(cscl(power, G), sb), lb);
            break;
        }
        case RZK_CLAMP_RADIANCE: {
            nc = cmul(cmul(cscl(power, G), sb), lb);
            float br = cval(nc);
            if (br > tau) r = cscl(nc, tau / br);
            else r = nc;
            break;
        }
        case RZK_CLAMP_FORM_FACTOR: {
            if (G > tau) r = cmul(cscl(cmul(lb, sb), tau), power);
            else r = cmul(cscl(cmul(lb, sb), G), power);
            nc = cmul(cmul(cscl(power, G), sb), lb);
            break;
        }
        default:
            nc = cmul(cmul(cscl(power, G), sb), lb);
            r = nc;
            break;
    }
    if (no_clamp) *no_clamp = nc;
    return r;
}

typedef struct { v3 p, ng, ns, wo; onb uvn; int mat; } recv_t;
typedef struct { v3 p, n, wi; onb uvn; rgb power; int mat; } vpl_t;

static recv_t load_recv(const rzk_receiver *r) {
    recv_t o;
    o.p = ld(r->p); o.ng = ld(r->ng); o.ns = ld(r->ns); o.wo = ld(r->wo);
    o.uvn.u = ld(r->u); o.uvn.v = ld(r->v); o.uvn.n = ld(r->n);
    o.mat = r->mat;
    return o;
}
static vpl_t load_vpl(const rzk_vpl *v) {
    vpl_t o;
    o.p = ld(v->p); o.n = ld(v->n); o.wi = ld(v->wi);
    o.uvn.u = ld(v->u); o.uvn.v = ld(v->v); o.uvn.n = ld(v->nn);
    o.power = crgb(v->contrib[0], v->contrib[1], v->contrib[2]);
    o.mat = v->mat;
    return o;
}

/* Shading part of gather_point after the visibility test (vpl.cc:676-687). */
static rgb shade_pair(const ro_scene *s, const recv_t *r, const vpl_t *l, int mode, float tau,
                      rgb *no_clamp) {
    float G = form_factor_abs(r->p, r->ns, l->p, l->n);
    v3 wi = unit(sub(l->p, r->p));
    rgb sb = brdf_eval(&s->mats[r->mat], &r->uvn, r->wo, wi);
    rgb lb = l->mat >= 0 ? brdf_eval(&s->mats[l->mat], &l->uvn, l->wi, neg(wi)) : WHITE;
    return radiance_terms(l->power, sb, lb, G, mode, tau, no_clamp);
}

static int occluded_pair(const ro_scene *s, v3 p, v3 q, ro_counters *c) {
    ray r = make_ray(p, sub(q, p));
    float tmax = len(sub(q, p)) - s->tmin;
    return any_hit(s, &r, s->tmin, tmax, c);
}

/* ---- double-precision shading for the FP64 reference image ---- */
typedef struct { double x, y, z; } d3;
static inline d3 dmk(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static inline d3 dfv(v3 a) { return dmk(a.x, a.y, a.z); }
static inline d3 dsub(d3 a, d3 b) { return dmk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 dadd(d3 a, d3 b) { return dmk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 dscl(d3 a, double t) { return dmk(a.x * t, a.y * t, a.z * t); }
static inline double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 dunit(d3 a) { double l = sqrt(ddot(a, a)); return dmk(a.x / l, a.y / l, a.z / l); }
typedef struct { double r, g, b; } drgb;

static drgb brdf_eval_d(const rzk_material *m, const onb *uvn, d3 wo, d3 wi) {
    drgb out = {0, 0, 0};
    d3 U = dfv(uvn->u), V = dfv(uvn->v), N = dfv(uvn->n);
    const double inv_pi = 1.0 / 3.14159265358979323846;
    if (m->type == RZK_BSDF_WARD) {
        double ax = m->p0, ay = m->p1;
        d3 lwi = dmk(ddot(U, wi), ddot(V, wi), ddot(N, wi));
        d3 lwo = dmk(ddot(U, wo), ddot(V, wo), ddot(N, wo));
        if (lwi.z <= 1e-6 || lwo.z <= 1e-6) return out;
        d3 wh = dadd(lwi, lwo);
        double expo = exp(-(wh.x * wh.x / (ax * ax) + wh.y * wh.y / (ay * ay)) / (wh.z * wh.z));
        double sp = 1.0 / (4.0 * 3.14159265358979323846 * ax * ay) / sqrt(lwi.z * lwo.z) * expo;
        out.r = m->kd[0] * inv_pi + m->ks[0] * sp;
        out.g = m->kd[1] * inv_pi + m->ks[1] * sp;
        out.b = m->kd[2] * inv_pi + m->ks[2] * sp;
        return out;
    }
    if (ddot(wi, N) <= 1e-6 || ddot(wo, N) <= 1e-6) return out;
    out.r = m->kd[0] * inv_pi; out.g = m->kd[1] * inv_pi; out.b = m->kd[2] * inv_pi;
    if (m->type == RZK_BSDF_PHONG) {
        double n = m->p0;
        d3 wr = dsub(dscl(N, 2.0 * ddot(wi, N)), wi);
        double ca = ddot(wo, wr);
        if (ca > 0.0) {
            double sp = (n + 2.0) / (2.0 * 3.14159265358979323846) * pow(ca, n);
            out.r += m->ks[0] * sp; out.g += m->ks[1] * sp; out.b += m->ks[2] * sp;
        }
    }
    return out;
}

static drgb shade_pair_d(const ro_scene *s, const recv_t *r, const vpl_t *l, int mode, double tau) {
    d3 p = dfv(r->p), pn = dfv(r->ns), q = dfv(l->p), qn = dfv(l->n);
    d3 pq = dsub(q, p);
    double dpq = ddot(pq, pq);
    double G = fabs((ddot(pn, pq) * -ddot(qn, pq)) / (dpq * dpq));
    d3 wi = dunit(pq);
    drgb sb = brdf_eval_d(&s->mats[r->mat], &r->uvn, dfv(r->wo), wi);
    drgb lb = {1, 1, 1};
    if (l->mat >= 0) lb = brdf_eval_d(&s->mats[l->mat], &l->uvn, dfv(l->wi), dscl(wi, -1.0));
    drgb P = {l->power.r, l->power.g, l->power.b};
    drgb nc = {P.r * G * sb.r * lb.r, P.g * G * sb.g * lb.g, P.b * G * sb.b * lb.b};
    drgb out = nc;
    if (mode == RZK_CLAMP_RADIANCE) {
        double br = sqrt(nc.r * nc.r + nc.g * nc.g + nc.b * nc.b);
        if (br > tau) { double w = tau / br; out.r *= w; out.g *= w; out.b *= w; }
    } else if (mode == RZK_CLAMP_FORM_FACTOR) {
        if (G > tau) { double w = tau / G; out.r *= w; out.g *= w; out.b *= w; }
    } else if (mode == RZK_CLAMP_REFLECTIVITY) {
        double rr = G * sb.r * lb.r, rg = G * sb.g * lb.g, rb = G * sb.b * lb.b;
        double lum = sqrt(rr * rr + rg * rg + rb * rb);
        if (lum > tau) { double w = tau / lum; out.r *= w; out.g *= w; out.b *= w; }
    }
    return out;
}

/* ------------------------------------------------------------------------------ */
/* Gather (vpl.cc:661-688 per pair; light_transport_matrix.cc:16-48 for matrices).  */
/* ------------------------------------------------------------------------------ */
typedef struct {
    const ro_scene *s;
    const rzk_receiver *recv;
    const vpl_t *vpls;
    int n_vpl, r0, r1, mode, cull;
    float tau, scale;
    float *out32;
    double *out64;
    ro_counters cnt;
} gather_job;

static void *gather_worker(void *arg) {
    gather_job *jb = (gather_job *)arg;
    const ro_scene *s = jb->s;
    for (int i = jb->r0; i < jb->r1; ++i) {
        recv_t r = load_recv(&jb->recv[i]);
        rgb sum = BLACK;
        double sr = 0, sg = 0, sbl = 0;
        if (r.mat >= 0) {
            for (int j = 0; j < jb->n_vpl; ++j) {
                const vpl_t *l = &jb->vpls[j];
                jb->cnt.pairs++;
                rgb L = shade_pair(s, &r, l, jb->mode, jb->tau, NULL);
                if (jb->cull && cblack(L)) {
                    /* a zero shading term stays zero whatever the visibility */
                    jb->cnt.culled++;
                    if (jb->out64) {
                        drgb D = shade_pair_d(s, &r, l, jb->mode, jb->tau);
                        (void)D;   /* the double term of a culled pair is not added */
                    }
                    continue;
                }
                if (occluded_pair(s, r.p, l->p, &jb->cnt)) continue;
                sum = cadd(sum, L);
                if (jb->out64) {
                    drgb D = shade_pair_d(s, &r, l, jb->mode, jb->tau);
                    sr += D.r; sg += D.g; sbl += D.b;
                }
            }
        }
        if (jb->out32) {
            jb->out32[3 * i] = sum.r * jb->scale;
            jb->out32[3 * i + 1] = sum.g * jb->scale;
            jb->out32[3 * i + 2] = sum.b * jb->scale;
        }
        if (jb->out64) {
            jb->out64[3 * i] = sr * jb->scale;
            jb->out64[3 * i + 1] = sg * jb->scale;
            jb->out64[3 * i + 2] = sbl * jb->scale;
        }
    }
    return NULL;
}

void ro_gather(const ro_scene *s, const rzk_receiver *recv, int n_recv, const rzk_vpl *vpls,
               int n_vpl, int clamp_mode, float tau, float scale, int cull, float *out_f32,
               double *out_f64, int n_threads, ro_counters *cnt) {
    vpl_t *vv = (vpl_t *)malloc(sizeof(vpl_t) * (n_vpl > 0 ? n_vpl : 1));
    for (int j = 0; j < n_vpl; ++j) vv[j] = load_vpl(&vpls[j]);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > 256) n_threads = 256;
    gather_job *jobs = (gather_job *)calloc(n_threads, sizeof(gather_job));
    pthread_t *th = (pthread_t *)calloc(n_threads, sizeof(pthread_t));
    for (int t = 0; t < n_threads; ++t) {
        gather_job *jb = &jobs[t];
        jb->s = s; jb->recv = recv; jb->vpls = vv; jb->n_vpl = n_vpl;
        jb->r0 = (int)((int64_t)n_recv * t / n_threads);
        jb->r1 = (int)((int64_t)n_recv * (t + 1) / n_threads);
        jb->mode = clamp_mode; jb->tau = tau; jb->scale = scale; jb->cull = cull;
        jb->out32 = out_f32; jb->out64 = out_f64;
        if (n_threads == 1) gather_worker(jb);
        else pthread_create(&th[t], NULL, gather_worker, jb);
    }
    if (n_threads > 1) for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
    if (cnt) {
        for (int t = 0; t < n_threads; ++t) {
            cnt->rays += jobs[t].cnt.rays; cnt->root_tests += jobs[t].cnt.root_tests;
            cnt->inner_pops += jobs[t].cnt.inner_pops; cnt->leaf_tests += jobs[t].cnt.leaf_tests;
            cnt->overflows += jobs[t].cnt.overflows; cnt->pairs += jobs[t].cnt.pairs;
            cnt->culled += jobs[t].cnt.culled;
        }
    }
    free(jobs); free(th); free(vv);
}

void ro_gather_pairs(const ro_scene *s, const rzk_receiver *recv, int n_recv,
                     const rzk_vpl *vpls, int n_vpl, int clamp_mode, float tau,
                     float *pair_rgb, uint8_t *pair_vis) {
    for (int j = 0; j < n_vpl; ++j) {
        vpl_t l = load_vpl(&vpls[j]);
        for (int i = 0; i < n_recv; ++i) {
            size_t k = (size_t)j * n_recv + i;
            recv_t r = load_recv(&recv[i]);
            rgb L = BLACK;
            int vis = 0;
            if (r.mat >= 0 && !occluded_pair(s, r.p, l.p, NULL)) {
                vis = 1;
                L = shade_pair(s, &r, &l, clamp_mode, tau, NULL);
            }
            if (pair_rgb) { pair_rgb[3 * k] = L.r; pair_rgb[3 * k + 1] = L.g; pair_rgb[3 * k + 2] = L.b; }
            if (pair_vis) pair_vis[k] = (uint8_t)vis;
        }
    }
}

void ro_incident(const ro_scene *s, const rzk_receiver *recv, int n_recv,
                 const rzk_vpl *vpls, int n_vpl, int clamp_mode, float tau, float *pair_rgb) {
    for (int j = 0; j < n_vpl; ++j) {
        vpl_t l = load_vpl(&vpls[j]);
        for (int i = 0; i < n_recv; ++i) {
            recv_t r = load_recv(&recv[i]);
            /* incident_radiance uses the geometric normal r.n (vpl.cc:413) */
            float G = form_factor_abs(r.p, r.ng, l.p, l.n);
            v3 wi = unit(sub(l.p, r.p));
            rgb lb = l.mat >= 0 ? brdf_eval(&s->mats[l.mat], &l.uvn, l.wi, neg(wi)) : WHITE;
            rgb L = radiance_terms(l.power, WHITE, lb, G, clamp_mode, tau, NULL);
            size_t k = (size_t)j * n_recv + i;
            pair_rgb[3 * k] = L.r; pair_rgb[3 * k + 1] = L.g; pair_rgb[3 * k + 2] = L.b;
        }
    }
}

void ro_brdf_eval(const ro_scene *s, const int32_t *mat, const float *uvn9, const float *wo,
                  const float *wi, int n, float *out) {
    for (int i = 0; i < n; ++i) {
        onb o = {ld(uvn9 + 9 * i), ld(uvn9 + 9 * i + 3), ld(uvn9 + 9 * i + 6)};
        rgb c = brdf_eval(&s->mats[mat[i]], &o, ld(wo + 3 * i), ld(wi + 3 * i));
        out[3 * i] = c.r; out[3 * i + 1] = c.g; out[3 * i + 2] = c.b;
    }
}

double ro_mean_contribution(const ro_scene *s, const rzk_receiver *recv,
                            const int32_t *recv_idx, const int32_t *vpl_idx, int n_pairs,
                            const rzk_vpl *vpls) {
    double acc = 0.0;
    for (int k = 0; k < n_pairs; ++k) {
        recv_t r = load_recv(&recv[recv_idx[k]]);
        vpl_t l = load_vpl(&vpls[vpl_idx[k]]);
        if (r.mat < 0) continue;
        if (occluded_pair(s, r.p, l.p, NULL)) continue;
        rgb nc;
        radiance_terms(l.power, BLACK, BLACK, 0.0f, RZK_CLAMP_NONE, 0.0f, NULL);
        shade_pair(s, &r, &l, RZK_CLAMP_NONE, 0.0f, &nc);
        acc += cval(nc);
    }
    return n_pairs > 0 ? acc / n_pairs : 0.0;
}

/* ------------------------------------------------------------------------------ */
/* Random stream: Philox4x32-10.                                                    */
/* ------------------------------------------------------------------------------ */
static inline void philox_round(uint32_t c[4], const uint32_t k[2]) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k[0];
    uint32_t n2 = hi0 ^ c[3] ^ k[1];
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
}

uint32_t ro_draw_u32(uint32_t seed, uint32_t stream, uint32_t path, uint32_t d) {
    uint32_t c[4] = {d >> 2, path, stream, 0x52454e5au};
    uint32_t k[2] = {seed, 0x4b5a4f52u};
    for (int r = 0; r < 10; ++r) {
        philox_round(c, k);
        k[0] += 0x9E3779B9u;
        k[1] += 0xBB67AE85u;
    }
    return c[d & 3];
}

typedef struct { uint32_t seed, stream, path, d; } rng_t;
/* Random::operator() and rand_exclude_01 (random.h:60-71) */
static inline float rnd(rng_t *g) {
    uint32_t r = ro_draw_u32(g->seed, g->stream, g->path, g->d++);
    return (r & 0x00ffffffu) * INV_TWO_POW_24;
}
static inline float rnd_ex01(rng_t *g) {
    uint32_t r = ro_draw_u32(g->seed, g->stream, g->path, g->d++);
    return (r & 0x00ffffffu) * INV_TWO_POW_24 + INV_TWO_POW_25;
}

/* ------------------------------------------------------------------------------ */
/* BRDF sampling (lambertian.cc:5-26, phong.cc:21-72, ward.cc:26-99) and pdfs.       */
/* ------------------------------------------------------------------------------ */
static float brdf_pdf(const rzk_material *m, const onb *uvn, v3 wo, v3 wi, float rho_d, float rho_s) {
    if (dot(wi, uvn->n) <= ZERO_EPSILON || dot(wo, uvn->n) <= ZERO_EPSILON) return 0.0f;
    if (m->type == RZK_BSDF_LAMBERTIAN) return dot(uvn->n, wi) * INV_PI;
    if (m->type == RZK_BSDF_PHONG) {   /* phong.cc:89-103 */
        float n = m->p0;
        v3 nn = uvn->n;
        float pdf = rho_d * (dot(nn, wi) * INV_PI);
        v3 wr = sub(scl(nn, 2 * dot(wi, nn)), wi);
        float ca = dot(wo, wr);
        if (ca > 0.0f) pdf += rho_s * (n + 1) * INV_2PI * powf(ca, n);
        return pdf;
    }
    /* ward.cc:118-134 */
    float ax = m->p0, ay = m->p1;
    float ax2 = ax * ax, ay2 = ay * ay;
    float inv4 = 1.0f / (4 * A_PI * ax * ay);
    float z = dot(uvn->n, wi);
    v3 wh = unit(w2l(uvn, add(wi, wo)));
    float expo = expf(-(wh.x * wh.x / ax2 + wh.y * wh.y / ay2) / (wh.z * wh.z));
    float ct = wh.z;
    v3 lwo = unit(w2l(uvn, wo));
    float ct3 = ct * ct * ct;
    return rho_d * (z * INV_PI) + rho_s * (inv4 / (dot(wh, lwo) * ct3) * expo);
}

static void rho_terms(const rzk_material *m, float *rho_d, float *rho_s) {
    /* ModifiedPhong / Ward constructors (phong.cc:6-16, ward.cc:5-24) */
    float kd = smax(smax(m->kd[0], m->kd[1]), m->kd[2]);
    float ks = smax(smax(m->ks[0], m->ks[1]), m->ks[2]);
    /* Rgb::max keeps the first of equals: tmp = r; if (g > tmp) ...; same as above */
    float rd = m->kd[0]; if (m->kd[1] > rd) rd = m->kd[1]; if (m->kd[2] > rd) rd = m->kd[2];
    float rs = m->ks[0]; if (m->ks[1] > rs) rs = m->ks[1]; if (m->ks[2] > rs) rs = m->ks[2];
    (void)kd; (void)ks;
    float total = rd + rs;
    if (total > 0.0f) { rd /= total; rs /= total; }
    *rho_d = rd; *rho_s = rs;
}

static v3 cosine_dir(const onb *uvn, float sx, float sy, float *z_out) {
    float phi = TWO_PI * sx;
    float sin_theta = sqrtf(sy);
    float x = sin_theta * cosf(phi);
    float y = sin_theta * sinf(phi);
    float z = sqrtf(1 - sin_theta * sin_theta);
    *z_out = z;
    return unit(l2w(uvn, mk(x, y, z)));
}

/* Material::sample; returns the BRDF value, pdf through *pdf (0 on rejection). */
static rgb brdf_sample(const rzk_material *m, const onb *uvn, v3 wo, rng_t *g, v3 *wi, float *pdf) {
    if (dot(wo, uvn->n) <= ZERO_EPSILON) { *wi = mk(0, 0, 0); *pdf = 0.0f; return BLACK; }
    if (m->type == RZK_BSDF_LAMBERTIAN) {
        float sx = rnd(g), sy = rnd(g);
        float z;
        *wi = cosine_dir(uvn, sx, sy, &z);
        *pdf = z * INV_PI;
        return cscl(crgb(m->kd[0], m->kd[1], m->kd[2]), INV_PI);
    }
    float rho_d, rho_s;
    rho_terms(m, &rho_d, &rho_s);
    float eps = rnd(g);
    if (eps < rho_d) {
        float sx = rnd(g), sy = rnd(g);
        float phi = TWO_PI * sx;
        float sin_theta = sqrtf(sy);
        float x = sin_theta * cosf(phi);
        float y = sin_theta * sinf(phi);
        float z = m->type == RZK_BSDF_PHONG ? sqrtf(1.0f - sin_theta * sin_theta)
                                            : sqrtf(1 - sin_theta * sin_theta);
        *wi = unit(l2w(uvn, mk(x, y, z)));
    } else if (m->type == RZK_BSDF_PHONG) {   /* phong.cc:46-68 */
        float sx = rnd(g), sy = rnd(g);
        onb o = onb_from_nu(wo, uvn->n);
        float phi = TWO_PI * sx;
        float alpha = acosf(powf(sy, 1.0f / (m->p0 + 1)));
        /* Onb::spherical_to_world (onb.cc:157-164) */
        float st_ = sinf(alpha), ct_ = cosf(alpha), sp = sinf(phi), cp = cosf(phi);
        v3 wr = l2w(&o, mk(st_ * cp, st_ * sp, ct_));
        v3 nn = uvn->n;
        float d = dot(wr, nn);
        if (d < 0.0f) { *wi = mk(0, 0, 0); *pdf = 0.0f; return BLACK; }
        *wi = sub(scl(nn, 2 * d), wr);
    } else {                                    /* ward.cc:48-97 */
        /* Vec2 sampler(rd.rand_exclude_01(), rd.rand_exclude_01()) (ward.cc:58): C++ leaves
           argument order unspecified; g++ on x86-64 evaluates right to left, so the
           second coordinate takes the first draw. */
        float sy = rnd_ex01(g);
        float sx = rnd_ex01(g);
        float ax = m->p0, ay = m->p1;
        float ax2 = ax * ax, ay2 = ay * ay, ay_ax = ay / ax;
        v3 lwo = unit(w2l(uvn, wo));
        float angle = TWO_PI * sx;
        float phi = atanf(ay_ax * tanf(angle));
        if (sinf(phi) * sinf(angle) < 0 || cosf(phi) * cosf(angle) < 0) phi += A_PI;
        float cp = cosf(phi), sp = sinf(phi);
        float theta = atanf(sqrtf(-logf(sy) / (cp * cp / ax2 + sp * sp / ay2)));
        float st_ = sinf(theta), ct_ = cosf(theta);
        v3 wh = mk(st_ * cp, st_ * sp, ct_);
        v3 lwi = sub(scl(wh, 2 * dot(lwo, wh)), lwo);
        *wi = l2w(uvn, lwi);
    }
    *pdf = brdf_pdf(m, uvn, wo, *wi, rho_d, rho_s);
    return brdf_eval(m, uvn, wo, *wi);
}

/* Closest hit with the local geometry, for the light-path tracer. */
static int trace_closest(const ro_scene *s, const ray *r, hitgeo *h) {
    float t, b, g;
    int slot = closest_hit(s, r, s->tmin, RAY_TMAX, &t, &b, &g, NULL);
    if (slot < 0) return 0;
    fill_hit(s, r, slot, t, b, g, h);
    return 1;
}

static void push_vpl(rzk_vpl *out, int cap, int *n, const hitgeo *h, v3 wi, rgb contrib,
                     int bounce, int path) {
    if (*n < cap) {
        rzk_vpl *o = &out[*n];
        memset(o, 0, sizeof(*o));
        st(o->p, h->p);
        st(o->n, h->ns);
        st(o->u, h->uvn.u);
        st(o->v, h->uvn.v);
        st(o->nn, h->uvn.n);
        st(o->wi, wi);
        o->contrib[0] = contrib.r; o->contrib[1] = contrib.g; o->contrib[2] = contrib.b;
        o->mat = h->mat;
        o->bounce = bounce;
        o->path = path;
    }
    (*n)++;
}

int ro_vpl_generate(const ro_scene *s, uint32_t seed, int n_particles, int max_bounce,
                    rzk_vpl *out, int cap) {
    int n = 0;
    if (s->n_lights == 0) return 0;
    for (int k = 0; k < n_particles; ++k) {
        rng_t g = {seed, 0u, (uint32_t)k, 0u};
        /* SubpathGenerator::sample_direct_vertex (path.cc:171-334), area light branch */
        float sx = rnd(&g);
        (void)rnd(&g);                                 /* Vec2::random draws two */
        int li = -1;
        float light_pdf = 0.0f;
        for (int i = 0; i < s->n_lights; ++i)
            if (sx < s->light_cdf[i]) { li = i; light_pdf = s->light_pdf[i]; break; }
        if (li < 0) continue;
        const ro_surf *ls = &s->surfs[s->lights[li]];
        /* AreaLight::sample (area_light.cc:27-46): Surface::sample -> Quad / Triangle */
        v3 q, qn;
        float pdf_q;
        {
            int which = 0;
            float pdf_sel = 1.0f;
            if (ls->kind == RZK_PRIM_QUAD) {
                float t = rnd(&g);
                if (t <= ls->t0_ratio) { which = 0; pdf_sel = ls->t0_ratio; }
                else { which = 1; pdf_sel = 1.0f - ls->t0_ratio; }
            }
            const ro_tri *tr = &s->tris[ls->first_tri + which];
            float u0 = rnd(&g), u1 = rnd(&g);          /* triangle.cc:296-306 */
            float tmp = sqrtf(1.0f - u0);
            float b = 1.0f - tmp;
            float c = u1 * tmp;
            float a = 1.0f - b - c;
            q = add(add(scl(tr->p0, a), scl(tr->p1, b)), scl(tr->p2, c));
            qn = tr->n;
            float pdf_t = 1.0f / tr->area;
            pdf_q = ls->kind == RZK_PRIM_QUAD ? pdf_sel * pdf_t : pdf_t;
            if (ls->flags & RZK_SURF_FLIPPED) qn = neg(qn);
        }
        float cx = rnd(&g), cy = rnd(&g);
        float phi = TWO_PI * cx;
        float sin_theta = sqrtf(cy);
        float x = sin_theta * cosf(phi);
        float y = sin_theta * sinf(phi);
        float z = sqrtf(1.f - sin_theta * sin_theta);
        /* Surface::get_basis uses the shape's unflipped normal and tangent (surface.h:170-176);
           Quad::normal / tangent come from its larger triangle (quad.h:114-120) */
        const ro_tri *bt = &s->tris[ls->first_tri + ls->first];
        onb luvn = onb_from_nu(bt->n, bt->u);
        v3 wo_q = unit(l2w(&luvn, mk(x, y, z)));
        rgb Le = ls->emit;
        float pdf_wo = z * INV_PI;
        if (pdf_q <= 0.0f || pdf_wo <= 0.0f) continue;
        float acc_pdf = light_pdf;
        acc_pdf *= pdf_q * pdf_wo;
        rgb contrib = cdiv(cscl(Le, fabsf(dot(qn, wo_q))), acc_pdf);
        rgb v1_thr = cscl(Le, fabsf(dot(qn, wo_q)));
        float v1_pdf = pdf_wo;
        ray r = make_ray(q, wo_q);
        hitgeo h;
        if (!trace_closest(s, &r, &h)) continue;
        if (h.light >= 0) continue;
        float cosr = fabsf(dot(h.ns, r.d)) / (h.t * h.t);
        v1_thr = cscl(v1_thr, cosr);
        v1_pdf *= cosr;
        acc_pdf *= cosr;
        (void)v1_thr; (void)v1_pdf;
        v3 actual_wi = neg(r.d);
        /* VplGenerator::generate_vpl (vpl_generator.cc:127-181) */
        if (acc_pdf == 0.0f) continue;
        if (max_bounce <= 1) continue;
        push_vpl(out, cap, &n, &h, actual_wi, contrib, 1, k);
        const rzk_material *m = &s->mats[h.mat];
        v3 wi;
        float pdf_wi;
        rgb brdf = brdf_sample(m, &h.uvn, actual_wi, &g, &wi, &pdf_wi);
        if (pdf_wi <= 0.0f || cblack(brdf)) continue;
        float cs = fabsf(dot(wi, h.ns));
        rgb T = cdiv(cscl(cmul(contrib, brdf), cs), pdf_wi);
        /* VplGenerator::trace_vpl (vpl_generator.cc:43-110), iterated */
        ray rr = make_ray(h.p, wi);
        for (int bounce = 2; bounce < max_bounce; ++bounce) {
            hitgeo hh;
            if (!trace_closest(s, &rr, &hh)) break;
            if (hh.light >= 0) break;
            v3 wi2 = unit(neg(rr.d));
            push_vpl(out, cap, &n, &hh, wi2, T, bounce, k);
            float continuation = 1.0f;
            if (bounce >= 4) {
                /* Material::get_representative_color() is white for BsdfMaterial */
                continuation = smin(1.0f, 0.99f);
                if (rnd(&g) > continuation) break;
            }
            v3 wo;
            float pdf;
            rgb b2 = brdf_sample(&s->mats[hh.mat], &hh.uvn, wi2, &g, &wo, &pdf);
            if (pdf <= 0.0f || cblack(b2)) break;
            pdf *= continuation;
            rgb f = cdiv(cscl(b2, fabsf(dot(hh.ns, wo))), pdf);
            T = cmul(T, f);
            rr = make_ray(hh.p, wo);
        }
    }
    return n;
}

/* ------------------------------------------------------------------------------ */
/* Light-transport-matrix statistics and column clustering.                        */
/* Matrix layout: column-major [cols][rows][3] (MatrixC<Rgb>, matrix_c.h:177-184).  */
/* ------------------------------------------------------------------------------ */

/* LightTransportMatrix::generate_alphas_for_clustering (light_transport_matrix.cc:72-106)
   and get_column_norms (light_transport_matrix.cc:118-130). */
void ro_ltm_alphas(const float *mat, int rows, int cols, float *alphas, float *norms) {
    float *R = (float *)malloc(sizeof(float) * (size_t)rows * cols + 4);
    for (int j = 0; j < cols; ++j)
        for (int i = 0; i < rows; ++i) {      /* MatrixC<Rgb>::flatten_magnitude (matrix_c.cc:49-58) */
            const float *c = mat + 3 * ((size_t)j * rows + i);
            R[(size_t)j * rows + i] = sqrtf(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        }
    float *cn = (float *)malloc(sizeof(float) * (cols + 1));
    for (int j = 0; j < cols; ++j) {
        float sum = 0.0f;
        for (int i = 0; i < rows; ++i) sum += R[(size_t)j * rows + i] * R[(size_t)j * rows + i];
        cn[j] = sqrtf(sum);
    }
    float *u = (float *)calloc(rows + 1, sizeof(float));   /* R.row_sum (matrix_c.h:236-245) */
    for (int j = 0; j < cols; ++j)
        for (int i = 0; i < rows; ++i) u[i] += R[(size_t)j * rows + i];
    float c0 = 0.0f;                                      /* column_norms.row_sum */
    for (int j = 0; j < cols; ++j) c0 += cn[j];
    for (int j = 0; j < cols; ++j) {                      /* v = Rt * u (matrix_c.h:224-233) */
        float v = 0.0f;
        for (int i = 0; i < rows; ++i) v += R[(size_t)j * rows + i] * u[i];
        alphas[j] = cn[j] * c0 - v;
    }
    if (norms) {
        for (int j = 0; j < cols; ++j) {
            float m = 0.0f;
            for (int i = 0; i < rows; ++i) {
                const float *c = mat + 3 * ((size_t)j * rows + i);
                m += c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
            }
            norms[j] = sqrtf(m);
        }
    }
    free(R); free(cn); free(u);
}

/* DiscretePdf (pdf.cc:18-77): pdf / cdf from an array, sample by linear scan. */
typedef struct { int n, zero; float *pdf, *cdf; } dpdf;
static void dpdf_set(dpdf *d, const float *a, int n) {
    d->n = n; d->zero = 0;
    d->pdf = (float *)malloc(sizeof(float) * (n > 0 ? n : 1));
    d->cdf = (float *)malloc(sizeof(float) * (n > 0 ? n : 1));
    if (n == 0) { d->zero = 1; return; }
    float sum = 0.0f;
    for (int i = 0; i < n; ++i) sum += a[i];
    if (sum == 0.0f) {
        for (int i = 0; i < n; ++i) d->pdf[i] = d->cdf[i] = 0.0f;
        d->zero = 1;
        return;
    }
    for (int i = 0; i < n; ++i) d->pdf[i] = a[i] / sum;
    d->cdf[0] = d->pdf[0];
    for (int i = 1; i < n; ++i) d->cdf[i] = d->cdf[i - 1] + d->pdf[i];
    d->cdf[n - 1] = 1.0f;
}
static void dpdf_sample(const dpdf *d, float v, int *k, float *pk) {
    for (int i = 0; i < d->n; ++i)
        if (v < d->cdf[i]) { *k = i; *pk = d->pdf[i]; return; }
    *k = -1; *pk = 0.0f;
}
static void dpdf_free(dpdf *d) { free(d->pdf); free(d->cdf); }

/* ClusterBuilder::cluster_by_sampling (cluster_builder.cc:82-273), draws from stream
   (seed, 1, 0).  Returns the number of final clusters; assign[col] = final cluster or -1. */
int ro_cluster_by_sampling(const float *mat, int rows, int cols, int num_clusters, uint32_t seed,
                           int32_t *center, int32_t *rep, float *weight, int32_t *assign) {
    for (int j = 0; j < cols; ++j) assign[j] = -1;
    if (cols < num_clusters) {
        for (int i = 0; i < cols; ++i) { center[i] = i; weight[i] = 1.0f; rep[i] = -1; }
        return cols;
    }
    rng_t g = {seed, 1u, 0u, 0u};
    float *alphas = (float *)malloc(sizeof(float) * (cols + 1));
    ro_ltm_alphas(mat, rows, cols, alphas, NULL);
    dpdf pa;
    dpdf_set(&pa, alphas, cols);
    int *cen = (int *)malloc(sizeof(int) * num_clusters);
    float *w = (float *)malloc(sizeof(float) * num_clusters);
    int count = 0;
    /* the reference's loop never ends when fewer than num_clusters columns can be drawn;
       cap the target at the drawable count and bound the draws (as the CUDA build does) */
    int drawable = 0;
    for (int i = 0; i < cols; ++i) drawable += pa.pdf[i] > 0.0f;
    const int target = drawable < num_clusters ? drawable : num_clusters;
    long long draws = 0;
    while (count < target && draws++ < 100000000LL) {
        int k; float pk;
        dpdf_sample(&pa, rnd(&g), &k, &pk);
        if (pk == 0.0f) continue;
        int idx = -1;
        for (int i = 0; i < count; ++i) if (cen[i] == k) { idx = i; break; }
        if (idx < 0) { cen[count] = k; w[count] = 1.0f / pk; count++; }
        else w[idx] += 1.0f / pk;
    }
    size_t n3 = 3 * (size_t)rows;
    float *K = (float *)malloc(sizeof(float) * n3 * count + 4);
    float *kn = (float *)malloc(sizeof(float) * count);
    for (int c = 0; c < count; ++c) {
        const float *src = mat + (size_t)cen[c] * n3;
        for (size_t e = 0; e < n3; ++e) K[c * n3 + e] = src[e] * w[c];
        float m = 0.0f;      /* get_column_norms */
        for (int i = 0; i < rows; ++i) {
            const float *v = K + c * n3 + 3 * i;
            m += v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        }
        kn[c] = sqrtf(m);
    }
    float *mags = (float *)malloc(sizeof(float) * (cols + 1));
    int *owner = (int *)malloc(sizeof(int) * (cols + 1));
    int *cnt = (int *)calloc(count, sizeof(int));
    for (int i = 0; i < cols; ++i) {
        const float *mi = mat + (size_t)i * n3;
        float s2 = 0.0f;                 /* magnitude(mi) (cluster_builder.cc:14-19) */
        for (size_t e = 0; e < n3; ++e) s2 += mi[e] * mi[e];
        float norm_mi = sqrtf(s2);
        int min_c = -1; float min_d = 3.402823466e+38f;
        for (int j = 0; j < count; ++j) {
            const float *mk = K + j * n3;
            float d = 0.0f;
            for (size_t e = 0; e < n3; ++e) d += mi[e] * mk[e];
            float dist = fabsf(kn[j] * norm_mi - d);
            if (dist < min_d) { min_c = j; min_d = dist; }
        }
        owner[i] = min_c;
        mags[i] = norm_mi;
        if (min_c >= 0) cnt[min_c]++;
    }
    /* per-cluster member lists in column order, pdf over magnitudes, representative */
    int n_final = 0;
    int *map = (int *)malloc(sizeof(int) * count);
    int **members = (int **)malloc(sizeof(int *) * count);
    for (int c = 0; c < count; ++c) { members[c] = (int *)malloc(sizeof(int) * (cnt[c] + 1)); cnt[c] = 0; }
    for (int i = 0; i < cols; ++i) if (owner[i] >= 0) members[owner[i]][cnt[owner[i]]++] = i;
    int *r = (int *)malloc(sizeof(int) * count);
    float *wf = (float *)malloc(sizeof(float) * count);
    for (int c = 0; c < count; ++c) {
        float *mm = (float *)malloc(sizeof(float) * (cnt[c] + 1));
        for (int t = 0; t < cnt[c]; ++t) mm[t] = mags[members[c][t]];
        dpdf pc;
        dpdf_set(&pc, mm, cnt[c]);
        int j; float pj;
        dpdf_sample(&pc, rnd(&g), &j, &pj);
        if (j < 0) {
            r[c] = cnt[c] > 0 ? members[c][cnt[c] / 2] : -1;
            wf[c] = 0.0f;
        } else {
            r[c] = members[c][j];
            wf[c] = 1.0f / pj;
        }
        dpdf_free(&pc);
        free(mm);
    }
    for (int c = 0; c < count; ++c) {
        map[c] = -1;
        if (r[c] >= 0) {
            map[c] = n_final;
            center[n_final] = cen[c]; rep[n_final] = r[c]; weight[n_final] = wf[c];
            n_final++;
        }
    }
    for (int i = 0; i < cols; ++i) assign[i] = owner[i] >= 0 ? map[owner[i]] : -1;
    for (int c = 0; c < count; ++c) free(members[c]);
    free(members); free(map); free(r); free(wf); free(cnt); free(owner); free(mags);
    free(K); free(kn); free(cen); free(w); free(alphas); dpdf_free(&pa);
    return n_final;
}
