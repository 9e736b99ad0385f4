/*
 * ref_harness.cc - TEST INFRASTRUCTURE ONLY.
 *
 * Drives the reference's own C++ classes, compiled from the reference sources by
 * oracle/Makefile into oracle/_ref/librzk_ref.so, so that tests can pin the CPU oracle
 * (oracle/rzk_oracle.c) and the CUDA path against the reference's actual behaviour.
 * Nothing in the product links or loads this file.
 *
 * What runs here is reference code:
 *   - AggregateBvh::build / hit (aggregate_bvh.cc:48-478), Aggregate::hit(p,q)
 *     (aggregate.cc:84-90), Triangle / Quad / Surface (triangle.cc, quad.cc, surface.cc)
 *   - BsdfMaterial + Lambertian / ModifiedPhong / Ward eval (material.h, lambertian.cc,
 *     phong.cc, ward.cc), BrdfPointLight::brdf (brdf_point_light.h:235-240),
 *     FormFactor (form_factor.h), RadianceTerms (vpl_interface.h:50-123)
 *   - Camera::shoot_ray (camera.cc:52-65), Sensor (sensor.cc)
 *   - VplGenerator::generate_vpl (vpl_generator.cc:127-181); its Random draws come
 *     from rng_shim.c, which stands in for mtwist.c and serves the counter-based
 *     stream the CUDA kernels use, so particle k sees the same draws everywhere
 * The only restated lines are VirtualPointLight::gather_point (vpl.cc:661-688),
 * VirtualPointLight::incident_radiance (vpl.cc:411-440) and the static clamp_term
 * (vpl.cc:214-230): they are members of VirtualPointLight, whose translation unit
 * drags in the closed LibImportance headers, so their few lines are repeated here
 * calling the reference's own Aggregate, FormFactor, Material and RadianceTerms.
 */
#include <iostream>

#include "ref_common.h"

using namespace rref;

namespace rref {

Vec3 v3(const float *f) { return Vec3(f[0], f[1], f[2]); }
void put3(float *dst, const Vec3 &v) { dst[0] = v.x(); dst[1] = v.y(); dst[2] = v.z(); }
void put3(float *dst, const Rgb &c) { dst[0] = c.red(); dst[1] = c.green(); dst[2] = c.blue(); }

/* vpl.cc:214-230 (static in the reference TU). */
void clamp_term(RadianceTerms &term, Float threshold, int mode) {
    switch (mode) {
        case VplRadianceClamp::REFLECTIVITY: term.eval_clamp_reflectivity(threshold); break;
        case VplRadianceClamp::RADIANCE:     term.eval_clamp_radiance(threshold); break;
        case VplRadianceClamp::FORM_FACTOR:  term.eval_clamp_form_factor(threshold); break;
        case VplRadianceClamp::NONE:
        default:                             term.eval_no_clamp(); break;
    }
}

Receiver to_receiver(const RefScene *s, const rzk_receiver &r) {
    Receiver rc;
    rc.p = v3(r.p);
    rc.n = v3(r.ng);
    rc.wo = v3(r.wo);
    rc.m = r.mat >= 0 ? (*s->materials)[r.mat] : nullptr;
    rc.light = nullptr;
    rc.uv = Vec2(0.0f, 0.0f);
    rc.tangent = Vec3(0.0f);
    rc.shading_n = v3(r.ns);
    rc.shading_uvn = Onb(v3(r.u), v3(r.v), v3(r.n));
    return rc;
}

BrdfPointLight to_vpl(const RefScene *s, const rzk_vpl &v) {
    LocalGeometry dg(v3(v.p), v3(v.n), v3(v.n), Onb(v3(v.u), v3(v.v), v3(v.nn)),
                     Vec3(0.0f), Vec2(0.0f, 0.0f));
    Material *m = v.mat >= 0 ? (*s->materials)[v.mat] : nullptr;
    BrdfPointLight pl(dg, Rgb(v.contrib[0], v.contrib[1], v.contrib[2]), m, v3(v.wi),
                      BrdfPointLightRef());
    pl.set_bounce(v.bounce);
    return pl;
}

/* VirtualPointLight::gather_point (vpl.cc:661-688), restated against reference types. */
Rgb gather_point(const RefScene *s, const LocalGeometry &dg, const Vec3 &wo, Material *m,
                 const BrdfPointLight *vpl, int clamp_mode, Float clamp_threshold,
                 bool &visible) {
    if (!m) { visible = false; return DefaultRgb::black; }
    Vec3 p = dg.p;
    Vec3 pn = dg.n;
    Vec3 q = vpl->org();
    Vec3 qn = vpl->normal();
    Aggregate *agg = s->scene->get_aggregate();
    Float tmin = s->scene->get_tmin();
    Float tick = s->scene->get_tick();
    if (agg->hit(p, q, tmin, tick)) {
        visible = false;
        return DefaultRgb::black;
    }
    visible = true;
    Float G = FormFactor::form_factor_abs(p, pn, q, qn);
    Vec3 wi = unit_vector(q - p);
    Rgb brdf = m->eval(dg, wo, wi);
    Rgb light_brdf = vpl->brdf(-wi);
    Rgb light_power = vpl->power();
    RadianceTerms term(light_power, brdf, light_brdf, G);
    clamp_term(term, clamp_threshold, clamp_mode);
    return term.radiance;
}

/* VirtualPointLight::incident_radiance (vpl.cc:411-440), restated. */
Rgb incident_radiance(const Receiver &r, const BrdfPointLight &vpl, int clamp_mode,
                      Float threshold) {
    Vec3 p = r.p;
    Vec3 pn = r.n;
    Vec3 q = vpl.org();
    Vec3 qn = vpl.normal();
    Float G = FormFactor::form_factor_abs(p, pn, q, qn);
    Vec3 wi = unit_vector(q - p);
    Rgb light_brdf = vpl.brdf(-wi);
    Rgb light_power = vpl.power();
    RadianceTerms term(light_power, DefaultRgb::white, light_brdf, G);
    clamp_term(term, threshold, clamp_mode);
    return term.radiance;
}

void fill_receiver(const Ray &r, const HitRecord &rec, rzk_receiver &out,
                   const RefScene *s) {
    std::memset(&out, 0, sizeof(out));
    out.mat = -1;
    out.light = -1;
    if (!rec.hit) return;
    Receiver rc(r, rec);
    put3(out.p, rc.p);
    put3(out.ng, rc.n);
    put3(out.ns, rc.shading_n);
    put3(out.wo, rc.wo);
    put3(out.u, rc.shading_uvn.u());
    put3(out.v, rc.shading_uvn.v());
    put3(out.n, rc.shading_uvn.n());
    out.mat = rc.m ? rc.m->get_material_index() : -1;
    if (rc.light) {
        for (size_t i = 0; i < s->lights->size(); ++i)
            if ((*s->lights)[i] == rc.light) out.light = (int)i;
    }
    out.flags = 1;
}

}  // namespace rref

/* Camera request for the harness: eye, lookat, up, vertical fov in degrees,
 * image and film sizes.  The harness builds the reference Camera from it the way
 * JsonImporter::load_cameras does (json_importer.cc:398-441). */
extern "C" {

struct RefCameraDesc {
    float eye[3], lookat[3], up[3];
    float fov;
    int32_t width, height;
    float film_w, film_h;
};

void *rref_create(const rzk_scene_desc *d, const RefCameraDesc *cd, uint32_t seed) {
    {   // Log::info() etc. print their level tag before returning the stream: keep those
        // tags off stdout, where callers print their own results
        std::streambuf *sb = std::cout.rdbuf(nullptr);
        Log::info().set_enable(false);
        Log::warn().set_enable(false);
        Log::debug().set_enable(false);
        std::cout.rdbuf(sb);
        std::cout.clear();
    }
    RefScene *s = new RefScene();
    s->shapes = new Shapes();
    s->materials = new Materials();
    s->textures = new Textures();
    s->surfaces = new Surfaces();
    s->lights = new Lights();
    for (int i = 0; i < d->n_mats; ++i) {
        const rzk_material &m = d->mats[i];
        Rgb kd(m.kd[0], m.kd[1], m.kd[2]);
        Rgb ks(m.ks[0], m.ks[1], m.ks[2]);
        Bsdf *b = nullptr;
        if (m.type == RZK_BSDF_LAMBERTIAN) b = new Lambertian(kd);
        else if (m.type == RZK_BSDF_PHONG) b = new ModifiedPhong(kd, ks, m.p0);
        else b = new Ward(kd, ks, m.p0, m.p1);
        s->materials->push_back(new BsdfMaterial(b));
    }
    int tri = 0;
    for (int i = 0; i < d->n_prims; ++i) {
        const float *v = d->prim_v + 12 * i;
        Shape *shape;
        if (d->prim_kind[i] == RZK_PRIM_QUAD)
            shape = new Quad(v3(v), v3(v + 3), v3(v + 6), v3(v + 9));
        else
            shape = new Triangle(v3(v), v3(v + 3), v3(v + 6));
        s->shapes->push_back(shape);
        s->tri_first.push_back(tri);
        s->tri_count.push_back(shape->get_triangle_count());
        tri += shape->get_triangle_count();
        if (d->prim_mat[i] >= 0) {
            Surface surf(shape, (*s->materials)[d->prim_mat[i]]);
            if (d->prim_flags) {
                surf.reverse_normal((d->prim_flags[i] & RZK_SURF_FLIPPED) != 0);
                surf.set_two_sided((d->prim_flags[i] & RZK_SURF_TWO_SIDED) != 0);
            }
            s->surfaces->append(surf);
        } else {
            const float *e = d->prim_emit + 3 * i;
            Surface surf(shape, Rgb(e[0], e[1], e[2]));
            if (d->prim_flags) {
                surf.reverse_normal((d->prim_flags[i] & RZK_SURF_FLIPPED) != 0);
                surf.set_two_sided((d->prim_flags[i] & RZK_SURF_TWO_SIDED) != 0);
            }
            s->surfaces->append(surf);
        }
    }
    /* Surface's copy constructor re-points the light at the copy (surface.cc:36-41);
       collect the lights after the vector has stopped moving. */
    for (size_t i = 0; i < s->surfaces->size(); ++i) {
        Surface &surf = (*s->surfaces)[i];
        if (surf.get_area_light()) {
            surf.get_area_light()->set_surface(&surf);
            s->lights->push_back(surf.get_area_light());
        }
    }
    s->sensor = new Sensor(Size2((Float)cd->width, (Float)cd->height),
                           Size2(cd->film_w, cd->film_h));
    s->camera = new Camera();
    Float focal = Camera::focal_length_from_fov(cd->fov, cd->film_h);
    s->camera->set_perspective(v3(cd->eye), v3(cd->lookat), v3(cd->up), focal, s->sensor);
    s->rd = new Random(seed);
    s->bvh = new BvhProbe(*s->surfaces);
    s->scene = new Scene("rzk", s->bvh, s->shapes, s->materials, s->textures, s->surfaces,
                         s->lights, s->camera, s->rd);
    if (d->tmin > 0.0f) s->scene->set_tmin(d->tmin);
    s->tmin = s->scene->get_tmin();
    return s;
}

void rref_destroy(void *h) {
    /* The reference objects hold raw pointers to one another; the harness lives for
       the duration of a test process, so only the handle is released. */
    delete (RefScene *)h;
}

int rref_num_triangles(void *h) { return ((RefScene *)h)->bvh->tri_count(); }
int rref_num_nodes(void *h) { return ((RefScene *)h)->bvh->node_count(); }

/* Sorted Morton codes, the permutation (sorted slot -> flattened triangle index) and the
 * BVH nodes in the reference's BFS numbering. */
int rref_bvh_dump(void *h, uint32_t *morton_sorted, int32_t *perm, rzk_bvh_node *nodes,
                  int cap_nodes) {
    RefScene *s = (RefScene *)h;
    const BvhProbe *b = s->bvh;
    int n = b->tri_count();
    for (int i = 0; i < n; ++i) {
        morton_sorted[i] = b->morton()[i];
        int sid = b->surface_ids()[i];
        int first = s->tri_first[sid];
        int cnt = s->tri_count[sid];
        int found = -1;
        for (int k = 0; k < cnt; ++k) {
            std::vector<Triangle> tris;
            (*s->surfaces)[sid].get_shape()->get_triangles(tris);
            const Triangle &a = tris[k];
            const Triangle &c = b->tris()[i];
            if (a.p0 == c.p0 && a.p1 == c.p1 && a.p2 == c.p2) { found = first + k; break; }
        }
        perm[i] = found;
    }
    int nn = b->node_count();
    if (nn > cap_nodes) return -nn;
    for (int i = 0; i < nn; ++i) {
        const BvhNode &bn = b->node_array()[i];
        put3(nodes[i].bmin, bn.box.v_min);
        put3(nodes[i].bmax, bn.box.v_max);
        nodes[i].start = bn.start;
        nodes[i].end = bn.end;
        nodes[i].left = bn.index_left;
        nodes[i].right = bn.index_right;
        nodes[i].level = bn.level;
        nodes[i].pad = 0;
    }
    return nn;
}

/* Camera as the reference computed it: eye, onb, focal, cop, scale. */
void rref_camera(void *h, rzk_camera *out) {
    RefScene *s = (RefScene *)h;
    Camera *c = s->camera;
    Onb onb = c->get_onb();
    put3(out->eye, c->get_eye());
    put3(out->u, onb.u());
    put3(out->v, onb.v());
    put3(out->n, onb.n());
    out->focal = c->get_focal_length();
    Vec2 cop = s->sensor->get_cop();
    Vec2 sc = s->sensor->get_image_film_ratio();
    out->cop[0] = cop.x(); out->cop[1] = cop.y();
    out->scale[0] = sc.x(); out->scale[1] = sc.y();
    out->width = (int)s->sensor->get_image_size().width;
    out->height = (int)s->sensor->get_image_size().height;
    out->pad = 0;
}

/* Aggregate::hit(p, q, tmin, time) for n segments: 1 = occluded. */
void rref_occluded(void *h, const float *p, const float *q, int n, uint8_t *out) {
    RefScene *s = (RefScene *)h;
    Aggregate *agg = s->scene->get_aggregate();
    for (int i = 0; i < n; ++i)
        out[i] = agg->hit(v3(p + 3 * i), v3(q + 3 * i), s->tmin, 0.0f) ? 1 : 0;
}

/* Closest hit of Ray(o, d) over [tmin, RAY_TMAX]; fills receivers and the hit distance. */
void rref_closest(void *h, const float *o, const float *d, int n, float *t_out,
                  rzk_receiver *recv) {
    RefScene *s = (RefScene *)h;
    Aggregate *agg = s->scene->get_aggregate();
    for (int i = 0; i < n; ++i) {
        Ray r(v3(o + 3 * i), v3(d + 3 * i));
        HitRecord rec;
        bool hit = agg->hit(r, s->tmin, s->scene->get_max_tmax(), 0.0f, rec);
        t_out[i] = hit ? rec.t : -1.0f;
        fill_receiver(r, rec, recv[i], s);
    }
}

/* One pixel-centre primary hit per pixel (camera.cc:52-65), row-major, row 0 at top. */
void rref_primary(void *h, rzk_receiver *out) {
    RefScene *s = (RefScene *)h;
    Aggregate *agg = s->scene->get_aggregate();
    int W = (int)s->sensor->get_image_size().width;
    int H = (int)s->sensor->get_image_size().height;
    for (int i = 0; i < H; ++i)
        for (int j = 0; j < W; ++j) {
            Ray r = s->camera->shoot_ray(i, j);
            HitRecord rec;
            agg->hit(r, s->tmin, s->scene->get_max_tmax(), 0.0f, rec);
            fill_receiver(r, rec, out[i * W + j], s);
        }
}

/* Primary rays only (origin, direction) for the same pixels. */
void rref_primary_rays(void *h, float *o, float *d) {
    RefScene *s = (RefScene *)h;
    int W = (int)s->sensor->get_image_size().width;
    int H = (int)s->sensor->get_image_size().height;
    for (int i = 0; i < H; ++i)
        for (int j = 0; j < W; ++j) {
            Ray r = s->camera->shoot_ray(i, j);
            put3(o + 3 * (i * W + j), r.o);
            put3(d + 3 * (i * W + j), r.d);
        }
}

/* VplGenerator::generate_vpl over n_particles light particles with the reference's
 * global MT19937 stream (reseeded by Random(seed)).  Particles are generated one at a
 * time through VplGenerator::spawn (vpl_generator.cc:183-204) so the particle index of
 * each VPL is known; each particle k draws from stream (seed, 0, k). */
int rref_vpl_generate(void *h, uint32_t seed, int n_particles, int max_bounce,
                      rzk_vpl *out, int cap) {
    RefScene *s = (RefScene *)h;
    VplGenerator gen;
    BrdfPointLights vpls;
    std::vector<int> path;
    for (int k = 0; k < n_particles; ++k) {
        size_t before = vpls.size();
        rref_rng_stream(seed, 0u, (uint32_t)k);
        gen.spawn(s->scene, 1, max_bounce, vpls, false);
        for (size_t i = before; i < vpls.size(); ++i) path.push_back(k);
    }
    int n = (int)vpls.size();
    int m = n < cap ? n : cap;
    for (int i = 0; i < m; ++i) {
        const BrdfPointLight &v = vpls[i];
        LocalGeometry dg = v.get_dg();
        rzk_vpl &o = out[i];
        std::memset(&o, 0, sizeof(o));
        put3(o.p, dg.p);
        put3(o.n, dg.n);
        put3(o.u, dg.uvn.u());
        put3(o.v, dg.uvn.v());
        put3(o.nn, dg.uvn.n());
        put3(o.wi, v.get_wi());
        put3(o.contrib, v.power());
        o.mat = v.get_material() ? v.get_material()->get_material_index() : -1;
        o.bounce = v.get_bounce();
        o.path = path[i];
    }
    return n;
}

/* Full gather: out[r] = sum over VPLs of gather_point(...) in VPL order (float), and
 * optionally the same sum in double, the per-pair radiance matrix (column-major
 * rows x cols like MatrixC, light_transport_matrix.cc:16-48) and visibility. */
void rref_gather(void *h, const rzk_receiver *recv, int n_recv, const rzk_vpl *vpls,
                 int n_vpl, int clamp_mode, float tau, float *out_rgb,
                 float *pair_rgb, uint8_t *pair_vis) {
    RefScene *s = (RefScene *)h;
    std::vector<BrdfPointLight> pls;
    pls.reserve(n_vpl);
    for (int j = 0; j < n_vpl; ++j) pls.push_back(to_vpl(s, vpls[j]));
    for (int i = 0; i < n_recv; ++i) {
        Receiver rc = to_receiver(s, recv[i]);
        LocalGeometry dg(rc);
        Rgb sum = DefaultRgb::black;
        for (int j = 0; j < n_vpl; ++j) {
            bool visible = false;
            Rgb L = gather_point(s, dg, rc.wo, rc.m, &pls[j], clamp_mode, tau, visible);
            sum += L;
            if (pair_rgb) put3(pair_rgb + 3 * ((size_t)j * n_recv + i), L);
            if (pair_vis) pair_vis[(size_t)j * n_recv + i] = visible ? 1 : 0;
        }
        put3(out_rgb + 3 * i, sum);
    }
}

/* The same gather over receivers split across n_threads std::threads (the reference's
 * AggregateBvh::hit and BRDF evaluation are const and keep no shared state), for timing
 * the reference CPU path on all host cores.  out_rgb[r] = scale * sum. */
void rref_gather_mt(void *h, const rzk_receiver *recv, int n_recv, const rzk_vpl *vpls, int n_vpl,
                    int clamp_mode, float tau, float scale, float *out_rgb, int n_threads) {
    RefScene *s = (RefScene *)h;
    std::vector<BrdfPointLight> pls;
    pls.reserve(n_vpl);
    for (int j = 0; j < n_vpl; ++j) pls.push_back(to_vpl(s, vpls[j]));
    if (n_threads < 1) n_threads = 1;
    auto work = [&](int t) {
        int r0 = (int)((long long)n_recv * t / n_threads), r1 = (int)((long long)n_recv * (t + 1) / n_threads);
        for (int i = r0; i < r1; ++i) {
            Receiver rc = to_receiver(s, recv[i]);
            LocalGeometry dg(rc);
            Rgb sum = DefaultRgb::black;
            for (int j = 0; j < n_vpl; ++j) {
                bool visible = false;
                sum += gather_point(s, dg, rc.wo, rc.m, &pls[j], clamp_mode, tau, visible);
            }
            put3(out_rgb + 3 * i, sum * scale);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < n_threads; ++t) th.emplace_back(work, t);
    work(0);
    for (auto &x : th) x.join();
}

/* LightTransportMatrix::generate_alphas_for_clustering (light_transport_matrix.cc:72-106)
 * and get_column_norms (light_transport_matrix.cc:118-130) on a column-major matrix
 * [cols][rows][3] (MatrixC<Rgb> layout). */
static LightTransportMatrix *make_ltm(const float *mat, int rows, int cols) {
    LightTransportMatrix *R = new LightTransportMatrix(rows, cols);
    std::vector<Float> col(3 * (size_t)rows);
    for (int j = 0; j < cols; ++j) {
        for (int k = 0; k < 3 * rows; ++k) col[k] = mat[(size_t)j * rows * 3 + k];
        R->set_column(j, col);
    }
    return R;
}

void rref_ltm_alphas(const float *mat, int rows, int cols, float *alphas, float *norms) {
    LightTransportMatrix *R = make_ltm(mat, rows, cols);
    std::vector<Float> a;
    R->generate_alphas_for_clustering(a);
    for (int j = 0; j < cols; ++j) alphas[j] = a[j];
    std::vector<Float> n;
    R->get_column_norms(n);
    for (int j = 0; j < cols; ++j) norms[j] = n[j];
    delete R;
}

/* LightTransportMatrix::save -> MatrixC<Rgb>::save (light_transport_matrix.cc:144-146,
 * matrix_c.cc:6-23) of a column-major matrix [cols][rows][3]. */
void rref_matrix_save(const float *mat, int rows, int cols, const char *path) {
    LightTransportMatrix *R = make_ltm(mat, rows, cols);
    R->save(path);
    delete R;
}

/* ClusterBuilder::cluster_by_sampling (cluster_builder.cc:82-273) with its random draws from
 * stream (seed, 1, 0).  Outputs the final clusters in order and, per column, the index of
 * the final cluster holding it (-1 if none).  Returns the number of clusters. */
int rref_cluster_by_sampling(void *h, const float *mat, int rows, int cols, int num_clusters, uint32_t seed,
                             int32_t *center, int32_t *rep, float *weight, int32_t *assign) {
    RefScene *s = (RefScene *)h;
    LightTransportMatrix *R = make_ltm(mat, rows, cols);
    BrdfPointLights vpls(cols);
    Pixels pixels(rows);
    Clusters cl;
    ClusterBuilder cb;
    rref_rng_stream(seed, 1u, 0u);
    cb.cluster_by_sampling(s->scene, nullptr, *R, num_clusters, cl, vpls, pixels);
    for (int j = 0; j < cols; ++j) assign[j] = -1;
    for (size_t c = 0; c < cl.size(); ++c) {
        center[c] = cl[c].center;
        rep[c] = cl[c].representative;
        weight[c] = cl[c].weight;
        for (int idx : cl[c].indices) assign[idx] = (int32_t)c;
    }
    delete R;
    return (int)cl.size();
}

/* incident_radiance for every (receiver, VPL) pair, column-major like rref_gather. */
void rref_incident(void *h, const rzk_receiver *recv, int n_recv, const rzk_vpl *vpls,
                   int n_vpl, int clamp_mode, float tau, float *pair_rgb) {
    RefScene *s = (RefScene *)h;
    for (int j = 0; j < n_vpl; ++j) {
        BrdfPointLight pl = to_vpl(s, vpls[j]);
        for (int i = 0; i < n_recv; ++i) {
            Receiver rc = to_receiver(s, recv[i]);
            put3(pair_rgb + 3 * ((size_t)j * n_recv + i),
                 incident_radiance(rc, pl, clamp_mode, tau));
        }
    }
}

/* Material::eval for a batch of (material, basis, wo, wi): rgb out. */
void rref_brdf_eval(void *h, const int32_t *mat, const float *uvn9, const float *wo,
                    const float *wi, int n, float *out) {
    RefScene *s = (RefScene *)h;
    for (int i = 0; i < n; ++i) {
        LocalGeometry dg;
        const float *b = uvn9 + 9 * i;
        dg.uvn = Onb(v3(b), v3(b + 3), v3(b + 6));
        Rgb c = (*s->materials)[mat[i]]->eval(dg, v3(wo + 3 * i), v3(wi + 3 * i));
        put3(out + 3 * i, c);
    }
}

}  // extern "C"
