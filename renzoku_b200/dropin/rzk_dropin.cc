// rzk_dropin.cc - AggregateCuda, VplGeneratorCuda, VirtualPointLightCuda and the scene-file
// factory: the reference's C++ interfaces implemented over librzk_cuda.so's C ABI.
#include "rzk_dropin.h"

#include <cstring>
#include <stdexcept>
#include <unordered_map>

#include <cuda_runtime.h>

#include "area_light.h"
#include "aggregate_bvh.h"
#include "camera.h"
#include "frame.h"
#include "hitrecord.h"
#include "image.h"
#include "lambertian.h"
#include "local_geometry.h"
#include "material.h"
#include "phong.h"
#include "quad.h"
#include "random.h"
#include "sensor.h"
#include "surface.h"
#include "triangle.h"
#include "ward.h"

namespace Renzoku {

namespace {

void ensure(rzk_status st, const char *what) {
    if (st != RZK_OK) throw std::runtime_error(std::string(what) + ": " + rzk_status_string(st));
}

void ensure_cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

void put3(float *dst, const Vec3 &v) {
    dst[0] = v.x();
    dst[1] = v.y();
    dst[2] = v.z();
}

Vec3 get3(const float *s) { return Vec3(s[0], s[1], s[2]); }

// The device material record of a reference material: BsdfMaterial over the three BRDFs
// of the gather (material.h:67-135); anything else has no device form.
bool material_record(Material *m, rzk_material &out) {
    std::memset(&out, 0, sizeof(out));
    if (!m || m->get_material_type() != Material::BSDF) return false;
    Bsdf *b = m->get_bsdf();
    if (!b) return false;
    switch (b->get_bsdf_type()) {
        case Bsdf::LAMBERTIAN: {
            const Rgb kd = static_cast<Lambertian *>(b)->get_diffuse_component();
            out.type = RZK_BSDF_LAMBERTIAN;
            out.kd[0] = kd.red(); out.kd[1] = kd.green(); out.kd[2] = kd.blue();
            return true;
        }
        case Bsdf::PHONG: {
            ModifiedPhong *p = static_cast<ModifiedPhong *>(b);
            const Rgb kd = p->get_diffuse_component(), ks = p->get_specular_component();
            out.type = RZK_BSDF_PHONG;
            out.kd[0] = kd.red(); out.kd[1] = kd.green(); out.kd[2] = kd.blue();
            out.ks[0] = ks.red(); out.ks[1] = ks.green(); out.ks[2] = ks.blue();
            out.p0 = p->get_glossy_coefficients().x();
            return true;
        }
        case Bsdf::WARD: {
            Ward *w = static_cast<Ward *>(b);
            const Rgb kd = w->get_diffuse_component(), ks = w->get_specular_component();
            const Vec2 a = w->get_glossy_coefficients();
            out.type = RZK_BSDF_WARD;
            out.kd[0] = kd.red(); out.kd[1] = kd.green(); out.kd[2] = kd.blue();
            out.ks[0] = ks.red(); out.ks[1] = ks.green(); out.ks[2] = ks.blue();
            out.p0 = a.x();
            out.p1 = a.y();
            return true;
        }
        default:
            return false;
    }
}

// The radiance an area light emits: AreaLight::query along its own normal returns it
// (area_light.cc:19-25 with AreaLight::pdf positive for wo = n, area_light.h:120-131).
Rgb emitted_radiance(AreaLight *l) {
    const Vec3 n(0.0f, 0.0f, 1.0f);
    Rgb L;
    l->query(Vec3(0.0f), n, n, L);
    return L;
}

rzk_ray ray_record(const Ray &r, Float tmin, Float tmax) {
    rzk_ray q;
    std::memset(&q, 0, sizeof(q));
    put3(q.o, r.o);
    put3(q.d, r.d);
    put3(q.inv_d, r.inv_d);
    put3(q.org_inv_d, r.org_inv_d);
    q.tmin = tmin;
    q.tmax = tmax;
    return q;
}

// Device scratch for a batch: grown on demand, owned by the caller.
void grow(void *&buf, size_t &cap, size_t need) {
    if (need <= cap) return;
    if (buf) cudaFree(buf);
    buf = nullptr;
    cap = 0;
    ensure_cuda(cudaMalloc(&buf, need), "cudaMalloc");
    cap = need;
}

}  // namespace

// ------------------------------------------------------------------------------------
// AggregateCuda

AggregateCuda::AggregateCuda(const Surfaces &surfaces, Float tmin, int device) : Aggregate(surfaces), dev(device) {
    // AggregateBvh::build's flattening (aggregate_bvh.cc:58-76): surfaces in order, each
    // shape's triangles in order; a quad's two triangles travel as one quad primitive
    std::vector<int32_t> kind, mat, flags;
    std::vector<float> v, emit;
    std::vector<rzk_material> mats;
    std::unordered_map<const Material *, int> mat_of;
    for (int i = 0; i < (int)surfaces.size(); ++i) {
        const Surface &s = surfaces[i];
        Shape *shape = s.get_shape();
        const int nt = shape->get_triangle_count();
        if (nt == 0) continue;   // analytic shapes: AggregateBvh skips them too
        float pv[12] = {0};
        if (Quad *q = dynamic_cast<Quad *>(shape)) {
            put3(pv, q->p0); put3(pv + 3, q->p1); put3(pv + 6, q->p2); put3(pv + 9, q->p3);
            kind.push_back(RZK_PRIM_QUAD);
        } else if (Triangle *t = dynamic_cast<Triangle *>(shape)) {
            put3(pv, t->p0); put3(pv + 3, t->p1); put3(pv + 6, t->p2);
            kind.push_back(RZK_PRIM_TRIANGLE);
        } else {
            throw std::runtime_error("AggregateCuda: only triangle and quad shapes have a device form");
        }
        v.insert(v.end(), pv, pv + 12);
        for (int k = 0; k < nt; ++k) {
            tri_surface.push_back(i);
            tri_local.push_back(k);
        }
        flags.push_back((s.is_reverse_normal() ? RZK_SURF_FLIPPED : 0) | (s.get_two_sided() ? RZK_SURF_TWO_SIDED : 0));
        if (s.get_area_light()) {
            const Rgb L = emitted_radiance(s.get_area_light());
            mat.push_back(-1);
            emit.push_back(L.red()); emit.push_back(L.green()); emit.push_back(L.blue());
        } else {
            Material *m = s.get_material();
            auto it = mat_of.find(m);
            int idx = it == mat_of.end() ? -1 : it->second;
            if (idx < 0) {
                rzk_material rec;
                if (!material_record(m, rec))
                    throw std::runtime_error("AggregateCuda: a surface's material has no device form "
                                             "(Lambertian, modified Phong and Ward do)");
                idx = (int)mats.size();
                mats.push_back(rec);
                mat_ptrs.push_back(m);
                mat_of[m] = idx;
            }
            mat.push_back(idx);
            emit.push_back(0.0f); emit.push_back(0.0f); emit.push_back(0.0f);
        }
    }
    rzk_scene_desc d;
    std::memset(&d, 0, sizeof(d));
    d.n_prims = (int32_t)kind.size();
    d.prim_kind = kind.data();
    d.prim_v = v.data();
    d.prim_mat = mat.data();
    d.prim_emit = emit.data();
    d.prim_flags = flags.data();
    d.n_mats = (int32_t)mats.size();
    d.mats = mats.data();
    d.tmin = tmin;
    ensure(rzk_context_create(device, &ctx), "rzk_context_create");
    rzk_status st = rzk_scene_create(ctx, &d, nullptr, &scene_h);
    if (st != RZK_OK) {
        rzk_context_destroy(ctx);
        ctx = nullptr;
        ensure(st, "rzk_scene_create");
    }
}

AggregateCuda::~AggregateCuda() {
    if (d_stage) cudaFree(d_stage);
    if (scene_h) rzk_scene_destroy(scene_h);
    if (ctx) rzk_context_destroy(ctx);
}

Material *AggregateCuda::material(int index) const {
    return index >= 0 && index < (int)mat_ptrs.size() ? mat_ptrs[index] : nullptr;
}

int AggregateCuda::material_index(const Material *m) const {
    for (size_t i = 0; i < mat_ptrs.size(); ++i)
        if (mat_ptrs[i] == m) return (int)i;
    return -1;
}

void AggregateCuda::query(const std::vector<rzk_ray> &rays, bool closest, std::vector<rzk_ray_hit> &out) const {
    const int n = (int)rays.size();
    out.resize(n);
    if (n == 0) return;
    std::lock_guard<std::mutex> lk(mu);
    ensure_cuda(cudaSetDevice(dev), "cudaSetDevice");
    const size_t rb = sizeof(rzk_ray) * (size_t)n, hb = sizeof(rzk_ray_hit) * (size_t)n;
    grow(d_stage, stage_bytes, rb + hb);
    char *base = (char *)d_stage;
    ensure_cuda(cudaMemcpy(base, rays.data(), rb, cudaMemcpyHostToDevice), "cudaMemcpy");
    ensure(rzk_ray_query_batch(scene_h, (const rzk_ray *)base, n, closest ? 1 : 0, (rzk_ray_hit *)(base + rb),
                               nullptr),
           "rzk_ray_query_batch");
    ensure_cuda(cudaMemcpy(out.data(), base + rb, hb, cudaMemcpyDeviceToHost), "cudaMemcpy");
    ensure(rzk_context_check(ctx, nullptr), "device error word");
}

// The record as AggregateBvh::hit completes it (aggregate_bvh.cc:440-445): the reference's
// own Triangle::fill_hit_record from the GeometryHit, then Surface::fill_hit_record.
void AggregateCuda::fill_record(const Ray &r, const rzk_ray_hit &h, HitRecord &record) const {
    const int s = tri_surface[h.tri];
    const Surface &surf = surfaces[s];
    // the shape's own triangle (a quad's t0 / t1): AggregateBvh fills from its sorted copy
    // of the same triangle, so the record is the same, its shape pointer the original's
    const Triangle &tri = *surf.get_shape()->get_triangle_pointer(tri_local[h.tri]);
    GeometryHit gh;
    gh.hit = true;
    gh.t = h.t;
    gh.beta = h.beta;
    gh.gamma = h.gamma;
    gh.shape = (Shape *)&tri;
    tri.fill_hit_record(r, gh, record);
    surf.fill_hit_record(r, record);
}

bool AggregateCuda::hit(const Ray &r, Float tmin, Float tmax, Float time, HitRecord &record) const {
    (void)time;
    std::vector<rzk_ray_hit> out;
    query(std::vector<rzk_ray>{ray_record(r, tmin, tmax)}, true, out);
    if (!out[0].hit) return false;
    fill_record(r, out[0], record);
    return true;
}

bool AggregateCuda::hit(const Ray &r, Float tmin, Float tmax, Float time) const {
    (void)time;
    std::vector<rzk_ray_hit> out;
    query(std::vector<rzk_ray>{ray_record(r, tmin, tmax)}, false, out);
    return out[0].hit != 0;
}

// Aggregate::hit(p, q, tmin, time) (aggregate.cc:84-90): Ray(p, q - p) over
// [tmin, |q - p| - tmin], the ray built by the reference's own Ray constructor.
bool AggregateCuda::hit(const Vec3 &p, const Vec3 &q, Float tmin, Float time) const {
    Ray r(p, q - p);
    Float tmax = (q - p).length() - tmin;
    return hit(r, tmin, tmax, time);
}

void AggregateCuda::hit_batch(const Ray *rays, const Float *tmin, const Float *tmax, int n, bool *hits,
                              HitRecord *records) const {
    std::vector<rzk_ray> q(n);
    for (int i = 0; i < n; ++i) q[i] = ray_record(rays[i], tmin[i], tmax[i]);
    std::vector<rzk_ray_hit> out;
    query(q, records != nullptr, out);
    for (int i = 0; i < n; ++i) {
        hits[i] = out[i].hit != 0;
        if (records && hits[i]) fill_record(rays[i], out[i], records[i]);
    }
}

void AggregateCuda::hit_segments(const Vec3 *p, const Vec3 *q, int n, Float tmin, bool *occluded) const {
    std::vector<rzk_ray> rq(n);
    for (int i = 0; i < n; ++i) {
        Ray r(p[i], q[i] - p[i]);
        rq[i] = ray_record(r, tmin, (q[i] - p[i]).length() - tmin);
    }
    std::vector<rzk_ray_hit> out;
    query(rq, false, out);
    for (int i = 0; i < n; ++i) occluded[i] = out[i].hit != 0;
}

// ------------------------------------------------------------------------------------
// VplGeneratorCuda

void VplGeneratorCuda::spawn(Scene *scene, int num_start_samples, int max_bounce, BrdfPointLights &lights,
                             bool is_photon) {
    (void)is_photon;
    AggregateCuda *agg = dynamic_cast<AggregateCuda *>(scene->get_aggregate());
    if (!agg) throw std::runtime_error("VplGeneratorCuda: the scene's aggregate is not an AggregateCuda");
    emitted = 0;
    if (num_start_samples <= 0) return;
    ensure_cuda(cudaSetDevice(agg->device()), "cudaSetDevice");
    // at most (max_bounce - 1) VPLs per particle (bounces 1 .. max_bounce - 1)
    const int cap = num_start_samples * std::max(1, max_bounce - 1);
    void *buf = nullptr;
    ensure_cuda(cudaMalloc(&buf, sizeof(rzk_vpl) * (size_t)cap + 256), "cudaMalloc");
    int made = 0;
    std::vector<rzk_vpl> h;
    rzk_status st = rzk_vpl_generate(agg->handle(), seed, num_start_samples, max_bounce, (rzk_vpl *)buf, cap,
                                     (int *)((char *)buf + sizeof(rzk_vpl) * (size_t)cap), nullptr);
    cudaError_t e = cudaSuccess;
    if (st == RZK_OK)
        e = cudaMemcpy(&made, (char *)buf + sizeof(rzk_vpl) * (size_t)cap, sizeof(int), cudaMemcpyDeviceToHost);
    if (st == RZK_OK && e == cudaSuccess) {
        h.resize(std::min(made, cap));
        e = cudaMemcpy(h.data(), buf, sizeof(rzk_vpl) * h.size(), cudaMemcpyDeviceToHost);
    }
    cudaFree(buf);
    ensure(st, "rzk_vpl_generate");
    ensure_cuda(e, "cudaMemcpy");
    emitted = num_start_samples;
    // BrdfPointLight(dg, T, m, wi, prev) with its bounce, as trace_vpl pushes it
    // (vpl_generator.cc:61-66); prev is the VPL before it on the same path
    const size_t base = lights.size();
    for (size_t i = 0; i < h.size(); ++i) {
        const rzk_vpl &v = h[i];
        LocalGeometry dg(get3(v.p), get3(v.n), get3(v.n), Onb(get3(v.u), get3(v.v), get3(v.nn)), Vec3(0.0f),
                         Vec2(0.0f, 0.0f));
        BrdfPointLightRef prev;
        if (i > 0 && h[i - 1].path == v.path && h[i - 1].bounce == v.bounce - 1)
            prev = BrdfPointLightRef((int)(base + i - 1));
        BrdfPointLight pl(dg, Rgb(v.contrib[0], v.contrib[1], v.contrib[2]), agg->material(v.mat), get3(v.wi), prev);
        pl.set_bounce(v.bounce);
        lights.push_back(pl);
    }
}

// ------------------------------------------------------------------------------------
// VirtualPointLightCuda

VirtualPointLightCuda::VirtualPointLightCuda() { suffix = "vpl_cuda"; }

VirtualPointLightCuda::~VirtualPointLightCuda() { release(); }

void VirtualPointLightCuda::release() {
    if (d_recv) cudaFree(d_recv);
    if (d_vpls) cudaFree(d_vpls);
    if (d_rgb) cudaFree(d_rgb);
    d_recv = nullptr;
    d_vpls = nullptr;
    d_rgb = nullptr;
}

void VirtualPointLightCuda::initialize(Scene *scene) {
    MonteCarloIntegrator::initialize(scene);
    agg = dynamic_cast<AggregateCuda *>(scene->get_aggregate());
    if (!agg) throw std::runtime_error("VirtualPointLightCuda: the scene's aggregate is not an AggregateCuda");
    release();
    ensure_cuda(cudaSetDevice(agg->device()), "cudaSetDevice");
    Camera *cam = scene->get_camera();
    const Size2 img = cam->get_image_size(), film = cam->get_film_size();
    w = (int)img.width;
    h = (int)img.height;
    rzk_camera rc;
    float eye[3], lookat[3], up[3];
    put3(eye, cam->get_eye());
    put3(lookat, cam->get_lookat());
    put3(up, cam->get_up());
    ensure(rzk_camera_setup_focal(eye, lookat, up, cam->get_focal_length(), w, h, film.width, film.height, &rc),
           "rzk_camera_setup_focal");
    ensure_cuda(cudaMalloc((void **)&d_recv, sizeof(rzk_receiver) * (size_t)w * h), "cudaMalloc");
    ensure_cuda(cudaMalloc((void **)&d_rgb, sizeof(float) * 3 * (size_t)w * h), "cudaMalloc");
    ensure(rzk_primary(agg->handle(), &rc, d_recv, nullptr), "rzk_primary");
    // the VPLs: the first max_vpls in push order of start_particles light particles
    const int cap = start_particles * std::max(1, max_bounce - 1);
    ensure_cuda(cudaMalloc((void **)&d_vpls, sizeof(rzk_vpl) * (size_t)cap + 256), "cudaMalloc");
    int *d_count = (int *)((char *)d_vpls + sizeof(rzk_vpl) * (size_t)cap);
    ensure(rzk_vpl_generate(agg->handle(), seed, start_particles, max_bounce, d_vpls, cap, d_count, nullptr),
           "rzk_vpl_generate");
    int made = 0;
    ensure_cuda(cudaMemcpy(&made, d_count, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy");
    n_vpl = std::min(std::min(made, cap), max_vpls);
    emitted = start_particles;
    if (n_vpl > 0 && n_vpl < std::min(made, cap)) {
        // num_emitted: the particles whose VPLs are kept (the path of the last kept VPL + 1)
        rzk_vpl last;
        ensure_cuda(cudaMemcpy(&last, d_vpls + (n_vpl - 1), sizeof(rzk_vpl), cudaMemcpyDeviceToHost), "cudaMemcpy");
        emitted = last.path + 1;
    }
    tau = 0.0f;
    if (clamp_mode == RZK_CLAMP_RADIANCE && n_vpl > 0) {
        double mean = 0.0;
        ensure(rzk_mean_contribution(agg->context(), agg->handle(), d_recv, w * h, d_vpls, n_vpl, seed, 65536, &mean,
                                     nullptr),
               "rzk_mean_contribution");
        tau = (float)(clamp_scale * mean);
    } else if (clamp_mode == RZK_CLAMP_FORM_FACTOR) {
        tau = clamp_scale;
    }
}

void VirtualPointLightCuda::integrate() {
    if (!agg || !d_recv) throw std::runtime_error("VirtualPointLightCuda: integrate before initialize");
    ensure_cuda(cudaSetDevice(agg->device()), "cudaSetDevice");
    const float scale = emitted > 0 ? 1.0f / (float)emitted : 0.0f;
    ensure(rzk_gather_cfg(agg->context(), agg->handle(), d_recv, w * h, w, d_vpls, n_vpl, clamp_mode, tau, scale,
                          d_rgb, 0, 0, nullptr),
           "rzk_gather_cfg");
    img.resize(3 * (size_t)w * h);
    ensure_cuda(cudaMemcpy(img.data(), d_rgb, sizeof(float) * img.size(), cudaMemcpyDeviceToHost), "cudaMemcpy");
    ensure(rzk_context_check(agg->context(), nullptr), "device error word");
}

void VirtualPointLightCuda::transfer_to_frame() {
    FrameBuffer *frame = scene ? scene->get_frame_buffer() : nullptr;
    if (!frame || img.empty()) return;
    ImageFloat *out = frame->get_current_buffer();
    for (int i = 0; i < h; ++i)
        for (int j = 0; j < w; ++j)
            for (int c = 0; c < 3; ++c) (*out)(i, j, c) = img[3 * ((size_t)i * w + j) + c];
}

// ------------------------------------------------------------------------------------
// Scene files

namespace {

// A Scene whose integrator starts unset: the reference's get_scene always installs the
// first view's integrator, but an integrator type this library does not provide is left
// to the caller, and Scene's constructor leaves the pointer uninitialised.
class SceneCuda : public Scene {
public:
    SceneCuda(string name, Aggregate *agg, Shapes *shapes, Materials *materials, Textures *textures,
              Surfaces *surfaces, Lights *lights, Camera *camera, Random *rd)
        : Scene(name, agg, shapes, materials, textures, surfaces, lights, camera, rd) {
        integrator = nullptr;
    }
};

}  // namespace

Scene *load_scene_cuda(const std::string &path, int device) {
    rzk_json *js = nullptr;
    ensure(rzk_json_import(path.c_str(), &js), "rzk_json_import");
    rzk_json_info info;
    rzk_scene_desc d;
    rzk_status st = rzk_json_get_info(js, &info);
    if (st == RZK_OK) st = rzk_json_scene_desc(js, &d);
    if (st != RZK_OK) {
        rzk_json_destroy(js);
        ensure(st, "rzk_json_get_info");
    }
    // the reference's objects, as JsonImporter builds them (json_importer.cc:212-305, 590-760)
    Shapes *shapes = new Shapes();
    Materials *materials = new Materials();
    Textures *textures = new Textures();
    Surfaces *surfaces = new Surfaces();
    Lights *lights = new Lights();
    for (int i = 0; i < d.n_mats; ++i) {
        const rzk_material &m = d.mats[i];
        const Rgb kd(m.kd[0], m.kd[1], m.kd[2]), ks(m.ks[0], m.ks[1], m.ks[2]);
        Bsdf *b = m.type == RZK_BSDF_LAMBERTIAN ? (Bsdf *)new Lambertian(kd)
                : m.type == RZK_BSDF_PHONG      ? (Bsdf *)new ModifiedPhong(kd, ks, m.p0)
                                                : (Bsdf *)new Ward(kd, ks, m.p0, m.p1);
        materials->push_back(new BsdfMaterial(b));
    }
    for (int i = 0; i < d.n_prims; ++i) {
        const float *v = d.prim_v + 12 * i;
        Shape *shape = d.prim_kind[i] == RZK_PRIM_QUAD
                           ? (Shape *)new Quad(get3(v), get3(v + 3), get3(v + 6), get3(v + 9))
                           : (Shape *)new Triangle(get3(v), get3(v + 3), get3(v + 6));
        shapes->push_back(shape);
        Surface surf = d.prim_mat[i] >= 0
                           ? Surface(shape, (*materials)[d.prim_mat[i]])
                           : Surface(shape, Rgb(d.prim_emit[3 * i], d.prim_emit[3 * i + 1], d.prim_emit[3 * i + 2]));
        const int f = d.prim_flags ? d.prim_flags[i] : 0;
        surf.reverse_normal((f & RZK_SURF_FLIPPED) != 0);
        surf.set_two_sided((f & RZK_SURF_TWO_SIDED) != 0);
        surfaces->append(surf);
    }
    // Surface's copy re-points its area light at the copy: collect the lights once the
    // vector has stopped moving
    for (size_t i = 0; i < surfaces->size(); ++i) {
        Surface &surf = (*surfaces)[i];
        if (AreaLight *l = surf.get_area_light()) {
            l->set_surface(&surf);
            lights->push_back(l);
        }
    }
    const Float tmin = d.tmin;
    Camera *camera = nullptr;
    if (info.has_camera) {
        Sensor *sensor = new Sensor(Size2((Float)info.width, (Float)info.height), Size2(info.film_w, info.film_h));
        camera = new Camera();
        camera->set_perspective(get3(info.eye), get3(info.lookat), get3(info.up), info.focal, sensor);
    }
    // the aggregate: json_importer.cc:857-883 with "cuda_lbvh" added
    Aggregate *agg = nullptr;
    try {
        if (info.traversal == RZK_TRAVERSAL_CUDA_LBVH) agg = new AggregateCuda(*surfaces, tmin, device);
        else if (info.traversal == RZK_TRAVERSAL_NONE) agg = new Aggregate(*surfaces);
        else agg = new AggregateBvh(*surfaces);
    } catch (...) {
        rzk_json_destroy(js);
        throw;
    }
    Scene *scene = new SceneCuda(path, agg, shapes, materials, textures, surfaces, lights, camera, new Random());
    scene->set_tmin(tmin);
    if (info.integrator == RZK_JSON_VPL_CUDA) {
        VirtualPointLightCuda *vpl = new VirtualPointLightCuda();
        vpl->set_max_bounce(info.max_bounce);
        if (info.samples > 0) vpl->set_start_particles(info.samples);
        scene->set_integrator(vpl);
    }
    rzk_json_destroy(js);
    return scene;
}

}  // namespace Renzoku
