/*
 * dropin_harness.cc - TEST INFRASTRUCTURE ONLY.
 *
 * Drives the drop-in classes of librzk_dropin.so (renzoku_b200/dropin) through the
 * reference's own interfaces - a Scene from load_scene_cuda, its Aggregate* and
 * Integrator*, an IVplGenerator* - next to the reference's AggregateBvh over the same
 * surfaces, so that tests can compare them.  Linked with the reference's translation units
 * (librzk_ref.so) and librzk_dropin.so.
 */
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "aggregate_bvh.h"
#include "hitrecord.h"
#include "scene.h"
#include "surface.h"
#include "vpl_generator.h"

#include "../../renzoku_b200/dropin/rzk_dropin.h"

using namespace Renzoku;

namespace {

struct DropinScene {
    Scene *scene = nullptr;
    AggregateBvh *bvh = nullptr;   // the reference's BVH over the same surfaces
};

void put3(float *d, const Vec3 &v) { d[0] = v.x(); d[1] = v.y(); d[2] = v.z(); }
Vec3 v3(const float *s) { return Vec3(s[0], s[1], s[2]); }

}  // namespace

extern "C" {

/* load_scene_cuda(path); NULL if it threw. */
void *rdi_load(const char *path, int device) {
    try {
        DropinScene *h = new DropinScene();
        h->scene = load_scene_cuda(path, device);
        h->bvh = new AggregateBvh(*h->scene->get_surfaces());
        return h;
    } catch (const std::exception &) {
        return nullptr;
    }
}

/* What the file selected: bit 0 the aggregate is an AggregateCuda, bit 1 the integrator is
 * a VirtualPointLightCuda. */
int rdi_kinds(void *hp) {
    DropinScene *h = (DropinScene *)hp;
    int k = 0;
    if (dynamic_cast<AggregateCuda *>(h->scene->get_aggregate())) k |= 1;
    if (dynamic_cast<VirtualPointLightCuda *>(h->scene->get_integrator())) k |= 2;
    return k;
}

/* Aggregate::hit(p, q, tmin, time) per segment through the scene's Aggregate* (the
 * virtual call the reference's integrators make), the batched hit_segments, and the
 * reference AggregateBvh's answer. */
int rdi_segments(void *hp, const float *p, const float *q, int n, uint8_t *virt, uint8_t *batch, uint8_t *ref) {
    DropinScene *h = (DropinScene *)hp;
    try {
        Aggregate *agg = h->scene->get_aggregate();
        const Float tmin = h->scene->get_tmin(), tick = h->scene->get_tick();
        std::vector<Vec3> P(n), Q(n);
        for (int i = 0; i < n; ++i) {
            P[i] = v3(p + 3 * i);
            Q[i] = v3(q + 3 * i);
            virt[i] = agg->hit(P[i], Q[i], tmin, tick) ? 1 : 0;
            ref[i] = static_cast<Aggregate *>(h->bvh)->hit(P[i], Q[i], tmin, tick) ? 1 : 0;
        }
        std::vector<char> b(n);
        AggregateCuda *cuda = dynamic_cast<AggregateCuda *>(agg);
        if (cuda) cuda->hit_segments(P.data(), Q.data(), n, tmin, (bool *)b.data());
        for (int i = 0; i < n; ++i) batch[i] = cuda ? (uint8_t)b[i] : 0;
        return 0;
    } catch (const std::exception &) {
        return -1;
    }
}

/* Closest hits of rays Ray(o, d) over [tmin, max_tmax]: per ray the hit flag, t, position,
 * geometric and shading normals, material index (-1 none) and area-light flag, from the
 * scene's Aggregate* and from the reference AggregateBvh (rec[2 * i] and rec[2 * i + 1],
 * 14 floats each). */
int rdi_closest(void *hp, const float *o, const float *d, int n, float *rec) {
    DropinScene *h = (DropinScene *)hp;
    try {
        Aggregate *agg = h->scene->get_aggregate();
        const Float tmin = h->scene->get_tmin(), tmax = h->scene->get_max_tmax(), tick = h->scene->get_tick();
        Materials *mats = h->scene->get_materials();
        for (int i = 0; i < n; ++i) {
            Ray r(v3(o + 3 * i), v3(d + 3 * i));
            for (int side = 0; side < 2; ++side) {
                HitRecord hr;
                const bool hit = side == 0 ? agg->hit(r, tmin, tmax, tick, hr) : h->bvh->hit(r, tmin, tmax, tick, hr);
                float *x = rec + 14 * (2 * (size_t)i + side);
                std::memset(x, 0, 14 * sizeof(float));
                x[0] = hit ? 1.0f : 0.0f;
                if (!hit) continue;
                x[1] = hr.t;
                put3(x + 2, r.point(hr.t));
                put3(x + 5, hr.normal);
                put3(x + 8, hr.shading_normal);
                int m = -1;
                for (size_t k = 0; k < mats->size(); ++k)
                    if ((*mats)[k] == hr.material) m = (int)k;
                x[11] = (float)m;
                x[12] = hr.light ? 1.0f : 0.0f;
                x[13] = hr.beta + hr.gamma;
            }
        }
        return 0;
    } catch (const std::exception &) {
        return -1;
    }
}

/* IVplGenerator::spawn through VplGeneratorCuda: positions, powers, bounces and the
 * previous-VPL references of what it appended; returns the count (-1 on error). */
int rdi_vpls(void *hp, uint32_t seed, int particles, int max_bounce, float *p, float *contrib, int32_t *bounce,
             int32_t *prev, int cap) {
    DropinScene *h = (DropinScene *)hp;
    try {
        VplGeneratorCuda gen(seed);
        IVplGenerator *g = &gen;
        BrdfPointLights out;
        g->spawn(h->scene, particles, max_bounce, out);
        const int n = std::min((int)out.size(), cap);
        for (int i = 0; i < n; ++i) {
            put3(p + 3 * i, out[i].org());
            const Rgb c = out[i].power();
            contrib[3 * i] = c.red(); contrib[3 * i + 1] = c.green(); contrib[3 * i + 2] = c.blue();
            bounce[i] = out[i].get_bounce();
            prev[i] = out[i].get_prev().index;
        }
        return (int)out.size();
    } catch (const std::exception &) {
        return -1;
    }
}

/* One frame through the scene's Integrator* (initialize, integrate, transfer_to_frame):
 * the image [h][w][3] (cap floats at most) and the integrator's size, VPL count, emitted
 * particles and clamp threshold in info[5]. */
int rdi_render(void *hp, int start_particles, int max_vpls, uint32_t seed, float *img, int cap, float *info) {
    DropinScene *h = (DropinScene *)hp;
    try {
        VirtualPointLightCuda *vpl = dynamic_cast<VirtualPointLightCuda *>(h->scene->get_integrator());
        if (!vpl) return -1;
        vpl->set_start_particles(start_particles);
        vpl->set_max_vpls(max_vpls);
        vpl->set_seed(seed);
        Integrator *it = vpl;
        it->initialize(h->scene);
        it->integrate();
        it->transfer_to_frame();
        const std::vector<float> &im = vpl->image();
        std::memcpy(img, im.data(), sizeof(float) * std::min((size_t)cap, im.size()));
        info[0] = (float)vpl->width();
        info[1] = (float)vpl->height();
        info[2] = (float)vpl->num_vpls();
        info[3] = (float)vpl->num_emitted();
        info[4] = vpl->clamping_threshold();
        return 0;
    } catch (const std::exception &) {
        return -2;
    }
}

}  // extern "C"
