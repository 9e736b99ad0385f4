/*
 * ref_common.h - TEST INFRASTRUCTURE ONLY: the pieces the reference harness translation
 * units share (the scene bundle and the restated VirtualPointLight members).
 */
#ifndef RZK_REF_COMMON_H_
#define RZK_REF_COMMON_H_

#include <cstdint>
#include <cstring>
#include <vector>
#include <string>
#include <thread>

#include "common.h"
#include "vec3.h"
#include "rgb.h"
#include "triangle.h"
#include "quad.h"
#include "surface.h"
#include "material.h"
#include "lambertian.h"
#include "phong.h"
#include "ward.h"
#include "area_light.h"
#include "aggregate_bvh.h"
#include "camera.h"
#include "sensor.h"
#include "scene.h"
#include "random.h"
#include "form_factor.h"
#include "vpl_interface.h"
#include "vpl_generator.h"
#include "local_geometry.h"
#include "hitrecord.h"
#include "log.h"
#include "light_transport_matrix.h"
#include "cluster_builder.h"
#include "image_sampler.h"

#include "../../include/rzk_types.h"
#include "../../include/rzk_scene.h"

using namespace Renzoku;

extern "C" void rref_rng_stream(uint32_t seed, uint32_t stream, uint32_t path);

namespace rref {

/* Exposes the protected build products of the reference BVH for dumping. */
class BvhProbe : public AggregateBvh {
public:
    explicit BvhProbe(Surfaces &s) : AggregateBvh(s) {}
    const BvhNode *node_array() const { return nodes; }
    int node_count() const { return num_nodes; }
    const unsigned int *morton() const { return sorted_morton; }
    const int *surface_ids() const { return sorted_surface_id; }
    const Triangle *tris() const { return sorted_triangles; }
    int tri_count() const { return num_triangles; }
};

struct RefScene {
    Shapes *shapes = nullptr;
    Materials *materials = nullptr;
    Textures *textures = nullptr;
    Surfaces *surfaces = nullptr;
    Lights *lights = nullptr;
    Camera *camera = nullptr;
    Sensor *sensor = nullptr;
    Random *rd = nullptr;
    BvhProbe *bvh = nullptr;
    Scene *scene = nullptr;
    std::vector<int> tri_first;   /* first flattened triangle of each primitive */
    std::vector<int> tri_count;
    float tmin = RAY_TMIN;
};

Vec3 v3(const float *f);
void put3(float *dst, const Vec3 &v);
void put3(float *dst, const Rgb &c);
void clamp_term(RadianceTerms &term, Float threshold, int mode);
Receiver to_receiver(const RefScene *s, const rzk_receiver &r);
BrdfPointLight to_vpl(const RefScene *s, const rzk_vpl &v);
Rgb gather_point(const RefScene *s, const LocalGeometry &dg, const Vec3 &wo, Material *m,
                 const BrdfPointLight *vpl, int clamp_mode, Float clamp_threshold, bool &visible);
Rgb incident_radiance(const Receiver &r, const BrdfPointLight &vpl, int clamp_mode, Float threshold);

/* The evaluator that LightSlice and MatrixRowColumnSampling call: VirtualPointLight's
 * radiance and incident radiance, as restated in ref_harness.cc against the reference's
 * own types. */
struct HarnessEval : public IVirtualPointLightEvaluator {
    RefScene *s = nullptr;
    int mode = 0, inc_mode = 0;
    float tau = 0.0f, inc_tau = 0.0f;
    Rgb radiance(Scene *, const Receiver &r, const BrdfPointLight &l, bool &visible) override {
        LocalGeometry dg(r);
        return gather_point(s, dg, r.wo, r.m, &l, mode, tau, visible);
    }
    Rgb incident_radiance(Scene *, const Receiver &r, const BrdfPointLight &l) override {
        return rref::incident_radiance(r, l, inc_mode, inc_tau);
    }
};
void fill_receiver(const Ray &r, const HitRecord &rec, rzk_receiver &out, const RefScene *s);
/* obj_harness.cc: per surface whose shape is a triangle or quad, in order (at most cap):
 * kind, 12 vertex floats, light flag, radiance, Bsdf::Type or -1, kd, ks, glossy pair;
 * returns how many were written */
int flatten_surfaces(Surfaces &surfaces, int cap, int32_t *kind, float *v, int32_t *is_light, float *emit,
                     int32_t *mtype, float *kd, float *ks, float *gl);
Rgb area_light_radiance(const AreaLight *l);
/* obj_harness.cc: a Camera as rzk_camera */
void camera_record(Camera *c, rzk_camera *cam);

}  // namespace rref

#endif  // RZK_REF_COMMON_H_
