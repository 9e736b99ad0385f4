/*
 * obj_harness.cc - TEST INFRASTRUCTURE ONLY.
 *
 * Runs the reference's own OBJ importer (ObjImporter::load, obj_importer.cc, over its
 * parser obj_parser.cpp), compiled here from the reference sources, and flattens what it
 * builds - the surfaces in order, each shape's vertices, each material's BSDF parameters
 * and each area light's radiance, and the camera - so that tests can compare the B200
 * library's OBJ import (rzk_obj_import) with it field by field.
 */
#include "ref_common.h"
#include "obj_importer.h"

using namespace rref;

namespace {

/* Reads the radiance an AreaLight was built with. */
class LightProbe : public AreaLight {
public:
    static Rgb radiance_of(const AreaLight *l) { return static_cast<const LightProbe *>(l)->radiance; }
};

}  // namespace

namespace rref {

int flatten_surfaces(Surfaces &surfaces, int cap, int32_t *kind, float *v, int32_t *is_light, float *emit,
                     int32_t *mtype, float *kd, float *ks, float *gl) {
    int k = 0;
    for (int i = 0; i < surfaces.size() && k < cap; ++i) {
        Surface &sf = surfaces[i];
        Shape *sh = sf.get_shape();
        std::vector<Vec3> pos;
        sh->get_vertex_positions(pos);
        if (pos.size() != 3 && pos.size() != 4) continue;
        kind[k] = (int32_t)pos.size();
        for (int c = 0; c < 12; ++c) v[12 * k + c] = 0.0f;
        for (size_t j = 0; j < pos.size(); ++j) put3(v + 12 * k + 3 * j, pos[j]);
        is_light[k] = sf.is_light() ? 1 : 0;
        for (int c = 0; c < 3; ++c) { emit[3 * k + c] = 0.0f; kd[3 * k + c] = 0.0f; ks[3 * k + c] = 0.0f; }
        gl[2 * k] = gl[2 * k + 1] = 0.0f;
        mtype[k] = -1;
        if (sf.is_light()) {
            put3(emit + 3 * k, LightProbe::radiance_of(sf.get_area_light()));
        } else if (Material *m = sf.get_material()) {
            Bsdf *b = m->get_bsdf();
            if (Lambertian *l = dynamic_cast<Lambertian *>(b)) {
                mtype[k] = (int32_t)l->get_bsdf_type();
                put3(kd + 3 * k, l->get_diffuse_component());
            } else if (ModifiedPhong *p = dynamic_cast<ModifiedPhong *>(b)) {
                mtype[k] = (int32_t)p->get_bsdf_type();
                put3(kd + 3 * k, p->get_diffuse_component());
                put3(ks + 3 * k, p->get_specular_component());
                Vec2 g = p->get_glossy_coefficients();
                gl[2 * k] = g.x(); gl[2 * k + 1] = g.y();
            } else if (Ward *w = dynamic_cast<Ward *>(b)) {
                mtype[k] = (int32_t)w->get_bsdf_type();
                put3(kd + 3 * k, w->get_diffuse_component());
                put3(ks + 3 * k, w->get_specular_component());
                Vec2 g = w->get_glossy_coefficients();
                gl[2 * k] = g.x(); gl[2 * k + 1] = g.y();
            }
        }
        k++;
    }
    return k;
}

Rgb area_light_radiance(const AreaLight *l) { return LightProbe::radiance_of(l); }

void camera_record(Camera *c, rzk_camera *cam) {
    Sensor *sn = c->get_sensor();
    Onb onb = c->get_onb();
    put3(cam->eye, c->get_eye());
    put3(cam->u, onb.u());
    put3(cam->v, onb.v());
    put3(cam->n, onb.n());
    cam->focal = c->get_focal_length();
    Vec2 cop = sn->get_cop();
    Vec2 sc = sn->get_image_film_ratio();
    cam->cop[0] = cop.x(); cam->cop[1] = cop.y();
    cam->scale[0] = sc.x(); cam->scale[1] = sc.y();
    cam->width = (int)sn->get_image_size().width;
    cam->height = (int)sn->get_image_size().height;
    cam->pad = 0;
}

}  // namespace rref

extern "C" {

/* Imports `path` and writes, per surface whose shape is a triangle or quad (in surface
 * order, at most `cap`): kind (3 or 4), 12 vertex floats (p3 = 0 for a triangle), whether
 * it is a light, the light's radiance, and for a material its Bsdf::Type (0 Lambertian,
 * 1 Ward, 2 Phong; -1 any other BSDF), kd, ks and (n, 0) or (ax, ay).  cam (may be NULL) receives
 * the camera as rzk_camera when the scene has one.  Returns the number of such surfaces,
 * and the total surface count in *n_surfaces. */
int rref_obj_import(const char *path, int cap, int32_t *kind, float *v, int32_t *is_light, float *emit,
                    int32_t *mtype, float *kd, float *ks, float *gl, rzk_camera *cam, int32_t *has_cam,
                    int32_t *n_surfaces) {
    ObjImporter imp;
    imp.load(path);
    Surfaces surfaces;
    imp.get_surfaces(surfaces);
    *n_surfaces = (int32_t)surfaces.size();
    const int k = flatten_surfaces(surfaces, cap, kind, v, is_light, emit, mtype, kd, ks, gl);
    *has_cam = 0;
    Scene *scene = imp.get_scene();   // NULL without a light or a camera
    if (scene && cam) {
        camera_record(scene->get_camera(), cam);
        *has_cam = 1;
    }
    return k;
}

}  // extern "C"
