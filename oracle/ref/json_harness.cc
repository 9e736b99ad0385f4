/*
 * json_harness.cc - TEST INFRASTRUCTURE ONLY.
 *
 * Runs the reference's own JSON scene importer (JsonImporter::load and get_scene,
 * json_importer.cc, over JsonParser, json_parser.cc, and the libjson stand-in under shim/),
 * compiled here from the reference sources, and flattens the scene it builds - the surfaces
 * in order, the lights by kind, the first view's camera and integrator, tmin and the
 * two-sided flag - so that tests can compare the B200 library's JSON import
 * (rzk_json_import) with it field by field.
 *
 * json_importer.cc creates a VirtualPointLight for a "vpl" view.  vpl.cc needs the
 * LibImportance library, which is absent, so within this translation unit that name stands
 * for a PathTracing subclass that only marks the view's integrator type; nothing else of the
 * file is changed.
 */
#include "ref_common.h"
#include "path_tracing.h"
#include "vpl.h"
#include "point_light.h"
#include "spot_light.h"
#include "dir_light.h"

namespace Renzoku {
class RrefVplTag : public PathTracing {};
}
#define VirtualPointLight RrefVplTag
#include "json_importer.cc"
#undef VirtualPointLight

using namespace rref;

extern "C" {

/* Imports `path` and writes, per triangle or quad surface in order (at most `cap`), the
 * fields rref_obj_import writes plus each surface's two-sided flag; the first view's camera
 * (cam) and, in meta: [0] surface count, [1] has camera, [2] integrator (1 path, 2 vpl),
 * [3] max_bounce, [4] samples, [5] point, [6] spot, [7] directional and [8] area lights,
 * [9] two-sided surfaces option; fmeta: [0] tmin, [1] near plane, [2] far plane.
 * light_emit receives each area light's radiance in light-list order (at most light_cap).
 * Returns the number of surfaces written. */
int rref_json_import(const char *path, int cap, int32_t *kind, float *v, int32_t *is_light, float *emit,
                     int32_t *mtype, float *kd, float *ks, float *gl, int32_t *two_sided, rzk_camera *cam,
                     int32_t *meta, float *fmeta, float *light_emit, int light_cap) {
    JsonImporter imp;
    imp.load(path);
    Scene *scene = imp.get_scene();
    Surfaces &surfaces = *scene->get_surfaces();
    const int k = flatten_surfaces(surfaces, cap, kind, v, is_light, emit, mtype, kd, ks, gl);
    int j = 0;
    for (int i = 0; i < surfaces.size() && j < k; ++i) {
        std::vector<Vec3> pos;
        surfaces[i].get_shape()->get_vertex_positions(pos);
        if (pos.size() != 3 && pos.size() != 4) continue;
        two_sided[j++] = surfaces[i].get_two_sided() ? 1 : 0;
    }
    for (int i = 0; i < 16; ++i) meta[i] = 0;
    meta[0] = (int32_t)surfaces.size();
    Camera *c = scene->get_camera();
    if (c) {
        camera_record(c, cam);
        meta[1] = 1;
        fmeta[1] = c->get_near_plane();
        fmeta[2] = c->get_far_plane();
    }
    Integrator *in = scene->get_integrator();
    if (dynamic_cast<RrefVplTag *>(in)) meta[2] = 2;
    else if (dynamic_cast<PathTracing *>(in)) meta[2] = 1;
    if (in) meta[3] = in->get_max_bounce();
    if (MonteCarloIntegrator *mc = dynamic_cast<MonteCarloIntegrator *>(in)) meta[4] = mc->get_num_samples();
    Lights &lights = *scene->get_lights();
    int n_area = 0;
    for (size_t i = 0; i < lights.size(); ++i) {
        Light *l = lights[i];
        if (dynamic_cast<SpotLight *>(l)) meta[6]++;
        else if (dynamic_cast<DirectionalLight *>(l)) meta[7]++;
        else if (dynamic_cast<PointLight *>(l)) meta[5]++;
        else if (AreaLight *a = dynamic_cast<AreaLight *>(l)) {
            if (n_area < light_cap) put3(light_emit + 3 * n_area, area_light_radiance(a));
            n_area++;
            meta[8]++;
        }
    }
    meta[9] = scene->get_two_sided_surfaces() ? 1 : 0;
    fmeta[0] = scene->get_tmin();
    return k;
}

}  // extern "C"
