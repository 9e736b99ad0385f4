// rzk_json.cu - the reference's JSON scene files, as a scene description for rzk_scene_create.
// Host code only.
//
// The file is read as the reference reads it (JsonParser over libjson's event parser,
// json_parser.cc:11-253, json_parser.h): an object at the first level under the root whose
// key is "geometry", "materials", "light_specs", "cameras" or "scene" is handed to the
// importer as soon as it is complete, so later sections see only what earlier ones defined;
// a null value adds no value (keys and values of that object no longer pair up, as there);
// integers and reals keep their text and are read with atoi / atof, a real cast to float.
//
// The scene follows JsonImporter (json_importer.cc:36-899): OBJ meshes under
// <scene directory>/mesh/ named by their key (and "<key>.<object>" per `o` object, matched by
// prefix), Lambertian / Ward / Phong materials built from the given parameters as they are,
// area lights bound to meshes, the pinhole camera of the first usable view, its integrator's
// max_bounce and samples, and the geometry options tmin and two_sided_surfaces.  What this
// path does not model - glass and mirror materials, spheres, point, spot and directional
// lights - is counted in rzk_json_info and left out.  Where the reference stops (a missing
// file, a syntax error, a missing key that it dereferences, a value of the wrong type) the
// import fails with RZK_ERR_INVALID; where it logs an error and goes on, so does this, and
// the entry is counted in `skipped`.
#include "rzk_internal.cuh"
#include "rzk_scenefile.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

// ---------------------------------------------------------------------------------------
// JSON values (json_parser.h): objects keep keys and values in two lists, as there.
struct JVal {
    enum Kind { OBJ, ARR, STR, INT, REAL, BOOL } kind = OBJ;
    std::string text;                 // STR: the string; INT / REAL: the number's text; BOOL: "1" / "0"
    std::vector<std::string> keys;    // OBJ
    std::vector<JVal> vals;           // OBJ values (a null adds none) or ARR items
};

struct Fail : std::runtime_error {
    explicit Fail(const std::string &s) : std::runtime_error(s) {}
};

// JsonValue / JsonPrimitive / JsonArray / JsonObject accessors: a wrong type throws there
// (JsonException), a missing key dereferences null; both end the import here.
const JVal &need(const JVal *v, const char *what) {
    if (!v) throw Fail(std::string("missing ") + what);
    return *v;
}
const JVal *get(const JVal &o, const std::string &key) {   // JsonObject::get_value
    if (o.kind != JVal::OBJ) throw Fail("not an object");
    for (size_t i = 0; i < o.keys.size(); ++i)
        if (o.keys[i] == key) return i < o.vals.size() ? &o.vals[i] : nullptr;
    return nullptr;
}
bool has(const JVal &o, const std::string &key) {          // JsonObject::has_key
    for (const std::string &k : o.keys)
        if (k == key) return true;
    return false;
}
const JVal &strict(const JVal &o, const char *key) { return need(get(o, key), key); }
const JVal &as_object(const JVal &v) {
    if (v.kind != JVal::OBJ) throw Fail("not an object");
    return v;
}
const JVal &as_array(const JVal &v) {
    if (v.kind != JVal::ARR) throw Fail("not an array");
    return v;
}
std::string as_string(const JVal &v) {
    if (v.kind != JVal::STR) throw Fail("not a string");
    return v.text;
}
int as_int(const JVal &v) {
    if (v.kind != JVal::INT) throw Fail("not an integer");
    return std::atoi(v.text.c_str());
}
float as_numeric(const JVal &v) {                            // JsonValue::to_numeric
    if (v.kind == JVal::INT) return (float)std::atoi(v.text.c_str());
    if (v.kind == JVal::REAL) return (float)std::atof(v.text.c_str());
    throw Fail("not a number");
}
bool as_bool(const JVal &v) {
    if (v.kind != JVal::BOOL) throw Fail("not a boolean");
    return v.text[0] != '0';
}
void as_vec3(const JVal &v, float *out) {                    // JsonArray::to_vec3 / to_rgb
    const JVal &a = as_array(v);
    if (a.vals.size() < 3) throw Fail("short array");
    for (int c = 0; c < 3; ++c) out[c] = as_numeric(a.vals[c]);
}
void as_size2(const JVal &v, float *out) {
    const JVal &a = as_array(v);
    if (a.vals.size() < 2) throw Fail("short array");
    for (int c = 0; c < 2; ++c) out[c] = as_numeric(a.vals[c]);
}

// ---------------------------------------------------------------------------------------
// The scene as JsonImporter builds it.
struct Shape {
    std::string name;
    bool sphere = false;
    int kind = 0;
    float v[12] = {0};
    int surface = -1;   // Shape::surface_index
    int shading = 0;    // ObjShape::shading
};
enum { S_MATERIAL, S_LIGHT, S_UNSUPPORTED, S_SPHERE };
struct Surf {
    int type = S_MATERIAL;
    int shape = -1;     // -1: an OBJ light quad or sphere that is in no shape list
    int kind = 0;
    float v[12] = {0};
    int mat = -1;       // index into Importer::mats
    float emit[3] = {0, 0, 0};
};
struct Mat {
    std::string name;
    bool modelled = false;
    rzk_material m;
};
enum { L_AREA, L_POINT, L_SPOT, L_DIRECTIONAL };
struct LightSpec {
    std::string name;
    int type = L_AREA;
    float radiance[3] = {0, 0, 0};
};
struct Cam {
    std::string name;
    float eye[3], lookat[3], up[3], focal, image[2], film[2], near_plane, far_plane;
};
struct View {
    int integrator, max_bounce, samples, camera;
};

struct Importer {
    std::string scene_path;
    std::vector<Shape> shapes;
    std::vector<Surf> surfaces;
    std::vector<Mat> mats;
    std::vector<LightSpec> specs;
    std::vector<Cam> cams;
    std::vector<View> views;
    const JVal *options = nullptr;
    JVal options_copy;
    int lights[4] = {0, 0, 0, 0};
    rzk_json_info info;

    Importer() { std::memset(&info, 0, sizeof(info)); }

    // JsonImporter::process_object (json_importer.cc:55-86)
    bool process(const std::string &key, const JVal &obj) {
        if (key == "geometry") { load_geometry(obj); return true; }
        if (key == "materials") { load_materials(obj); return true; }
        if (key == "light_specs") { load_light_specs(obj); return true; }
        if (key == "cameras") { load_cameras(obj); return true; }
        if (key == "scene") { load_scene(obj); return true; }
        return false;
    }

    // an object's i-th value (JsonObject::values[i]); its keys and values may not pair up
    static const JVal &value_at(const JVal &o, size_t i) {
        if (i >= o.vals.size()) throw Fail("key without a value");
        return o.vals[i];
    }

    // ObjImporter::load of <scene>/mesh/<file> and load_shapes_from_obj
    // (json_importer.cc:131-152): the shapes named by the key
    int load_obj(const std::string &key, const std::string &file, rzk::ObjModel &m) {
        const std::string path = scene_path + "mesh/" + file;
        if (rzk::obj_load(path.c_str(), m) != RZK_OK) throw Fail("cannot read " + path);
        info.obj_files++;
        const int base = (int)shapes.size();
        for (const rzk::ObjShape &s : m.shapes) {
            Shape sh;
            sh.name = s.object >= 0 ? key + "." + m.object_names[s.object] : key;
            sh.kind = s.kind;
            std::memcpy(sh.v, s.v, sizeof(sh.v));
            sh.surface = s.surface;   // the OBJ importer's own surface index
            sh.shading = s.shading;
            shapes.push_back(sh);
        }
        return base;
    }

    // JsonImporter::load_geometry (json_importer.cc:154-209)
    void load_geometry(const JVal &obj) {
        for (size_t i = 0; i < obj.keys.size(); ++i) {
            const JVal &v = value_at(obj, i);
            const std::string &name = obj.keys[i];
            if (v.kind == JVal::ARR) { info.skipped++; continue; }
            if (v.kind != JVal::OBJ) {
                if (v.kind != JVal::STR) { info.skipped++; continue; }
                rzk::ObjModel m;
                load_obj(name, v.text, m);
                continue;
            }
            const std::string type = as_string(strict(v, "type"));
            if (type == "sphere") {
                float c[3];
                as_vec3(strict(v, "center"), c);
                (void)as_numeric(strict(v, "radius"));
                Shape sh;
                sh.name = name;
                sh.sphere = true;
                shapes.push_back(sh);
            } else {
                info.skipped++;
            }
        }
    }

    // JsonImporter::load_materials (json_importer.cc:211-310): BSDFs from their parameters
    // as given (no scaling of kd and ks, unlike the OBJ importer)
    void load_materials(const JVal &obj) {
        for (size_t i = 0; i < obj.keys.size(); ++i) {
            const JVal &spec = as_object(value_at(obj, i));
            const std::string type = as_string(need(get(spec, "type"), "type"));
            Mat mt;
            mt.name = obj.keys[i];
            std::memset(&mt.m, 0, sizeof(mt.m));
            if (type == "lambertian") {
                as_vec3(need(get(spec, "kd"), "kd"), mt.m.kd);
                mt.m.type = RZK_BSDF_LAMBERTIAN;
                mt.modelled = true;
            } else if (type == "ward") {
                as_vec3(need(get(spec, "kd"), "kd"), mt.m.kd);
                as_vec3(need(get(spec, "ks"), "ks"), mt.m.ks);
                mt.m.p0 = as_numeric(need(get(spec, "ax"), "ax"));
                mt.m.p1 = as_numeric(need(get(spec, "ay"), "ay"));
                mt.m.type = RZK_BSDF_WARD;
                mt.modelled = true;
            } else if (type == "phong") {
                as_vec3(need(get(spec, "kd"), "kd"), mt.m.kd);
                as_vec3(need(get(spec, "ks"), "ks"), mt.m.ks);
                mt.m.p0 = as_numeric(need(get(spec, "n"), "n"));
                mt.m.type = RZK_BSDF_PHONG;
                mt.modelled = true;
            } else if (type == "glass") {
                (void)as_numeric(strict(spec, "n"));
                if (has(spec, "kd")) { float kd[3]; as_vec3(strict(spec, "kd"), kd); }
            } else if (type == "mirror") {
                if (has(spec, "kd")) { float kd[3]; as_vec3(need(get(spec, "kd"), "kd"), kd); }
            } else {
                info.skipped++;
                continue;
            }
            mats.push_back(mt);
        }
    }

    // JsonImporter::load_light_specs (json_importer.cc:312-409)
    void load_light_specs(const JVal &obj) {
        for (size_t i = 0; i < obj.keys.size(); ++i) {
            const JVal &spec = as_object(value_at(obj, i));
            const std::string type = as_string(need(get(spec, "type"), "type"));
            LightSpec ls;
            ls.name = obj.keys[i];
            float tmp[3];
            if (type == "area") {
                ls.type = L_AREA;
                as_vec3(need(get(spec, "radiance"), "radiance"), ls.radiance);
            } else if (type == "directional") {
                ls.type = L_DIRECTIONAL;
                as_vec3(strict(spec, "radiance"), ls.radiance);
                as_vec3(strict(spec, "direction"), tmp);
            } else if (type == "point") {
                ls.type = L_POINT;
                as_vec3(need(get(spec, "radiance"), "radiance"), ls.radiance);
                as_vec3(need(get(spec, "position"), "position"), tmp);
            } else if (type == "spot") {
                ls.type = L_SPOT;
                as_vec3(need(get(spec, "radiance"), "radiance"), ls.radiance);
                as_vec3(need(get(spec, "position"), "position"), tmp);
                as_vec3(need(get(spec, "direction"), "direction"), tmp);
                (void)as_numeric(need(get(spec, "phi"), "phi"));
                (void)as_numeric(need(get(spec, "theta"), "theta"));
                (void)as_numeric(need(get(spec, "falloff"), "falloff"));
            } else {
                info.skipped++;
                continue;
            }
            specs.push_back(ls);
        }
    }

    // JsonImporter::load_cameras (json_importer.cc:411-448): the focal length as given, or
    // from the field of view over the film height (Camera::focal_length_from_fov,
    // camera.h:228-230)
    void load_cameras(const JVal &obj) {
        for (size_t i = 0; i < obj.keys.size(); ++i) {
            const JVal &spec = as_object(value_at(obj, i));
            const std::string type = as_string(need(get(spec, "type"), "type"));
            if (type != "pinhole") { info.skipped++; continue; }
            Cam c;
            c.name = obj.keys[i];
            as_vec3(need(get(spec, "pos"), "pos"), c.eye);
            as_vec3(need(get(spec, "lookat"), "lookat"), c.lookat);
            as_vec3(need(get(spec, "up"), "up"), c.up);
            c.near_plane = as_numeric(need(get(spec, "near"), "near"));
            c.far_plane = as_numeric(need(get(spec, "far"), "far"));
            as_size2(need(get(spec, "image"), "image"), c.image);
            as_size2(need(get(spec, "film"), "film"), c.film);
            if (const JVal *f = get(spec, "focal")) {
                c.focal = as_numeric(*f);
            } else if (const JVal *fov = get(spec, "fov")) {
                const float DEGREE_TO_RADIAN = rzk::A_PI / 180.0f;
                const float deg = as_numeric(*fov);
                c.focal = c.film[1] / (2.0f * tanf(deg / 2 * DEGREE_TO_RADIAN));
            } else {
                throw Fail("camera without focal length or field of view");
            }
            cams.push_back(c);
        }
    }

    int camera_index(const std::string &name) const {   // JsonImporter::get_camera
        for (size_t i = 0; i < cams.size(); ++i)
            if (cams[i].name == name) return (int)i;
        return -1;
    }
    int material_index(const std::string &name) const {   // JsonImporter::get_material
        for (size_t i = 0; i < mats.size(); ++i)
            if (mats[i].name == name) return (int)i;
        return -1;
    }
    const LightSpec *light_spec(const std::string &name) const {
        for (const LightSpec &s : specs)
            if (s.name == name) return &s;
        return nullptr;
    }
    // JsonImporter::get_shape (json_importer.cc:98-111): the name itself, or any name that
    // begins with "<name>."
    std::vector<int> matching_shapes(const std::string &name) const {
        std::vector<int> out;
        const std::string prefix = name + ".";
        for (size_t i = 0; i < shapes.size(); ++i)
            if (shapes[i].name == name || shapes[i].name.compare(0, prefix.size(), prefix) == 0)
                out.push_back((int)i);
        return out;
    }

    // JsonImporter::load_scene / load_world (json_importer.cc:450-495)
    void load_scene(const JVal &obj) {
        const JVal &world = as_object(strict(obj, "world"));
        load_surfaces(as_object(need(get(world, "surfaces"), "surfaces")));
        load_lights(as_object(need(get(world, "lights"), "lights")));
        load_views(as_object(strict(obj, "views")));
        if (const JVal *o = get(obj, "options")) {
            options_copy = as_object(*o);
            options = &options_copy;
        }
    }

    // JsonImporter::load_camera_views / load_integrator (json_importer.cc:497-595)
    void load_views(const JVal &list) {
        for (size_t i = 0; i < list.keys.size(); ++i) {
            const JVal &view = as_object(value_at(list, i));
            const JVal &spec = as_object(need(get(view, "integrator"), "integrator"));
            View vw;
            vw.max_bounce = as_int(need(get(spec, "max_bounce"), "max_bounce"));
            const std::string type = as_string(need(get(spec, "type"), "type"));
            // "vpl_cuda" is this library's extension of the seam: the device gather, read with
            // the keys of "vpl"
            if (type != "path" && type != "vpl" && type != "vpl_cuda") { info.skipped++; continue; }
            vw.samples = as_int(need(get(spec, "samples"), "samples"));
            vw.integrator = type == "path" ? RZK_JSON_PATH : type == "vpl" ? RZK_JSON_VPL : RZK_JSON_VPL_CUDA;
            vw.camera = camera_index(as_string(need(get(view, "camera"), "camera")));
            if (vw.camera < 0) { info.skipped++; continue; }
            views.push_back(vw);
        }
    }

    void append(Surf sf) {   // Surfaces::append (surface.h:123-127)
        if (sf.shape >= 0) shapes[sf.shape].surface = (int)surfaces.size();
        surfaces.push_back(sf);
    }
    Surf surface_of(int shape) const {
        Surf sf;
        sf.shape = shape;
        sf.kind = shapes[shape].kind;
        std::memcpy(sf.v, shapes[shape].v, sizeof(sf.v));
        return sf;
    }

    // JsonImporter::load_surfaces (json_importer.cc:597-692)
    void load_surfaces(const JVal &obj) {
        for (size_t i = 0; i < obj.keys.size(); ++i) {
            const std::string &name = obj.keys[i];
            const JVal &v = value_at(obj, i);
            if (v.kind == JVal::STR) {
                // a whole OBJ scene: its shapes, materials, surfaces and lights appended; the
                // shapes keep the OBJ importer's own surface indices
                rzk::ObjModel m;
                const int base = load_obj(name, v.text, m);
                const int mat_base = (int)mats.size();
                std::vector<int> mtl_of_mat(m.mats.size(), -1);
                for (size_t k = 0; k < m.mtl_names.size(); ++k) {
                    Mat mt;
                    mt.name = m.mtl_names[k];
                    mt.modelled = m.mtl_mats[k] >= 0;
                    if (mt.modelled) {
                        mt.m = m.mats[m.mtl_mats[k]];
                        mtl_of_mat[m.mtl_mats[k]] = (int)k;
                    } else {
                        std::memset(&mt.m, 0, sizeof(mt.m));
                    }
                    mats.push_back(mt);
                }
                for (const rzk::ObjSurface &s : m.surfaces) {
                    Surf sf;
                    sf.shape = s.shape >= 0 ? base + s.shape : -1;
                    sf.kind = s.kind;
                    std::memcpy(sf.v, s.v, sizeof(sf.v));
                    std::memcpy(sf.emit, s.emit, sizeof(sf.emit));
                    switch (s.type) {
                    case rzk::OBJ_SURF_MATERIAL: sf.type = S_MATERIAL; sf.mat = mat_base + mtl_of_mat[s.mat]; break;
                    case rzk::OBJ_SURF_LIGHT: sf.type = S_LIGHT; lights[L_AREA]++; break;
                    case rzk::OBJ_SURF_UNSUPPORTED: sf.type = S_UNSUPPORTED; break;
                    default: sf.type = S_SPHERE; break;
                    }
                    surfaces.push_back(sf);   // vector::insert: no surface index is set
                }
                lights[L_POINT] += m.info.point_lights;
                continue;
            }
            const JVal &surf = as_object(v);
            if (has(surf, "visible") && !as_bool(need(get(surf, "visible"), "visible"))) continue;
            const std::string mesh = as_string(need(get(surf, "mesh"), "mesh"));
            if (mesh.empty()) { info.skipped++; continue; }
            const std::string bsdf = as_string(need(get(surf, "bsdf"), "bsdf"));
            if (bsdf.empty()) { info.skipped++; continue; }
            const std::vector<int> pieces = matching_shapes(mesh);
            const int mat = material_index(bsdf);
            if (mat < 0) { info.skipped++; continue; }
            for (int p : pieces) {
                Surf sf = surface_of(p);
                sf.type = shapes[p].sphere ? S_SPHERE : (mats[mat].modelled ? S_MATERIAL : S_UNSUPPORTED);
                sf.mat = mat;
                const int k = shapes[p].surface;
                if (k >= 0) {
                    // replaces the shape's surface in place when the index names it, else the
                    // reference reports a surface/shape index error and binds nothing
                    if (k < (int)surfaces.size() && surfaces[k].shape == p) surfaces[k] = sf;
                    else info.skipped++;
                } else {
                    append(sf);
                }
            }
        }
    }

    // JsonImporter::load_lights (json_importer.cc:694-775)
    void load_lights(const JVal &obj) {
        for (size_t i = 0; i < obj.keys.size(); ++i) {
            const JVal &v = value_at(obj, i);
            if (v.kind == JVal::STR) {
                const LightSpec *s = light_spec(v.text);
                if (!s || s->type == L_AREA) { info.skipped++; continue; }
                lights[s->type]++;
            } else if (v.kind == JVal::OBJ) {
                const LightSpec *s = light_spec(as_string(strict(v, "light")));
                if (!s || s->type != L_AREA) { info.skipped++; continue; }
                const std::vector<int> pieces = matching_shapes(as_string(strict(v, "mesh")));
                for (int p : pieces) {
                    Surf sf = surface_of(p);
                    sf.type = shapes[p].sphere ? S_SPHERE : S_LIGHT;
                    std::memcpy(sf.emit, s->radiance, sizeof(sf.emit));
                    append(sf);
                    lights[L_AREA]++;
                }
            }
        }
    }

    // JsonImporter::get_scene / apply_scene_options (json_importer.cc:777-899): the first
    // view's camera and integrator, tmin and two-sided surfaces; then the surfaces in order
    void finish(rzk::SceneArrays &out) {
        info.tmin = 1e-3f;   // RAY_TMIN (common.h:48)
        if (options) {
            if (const JVal *g = get(*options, "geometry")) {
                const JVal &geo = as_object(*g);
                if (has(geo, "traversal")) {
                    // json_importer.cc:862-876: "bvh", "none", anything else reverts to BVH;
                    // "cuda_lbvh" selects this library's device LBVH
                    const std::string t = as_string(need(get(geo, "traversal"), "traversal"));
                    info.traversal = t == "none" ? RZK_TRAVERSAL_NONE
                                   : t == "cuda_lbvh" ? RZK_TRAVERSAL_CUDA_LBVH : RZK_TRAVERSAL_BVH;
                }
                if (has(geo, "tmin")) info.tmin = as_numeric(need(get(geo, "tmin"), "tmin"));
                if (has(geo, "two_sided_surfaces"))
                    info.two_sided = as_bool(need(get(geo, "two_sided_surfaces"), "two_sided_surfaces")) ? 1 : 0;
            }
            // the OpenGL viewer's options are read (and required where the reference requires
            // them) though nothing here uses them (json_importer.cc:810-829)
            if (const JVal *o = get(*options, "opengl")) {
                const JVal &gl = as_object(*o);
                if (const JVal *v = get(gl, "shadow_map")) {
                    const JVal &sm = as_object(*v);
                    (void)as_numeric(strict(sm, "polygon_offset_factor"));
                    (void)as_numeric(strict(sm, "polygon_offset_unit"));
                }
                if (const JVal *v = get(gl, "sensor")) {
                    const JVal &so = as_object(*v);
                    (void)as_string(strict(so, "multi_sample"));
                    (void)as_int(strict(so, "num_antialiased_samples"));
                }
            }
            if (const JVal *e = get(*options, "experimental")) (void)as_object(*e);
        }
        if (!views.empty()) {
            const View &vw = views[0];
            const Cam &c = cams[vw.camera];
            info.has_camera = 1;
            std::memcpy(info.eye, c.eye, sizeof(info.eye));
            std::memcpy(info.lookat, c.lookat, sizeof(info.lookat));
            std::memcpy(info.up, c.up, sizeof(info.up));
            info.focal = c.focal;
            info.width = (int32_t)c.image[0];
            info.height = (int32_t)c.image[1];
            info.film_w = c.film[0];
            info.film_h = c.film[1];
            info.near_plane = c.near_plane;
            info.far_plane = c.far_plane;
            info.integrator = vw.integrator;
            info.max_bounce = vw.max_bounce;
            info.samples = vw.samples;
        }
        std::vector<int> scene_mat(mats.size(), -1);
        const int flags = info.two_sided ? RZK_SURF_TWO_SIDED : 0;
        for (const Surf &sf : surfaces) {
            if ((sf.type == S_MATERIAL || sf.type == S_LIGHT) && sf.shape >= 0) {
                if (shapes[sf.shape].shading == 1) info.faces_with_vertex_normals++;
                else if (shapes[sf.shape].shading == 2) info.smoothed_faces++;
            }
            if (sf.type == S_MATERIAL) {
                if (scene_mat[sf.mat] < 0) {
                    scene_mat[sf.mat] = (int)out.mats.size();
                    out.mats.push_back(mats[sf.mat].m);
                }
                out.add(sf.kind, sf.v, scene_mat[sf.mat], nullptr, flags);
            } else if (sf.type == S_LIGHT) {
                out.add(sf.kind, sf.v, -1, sf.emit, flags);
                info.n_lights++;
            } else if (sf.type == S_UNSUPPORTED) {
                info.surfaces_unsupported_material++;
            } else {
                info.spheres++;
            }
        }
        info.n_prims = (int32_t)out.kind.size();
        info.n_mats = (int32_t)out.mats.size();
        info.point_lights = lights[L_POINT];
        info.spot_lights = lights[L_SPOT];
        info.directional_lights = lights[L_DIRECTIONAL];
    }
};

// ---------------------------------------------------------------------------------------
// RFC 8259 text into JVal, handing each complete first-level object of a root object to the
// importer (JsonParser::end_object, json_parser.cc:161-185).
struct Reader {
    const char *p, *end;
    Importer *imp;

    void ws() {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
    }
    [[noreturn]] void bad() { throw Fail("JSON syntax error"); }
    void expect(char c) {
        ws();
        if (p >= end || *p != c) bad();
        ++p;
    }
    static void utf8(std::string &s, unsigned cp) {
        if (cp < 0x80) {
            s += (char)cp;
        } else if (cp < 0x800) {
            s += (char)(0xc0 | (cp >> 6));
            s += (char)(0x80 | (cp & 0x3f));
        } else if (cp < 0x10000) {
            s += (char)(0xe0 | (cp >> 12));
            s += (char)(0x80 | ((cp >> 6) & 0x3f));
            s += (char)(0x80 | (cp & 0x3f));
        } else {
            s += (char)(0xf0 | (cp >> 18));
            s += (char)(0x80 | ((cp >> 12) & 0x3f));
            s += (char)(0x80 | ((cp >> 6) & 0x3f));
            s += (char)(0x80 | (cp & 0x3f));
        }
    }
    unsigned hex4() {
        if (end - p < 4) bad();
        unsigned v = 0;
        for (int i = 0; i < 4; ++i) {
            const char c = *p++;
            v <<= 4;
            if (c >= '0' && c <= '9') v |= (unsigned)(c - '0');
            else if (c >= 'a' && c <= 'f') v |= (unsigned)(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= (unsigned)(c - 'A' + 10);
            else bad();
        }
        return v;
    }
    // a string's text up to its first NUL (the reference copies it as a C string)
    std::string str() {
        expect('"');
        std::string s;
        while (true) {
            if (p >= end) bad();
            const unsigned char c = (unsigned char)*p++;
            if (c == '"') break;
            if (c < 0x20) bad();
            if (c != '\\') { s += (char)c; continue; }
            if (p >= end) bad();
            const char e = *p++;
            switch (e) {
            case '"': s += '"'; break;
            case '\\': s += '\\'; break;
            case '/': s += '/'; break;
            case 'b': s += '\b'; break;
            case 'f': s += '\f'; break;
            case 'n': s += '\n'; break;
            case 'r': s += '\r'; break;
            case 't': s += '\t'; break;
            case 'u': {
                unsigned cp = hex4();
                if (cp >= 0xd800 && cp < 0xdc00) {   // a surrogate pair
                    if (end - p < 6 || p[0] != '\\' || p[1] != 'u') bad();
                    p += 2;
                    const unsigned lo = hex4();
                    if (lo < 0xdc00 || lo >= 0xe000) bad();
                    cp = 0x10000 + ((cp - 0xd800) << 10) + (lo - 0xdc00);
                } else if (cp >= 0xdc00 && cp < 0xe000) {
                    bad();
                }
                utf8(s, cp);
                break;
            }
            default: bad();
            }
        }
        return std::string(s.c_str());
    }
    void number(JVal &v) {
        const char *s = p;
        bool real = false;
        if (p < end && *p == '-') ++p;
        if (p >= end) bad();
        if (*p == '0') {
            ++p;
        } else if (*p >= '1' && *p <= '9') {
            while (p < end && *p >= '0' && *p <= '9') ++p;
        } else {
            bad();
        }
        if (p < end && *p == '.') {
            real = true;
            ++p;
            if (p >= end || *p < '0' || *p > '9') bad();
            while (p < end && *p >= '0' && *p <= '9') ++p;
        }
        if (p < end && (*p == 'e' || *p == 'E')) {
            real = true;
            ++p;
            if (p < end && (*p == '+' || *p == '-')) ++p;
            if (p >= end || *p < '0' || *p > '9') bad();
            while (p < end && *p >= '0' && *p <= '9') ++p;
        }
        v.kind = real ? JVal::REAL : JVal::INT;
        v.text.assign(s, p);
    }
    bool word(const char *w) {
        const size_t n = std::strlen(w);
        if ((size_t)(end - p) < n || std::strncmp(p, w, n) != 0) return false;
        p += n;
        return true;
    }
    // one value; false for null (which adds nothing)
    bool value(JVal &v, int depth) {
        ws();
        if (p >= end) bad();
        if (depth > 512) bad();
        const char c = *p;
        if (c == '{') {
            ++p;
            v.kind = JVal::OBJ;
            ws();
            if (p < end && *p == '}') { ++p; return true; }
            while (true) {
                ws();
                v.keys.push_back(str());
                expect(':');
                JVal child;
                if (value(child, depth + 1)) {
                    if (depth == 0 && child.kind == JVal::OBJ && imp->process(v.keys.back(), child))
                        v.keys.pop_back();
                    else
                        v.vals.push_back(std::move(child));
                }
                ws();
                if (p < end && *p == ',') { ++p; continue; }
                expect('}');
                return true;
            }
        }
        if (c == '[') {
            ++p;
            v.kind = JVal::ARR;
            ws();
            if (p < end && *p == ']') { ++p; return true; }
            while (true) {
                JVal child;
                if (value(child, depth + 1)) v.vals.push_back(std::move(child));
                ws();
                if (p < end && *p == ',') { ++p; continue; }
                expect(']');
                return true;
            }
        }
        if (c == '"') {
            v.kind = JVal::STR;
            v.text = str();
            return true;
        }
        if (word("true")) { v.kind = JVal::BOOL; v.text = "1"; return true; }
        if (word("false")) { v.kind = JVal::BOOL; v.text = "0"; return true; }
        if (word("null")) return false;
        number(v);
        return true;
    }
};

}  // namespace

struct rzk_json {
    rzk::SceneArrays arrays;
    rzk_json_info info;
};

extern "C" {

rzk_status rzk_json_import(const char *path, rzk_json **out) {
    if (!path || !out) return RZK_ERR_INVALID;
    *out = nullptr;
    FILE *f = std::fopen(path, "rb");
    if (!f) return RZK_ERR_INVALID;
    std::string text;
    char buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
    std::fclose(f);
    Importer imp;
    // File::split_path (file.h:11-28): the scene directory is the file's, with its slash
    const std::string p(path);
    const size_t slash = p.find_last_of('/');
    imp.scene_path = slash == std::string::npos ? std::string() : p.substr(0, slash + 1);
    rzk_json *o = new rzk_json();
    try {
        Reader r{text.data(), text.data() + text.size(), &imp};
        // the root is an object (or an array, which the reference reports and leaves
        // unprocessed); a lone scalar has no container to go into there
        r.ws();
        if (r.p >= r.end || (*r.p != '{' && *r.p != '[')) r.bad();
        JVal root;
        r.value(root, 0);
        r.ws();
        if (r.p != r.end) r.bad();
        imp.finish(o->arrays);
    } catch (const std::exception &) {
        delete o;
        return RZK_ERR_INVALID;
    }
    o->info = imp.info;
    *out = o;
    return RZK_OK;
}

rzk_status rzk_json_get_info(const rzk_json *js, rzk_json_info *info) {
    if (!js || !info) return RZK_ERR_INVALID;
    *info = js->info;
    return RZK_OK;
}

rzk_status rzk_json_scene_desc(const rzk_json *js, rzk_scene_desc *desc) {
    if (!js || !desc) return RZK_ERR_INVALID;
    js->arrays.desc(desc, js->info.tmin);
    return RZK_OK;
}

rzk_status rzk_json_destroy(rzk_json *js) {
    if (!js) return RZK_ERR_INVALID;
    delete js;
    return RZK_OK;
}

}  // extern "C"
