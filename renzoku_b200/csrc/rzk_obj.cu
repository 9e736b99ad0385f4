// rzk_obj.cu - Wavefront OBJ / MTL scenes in the reference's dialect, as a scene
// description for rzk_scene_create.  Host code only.
//
// Reading follows the reference's parser (obj_parser.cpp): lines read in pieces of at most
// 511 characters, tokens split on white space, integers by atoi and reals by atof, indices
// 1-based or negative (relative to the list's current length) and 0 for "none", a face
// keeping its first four vertices, `usemtl` naming a material of the MTL file read so far.
// Its dialect adds `c` (camera: eye and look-at vertices, up normal, focal length),
// `lp` (point light), `lq` (quad area light) and `sp` (sphere).
//
// The scene follows ObjImporter::load (obj_importer.cc:212-553): light quads first, then
// the faces in file order - a face whose material's name contains "rz_light" becomes an
// area light with the material's diffuse colour as radiance, a face without a material
// becomes no surface - with each MTL material turned into a BSDF by load_material
// (obj_importer.cc:81-172): Kd and Ks scaled down together when Kd + Ks exceeds 1 in any
// channel (not for lights), Lambertian when Ks is black, else Phong with exponent Ns (1 when
// 0), or Ward with roughnesses 1 / Ns[0] and 1 / Ns[1] when Ns has two values.
//
// What this path does not model is counted and left out (rzk_obj_info): point lights and
// spheres, refractive (Ni > 1) and textured (map_Kd) materials.  Vertex normals and
// smoothing groups, which change the reference's shading normals, are counted and the
// faces imported with their facet normals.
#include "rzk_internal.cuh"
#include "rzk_scenefile.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

struct rzk_obj {
    rzk::SceneArrays arrays;
    rzk_obj_info info;
};

namespace {

constexpr int kLineBytes = 512;        // the reference parser's line buffer (OBJ_LINE_SIZE)
const char *const kSpace = " \t\n\r";

struct Mtl {
    std::string name;
    float diff[3] = {0, 0, 0}, spec[3] = {0, 0, 0};
    float shiny[2] = {0, 0};
    float refract_index = 1.0f;
    bool textured = false;
};

struct Face {
    int v[4], n[4];
    int count, mat, smooth, object;
};

struct LightQuad {
    int v[4];
    int count, mat;
};

// an OBJ index (1-based, negative = from the end of the list so far, 0 = none)
int list_index(int size, int idx) {
    if (idx == 0) return -1;
    if (idx < 0) return size + idx;
    return idx - 1;
}

float next_real(const char *delims) {
    const char *t = std::strtok(nullptr, delims);
    return t ? (float)std::atof(t) : 0.0f;
}

// the MTL file (obj_parse_mtl_file, obj_parser.cpp:224-369); false when it cannot be read
bool read_mtl(const std::string &path, std::vector<Mtl> &out) {
    FILE *f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    char line[kLineBytes];
    bool open = false;
    Mtl cur;
    while (std::fgets(line, kLineBytes, f)) {
        const char *tok = std::strtok(line, kSpace);
        if (!tok || !std::strcmp(tok, "//") || !std::strcmp(tok, "#")) continue;
        if (!std::strcmp(tok, "newmtl")) {
            if (open) out.push_back(cur);
            cur = Mtl();
            const char *name = std::strtok(nullptr, kSpace);
            cur.name = name ? std::string(name).substr(0, 255) : std::string();
            open = true;
        } else if (!open) {
            continue;
        } else if (!std::strcmp(tok, "Kd")) {
            for (float &x : cur.diff) x = next_real(" \t");
        } else if (!std::strcmp(tok, "Ks")) {
            for (float &x : cur.spec) x = next_real(" \t");
        } else if (!std::strcmp(tok, "Ns")) {
            cur.shiny[0] = next_real(" \t");
            const char *t = std::strtok(nullptr, " \t");   // a second value: Ward
            if (t) cur.shiny[1] = (float)std::atof(t);
        } else if (!std::strcmp(tok, "Ni")) {
            cur.refract_index = next_real(" \t");
        } else if (!std::strcmp(tok, "map_Kd")) {
            cur.textured = std::strtok(nullptr, kSpace) != nullptr;
        }
        // Ka, Ke, d, r, sharpness, illum, map_Disp: read by the reference, used by no BSDF here
    }
    if (open) out.push_back(cur);
    std::fclose(f);
    return true;
}

// vertex / texture / normal indices of a face or light line (obj_parse_vertex_index,
// obj_parser.cpp:68-112): at most four vertices are kept
int read_corners(int *v, int *n) {
    int count = 0;
    const char *tok;
    while ((tok = std::strtok(nullptr, kSpace)) != nullptr) {
        if (count >= 4) continue;
        v[count] = std::atoi(tok);
        int ni = 0;
        const char *s = std::strstr(tok, "//");
        if (s) {
            ni = std::atoi(s + 2);
        } else if ((s = std::strchr(tok, '/')) != nullptr) {
            const char *s2 = std::strchr(s + 1, '/');
            if (s2) ni = std::atoi(s2 + 1);
        }
        if (n) n[count] = ni;
        count++;
    }
    return count;
}

bool is_light_name(const std::string &name) { return name.find("rz_light") != std::string::npos; }

float rgb_max(const float *c) {   // Rgb::max (rgb.h:44-50)
    float m = c[0];
    if (c[1] > m) m = c[1];
    if (c[2] > m) m = c[2];
    return m;
}

// load_material (obj_importer.cc:81-172) for the BSDFs this path models; false for a
// refractive or textured material
bool to_material(const Mtl &m, rzk_material &out) {
    std::memset(&out, 0, sizeof(out));
    if (m.refract_index > 1.0f || m.textured) return false;
    float kd[3] = {m.diff[0], m.diff[1], m.diff[2]}, ks[3] = {m.spec[0], m.spec[1], m.spec[2]};
    if (!is_light_name(m.name)) {
        const float total[3] = {kd[0] + ks[0], kd[1] + ks[1], kd[2] + ks[2]};
        if (total[0] > 1.0f || total[1] > 1.0f || total[2] > 1.0f) {
            const float t = rgb_max(total);
            for (int c = 0; c < 3; ++c) { kd[c] = kd[c] / t; ks[c] = ks[c] / t; }
        }
    }
    for (int c = 0; c < 3; ++c) { out.kd[c] = kd[c]; out.ks[c] = ks[c]; }
    if (rgb_max(kd) != 0.0f && rgb_max(ks) == 0.0f) {
        out.type = RZK_BSDF_LAMBERTIAN;
    } else if (m.shiny[1] == 0.0f) {
        out.type = RZK_BSDF_PHONG;
        out.p0 = m.shiny[0] == 0.0f ? 1.0f : m.shiny[0];
    } else {
        out.type = RZK_BSDF_WARD;
        const float s0 = m.shiny[0] == 0.0f ? m.shiny[1] : m.shiny[0];
        out.p0 = 1.0f / s0;
        out.p1 = 1.0f / m.shiny[1];
    }
    return true;
}

void put_geometry(int count, const int *vi, const std::vector<float> &verts, int &kind, float *v) {
    kind = count == 4 ? RZK_PRIM_QUAD : RZK_PRIM_TRIANGLE;
    for (int k = 0; k < 4; ++k)
        for (int c = 0; c < 3; ++c) v[3 * k + c] = k < count ? verts[3 * vi[k] + c] : 0.0f;
}

}  // namespace

namespace rzk {

rzk_status obj_load(const char *path, ObjModel &o) {
    FILE *f = std::fopen(path, "r");
    if (!f) return RZK_ERR_INVALID;
    std::vector<float> verts, normals;   // 3 per vertex / normal
    std::vector<Face> faces;
    std::vector<LightQuad> lquads;
    std::vector<int> sphere_mats;
    std::vector<Mtl> mtls;
    int cur_mat = -1, cur_smooth = 0, cur_object = -1;
    bool have_cam = false, bad = false;
    int cam_idx[3] = {0, 0, 0};
    float focal = 0.0f;
    std::memset(&o.info, 0, sizeof(o.info));
    rzk_obj_info &info = o.info;
    std::string dir(path);
    const size_t slash = dir.find_last_of("/\\");
    dir = slash == std::string::npos ? std::string() : dir.substr(0, slash + 1);
    char line[kLineBytes];
    while (std::fgets(line, kLineBytes, f)) {
        const char *tok = std::strtok(line, kSpace);
        if (!tok || tok[0] == '#') continue;
        if (!std::strcmp(tok, "v") || !std::strcmp(tok, "vn")) {
            std::vector<float> &dst = tok[1] ? normals : verts;
            for (int c = 0; c < 3; ++c) dst.push_back(next_real(kSpace));
        } else if (!std::strcmp(tok, "f")) {
            Face fc;
            std::memset(&fc, 0, sizeof(fc));
            fc.count = read_corners(fc.v, fc.n);
            for (int k = 0; k < fc.count; ++k) {
                fc.v[k] = list_index((int)(verts.size() / 3), fc.v[k]);
                fc.n[k] = list_index((int)(normals.size() / 3), fc.n[k]);
            }
            fc.mat = cur_mat;
            fc.smooth = cur_smooth;
            fc.object = cur_object;
            faces.push_back(fc);
        } else if (!std::strcmp(tok, "lq")) {
            LightQuad q;
            q.count = read_corners(q.v, nullptr);
            for (int k = 0; k < q.count; ++k) q.v[k] = list_index((int)(verts.size() / 3), q.v[k]);
            q.mat = cur_mat;
            lquads.push_back(q);
        } else if (!std::strcmp(tok, "lp")) {
            info.point_lights++;
        } else if (!std::strcmp(tok, "sp")) {
            info.spheres++;
            sphere_mats.push_back(cur_mat);
        } else if (!std::strcmp(tok, "o")) {   // object name (obj_parser.cpp:527-532)
            const char *name = std::strtok(nullptr, kSpace);
            o.object_names.push_back(name ? name : "");
            cur_object++;
        } else if (!std::strcmp(tok, "c")) {
            int k = 0;
            const char *t;
            while (k < 3 && (t = std::strtok(nullptr, kSpace)) != nullptr) cam_idx[k++] = std::atoi(t);
            const char *ft = std::strtok(nullptr, kSpace);
            if (k < 3 || !ft) { bad = true; continue; }
            if (!have_cam) {   // the importer uses the first camera (obj_importer.cc:234-236)
                have_cam = true;
                cam_idx[0] = list_index((int)(verts.size() / 3), cam_idx[0]);
                cam_idx[1] = list_index((int)(verts.size() / 3), cam_idx[1]);
                cam_idx[2] = list_index((int)(normals.size() / 3), cam_idx[2]);
                focal = (float)std::atof(ft);
                for (int c = 0; c < 3; ++c) {
                    if (cam_idx[0] < 0 || cam_idx[1] < 0 || cam_idx[2] < 0 ||
                        cam_idx[0] >= (int)(verts.size() / 3) || cam_idx[1] >= (int)(verts.size() / 3) ||
                        cam_idx[2] >= (int)(normals.size() / 3)) {
                        bad = true;
                        break;
                    }
                    info.eye[c] = verts[3 * cam_idx[0] + c];
                    info.lookat[c] = verts[3 * cam_idx[1] + c];
                    info.up[c] = normals[3 * cam_idx[2] + c];
                }
                info.focal = focal;
            }
        } else if (!std::strcmp(tok, "usemtl")) {
            const char *name = std::strtok(nullptr, kSpace);
            cur_mat = -1;
            for (size_t i = 0; name && i < mtls.size(); ++i)
                if (mtls[i].name == name) { cur_mat = (int)i; break; }
        } else if (!std::strcmp(tok, "mtllib")) {
            const char *name = std::strtok(nullptr, kSpace);
            // an unreadable MTL file leaves the materials as they were (obj_parser.cpp:499-513)
            if (name && !read_mtl(dir + name, mtls)) info.mtl_files_missing++;
        } else if (!std::strcmp(tok, "s")) {
            const char *g = std::strtok(nullptr, kSpace);
            cur_smooth = (!g || !std::strcmp(g, "off")) ? 0 : (int)std::atof(g);
        }
        // vt, g, p, pl, ld and unknown commands: nothing this path reads
    }
    std::fclose(f);
    if (bad) return RZK_ERR_INVALID;
    info.has_camera = have_cam ? 1 : 0;
    info.width = 512;   // Sensor(Size2(512, 512), Size2(0.025, 0.025)) (obj_importer.cc:237)
    info.height = 512;
    info.film_w = 0.025f;
    info.film_h = 0.025f;
    // materials in file order; a modelled BSDF gets the next scene material index
    std::vector<int> mat_of(mtls.size(), -1);
    for (size_t i = 0; i < mtls.size(); ++i) {
        rzk_material m;
        if (to_material(mtls[i], m)) {
            mat_of[i] = (int)o.mats.size();
            o.mats.push_back(m);
        }
        o.mtl_names.push_back(mtls[i].name);
    }
    o.mtl_mats = mat_of;
    const int nv = (int)(verts.size() / 3);
    auto in_range = [&](int count, const int *vi) {
        for (int k = 0; k < count; ++k)
            if (vi[k] < 0 || vi[k] >= nv) return false;
        return true;
    };
    // light quads (obj_importer.cc:271-284): radiance = the material's diffuse colour
    for (const LightQuad &q : lquads) {
        if (q.count != 4 || q.mat < 0 || !in_range(4, q.v)) return RZK_ERR_INVALID;
        ObjSurface sf;
        std::memset(&sf, 0, sizeof(sf));
        sf.type = OBJ_SURF_LIGHT;
        sf.shape = -1;
        sf.mat = -1;
        put_geometry(4, q.v, verts, sf.kind, sf.v);
        for (int c = 0; c < 3; ++c) sf.emit[c] = mtls[q.mat].diff[c];
        o.surfaces.push_back(sf);
    }
    // faces (obj_importer.cc:306-452): each face of 3 or 4 vertices is a shape; one with a
    // material is also a surface
    for (const Face &fc : faces) {
        if (fc.count < 3) { info.short_faces++; continue; }
        if (!in_range(fc.count, fc.v)) return RZK_ERR_INVALID;
        ObjShape sh;
        put_geometry(fc.count, fc.v, verts, sh.kind, sh.v);
        sh.object = fc.object;
        sh.surface = -1;
        {
            bool normals_given = false;
            for (int k = 0; k < fc.count; ++k) normals_given |= fc.n[k] >= 0;
            sh.shading = normals_given ? 1 : (fc.smooth > 0 ? 2 : 0);
        }
        if (fc.mat < 0) {
            info.faces_without_material++;
            o.shapes.push_back(sh);
            continue;
        }
        const Mtl &m = mtls[fc.mat];
        ObjSurface sf;
        std::memset(&sf, 0, sizeof(sf));
        sf.kind = sh.kind;
        std::memcpy(sf.v, sh.v, sizeof(sf.v));
        sf.mat = -1;
        if (is_light_name(m.name)) {
            // a light needs a diffuse BSDF (obj_importer.cc:427-435): not a refractive one
            if (m.refract_index > 1.0f) {
                info.faces_unsupported_material++;
                o.shapes.push_back(sh);
                continue;
            }
            sf.type = OBJ_SURF_LIGHT;
            for (int c = 0; c < 3; ++c) sf.emit[c] = m.diff[c];
        } else if (mat_of[fc.mat] < 0) {
            info.faces_unsupported_material++;
            sf.type = OBJ_SURF_UNSUPPORTED;
        } else {
            sf.type = OBJ_SURF_MATERIAL;
            sf.mat = mat_of[fc.mat];
        }
        if (sf.type != OBJ_SURF_UNSUPPORTED) {
            if (sh.shading == 1) info.faces_with_vertex_normals++;
            else if (sh.shading == 2) info.smoothed_faces++;
        }
        sh.surface = (int)o.surfaces.size();
        sf.shape = (int)o.shapes.size();
        o.shapes.push_back(sh);
        o.surfaces.push_back(sf);
    }
    // spheres (obj_importer.cc:455-468): surfaces after the faces
    for (size_t i = 0; i < sphere_mats.size(); ++i) {
        ObjSurface sf;
        std::memset(&sf, 0, sizeof(sf));
        sf.type = OBJ_SURF_SPHERE;
        sf.shape = -1;
        sf.mat = -1;
        o.surfaces.push_back(sf);
    }
    for (const ObjSurface &sf : o.surfaces) {
        if (sf.type == OBJ_SURF_MATERIAL || sf.type == OBJ_SURF_LIGHT) info.n_prims++;
        if (sf.type == OBJ_SURF_LIGHT) info.n_lights++;
    }
    info.n_mats = (int)o.mats.size();
    return RZK_OK;
}

void SceneArrays::add(int k, const float *v12, int m, const float *e, int f) {
    kind.push_back(k);
    v.insert(v.end(), v12, v12 + 12);
    mat.push_back(m);
    flags.push_back(f);
    for (int c = 0; c < 3; ++c) emit.push_back(e ? e[c] : 0.0f);
}

void SceneArrays::desc(rzk_scene_desc *d, float tmin) const {
    std::memset(d, 0, sizeof(*d));
    d->n_prims = (int32_t)kind.size();
    d->prim_kind = kind.data();
    d->prim_v = v.data();
    d->prim_mat = mat.data();
    d->prim_emit = emit.data();
    d->prim_flags = flags.data();
    d->n_mats = (int32_t)mats.size();
    d->mats = mats.data();
    d->tmin = tmin;
}

}  // namespace rzk

extern "C" {

rzk_status rzk_obj_import(const char *path, rzk_obj **out) {
    if (!path || !out) return RZK_ERR_INVALID;
    *out = nullptr;
    rzk::ObjModel m;
    const rzk_status r = rzk::obj_load(path, m);
    if (r != RZK_OK) return r;
    rzk_obj *o = new rzk_obj();
    o->info = m.info;
    o->arrays.mats = m.mats;
    for (const rzk::ObjSurface &sf : m.surfaces) {
        if (sf.type == rzk::OBJ_SURF_MATERIAL) o->arrays.add(sf.kind, sf.v, sf.mat, nullptr, 0);
        else if (sf.type == rzk::OBJ_SURF_LIGHT) o->arrays.add(sf.kind, sf.v, -1, sf.emit, 0);
    }
    *out = o;
    return RZK_OK;
}

rzk_status rzk_obj_get_info(const rzk_obj *obj, rzk_obj_info *info) {
    if (!obj || !info) return RZK_ERR_INVALID;
    *info = obj->info;
    return RZK_OK;
}

rzk_status rzk_obj_scene_desc(const rzk_obj *obj, rzk_scene_desc *desc) {
    if (!obj || !desc) return RZK_ERR_INVALID;
    obj->arrays.desc(desc, 1e-3f);
    return RZK_OK;
}

rzk_status rzk_obj_destroy(rzk_obj *obj) {
    if (!obj) return RZK_ERR_INVALID;
    delete obj;
    return RZK_OK;
}

}  // extern "C"
