// rzk_scenefile.h - host-side scene files (OBJ, JSON) shared by rzk_obj.cu and rzk_json.cu.
#pragma once

#include <string>
#include <vector>

#include "../../include/rzk.h"

namespace rzk {

// A face of 3 or 4 vertices as ObjImporter::load keeps it in its shape list
// (obj_importer.cc:306-420): every such face, with or without a material.
struct ObjShape {
    int kind;       // RZK_PRIM_TRIANGLE or RZK_PRIM_QUAD
    float v[12];    // vertices; the fourth is zero for a triangle
    int object;     // index into ObjModel::object_names (the `o` line before it), -1 before any
    int surface;    // the importer's surface index (Surfaces::append, surface.h:123-127), -1 for none
    int shading;    // 1: vertex normals given, 2: in a smoothing group without them (the
                    // reference interpolates shading normals; facet normals here), 0: neither
};

// One entry of the importer's surface list.
enum { OBJ_SURF_MATERIAL = 0, OBJ_SURF_LIGHT = 1, OBJ_SURF_UNSUPPORTED = 2, OBJ_SURF_SPHERE = 3 };
struct ObjSurface {
    int type;       // OBJ_SURF_*
    int shape;      // index into ObjModel::shapes; -1 for a light quad or a sphere
    int kind;       // RZK_PRIM_* (a sphere: 0)
    float v[12];
    int mat;        // index into ObjModel::mats (OBJ_SURF_MATERIAL)
    float emit[3];  // radiance (OBJ_SURF_LIGHT)
};

// One OBJ file as ObjImporter::load (obj_importer.cc:212-553) builds it: the shape list, the
// object names, the surface list in its order (light quads, faces that have a material,
// spheres) and the materials this path models.
struct ObjModel {
    std::vector<ObjShape> shapes;
    std::vector<std::string> object_names;
    std::vector<ObjSurface> surfaces;
    std::vector<rzk_material> mats;
    std::vector<std::string> mtl_names;   // every MTL material in file order (Material::set_name)
    std::vector<int> mtl_mats;            // its index into mats, -1 where this path has no BSDF
    rzk_obj_info info;
};

// Reads `path` and its mtllib files; RZK_ERR_INVALID when a file cannot be read or an index
// points outside its list.
rzk_status obj_load(const char *path, ObjModel &m);

// The arrays behind an rzk_scene_desc, filled primitive by primitive.
struct SceneArrays {
    std::vector<int32_t> kind, mat, flags;
    std::vector<float> v, emit;
    std::vector<rzk_material> mats;
    // one primitive: kind, 12 vertex floats, material (-1 for an area light), radiance (null: 0)
    void add(int kind, const float *v12, int mat, const float *emit, int flags);
    // pointers into these arrays (valid while they are unchanged)
    void desc(rzk_scene_desc *d, float tmin) const;
};

}  // namespace rzk
