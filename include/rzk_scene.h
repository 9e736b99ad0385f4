/*
 * rzk_scene.h - the scene description that crosses the C ABI.
 *
 * A scene is a list of primitives; each primitive is one reference Surface
 * (surface.h:24-111) whose Shape is a Triangle (triangle.h:13) or a Quad (quad.h:9).
 * A primitive either carries a material (Surface(Shape*, Material*), surface.cc:13) or
 * an emission (Surface(Shape*, const Rgb&), surface.cc:19, which creates an AreaLight).
 * Area lights are numbered in primitive order.
 *
 * Triangles are flattened exactly as AggregateBvh::build collects them
 * (aggregate_bvh.cc:58-76): primitive order, and for a quad t0 = (p0,p1,p2) then
 * t1 = (p0,p2,p3) (quad.cc:5-28, quad.h:99-102), both with the quad's tangent
 * unit(p0 - p1).
 */
#ifndef RZK_SCENE_H_
#define RZK_SCENE_H_

#include "rzk_types.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { RZK_PRIM_TRIANGLE = 3, RZK_PRIM_QUAD = 4 };

typedef struct {
    int32_t n_prims;
    const int32_t *prim_kind;   /* RZK_PRIM_TRIANGLE or RZK_PRIM_QUAD, n_prims        */
    const float *prim_v;        /* n_prims x 12 floats: p0,p1,p2,p3 (p3 unused for a
                                   triangle)                                          */
    const int32_t *prim_mat;    /* material index, or -1 for an emitter, n_prims      */
    const float *prim_emit;     /* n_prims x 3 radiance; read only where prim_mat<0   */
    const int32_t *prim_flags;  /* RZK_SURF_* bits, n_prims (NULL = all zero)         */
    int32_t n_mats;
    const rzk_material *mats;
    float tmin;                 /* Scene::tmin, RAY_TMIN = 1e-3 by default (common.h:48) */
} rzk_scene_desc;

#ifdef __cplusplus
}
#endif

#endif /* RZK_SCENE_H_ */
