/*
 * rzk_types.h - plain-C record layouts shared by the CUDA library (librzk_cuda.so),
 * the C++ host classes, the CPU oracle and the Python bindings.
 *
 * Every record is a flat array of 32-bit words so that it can cross the C ABI, be
 * staged into shared memory with bulk copies (sizes are multiples of 16 bytes), and be
 * mirrored by numpy structured dtypes without packing surprises.
 *
 * The fields follow the reference's own types:
 *   rzk_receiver  <- Receiver / LocalGeometry   (local_geometry.h:11-33, 38-61)
 *   rzk_vpl       <- BrdfPointLight             (brdf_point_light.h:31-141)
 *   rzk_material  <- BsdfMaterial + Lambertian / ModifiedPhong / Ward
 *                    (material.h:67-135, lambertian.h:15, phong.h:29, ward.h:20)
 *   rzk_camera    <- Camera + Sensor pinhole model (camera.cc:52-65, sensor.h:176-182)
 */
#ifndef RZK_TYPES_H_
#define RZK_TYPES_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: every rzk_* entry point returns one of these (no exceptions cross
 * the ABI). */
typedef enum {
    RZK_OK = 0,
    RZK_ERR_INVALID = 1,     /* bad argument (null pointer, negative size, bad enum) */
    RZK_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    RZK_ERR_NOMEM = 3,       /* device allocation refused */
    RZK_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
    RZK_ERR_STACK = 5,       /* traversal stack overflowed (reference drops pushes) */
    RZK_ERR_CAPACITY = 6,    /* a fixed-size buffer is too small for the request */
    RZK_ERR_UNSUPPORTED = 7, /* feature not available in this build */
    RZK_ERR_BUSY = 8         /* admission refused: not enough free device memory */
} rzk_status;

/* Bsdf::Type values (bsdf.h:10-18). Only the three BRDFs on the gather path. */
enum { RZK_BSDF_LAMBERTIAN = 0, RZK_BSDF_WARD = 1, RZK_BSDF_PHONG = 2 };

/* VplRadianceClamp::Type (vpl_interface.h:155-162), same numbering. */
enum { RZK_CLAMP_NONE = 0, RZK_CLAMP_FORM_FACTOR = 1, RZK_CLAMP_REFLECTIVITY = 2,
       RZK_CLAMP_RADIANCE = 3 };

/* Surface flags (surface.h:109-110). */
enum { RZK_SURF_FLIPPED = 1, RZK_SURF_TWO_SIDED = 2 };

/* A material: 12 words. type is an RZK_BSDF_* value.
 *   Lambertian: kd
 *   Phong:      kd, ks, p0 = exponent n
 *   Ward:       kd, ks, p0 = ax, p1 = ay                                          */
typedef struct {
    int32_t type;
    float kd[3];
    float ks[3];
    float p0, p1;
    float pad[3];
} rzk_material;

/* One shading point (a primary hit): 24 words = 96 bytes.
 *   p     hit position            r.org() + t * r.dir()
 *   ng    geometric normal        HitRecord::normal after the surface flips
 *   ns    shading normal          HitRecord::shading_normal after the flips
 *   wo    -ray direction          Receiver::wo
 *   u,v,n shading basis           HitRecord::uvn (Onb::init_from_nu(ns, tangent))
 *   mat   material index, -1 when the surface has none (light or miss)
 *   light area-light index, -1 when none
 *   flags bit0: the primary ray hit something                                     */
typedef struct {
    float p[3];
    float ng[3];
    float ns[3];
    float wo[3];
    float u[3];
    float v[3];
    float n[3];
    int32_t mat;
    int32_t light;
    int32_t flags;
} rzk_receiver;

/* One virtual point light: 24 words = 96 bytes.
 *   p, n     LocalGeometry::p and ::n (shading normal) of the VPL    (org(), normal())
 *   u,v,nn   LocalGeometry::uvn
 *   wi       incident direction stored at creation                    (get_wi())
 *   contrib  power                                                    (power())
 *   mat      material index (-1 with flags bit0 set: VPL on a light, brdf() = white)
 *   bounce   BrdfPointLight::bounce
 *   path     index of the light particle that produced it                          */
typedef struct {
    float p[3];
    float n[3];
    float u[3];
    float v[3];
    float nn[3];
    float wi[3];
    float contrib[3];
    int32_t mat;
    int32_t bounce;
    int32_t path;
} rzk_vpl;

/* Pinhole camera, precomputed on the host exactly as Camera::set_perspective and
 * Sensor do (camera.cc:23-30, sensor.h:176-182): 20 words.                       */
typedef struct {
    float eye[3];
    float u[3], v[3], n[3];   /* Camera::onb after init_from_nv(eye - lookat, up) */
    float focal;
    float cop[2];             /* img_size / 2 */
    float scale[2];           /* img_size / film_size */
    int32_t width, height;
    int32_t pad;
} rzk_camera;

/* One ray exactly as a constructed reference Ray holds it (ray.h:17-36: origin, unit
 * direction, inverse direction after the ZERO_EPSILON substitution, -origin x inverse
 * direction) and the interval [tmin, tmax] of the query: 16 words.                  */
typedef struct {
    float o[3], d[3], inv_d[3], org_inv_d[3];
    float tmin, tmax;
    int32_t pad[2];
} rzk_ray;

/* Result of one ray query: 8 words.  hit = 1 when a triangle passes; for closest-hit
 * queries also the reference's GeometryHit (t, beta, gamma; triangle.cc:158-232) and the
 * hit triangle's index in the flattened order of rzk_scene.h (else -1).            */
typedef struct {
    int32_t hit;
    float t, beta, gamma;
    int32_t tri;
    int32_t pad[3];
} rzk_ray_hit;

/* Flat BVH node as the reference numbers it (BvhNode, aggregate_bvh.h:10-16):
 * used only for dumps and bit-exact comparison.                                 */
typedef struct {
    float bmin[3];
    float bmax[3];
    int32_t start, end, left, right, level;
    int32_t pad;
} rzk_bvh_node;

#ifdef __cplusplus
}
#endif

#endif /* RZK_TYPES_H_ */
