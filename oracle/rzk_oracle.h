/*
 * rzk_oracle.h - TEST INFRASTRUCTURE ONLY: the CPU oracle for the VPL gather path.
 *
 * A plain-C restatement of the reference's algorithms for this path, used by tests/,
 * the smoke check and bench.py's CPU-baseline leg as the checker.  The product
 * (librzk_cuda.so and the host classes) never links or calls it.  Each function in
 * rzk_oracle.c cites the reference file:line it follows.
 *
 * Floating-point discipline: compiled with -O2 -ffp-contract=off and no -march, so
 * every expression is evaluated as IEEE single-precision operations in the reference's
 * source order (x86-64 SSE, no FMA).  That makes Morton codes, the sorted order, the
 * BVH, ray/box/triangle predicates and primary hits bit-identical to the reference
 * built the same way.
 */
#ifndef RZK_ORACLE_H_
#define RZK_ORACLE_H_

#include <stdint.h>
#include "../include/rzk_types.h"
#include "../include/rzk_scene.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ro_scene ro_scene;

/* Traversal work counters (per call, summed over rays). */
typedef struct {
    int64_t rays;          /* shadow or closest-hit rays traced                       */
    int64_t root_tests;    /* root box tests                                          */
    int64_t inner_pops;    /* inner nodes popped (both child boxes read and tested)   */
    int64_t leaf_tests;    /* triangle tests                                          */
    int64_t overflows;     /* pushes dropped because the 64-entry stack was full      */
    int64_t pairs;         /* shading-point x VPL pairs evaluated                      */
    int64_t culled;        /* pairs whose shading term was exactly zero (no ray)       */
} ro_counters;

ro_scene *ro_scene_create(const rzk_scene_desc *d);
void ro_scene_destroy(ro_scene *s);
int ro_num_triangles(const ro_scene *s);
int ro_num_nodes(const ro_scene *s);
int ro_num_lights(const ro_scene *s);

/* Morton codes of the flattened triangles in input order (morton.h:98-102). */
void ro_morton_codes(const ro_scene *s, uint32_t *codes);
/* Sorted codes, sorted-slot -> triangle permutation, BFS nodes (aggregate_bvh.cc). */
void ro_bvh_dump(const ro_scene *s, uint32_t *morton_sorted, int32_t *perm,
                 rzk_bvh_node *nodes);

/* Camera::set_perspective + Sensor (camera.cc:23-30, camera.h:228-230, sensor.h). */
void ro_camera_setup(const float eye[3], const float lookat[3], const float up[3],
                     float fov_deg, int width, int height, float film_w, float film_h,
                     rzk_camera *out);
/* Camera::shoot_ray(i, j) for every pixel, after the Ray constructor. */
void ro_primary_rays(const rzk_camera *cam, float *o, float *d);

/* Aggregate::hit(p, q, tmin, time) (aggregate.cc:84-90): 1 = occluded. */
void ro_occluded(const ro_scene *s, const float *p, const float *q, int n, uint8_t *out,
                 ro_counters *cnt);
/* Closest hit of Ray(o, d) (aggregate_bvh.cc:402-448) + hit record (surface.cc:62-96). */
void ro_closest(const ro_scene *s, const float *o, const float *d, int n, float *t_out,
                rzk_receiver *recv, ro_counters *cnt);
/* One primary hit per pixel. */
void ro_primary(const ro_scene *s, const rzk_camera *cam, rzk_receiver *out,
                int n_threads);

/* Full gather: out[r] = scale * sum_j gather_point(r, vpl_j) summed in VPL order, in
 * float (out_f32) and, with the same visibility, in double (out_f64).  Either output may
 * be NULL.  cull != 0 skips the shadow ray where the shading term is exactly zero
 * (identical sum).  n_threads > 1 splits receivers over threads. */
void ro_gather(const ro_scene *s, const rzk_receiver *recv, int n_recv, const rzk_vpl *vpls,
               int n_vpl, int clamp_mode, float tau, float scale, int cull, float *out_f32,
               double *out_f64, int n_threads, ro_counters *cnt);
/* Per-pair radiance (column-major rows x cols, rgb) and visibility, as
 * LightTransportMatrix::fill stores it (light_transport_matrix.cc:16-48). */
void ro_gather_pairs(const ro_scene *s, const rzk_receiver *recv, int n_recv,
                     const rzk_vpl *vpls, int n_vpl, int clamp_mode, float tau,
                     float *pair_rgb, uint8_t *pair_vis);
/* incident_radiance for every pair (vpl.cc:411-440), column-major rgb. */
void ro_incident(const ro_scene *s, const rzk_receiver *recv, int n_recv,
                 const rzk_vpl *vpls, int n_vpl, int clamp_mode, float tau,
                 float *pair_rgb);
/* Material::eval for a batch. */
void ro_brdf_eval(const ro_scene *s, const int32_t *mat, const float *uvn9,
                  const float *wo, const float *wi, int n, float *out);
/* Mean of RadianceTerms::radiance_no_clamp.value() over the given pairs (visible ones
 * count with their value, occluded ones as zero), used for "0.1 x mean contribution". */
double ro_mean_contribution(const ro_scene *s, const rzk_receiver *recv,
                            const int32_t *recv_idx, const int32_t *vpl_idx, int n_pairs,
                            const rzk_vpl *vpls);

/* Counter-based random stream shared with the GPU and the reference harness:
 * Philox4x32-10 (Salmon et al., SC'11) on counter {d>>2, path, stream, 0x52454e5a} and
 * key {seed, 0x4b5a4f52}, word d&3. */
uint32_t ro_draw_u32(uint32_t seed, uint32_t stream, uint32_t path, uint32_t d);

/* VplGenerator::generate_vpl (vpl_generator.cc:43-181, path.cc:171-334) with draw d of
 * particle k taken from ro_draw_u32(seed, 0, k, d).  VPLs are written in push order
 * (particle-major, bounce-minor).  Returns the number generated (may exceed cap). */
int ro_vpl_generate(const ro_scene *s, uint32_t seed, int n_particles, int max_bounce,
                    rzk_vpl *out, int cap);

/* LightTransportMatrix::generate_alphas_for_clustering / get_column_norms on a
 * column-major [cols][rows][3] matrix (light_transport_matrix.cc:72-130). */
void ro_ltm_alphas(const float *mat, int rows, int cols, float *alphas, float *norms);
/* ClusterBuilder::cluster_by_sampling (cluster_builder.cc:82-273), draws from stream
 * (seed, 1, 0); returns the number of final clusters. */
int ro_cluster_by_sampling(const float *mat, int rows, int cols, int num_clusters, uint32_t seed,
                           int32_t *center, int32_t *rep, float *weight, int32_t *assign);

#ifdef __cplusplus
}
#endif

#endif /* RZK_ORACLE_H_ */
