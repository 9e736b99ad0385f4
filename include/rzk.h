/*
 * rzk.h - the C ABI of librzk_cuda.so, the B200 (sm_100a) implementation of Renzoku's
 * many-light VPL gather path.
 *
 * Conventions
 *   - Every entry point returns an rzk_status (rzk_types.h); nothing throws across the ABI.
 *   - Pointers named d_* are device pointers, h_* are host pointers; sizes are element
 *     counts.  `stream` is a cudaStream_t passed as void* (NULL = the legacy default
 *     stream); every device call is ordered on it and returns without synchronising
 *     unless its comment says otherwise.
 *   - Device memory owned by the library lives behind opaque handles (rzk_scene,
 *     rzk_context).  A context is single-threaded: use one per host thread.
 *
 * Each entry point names the reference interface it replaces (file:line in the
 * reference project).
 */
#ifndef RZK_H_
#define RZK_H_

#include <stddef.h>
#include <stdint.h>
#include "rzk_types.h"
#include "rzk_scene.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rzk_context rzk_context;
typedef struct rzk_scene rzk_scene;

/* Library / context ---------------------------------------------------------------- */

/* Human-readable name of a status code. */
const char *rzk_status_string(rzk_status s);

/* Creates a context on `device` (cudaSetDevice is called).  The context owns the
 * gather's reusable scratch buffers and an error word the kernels write on bounded-wait
 * timeouts.  No reference counterpart (the reference is single-process CPU). */
rzk_status rzk_context_create(int device, rzk_context **out);
rzk_status rzk_context_destroy(rzk_context *ctx);
/* Reads and clears the device error word (RZK_OK when no kernel reported a problem).
 * Synchronises `stream`. */
rzk_status rzk_context_check(rzk_context *ctx, void *stream);
/* Shadow rays the gather kernels of this context have traced since it was created or last
 * reset: every (receiver, VPL) pair that survives the exact-zero test (both BRDFs' own
 * early-outs, lambertian.cc:63-66, phong.cc:74-77, ward.cc:104-109) and so needs
 * Aggregate::hit(p, q) (aggregate.cc:84-90).  One atomic add per warp work item.  Reads
 * after `stream` has run; reset != 0 also zeroes the counter on `stream`. */
rzk_status rzk_context_rays(rzk_context *ctx, uint64_t *h_rays, int reset, void *stream);
/* Failure-path check of the bounded waits (no reference counterpart): one warp runs the
 * chunk ring's slot wait (rzk_gather_noalloc's persistent gather) on a slot that nothing
 * frees, limited to timeout_ms (1..4000).  The wait gives up, sets the timeout bit of the
 * context's error word (rzk_context_check then returns RZK_ERR_TIMEOUT) and the kernel
 * returns; *h_acquired = 0 (1 would mean the wait wrongly succeeded).  Synchronises
 * `stream`; the context stays usable. */
rzk_status rzk_debug_ring_wait(rzk_context *ctx, int timeout_ms, int *h_acquired, void *stream);

/* Aggregate ------------------------------------------------------------------------- */

/* Uploads a scene and builds its device-resident LBVH: replaces
 * AggregateBvh::AggregateBvh / build (aggregate_bvh.cc:20-240; aggregate_bvh.h:22) and the
 * scene-side tables of Scene::Scene (scene.cc:26-60, light selection pdf).
 * The Morton codes, sorted order and BFS node numbering are bit-identical to the
 * reference's.  Synchronises `stream` (the BFS build reads level sizes back). */
rzk_status rzk_scene_create(rzk_context *ctx, const rzk_scene_desc *desc, void *stream,
                            rzk_scene **out);
rzk_status rzk_scene_destroy(rzk_scene *scene);

/* Triangle, node and level counts and the device bytes the scene holds. */
rzk_status rzk_scene_info(const rzk_scene *scene, int *n_tris, int *n_nodes, int *n_levels,
                          size_t *device_bytes);
/* Aggregate::get_bounding_box (aggregate.cc:28-30): the box the Morton codes are taken
 * in, box[6] = min xyz, max xyz. */
rzk_status rzk_scene_bounding_box(const rzk_scene *scene, float *box);

/* Re-runs the LBVH build on the resident triangles (timing / rebuild after edits).
 * Same result as rzk_scene_create. Synchronises `stream`. */
rzk_status rzk_scene_rebuild(rzk_scene *scene, void *stream);

/* Copies the BVH to host buffers in the reference's layout (BvhNode,
 * aggregate_bvh.h:10-16): sorted Morton codes [n_tris], permutation sorted slot ->
 * flattened triangle [n_tris], nodes in BFS order [n_nodes].  Any pointer may be NULL.
 * Synchronises `stream`. */
rzk_status rzk_bvh_dump(rzk_scene *scene, uint32_t *h_morton_sorted, int32_t *h_perm,
                        rzk_bvh_node *h_nodes, int cap_nodes, void *stream);

/* Unsorted Morton codes of the flattened triangles (morton.h:98-102), host buffer. */
rzk_status rzk_morton_codes(rzk_scene *scene, uint32_t *h_codes, void *stream);

/* Aggregate::hit(p, q, tmin, time) for n segments (aggregate.cc:84-90 ->
 * AggregateBvh::hit any-hit, aggregate_bvh.cc:452-478).  d_out[i] = 1 when occluded. */
rzk_status rzk_occluded_batch(rzk_scene *scene, const float *d_p, const float *d_q, int n,
                              uint8_t *d_out, void *stream);

/* Aggregate::hit(ray, tmin, RAY_TMAX, time, HitRecord&) for n rays
 * (aggregate_bvh.cc:402-448, surface.cc:62-96): d_t[i] = hit distance or -1, and the
 * hit as a receiver (mat = -1 on a miss). d_recv may be NULL. */
rzk_status rzk_closest_batch(rzk_scene *scene, const float *d_o, const float *d_d, int n,
                             float *d_t, rzk_receiver *d_recv, void *stream);

/* AggregateBvh::hit for n rays given as constructed reference Rays with their own
 * [tmin, tmax] (no re-normalisation: the query sees the caller's Ray bit for bit):
 * closest = 0 is the any-hit query hit(ray, tmin, tmax, time) (aggregate_bvh.cc:452-478);
 * closest = 1 is hit(ray, tmin, tmax, time, HitRecord&) (aggregate_bvh.cc:402-448) up
 * to the record fill, returning what that fill starts from (t, beta, gamma, triangle). */
rzk_status rzk_ray_query_batch(rzk_scene *scene, const rzk_ray *d_rays, int n, int closest,
                               rzk_ray_hit *d_out, void *stream);

/* One pixel-centre primary hit per pixel: Camera::shoot_ray(i, j) (camera.cc:52-65)
 * then the closest hit; row-major, row 0 at the top of the image.  `h_cam` is a host
 * struct (use rzk_camera_setup). d_out has width*height receivers. */
rzk_status rzk_primary(rzk_scene *scene, const rzk_camera *h_cam, rzk_receiver *d_out,
                       void *stream);

/* Camera::set_perspective + Camera::focal_length_from_fov + Sensor (camera.cc:23-30,
 * camera.h:228-230, sensor.h:176-182) computed on the host: the pinhole parameters the
 * primary-ray kernel consumes. */
rzk_status rzk_camera_setup(const float eye[3], const float lookat[3], const float up[3],
                            float fov_deg, int width, int height, float film_w, float film_h,
                            rzk_camera *h_out);
/* The same from a focal length: Camera::set_perspective(eye, lookat, up, focal, sensor)
 * (camera.cc:23-30), as the OBJ importer's camera line gives it (obj_importer.cc:236-246). */
rzk_status rzk_camera_setup_focal(const float eye[3], const float lookat[3], const float up[3],
                                  float focal, int width, int height, float film_w, float film_h,
                                  rzk_camera *h_out);

/* OBJ / MTL scenes --------------------------------------------------------------------- */

/* A Wavefront OBJ scene in the reference's dialect, imported on the host: the reference
 * parser (obj_parser.cpp) and ObjImporter::load (obj_importer.cc:212-553), giving the
 * same surfaces in the same order (light quads, then faces in file order) with the same
 * BSDF parameters and light radiances.  What this path does not model is counted in
 * rzk_obj_info and left out; the scene equals the reference's where those counts are 0. */
typedef struct rzk_obj rzk_obj;
typedef struct {
    int32_t n_prims, n_mats, n_lights;   /* the scene description's primitives, materials,
                                            area lights */
    int32_t has_camera;                  /* the first `c` line: Camera::set_perspective(eye,
                                            lookat, up, focal) on a 512 x 512 sensor with a
                                            0.025 x 0.025 film (obj_importer.cc:234-252) */
    float eye[3], lookat[3], up[3], focal;
    int32_t width, height;
    float film_w, film_h;
    int32_t point_lights;                /* `lp` lines: point lights, not imported */
    int32_t spheres;                     /* `sp` lines: analytic spheres, not imported */
    int32_t faces_without_material;      /* no surface in the reference either */
    int32_t faces_unsupported_material;  /* refractive (Ni > 1) or textured (map_Kd): left out */
    int32_t short_faces;                 /* fewer than 3 vertices: skipped by the reference too */
    int32_t faces_with_vertex_normals;   /* imported with facet normals (the reference
                                            interpolates the given normals) */
    int32_t smoothed_faces;              /* smoothing group > 0: facet normals here */
    int32_t mtl_files_missing;           /* mtllib files that could not be read */
} rzk_obj_info;

/* Reads `path` (and its mtllib files, relative to its directory).  RZK_ERR_INVALID when the
 * file cannot be read or an index points outside its lists. */
rzk_status rzk_obj_import(const char *path, rzk_obj **out);
rzk_status rzk_obj_get_info(const rzk_obj *obj, rzk_obj_info *info);
/* Fills `desc` with pointers into the object (valid until rzk_obj_destroy), ready for
 * rzk_scene_create; tmin is the reference's RAY_TMIN. */
rzk_status rzk_obj_scene_desc(const rzk_obj *obj, rzk_scene_desc *desc);
rzk_status rzk_obj_destroy(rzk_obj *obj);

/* JSON scenes -------------------------------------------------------------------------- */

/* A scene file in the reference's JSON format, imported on the host: JsonImporter::load and
 * get_scene (json_importer.cc:36-899) over JsonParser (json_parser.cc).  Sections are read in
 * file order as the reference does ("geometry": OBJ meshes under <file's directory>/mesh/,
 * "materials", "light_specs", "cameras", "scene": world surfaces binding meshes to
 * materials, world lights binding meshes to area lights, views, options), giving the same
 * surfaces in the same order with the same BSDF parameters and light radiances.  What this
 * path does not model is counted and left out; the scene equals the reference's where those
 * counts are 0. */
typedef struct rzk_json rzk_json;
enum { RZK_JSON_NONE = 0, RZK_JSON_PATH = 1, RZK_JSON_VPL = 2, RZK_JSON_VPL_CUDA = 3 };
/* options.geometry.traversal (json_importer.cc:857-883): "bvh" (also the default and what an
 * unknown name reverts to), "none", and this library's "cuda_lbvh". */
enum { RZK_TRAVERSAL_BVH = 0, RZK_TRAVERSAL_NONE = 1, RZK_TRAVERSAL_CUDA_LBVH = 2 };
typedef struct {
    int32_t n_prims, n_mats, n_lights;   /* the scene description's primitives, materials,
                                            area lights */
    int32_t has_camera;                  /* the first view whose integrator and camera resolve */
    float eye[3], lookat[3], up[3];
    float focal;                         /* "focal", else from "fov" over the film height
                                            (Camera::focal_length_from_fov, camera.h:228-230) */
    int32_t width, height;               /* "image" */
    float film_w, film_h;                /* "film" */
    float near_plane, far_plane;
    int32_t integrator;                  /* that view's integrator: RZK_JSON_PATH, _VPL, or
                                            _VPL_CUDA ("vpl_cuda": this library's gather,
                                            which the reference's load_integrator lacks) */
    int32_t max_bounce, samples;
    float tmin;                          /* options.geometry.tmin, else RAY_TMIN (1e-3) */
    int32_t two_sided;                   /* options.geometry.two_sided_surfaces: every
                                            primitive carries RZK_SURF_TWO_SIDED */
    int32_t obj_files;                   /* OBJ files read */
    int32_t point_lights, spot_lights, directional_lights;   /* not imported */
    int32_t spheres;                     /* sphere surfaces and sphere area lights: not imported */
    int32_t surfaces_unsupported_material;   /* glass, mirror, or a refractive or textured
                                                OBJ material: left out */
    int32_t skipped;                     /* entries the reference reports and skips (unknown
                                            types, names that resolve to nothing) */
    int32_t faces_with_vertex_normals;   /* imported faces given vertex normals, and faces in a */
    int32_t smoothed_faces;              /* smoothing group without them: facet normals here,
                                            interpolated shading normals in the reference */
    int32_t traversal;                   /* RZK_TRAVERSAL_* from options.geometry.traversal */
} rzk_json_info;

/* Reads `path` and the OBJ and MTL files it names.  RZK_ERR_INVALID where the reference stops
 * with an error: a file that cannot be read, a syntax error, a missing key or a value of the
 * wrong type where the reference requires one. */
rzk_status rzk_json_import(const char *path, rzk_json **out);
rzk_status rzk_json_get_info(const rzk_json *js, rzk_json_info *info);
/* Fills `desc` with pointers into the object (valid until rzk_json_destroy), ready for
 * rzk_scene_create; tmin is the scene's. */
rzk_status rzk_json_scene_desc(const rzk_json *js, rzk_scene_desc *desc);
rzk_status rzk_json_destroy(rzk_json *js);

/* Warm restart: a built scene as one host blob (device arrays and host-side counts), and
 * back.  No reference counterpart (the reference rebuilds its BVH from the scene file on
 * every run, aggregate_bvh.cc:48-240).  A restored scene answers every query bit for bit
 * like the scene it was saved from, on any device of the same architecture. */
rzk_status rzk_scene_serialized_size(rzk_scene *scene, size_t *bytes);
/* Copies the scene into h_buf (cap bytes, at least rzk_scene_serialized_size); *written =
 * bytes used.  Synchronises `stream`. */
rzk_status rzk_scene_serialize(rzk_scene *scene, void *h_buf, size_t cap, size_t *written, void *stream);
/* A new scene on ctx's device from a blob; RZK_ERR_INVALID for a blob that is not one (bad
 * magic or version, truncated, sizes that disagree with its counts).  Synchronises
 * `stream`. */
rzk_status rzk_scene_deserialize(rzk_context *ctx, const void *h_buf, size_t size, void *stream,
                                 rzk_scene **out);

/* Transport-matrix files in MatrixC<Rgb>::save's format (matrix_c.cc:6-23): the text
 * header "rows cols\n" then every entry's RGB floats column by column - the device layout
 * [cols][rows][3] of rzk_gather_matrix.  rzk_matrix_save writes d_matrix to `path`;
 * rzk_matrix_file_info reads the header; rzk_matrix_load reads a file whose header matches
 * rows x cols into d_matrix (MatrixC::load reads every entry into its first element and
 * stores an unset value, matrix_c.cc:38-41; this reads what save wrote).  Synchronise
 * `stream`. */
rzk_status rzk_matrix_save(const char *path, const float *d_matrix, int rows, int cols, void *stream);
rzk_status rzk_matrix_file_info(const char *path, int *rows, int *cols);
rzk_status rzk_matrix_load(const char *path, float *d_matrix, int rows, int cols, void *stream);

/* IVplGenerator ----------------------------------------------------------------------- */

/* VplGenerator::spawn (vpl_generator.cc:183-204; generate_vpl 127-181, trace_vpl 43-110;
 * SubpathGenerator::sample_direct_vertex path.cc:171-334): one thread per light particle,
 * draw d of particle k from the counter-based stream (seed, 0, k).  VPLs are written to
 * d_out in the reference's push order (particle-major, bounce-minor), at most `cap`; the
 * total produced is written to *d_count (device int).  Bounce-0 VPLs are not stored
 * (vpl_generator.cc:150-151). */
rzk_status rzk_vpl_generate(rzk_scene *scene, uint32_t seed, int n_particles, int max_bounce,
                            rzk_vpl *d_out, int cap, int *d_count, void *stream);

/* IVirtualPointLightEvaluator / TransportMatrix ---------------------------------------- */

/* The full gather: d_rgb[r] = scale * sum_j radiance(receiver r, vpl j), where
 * radiance is VirtualPointLight::gather_point (vpl.cc:661-688) with clamp mode/threshold
 * (vpl.cc:214-230).  Receivers with mat < 0 get black.  This is the per-pixel sum of
 * LightTransportMatrix::fill (light_transport_matrix.cc:16-48) without materialising
 * the matrix, and connect_to_vpl's NONE / POWER_SAMPLING accumulation (vpl.cc:496-520)
 * over all VPLs.  The sum is deterministic: VPLs are grouped into chunks of nearby VPLs
 * (a stable sort along a Hilbert curve through their positions) and the chunk sums added in chunk
 * order, so only the float summation order differs from the reference's VPL order. */
rzk_status rzk_gather(rzk_context *ctx, rzk_scene *scene, const rzk_receiver *d_recv,
                      int n_recv, const rzk_vpl *d_vpls, int n_vpl, int clamp_mode, float tau,
                      float scale, float *d_rgb, void *stream);

/* Number of compiled gather tile configurations (threads per CTA x VPLs per shared-memory
 * tile); the autotuner searches these. */
int rzk_gather_variants(void);

/* rzk_gather with an explicit layout and tile configuration.  image_width > 0 declares
 * the receivers a row-major image of that width (as rzk_primary writes them): each warp
 * then takes an 8 x 4 pixel tile, whose shadow rays are more coherent than a 32-pixel
 * row; 0 = 32 consecutive receivers per warp.  `variant` in [0, rzk_gather_variants()),
 * `n_chunks` VPL chunks (0 = automatic).  Layout and variant never change the image;
 * n_chunks changes only the float summation order.  n_chunks = 1 sums in exactly the
 * reference's order; with more chunks each chunk is a run of the VPLs stably sorted by the
 * Hilbert-curve index of their positions' cells on a 256^3 grid over the scene box
 * (nearby VPLs trace coherent shadow rays), and the chunk sums are added in chunk order. */
rzk_status rzk_gather_cfg(rzk_context *ctx, rzk_scene *scene, const rzk_receiver *d_recv,
                          int n_recv, int image_width, const rzk_vpl *d_vpls, int n_vpl,
                          int clamp_mode, float tau, float scale, float *d_rgb, int variant,
                          int n_chunks, void *stream);

/* Same computation from host buffers: copies receivers and VPLs to the device, gathers
 * and copies the image back (the end-to-end drop-in call).  image_width as in
 * rzk_gather_cfg.  Synchronises `stream`. */
rzk_status rzk_gather_host(rzk_context *ctx, rzk_scene *scene, const rzk_receiver *h_recv,
                           int n_recv, int image_width, const rzk_vpl *h_vpls, int n_vpl,
                           int clamp_mode, float tau, float scale, float *h_rgb, void *stream);

/* Bytes of the fixed device array that rzk_gather_noalloc uses as scratch. */
#define RZK_NOALLOC_SCRATCH_BYTES (16u << 20)

/* rzk_gather without any device allocation.  No counterpart in the reference.
 * For callers that cannot let the library call cudaMalloc - their device memory is owned
 * by another framework's allocator or held to a fixed budget, or they run a frame loop in
 * which an allocation (which can synchronise the device or fail) is not acceptable.  The
 * scratch (a work counter, the spatially ordered VPL copy with its sort scratch when it
 * fits, and the chunk ring in which the gather sums each 8 x 4 tile's VPL chunks as soon
 * as the tile's last chunk is done) is a fixed static device array of
 * RZK_NOALLOC_SCRATCH_BYTES (16 MiB) that every GPU loading the library holds until the
 * process exits; the call itself allocates and frees nothing.
 *   - Size: the array holds the chunk sums of a window of tiles (about 1,000 tiles at 32
 *     chunks), not of the image, so any number of receivers is served in one launch.
 *   - The current device must be the scene's context's device (else RZK_ERR_INVALID).
 *   - The first call on a device looks up the array's device address there (once per
 *     device, with that device current); make that first call before any stream capture.
 *   - All calls share the one array, and it keeps the previous call's contents (the call
 *     clears what it uses first): calls whose work overlaps on the GPU (other streams,
 *     other host threads) race and must be serialised by the caller.
 *   - Result: rzk_gather's chunking (at most 32 chunks of >= 128 VPLs, the VPLs in the
 *     Hilbert order) wherever the ordered copy leaves room for a ring of 512 tiles (up to
 *     about 90,000 VPLs) - then the image is rzk_gather's bit for bit; beyond that the
 *     caller's VPL order changes only the float summation order.
 *   - Like every kernel of the library it reports a bounded wait that gave up in the
 *     context's error word, not in its return value: check rzk_context_check on the
 *     scene's context after the stream has run the call (the image is undefined after a
 *     reported error). */
rzk_status rzk_gather_noalloc(rzk_scene *scene, const rzk_receiver *d_recv, int n_recv,
                              int image_width, const rzk_vpl *d_vpls, int n_vpl, int clamp_mode,
                              float tau, float scale, float *d_rgb, void *stream);

/* LightTransportMatrix::fill (light_transport_matrix.cc:16-48): every pair's radiance
 * into a column-major rows x cols MatrixC<Rgb> (matrix_c.h:20-107) d_matrix
 * [n_vpl][n_recv][3], and optionally its visibility d_vis [n_vpl][n_recv]. */
rzk_status rzk_gather_matrix(rzk_scene *scene, const rzk_receiver *d_recv, int n_recv,
                             const rzk_vpl *d_vpls, int n_vpl, int clamp_mode, float tau,
                             float *d_matrix, uint8_t *d_vis, void *stream);

/* VirtualPointLight::incident_radiance (vpl.cc:411-440) for every pair, column-major
 * [n_vpl][n_recv][3].  No visibility. */
rzk_status rzk_incident_matrix(rzk_scene *scene, const rzk_receiver *d_recv, int n_recv,
                               const rzk_vpl *d_vpls, int n_vpl, int clamp_mode, float tau,
                               float *d_matrix, void *stream);

/* Mean over n_pairs seeded (receiver, VPL) pairs of RadianceTerms::radiance_no_clamp
 * .value() (vpl_interface.h:102-116), occluded pairs counted as zero: the base of the
 * "0.1 x mean contribution" RADIANCE clamp.  Pair k uses receiver
 * draw(seed,3,k,0) % n_recv and VPL draw(seed,3,k,1) % n_vpl.  *h_mean is written after
 * `stream` is synchronised. */
rzk_status rzk_mean_contribution(rzk_context *ctx, rzk_scene *scene,
                                 const rzk_receiver *d_recv, int n_recv,
                                 const rzk_vpl *d_vpls, int n_vpl, uint32_t seed,
                                 int n_pairs, double *h_mean, void *stream);

/* Batched gather ----------------------------------------------------------------------- */

/* One gather of a batch: the arguments of rzk_gather_cfg for one scene / image / VPL set. */
typedef struct {
    rzk_scene *scene;
    const rzk_receiver *d_recv;
    int32_t n_recv;
    int32_t image_width;        /* as in rzk_gather_cfg; 0 = 32 consecutive receivers/warp */
    const rzk_vpl *d_vpls;
    int32_t n_vpl;
    int32_t clamp_mode;
    float tau;
    float scale;
    float *d_rgb;               /* n_recv x 3 output */
} rzk_gather_job;

typedef struct rzk_batch rzk_batch;

/* Number of compiled batch tile configurations (warps per CTA, VPLs per tile, CTAs/SM,
 * warp tile shape). */
int rzk_batch_variants(void);
/* A batch variant's tile shape: warps per CTA (each warp one 32-receiver packet, one lane
 * per shadow ray), VPLs per shared-memory tile, resident CTAs per SM it is compiled for, and
 * the warp tile's width in pixels (8: 8 x 4 receivers; 4: 4 x 8; 16: 16 x 2; 32: 32 x 1). */
rzk_status rzk_batch_variant_info(int variant, int32_t *warps, int32_t *vpl_tile, int32_t *ctas_per_sm,
                                  int32_t *tile_width);

/* Describes a batch of independent gathers (the integrator's per-frame gather of
 * vpl.cc:496-520 for many scenes or requests at once): uploads a device job table and
 * allocates one partial-sum buffer.  chunk_len = VPLs per work item (a multiple of 128;
 * 0 = rzk_gather's default).  Synchronous.  No reference counterpart (the reference
 * renders one scene per process, integrator_scheduler.cc:54-229). */
rzk_status rzk_batch_create(rzk_context *ctx, const rzk_gather_job *jobs, int n_jobs, int variant,
                            int chunk_len, rzk_batch **out);
/* Runs every job of the batch: one memset, then per table of up to 128 jobs the spatial
 * ordering of its chunked jobs' VPLs (as rzk_gather_cfg orders them, in one sort), one
 * persistent launch and one reduction; no allocation and no synchronisation, so it can be
 * captured in a CUDA graph and replayed.
 * Each job's image equals rzk_gather_cfg's for the same chunk length, bit for bit. */
rzk_status rzk_batch_run(rzk_batch *batch, void *stream);
rzk_status rzk_batch_destroy(rzk_batch *batch);
/* Autotuner: times every batch variant (tile shape) x chunk length in {default (0), 512,
 * 1024, 2048} (best of two runs each) on up to max_probe_jobs evenly spaced jobs (0 = all)
 * and returns the fastest; h_probe_ms (NULL or rzk_batch_variants() x 4 floats, variant-major)
 * receives every probe's time.  Synchronises `stream`. */
rzk_status rzk_batch_autotune(rzk_context *ctx, const rzk_gather_job *jobs, int n_jobs,
                              int max_probe_jobs, int *best_variant, int *best_chunk_len,
                              float *best_ms, float *h_probe_ms, void *stream);

/* Clustering ------------------------------------------------------------------------- */

/* LightTransportMatrix::generate_alphas_for_clustering (light_transport_matrix.cc:72-106)
 * on the column-major matrix d_matrix [cols][rows][3] (MatrixC<Rgb>, as rzk_gather_matrix
 * writes it): d_alphas[cols]; optional d_col_norms[cols] = get_column_norms
 * (light_transport_matrix.cc:118-130).  Bit-identical to the reference (every sum in the
 * reference's order).  Synchronises `stream`. */
rzk_status rzk_ltm_alphas(const float *d_matrix, int rows, int cols, float *d_alphas,
                          float *d_col_norms, void *stream);

/* ClusterBuilder::cluster_by_sampling (cluster_builder.cc:82-273) on d_matrix: centre
 * sampling by alpha and the representatives are drawn on the host from the counter-based
 * stream (seed, 1, 0) in the reference's order; the column-to-cluster distances and the
 * nearest-cluster assignment run on the device.  Outputs (host): *h_n_clusters, and per
 * final cluster its centre column, representative column and weight (capacity
 * max(num_clusters, cols)); h_assign[cols] = final cluster of each column or -1.
 * Synchronises `stream`. */
rzk_status rzk_cluster_by_sampling(const float *d_matrix, int rows, int cols, int num_clusters,
                                   uint32_t seed, int *h_n_clusters, int32_t *h_center,
                                   int32_t *h_representative, float *h_weight,
                                   int32_t *h_assign, void *stream);

/* Matrix row-column sampling ---------------------------------------------------------- */

/* MatrixRowColumnSampling (mrcs.cc:16-186, mrcs.h:17-45). */
typedef struct rzk_mrcs rzk_mrcs;
typedef struct {
    int32_t block_size;     /* side of the pixel strata that give the matrix rows (32) */
    float cluster_ratio;    /* clusters per VPL (0.01) */
    int32_t max_clusters;   /* cap on the cluster count (1000) */
    int32_t max_columns;    /* more VPLs than this are resampled to this many columns (10000) */
    uint32_t seed;          /* the set-up's random stream is (seed, 7, 0) */
} rzk_mrcs_params;

/* MatrixRowColumnSampling's defaults (mrcs.cc:16-20; max_columns mrcs.cc:79). */
rzk_status rzk_mrcs_params_default(rzk_mrcs_params *params);
/* MatrixRowColumnSampling::initialize (mrcs.cc:43-186) for the camera's image and the
 * device VPLs: stratified pixels (ImageSampler::sample_stratified, image_sampler.cc:8-23),
 * the columns (every VPL, or max_columns resampled by average power), the reduced matrix
 * (LightTransportMatrix::fill) on the device, then ClusterBuilder::cluster_by_sampling.
 * All draws come from one stream in the reference's program order.  With more than
 * max_columns VPLs the reference assigns columns past the end of its reduced matrix and
 * gathers from all_vpls with reduced indices (cluster_builder.cc:189-199, mrcs.cc:36);
 * here the clustering and the representatives use the resampled columns.  The VPLs need
 * not outlive the call.  Synchronises `stream`. */
rzk_status rzk_mrcs_create(rzk_context *ctx, rzk_scene *scene, const rzk_camera *camera,
                           const rzk_vpl *d_vpls, int n_vpl, int clamp_mode, float tau,
                           const rzk_mrcs_params *params, void *stream, rzk_mrcs **out);
rzk_status rzk_mrcs_destroy(rzk_mrcs *mrcs);
/* Matrix rows (sampled pixels), columns, the target cluster count, the clusters found
 * (before dropping those without a representative) and the set-up stage times in ms
 * (pixels + columns, matrix, clustering, representatives).  Any pointer may be NULL. */
rzk_status rzk_mrcs_info(const rzk_mrcs *mrcs, int *n_rows, int *n_columns, int *num_clusters,
                         int *n_clusters, float *stage_ms);
/* The sampled pixels (x, y per row) and per cluster its centre column, representative
 * column (-1: none, the cluster never gathers) and weight.  Any pointer may be NULL. */
rzk_status rzk_mrcs_clusters(const rzk_mrcs *mrcs, int32_t *h_pixels, int32_t *h_center,
                             int32_t *h_representative, float *h_weight);
/* MatrixRowColumnSampling::gather_clusters (mrcs.cc:28-41) for every receiver:
 * d_rgb[r] = scale * sum over clusters of weight x radiance(r, representative), added in
 * cluster order (the integrator divides by num_emitted_photons, vpl.cc:481-484: pass
 * scale = 1 / num_emitted).  image_width as in rzk_gather_cfg.  Runs as a tracing pass
 * (visibility ballots, one 32-bit word per warp tile and representative, held by the
 * object and grown by the first gather of a larger image) and a summing pass. */
rzk_status rzk_mrcs_gather(rzk_mrcs *mrcs, const rzk_receiver *d_recv, int n_recv, int image_width,
                           float scale, float *d_rgb, void *stream);

/* LightSlice ------------------------------------------------------------------------- */

/* LightSlice's settings (lightslice.h:306-312, lightslice.cc:23-85). */
typedef struct {
    int32_t num_clusters;         /* global VPL clusters (num_clusters) */
    int32_t max_slice_size;       /* kd-tree leaf capacity that makes a slice (>= 2) */
    int32_t num_neighbor_slices;  /* rows of a slice's matrix L */
    int32_t max_slice_clusters;   /* per-slice refinement stops at this many clusters */
    int32_t map_resolution;       /* Jensen map side (luminance_map_resolution) */
    float map_epsilon;            /* luminance_map_epsilon */
    float density_radius;         /* estimate_sum's disk radius */
    int32_t incident_clamp_mode;  /* clamp of incident_radiance in the reduced matrix */
    float incident_tau;
    uint32_t seed;                /* streams (seed,4,0) slicing, (seed,1,0) clustering, (seed,5,s) refinement */
    int32_t n_threads;            /* host threads refining slices (0 = all cores) */
} rzk_lightslice_params;

typedef struct rzk_lightslice rzk_lightslice;

/* The reference's defaults (lightslice.cc:23-85; seed 2013 as random.h:21). */
rzk_status rzk_lightslice_params_default(rzk_lightslice_params *params);

/* LightSlice::initialize (lightslice.cc:589-1277) for one image: d_recv are the width x
 * height primary receivers (row-major, as rzk_primary writes them), d_vpls the VPL set (only
 * VPLs of bounce <= 1 are used, lightslice.cc:606-613).  Slices the shading points with the
 * 6-D kd-tree (lightslice.cc:252-303), traces the reduced matrix of the slice
 * representatives on the device, clusters its columns (cluster_builder.cc:82-273), refines
 * the clusters per slice (lightslice.cc:789-1060), and builds the per-slice Jensen maps
 * (lightslice.cc:2058-2151).  The maps are built for the slices whose VPL sum is positive:
 * the reference calls build_map before it sets the sampling records' is_valid (still
 * value-initialised false), which would leave every map empty.  Synchronous. */
rzk_status rzk_lightslice_create(rzk_context *ctx, rzk_scene *scene, const rzk_receiver *d_recv, int width,
                                 int height, const rzk_vpl *d_vpls, int n_vpl,
                                 const rzk_lightslice_params *params, rzk_lightslice **out, void *stream);
rzk_status rzk_lightslice_destroy(rzk_lightslice *ls);
/* Sizes and the host time of each build stage (h_ms[8]: points+filter, slicing, reduced
 * matrix, global clustering, refinement, maps, tables). */
rzk_status rzk_lightslice_info(const rzk_lightslice *ls, int32_t *n_points, int32_t *n_slices,
                               int32_t *n_vpl_used, int32_t *n_global_clusters, int32_t *n_slice_clusters,
                               double *h_ms);
/* Slicing dump: per kd-tree data position its pixel; per slice [start, end], representative
 * (a data position) and its nearest slices (num_neighbor_slices each, furthest first, -1
 * padded).  Any pointer may be NULL. */
rzk_status rzk_lightslice_slices(const rzk_lightslice *ls, int32_t *h_point_pixel, int32_t *h_start,
                                 int32_t *h_end, int32_t *h_rep, int32_t *h_neighbors);
/* Per-slice clusters, slice-major: h_count[n_slices]; per cluster its representative
 * (one-bounce VPL index), weight, upper-hemisphere flag, direction to the representative,
 * total incident radiance, probability in the slice's cluster distribution, member count;
 * h_members the members of every cluster in order.  Any pointer may be NULL. */
rzk_status rzk_lightslice_clusters(const rzk_lightslice *ls, int32_t *h_count, int32_t *h_rep, float *h_weight,
                                   uint8_t *h_upper, float *h_wi, float *h_incident, float *h_pdf,
                                   int32_t *h_size, int32_t *h_members);
/* The global clustering of the one-bounce VPL columns (ClusterBuilder::cluster_by_sampling,
 * cluster_builder.cc:82-273, as LightSlice::initialize runs it, lightslice.cc:756-762):
 * per global cluster (n_global_clusters of rzk_lightslice_info) its representative column
 * and weight, per column (n_vpl_used) its cluster.  Any pointer may be NULL. */
rzk_status rzk_lightslice_global(const rzk_lightslice *ls, int32_t *h_rep, float *h_weight, int32_t *h_assign);
/* Jensen maps [slice][res][res] (row-major, row = y), validity, VPL sum, row CDFs
 * [slice][res] and column CDFs [slice][res][res] (DiscretePdf2D, pdf.cc:195-229). */
rzk_status rzk_lightslice_maps(const rzk_lightslice *ls, float *h_maps, uint8_t *h_valid, float *h_sum,
                               float *h_row_cdf, float *h_col_cdf);
/* The reduced matrix (column-major [n_vpl_used][n_slices][3]) and visibility, copied to
 * device buffers, and the input index of every one-bounce VPL.  Any pointer may be NULL. */
rzk_status rzk_lightslice_matrix(const rzk_lightslice *ls, float *d_R, uint8_t *d_V, int32_t *h_vpl_index,
                                 void *stream);
/* KdTreeN::find_cluster with the plane bias (kdtree_n.h:486-518) for every receiver: its
 * slice, or -1 without a material. */
rzk_status rzk_lightslice_find_slice(rzk_lightslice *ls, const rzk_receiver *d_recv, int n_recv,
                                     int32_t *d_slice, void *stream);
/* Host-input forms of the two host stages, for callers that computed the points, the
 * reduced matrix or the global clusters elsewhere (and for checking those stages on their
 * own).  rzk_lightslice_host_slice: the 6-D points [n][6] with their pixels, in pixel order
 * -> slices, representatives, neighbours.  rzk_lightslice_host_refine: the reduced matrix
 * [n_vpl_used][n_slices][3] and visibility of that slicing, the used VPLs, each slice's
 * representative receiver, the global clusters (representative, weight), each column's
 * cluster and magnitude -> per-slice clusters, distributions and maps.  Objects made this
 * way have no device tables: gather and find_slice return RZK_ERR_INVALID on them. */
rzk_status rzk_lightslice_host_slice(const rzk_lightslice_params *params, const float *h_points,
                                     const int32_t *h_pixel, int n_points, rzk_lightslice **out);
rzk_status rzk_lightslice_host_refine(rzk_lightslice *ls, const float *h_R, const uint8_t *h_V, int n_vpl_used,
                                      const rzk_vpl *h_vpls_used, const rzk_receiver *h_rep_recv,
                                      int n_global, const int32_t *h_global_rep, const float *h_global_weight,
                                      const int32_t *h_assign, const float *h_mags);
/* KdTreeN::find_cluster (kdtree_n.h:486-518) on the host for 6-D points [n][6]. */
rzk_status rzk_lightslice_host_find(const rzk_lightslice *ls, const float *h_points, int n, int32_t *h_slice);
/* LightSlice::gather_clusters (lightslice.cc:1315-1345) for every receiver, times `scale`
 * (1 / num_emitted_photons, vpl.cc:487-490): the sum over its slice's clusters of
 * weight x radiance(representative) where visible, in cluster order.  Receivers without a
 * material get black. */
rzk_status rzk_lightslice_gather(rzk_lightslice *ls, const rzk_receiver *d_recv, int n_recv, int clamp_mode,
                                 float tau, float scale, float *d_rgb, void *stream);

/* Guided path tracing ---------------------------------------------------------------- */

typedef struct {
    int32_t spp;              /* samples per pixel (pixel-centre primary rays) */
    int32_t max_bounce;       /* VirtualPointLight max_bounce, 1..16 */
    int32_t rr_depth;         /* Russian roulette at vertices deeper than this; 0 = off */
    float rr_prob;            /* survival probability when Russian roulette applies */
    int32_t direct_lighting;  /* Integrator::is_direct_lighting */
    uint32_t seed;            /* sample s of pixel k draws from stream (seed, 6, k * spp + s) */
    int32_t sampler;          /* LightSlice's direction sampler: RZK_GUIDE_JENSEN (0) or
                                 RZK_GUIDE_METROPOLIS (1, the reference's default) */
    int32_t chain_samples;    /* METROPOLIS: chain states kept per slice after the warm-up
                                 (0: 4096) */
} rzk_guided_params;
enum { RZK_GUIDE_JENSEN = 0, RZK_GUIDE_METROPOLIS = 1 };

/* VirtualPointLight::guided_path_trace / trace_wellington with METRO_RANDOM
 * (vpl.cc:907-1040) guided by a LightSlice (LightSlice::sample / pdf, lightslice.cc:1569-2056)
 * with its JENSEN sampler (the slice's luminance map, lightslice.cc:2313-2377) or its
 * METROPOLIS sampler (Metropolis chains over each slice's incoming-radiance density,
 * lightslice.cc:1427-1517, 1709-1928: eight per slice, each with the reference's 1,024-state
 * warm-up, run before the paths from the streams (seed, 8, slice * 8 + chain), and a path
 * draws a state of its slice's chains uniformly, so the directions match the reference's in
 * distribution only) and FirstBounce::radiance for
 * direct light (first_bounce.h:54-71, area_light.cc:48-142).  Russian roulette (rr_depth,
 * rr_prob) has no reference counterpart: the reference recursion always runs to
 * max_bounce.  Writes the per-pixel mean over spp (d_rgb [W*H][3]) and optionally every
 * path's radiance (d_paths [W*H*spp][3], path = pixel * spp + sample). */
rzk_status rzk_guided_render(rzk_context *ctx, rzk_scene *scene, rzk_lightslice *ls, const rzk_camera *camera,
                             const rzk_guided_params *params, float *d_rgb, float *d_paths, void *stream);
/* LightSlice::eval_incoming_radiance (FIXED_RADIUS, lightslice.cc:1427-1517): the METROPOLIS
 * sampler's density of slice d_slice[i] at the point (d_xy[2i], d_xy[2i+1]) of the unit
 * square of that slice's sampling record, into d_out[i] (0 for a slice out of range). */
rzk_status rzk_lightslice_density(rzk_lightslice *ls, const int32_t *d_slice, const float *d_xy, int n, float *d_out,
                                  void *stream);
/* The METROPOLIS chains rzk_guided_render draws from (LightSlice::metropolis_sample,
 * lightslice.cc:1763-1911): per slice eight chains from the streams (seed, 8, slice * 8 +
 * chain), each 1,024 warm-up states (the first a cluster drawn from the slice's cluster
 * distribution) and then its eighth of the slice's n_samples states in order, each as
 * (x, y, density, 0) with (x, y) its point on the unit square of the slice's sampling record
 * (direction_to_square), into d_out [n_slices][n_samples][4]; zeros for a slice without a
 * valid sampling record. */
rzk_status rzk_lightslice_chains(rzk_lightslice *ls, uint32_t seed, int n_samples, float *d_out, void *stream);

/* Serving ---------------------------------------------------------------------------- */

enum { RZK_REQ_GATHER = 0, RZK_REQ_GUIDED = 1 };

/* One request: a gather (the VPL integrator's frame, vpl.cc:496-520) or a guided render
 * (vpl.cc:907-932) of a device-resident scene through the request's own camera. */
typedef struct {
    int32_t kind;                 /* RZK_REQ_GATHER or RZK_REQ_GUIDED */
    rzk_scene *scene;
    rzk_lightslice *lightslice;   /* guided: the scene's LightSlice */
    rzk_camera camera;            /* the image: camera.width x camera.height pixel-centre rays */
    const rzk_vpl *d_vpls;        /* gather: VPLs, count, clamp, 1 / num_emitted */
    int32_t n_vpl;
    int32_t clamp_mode;
    float tau;
    float scale;
    int32_t spp;                  /* guided: as rzk_guided_params */
    int32_t max_bounce;
    int32_t rr_depth;
    float rr_prob;
    uint32_t seed;
    float *d_rgb;                 /* caller-owned device output, width * height * 3 floats */
    int32_t sampler;              /* guided: RZK_GUIDE_JENSEN (0) or RZK_GUIDE_METROPOLIS (1) */
} rzk_request;

typedef struct {
    int64_t hbm_budget_bytes;  /* device memory admitted requests may hold (0 = 90% of free at create) */
    int32_t batching;          /* 1: each iteration's gathers run as one batched launch; 0: one request at a time */
    int32_t max_batch;         /* most requests taken per iteration (0 = 256) */
} rzk_server_params;

typedef struct rzk_server rzk_server;

/* A request loop with its own context, stream and worker thread on `device`.  No reference
 * counterpart: the reference renders one scene per process (integrator_scheduler.cc). */
rzk_status rzk_server_create(int device, const rzk_server_params *params, rzk_server **out);
/* Finishes every admitted request, then releases the server. */
rzk_status rzk_server_destroy(rzk_server *server);
/* Admits the request if the device memory it will hold in flight (receivers, and for a
 * gather its per-chunk partial sums and its spatially ordered VPL copy with the sort's
 * scratch) fits the budget next to the admitted ones, else
 * returns RZK_ERR_BUSY without queueing it.  Thread-safe.  The caller keeps the scene, the
 * VPLs, the LightSlice and d_rgb alive until the request is done. */
rzk_status rzk_server_submit(rzk_server *server, const rzk_request *request, uint64_t *ticket);
/* *state: 0 queued, 1 running, 2 done, 3 cancelled, 4 failed.  A finished request is
 * reported once (with its latency, submit to completion) and then forgotten; the return
 * value is the request's status. */
rzk_status rzk_server_poll(rzk_server *server, uint64_t ticket, int32_t *state, double *latency_ms);
/* Waits up to timeout_ms (< 0: no limit) for the request; RZK_ERR_TIMEOUT if it is still
 * pending.  Reports and forgets it like rzk_server_poll. */
rzk_status rzk_server_wait(rzk_server *server, uint64_t ticket, int32_t timeout_ms, double *latency_ms);
/* Withdraws a request that is still queued; RZK_ERR_BUSY once it has been launched. */
rzk_status rzk_server_cancel(rzk_server *server, uint64_t ticket);
/* Counters since creation; `launches` counts the kernels the server has launched. */
rzk_status rzk_server_stats(rzk_server *server, int64_t *submitted, int64_t *rejected, int64_t *completed,
                            int64_t *launches, int64_t *held_bytes, int64_t *budget_bytes);
/* Where each completed request's latency went, in completion order (the first `cap`, at
 * most 2^20 kept): its kind, the time from submit to the launch of its group (waiting for a
 * slot) and from that launch to completion (the group on its stream, behind the group
 * before it).  *n receives the number recorded. */
rzk_status rzk_server_timings(rzk_server *server, int32_t *h_kind, double *h_queue_ms, double *h_run_ms, int cap,
                              int32_t *n);

#ifdef __cplusplus
}
#endif

#endif /* RZK_H_ */
