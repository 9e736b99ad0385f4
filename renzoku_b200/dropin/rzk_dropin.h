/*
 * rzk_dropin.h - the B200 gather path behind the reference's own C++ interfaces.
 *
 * These classes implement Renzoku's Aggregate (aggregate.h:15-91), IVplGenerator
 * (vpl_generator.h:8-21) and Integrator (integrator.h:54-87, through
 * MonteCarloIntegrator, monte_carlo_integrator.h:28-48) on top of the C ABI of
 * librzk_cuda.so (include/rzk.h), so that the reference's renderer selects the device
 * path from a scene file: "options.geometry.traversal": "cuda_lbvh" picks AggregateCuda
 * and an integrator of type "vpl_cuda" picks VirtualPointLightCuda (load_scene_cuda
 * below extends the selection of JsonImporter::get_scene, json_importer.cc:854-897, and
 * JsonImporter::load_integrator, json_importer.cc:523-588).
 *
 * Compiled against the reference's headers (the reference tree on the quote-include
 * path) and linked with librzk_cuda.so and the CUDA runtime; the reference's own
 * translation units come from the program that loads it.
 */
#ifndef RZK_DROPIN_H_
#define RZK_DROPIN_H_

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "aggregate.h"
#include "monte_carlo_integrator.h"
#include "vpl_generator.h"
#include "scene.h"

#include "../../include/rzk.h"

namespace Renzoku {

/* The scene's surfaces as a device-resident LBVH (rzk_scene_create).  Every query answers
 * what AggregateBvh would (aggregate_bvh.cc:402-478) bit for bit: the device tests the
 * caller's constructed Ray over the caller's interval, and a closest hit's HitRecord is
 * filled by the reference's own Triangle::fill_hit_record and Surface::fill_hit_record
 * from the device's (t, beta, gamma, triangle).  The three virtual hit() overloads answer
 * one query per call (a device round trip, serialised across host threads); hit_batch and
 * hit_segments answer many in one launch.  Errors (an unsupported material, a CUDA
 * failure) throw std::runtime_error, as Aggregate::sample does (aggregate.cc:143). */
class AggregateCuda : public Aggregate {
public:
    explicit AggregateCuda(const Surfaces &surfaces, Float tmin = RAY_TMIN, int device = 0);
    virtual ~AggregateCuda();

    virtual bool hit(const Ray &r, Float tmin, Float tmax, Float time, HitRecord &record) const;
    virtual bool hit(const Ray &r, Float tmin, Float tmax, Float time) const;
    virtual bool hit(const Vec3 &p, const Vec3 &q, Float tmin, Float time) const;

    /* n rays with their intervals.  records == NULL: any-hit, hits[i] set; otherwise the
     * closest hit's record in records[i] and hits[i]. */
    void hit_batch(const Ray *rays, const Float *tmin, const Float *tmax, int n, bool *hits,
                   HitRecord *records) const;
    /* Aggregate::hit(p[i], q[i], tmin, time) for n segments (aggregate.cc:84-90). */
    void hit_segments(const Vec3 *p, const Vec3 *q, int n, Float tmin, bool *occluded) const;

    rzk_scene *handle() const { return scene_h; }
    rzk_context *context() const { return ctx; }
    int device() const { return dev; }
    /* the reference Material behind a device material index (rzk_vpl::mat, rzk_receiver::mat) */
    Material *material(int index) const;
    /* the device material index of a reference Material (-1 if the scene has none such) */
    int material_index(const Material *m) const;

private:
    void query(const std::vector<rzk_ray> &rays, bool closest, std::vector<rzk_ray_hit> &out) const;
    void fill_record(const Ray &r, const rzk_ray_hit &h, HitRecord &record) const;

    int dev = 0;
    rzk_context *ctx = nullptr;
    rzk_scene *scene_h = nullptr;
    std::vector<Material *> mat_ptrs;     // device material index -> reference material
    std::vector<int> tri_surface;         // flattened triangle -> surface index
    std::vector<int> tri_local;           // flattened triangle -> triangle of its shape
    // staging of the one-query calls (guarded by mu)
    mutable std::mutex mu;
    mutable void *d_stage = nullptr;
    mutable size_t stage_bytes = 0;
};

/* IVplGenerator::spawn on the device (rzk_vpl_generate): one thread per light particle,
 * particle k drawing from the counter-based stream (seed, 0, k) instead of the scene's one
 * sequential generator, VPLs appended in the reference's push order (particle-major,
 * bounce-minor; bounce-0 VPLs not stored, vpl_generator.cc:150-151), each VPL's previous
 * reference its parent on the same path.  The scene's aggregate must be an AggregateCuda. */
class VplGeneratorCuda : public IVplGenerator {
public:
    explicit VplGeneratorCuda(uint32_t seed = 2013) : seed(seed) {}
    virtual void spawn(Scene *scene, int num_start_samples, int max_bounce, BrdfPointLights &lights,
                       bool is_photon = false);
    /* light particles whose VPLs the last spawn produced (VirtualPointLight divides by it,
     * vpl.cc:487-490) */
    int num_emitted() const { return emitted; }

private:
    uint32_t seed;
    int emitted = 0;
};

/* The "vpl_cuda" integrator: the VPL gather of every pixel on the device.  initialize()
 * traces the pixel-centre primary hits (Camera::shoot_ray, camera.cc:52-65), generates
 * the VPLs (VplGeneratorCuda, keeping the first max_vpls in push order) and sets the
 * RADIANCE clamp threshold to clamp_scale x the mean unclamped contribution over seeded
 * pairs; integrate() gathers every pixel against every VPL (gather_point, vpl.cc:661-688,
 * divided by the emitted particles, vpl.cc:487-490) and keeps the image on the host;
 * transfer_to_frame() copies it into the scene's frame buffer.  Like the reference's GPU
 * integrators it outputs through the viewer (is_viewer_outputing), so Scene::start runs
 * it without the CPU scheduler. */
class VirtualPointLightCuda : public MonteCarloIntegrator {
public:
    VirtualPointLightCuda();
    virtual ~VirtualPointLightCuda();

    virtual void initialize(Scene *scene);
    virtual void integrate();
    virtual bool integrate_partial() { integrate(); return false; }
    virtual void transfer_to_frame();
    virtual string get_suffix() const { return "vpl_cuda"; }
    virtual bool is_viewer_outputing() const { return true; }

    void set_start_particles(int n) { start_particles = n; }
    void set_max_vpls(int n) { max_vpls = n; }
    void set_seed(uint32_t s) { seed = s; }
    void set_clamping(int mode, Float scale) { clamp_mode = mode; clamp_scale = scale; }

    int width() const { return w; }
    int height() const { return h; }
    int num_vpls() const { return n_vpl; }
    int num_emitted() const { return emitted; }
    Float clamping_threshold() const { return tau; }
    /* the last integrated image, row-major [height][width][3] */
    const std::vector<float> &image() const { return img; }
    /* device buffers of the receivers and VPLs the gather used (for callers that pass them
     * on to other entry points of the library) */
    const rzk_receiver *device_receivers() const { return d_recv; }
    const rzk_vpl *device_vpls() const { return d_vpls; }

private:
    void release();

    AggregateCuda *agg = nullptr;
    int start_particles = 24000, max_vpls = 32768;
    uint32_t seed = 2013;
    int clamp_mode = RZK_CLAMP_RADIANCE;
    Float clamp_scale = 0.1f, tau = 0.0f;
    int w = 0, h = 0, n_vpl = 0, emitted = 0;
    rzk_receiver *d_recv = nullptr;
    rzk_vpl *d_vpls = nullptr;
    float *d_rgb = nullptr;
    std::vector<float> img;
};

/* A scene file through the reference's JSON format with the device path selectable:
 * traversal "cuda_lbvh" -> AggregateCuda, "bvh" -> AggregateBvh, "none" -> Aggregate
 * (anything else: AggregateBvh, as json_importer.cc:873-876 reverts); the first view's
 * integrator "vpl_cuda" -> VirtualPointLightCuda (max_bounce and "samples" as the start
 * particles), other integrator types left to the caller (NULL).  The scene is read by the
 * library's own importer (rzk_json_import) and rebuilt as the reference's objects
 * (Triangle / Quad shapes, BsdfMaterial over Lambertian / ModifiedPhong / Ward, area
 * lights, a perspective Camera).  Throws std::runtime_error when the file cannot be read. */
Scene *load_scene_cuda(const std::string &path, int device = 0);

}  // namespace Renzoku

#endif  // RZK_DROPIN_H_
