// rzk_capi.cu - the C ABI of librzk_cuda.so (include/rzk.h): contexts, scene upload
// and LBVH build, and the batched Aggregate / VPL generator / gather entry points.
#include "rzk_internal.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace rzk {

static thread_local char g_last_error[512] = "";

void set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line) {
    snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%s:%d)", cudaGetErrorString(e), what,
             file, line);
}

rzk_status launch_occluded(const DevScene &s, const float *p, const float *q, int n, uint8_t *out,
                           cudaStream_t st);
rzk_status launch_ray_query(const DevScene &s, const int *perm, const rzk_ray *rays, int n, int closest,
                            rzk_ray_hit *out, cudaStream_t st);
rzk_status launch_closest(const DevScene &s, const float *o, const float *d, int n, float *t,
                          rzk_receiver *recv, cudaStream_t st);
rzk_status launch_primary(const DevScene &s, const rzk_camera &cam, rzk_receiver *out, cudaStream_t st);
rzk_status launch_gather(rzk_context *ctx, const DevScene &s, const float *box, const rzk_receiver *recv,
                         int n_recv, int img_w, const rzk_vpl *vpls, int n_vpl, int mode, float tau,
                         float scale, float *out, int variant, int n_chunks, cudaStream_t st);
int gather_variant_count();
rzk_status launch_mean(rzk_context *ctx, const DevScene &s, const rzk_receiver *recv, int n_recv,
                       const rzk_vpl *vpls, int n_vpl, uint32_t seed, int n_pairs, double *h_mean,
                       cudaStream_t st);
rzk_status setup_lights(rzk_scene *s, const std::vector<int> &first_tri, const std::vector<int> &n_tris,
                        const std::vector<int> &kind, const std::vector<int> &flags,
                        const std::vector<float> &emit, cudaStream_t st);
rzk_status launch_vplgen(rzk_scene *sc, uint32_t seed, int n_particles, int max_bounce, rzk_vpl *out,
                         int cap, int *d_count, cudaStream_t st);

}  // namespace rzk

using namespace rzk;


static inline cudaStream_t as_stream(void *s) { return (cudaStream_t)s; }
static inline bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

extern "C" {

const char *rzk_status_string(rzk_status s) {
    switch (s) {
        case RZK_OK: return "ok";
        case RZK_ERR_INVALID: return "invalid argument";
        case RZK_ERR_CUDA: return g_last_error[0] ? g_last_error : "CUDA error";
        case RZK_ERR_NOMEM: return "device allocation failed";
        case RZK_ERR_TIMEOUT: return "bounded device wait timed out";
        case RZK_ERR_STACK: return "traversal stack overflow";
        case RZK_ERR_CAPACITY: return "buffer capacity exceeded";
        case RZK_ERR_UNSUPPORTED: return "unsupported";
        case RZK_ERR_BUSY: return "admission refused: not enough free device memory";
    }
    return "unknown status";
}

rzk_status rzk_context_create(int device, rzk_context **out) {
    if (!out) return RZK_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    RZK_CUDA_TRY(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return RZK_ERR_INVALID;
    RZK_CUDA_TRY(cudaSetDevice(device));
    rzk_context *c = new rzk_context();
    c->device = device;
    // one 16-byte allocation: the error word, then (8-byte aligned) the ray counter
    cudaError_t e = cudaMalloc((void **)&c->d_err, 16);
    if (e == cudaSuccess) e = cudaMemset(c->d_err, 0, 16);
    c->d_rays = (unsigned long long *)((char *)c->d_err + 8);
    if (e != cudaSuccess) {
        set_last_cuda_error(e, "context", __FILE__, __LINE__);
        delete c;
        return RZK_ERR_CUDA;
    }
    *out = c;
    return RZK_OK;
}

rzk_status rzk_context_destroy(rzk_context *c) {
    if (!c) return RZK_ERR_INVALID;
    cudaSetDevice(c->device);
    if (c->d_err) cudaFree(c->d_err);
    if (c->d_partial) cudaFree(c->d_partial);
    if (c->d_stage) cudaFree(c->d_stage);
    if (c->d_work) cudaFree(c->d_work);
    if (c->d_order) cudaFree(c->d_order);
    delete c;
    return RZK_OK;
}

rzk_status rzk_context_check(rzk_context *c, void *stream) {
    if (!c) return RZK_ERR_INVALID;
    uint32_t w = 0;
    RZK_CUDA_TRY(cudaMemcpyAsync(&w, c->d_err, sizeof(w), cudaMemcpyDeviceToHost, as_stream(stream)));
    RZK_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));
    RZK_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(uint32_t), as_stream(stream)));
    if (w & ERR_TIMEOUT) return RZK_ERR_TIMEOUT;
    if (w & ERR_STACK) return RZK_ERR_STACK;
    if (w) return RZK_ERR_CUDA;
    return RZK_OK;
}

rzk_status rzk_debug_ring_wait(rzk_context *c, int timeout_ms, int *h_acquired, void *stream) {
    if (!c || !h_acquired || timeout_ms < 1 || timeout_ms > 4000) return RZK_ERR_INVALID;
    int dev = 0;
    RZK_CUDA_TRY(cudaGetDevice(&dev));
    if (dev != c->device) return RZK_ERR_INVALID;   // the context's buffers live on its device
    return launch_ring_wait_probe(c, timeout_ms, h_acquired, as_stream(stream));
}

rzk_status rzk_context_rays(rzk_context *c, uint64_t *h_rays, int reset, void *stream) {
    if (!c || !h_rays) return RZK_ERR_INVALID;
    unsigned long long n = 0;
    RZK_CUDA_TRY(cudaMemcpyAsync(&n, c->d_rays, sizeof(n), cudaMemcpyDeviceToHost, as_stream(stream)));
    RZK_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));
    if (reset) RZK_CUDA_TRY(cudaMemsetAsync(c->d_rays, 0, sizeof(n), as_stream(stream)));
    *h_rays = (uint64_t)n;
    return RZK_OK;
}

static void free_scene(rzk_scene *s) {
    void *ptrs[] = {s->d_v, s->d_tp, s->d_tri_surf, s->d_tri_n, s->d_tri_u, s->d_tri_area,
                    s->d_bmin, s->d_bmax, s->d_codes, s->d_sorted_codes, s->d_perm, s->d_start,
                    s->d_end, s->d_left, s->d_right, s->d_level, s->d_nbmin, s->d_nbmax,
                    s->d_nodes, s->d_tri_isect, s->d_tri_shade, s->d_surf, s->d_mats,
                    s->d_lights, s->d_light_pdf, s->d_light_cdf, s->d_wide, s->d_trav};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    delete s;
}

rzk_status rzk_scene_create(rzk_context *ctx, const rzk_scene_desc *d, void *stream, rzk_scene **out) {
    if (!ctx || !d || !out || d->n_prims < 0 || d->n_mats < 0) return RZK_ERR_INVALID;
    if (d->n_prims > 0 && (!d->prim_kind || !d->prim_v || !d->prim_mat)) return RZK_ERR_INVALID;
    if (d->n_mats > 0 && !d->mats) return RZK_ERR_INVALID;
    *out = nullptr;
    cudaStream_t st = as_stream(stream);
    RZK_CUDA_TRY(cudaSetDevice(ctx->device));
    // Flatten exactly as AggregateBvh::build collects triangles (aggregate_bvh.cc:58-76):
    // primitive order; a quad is t0 = (p0,p1,p2), t1 = (p0,p2,p3) with the quad's tangent
    // reference p1 (quad.cc:5-28).
    std::vector<float> v, tp;
    std::vector<int> tri_surf;
    std::vector<int4> surf(d->n_prims > 0 ? d->n_prims : 1);
    std::vector<int> l_first, l_n, l_kind, l_flags;
    std::vector<float> l_emit;
    for (int i = 0; i < d->n_prims; ++i) {
        const float *pv = d->prim_v + 12 * (size_t)i;
        int kind = d->prim_kind[i];
        int mat = d->prim_mat[i];
        int flags = d->prim_flags ? d->prim_flags[i] : 0;
        if (kind != RZK_PRIM_TRIANGLE && kind != RZK_PRIM_QUAD) return RZK_ERR_INVALID;
        if (mat >= d->n_mats) return RZK_ERR_INVALID;
        int first = (int)tri_surf.size();
        auto push = [&](int a, int b, int c) {
            for (int k : {a, b, c}) for (int x = 0; x < 3; ++x) v.push_back(pv[3 * k + x]);
            for (int x = 0; x < 3; ++x) tp.push_back(pv[3 * 1 + x]);
            tri_surf.push_back(i);
        };
        push(0, 1, 2);
        if (kind == RZK_PRIM_QUAD) push(0, 2, 3);
        int light = -1;
        if (mat < 0) {
            if (!d->prim_emit) return RZK_ERR_INVALID;
            light = (int)l_first.size();
            l_first.push_back(first);
            l_n.push_back(kind == RZK_PRIM_QUAD ? 2 : 1);
            l_kind.push_back(kind);
            l_flags.push_back(flags);
            for (int x = 0; x < 3; ++x) l_emit.push_back(d->prim_emit[3 * (size_t)i + x]);
        }
        surf[i] = make_int4(mat < 0 ? -1 : mat, flags, light, 0);
    }
    for (int i = 0; i < d->n_mats; ++i) {
        int t = d->mats[i].type;
        if (t != RZK_BSDF_LAMBERTIAN && t != RZK_BSDF_PHONG && t != RZK_BSDF_WARD) return RZK_ERR_INVALID;
    }
    rzk_scene *s = new rzk_scene();
    s->ctx = ctx;
    s->n_tris = (int)tri_surf.size();
    s->n_surfs = d->n_prims;
    s->n_mats = d->n_mats;
    s->tmin = d->tmin > 0.0f ? d->tmin : 1e-3f;
    s->light_surf = l_first;
    auto fail = [&](rzk_status e) { free_scene(s); return e; };
    auto up = [&](void **dst, const void *src, size_t bytes) -> rzk_status {
        cudaError_t e = cudaMalloc(dst, bytes > 0 ? bytes : 16);
        if (e != cudaSuccess) { set_last_cuda_error(e, "scene alloc", __FILE__, __LINE__); return RZK_ERR_NOMEM; }
        s->device_bytes += bytes;
        if (bytes > 0) {
            e = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) { set_last_cuda_error(e, "scene upload", __FILE__, __LINE__); return RZK_ERR_CUDA; }
        }
        return RZK_OK;
    };
    rzk_status e;
    if ((e = up((void **)&s->d_v, v.data(), sizeof(float) * v.size())) != RZK_OK) return fail(e);
    if ((e = up((void **)&s->d_tp, tp.data(), sizeof(float) * tp.size())) != RZK_OK) return fail(e);
    if ((e = up((void **)&s->d_tri_surf, tri_surf.data(), sizeof(int) * tri_surf.size())) != RZK_OK) return fail(e);
    if ((e = up((void **)&s->d_surf, surf.data(), sizeof(int4) * surf.size())) != RZK_OK) return fail(e);
    if ((e = up((void **)&s->d_mats, d->mats, sizeof(rzk_material) * d->n_mats)) != RZK_OK) return fail(e);
    if ((e = bvh_build(s, st)) != RZK_OK) return fail(e);
    if ((e = setup_lights(s, l_first, l_n, l_kind, l_flags, l_emit, st)) != RZK_OK) return fail(e);
    cudaError_t ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) { set_last_cuda_error(ce, "scene build", __FILE__, __LINE__); return fail(RZK_ERR_CUDA); }
    *out = s;
    return RZK_OK;
}

rzk_status rzk_scene_destroy(rzk_scene *s) {
    if (!s) return RZK_ERR_INVALID;
    free_scene(s);
    return RZK_OK;
}

rzk_status rzk_scene_info(const rzk_scene *s, int *n_tris, int *n_nodes, int *n_levels, size_t *bytes) {
    if (!s) return RZK_ERR_INVALID;
    if (n_tris) *n_tris = s->n_tris;
    if (n_nodes) *n_nodes = s->n_nodes;
    if (n_levels) *n_levels = s->n_levels;
    if (bytes) *bytes = s->device_bytes;
    return RZK_OK;
}

rzk_status rzk_scene_bounding_box(const rzk_scene *s, float *box) {
    if (!s || !box) return RZK_ERR_INVALID;
    for (int i = 0; i < 6; ++i) box[i] = s->box[i];
    return RZK_OK;
}

rzk_status rzk_scene_rebuild(rzk_scene *s, void *stream) {
    if (!s) return RZK_ERR_INVALID;
    return bvh_build(s, as_stream(stream));
}

rzk_status rzk_bvh_dump(rzk_scene *s, uint32_t *h_codes, int32_t *h_perm, rzk_bvh_node *h_nodes,
                        int cap_nodes, void *stream) {
    if (!s) return RZK_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    const int n = s->n_tris, nn = s->n_nodes;
    if (h_nodes && cap_nodes < nn) return RZK_ERR_CAPACITY;
    if (h_codes && n) RZK_CUDA_TRY(cudaMemcpyAsync(h_codes, s->d_sorted_codes, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
    if (h_perm && n) RZK_CUDA_TRY(cudaMemcpyAsync(h_perm, s->d_perm, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
    if (h_nodes && nn) {
        std::vector<int> a(nn), b(nn), l(nn), r(nn), lv(nn);
        std::vector<float> mn(3 * (size_t)nn), mx(3 * (size_t)nn);
        RZK_CUDA_TRY(cudaMemcpyAsync(a.data(), s->d_start, 4 * (size_t)nn, cudaMemcpyDeviceToHost, st));
        RZK_CUDA_TRY(cudaMemcpyAsync(b.data(), s->d_end, 4 * (size_t)nn, cudaMemcpyDeviceToHost, st));
        RZK_CUDA_TRY(cudaMemcpyAsync(l.data(), s->d_left, 4 * (size_t)nn, cudaMemcpyDeviceToHost, st));
        RZK_CUDA_TRY(cudaMemcpyAsync(r.data(), s->d_right, 4 * (size_t)nn, cudaMemcpyDeviceToHost, st));
        RZK_CUDA_TRY(cudaMemcpyAsync(lv.data(), s->d_level, 4 * (size_t)nn, cudaMemcpyDeviceToHost, st));
        RZK_CUDA_TRY(cudaMemcpyAsync(mn.data(), s->d_nbmin, 12 * (size_t)nn, cudaMemcpyDeviceToHost, st));
        RZK_CUDA_TRY(cudaMemcpyAsync(mx.data(), s->d_nbmax, 12 * (size_t)nn, cudaMemcpyDeviceToHost, st));
        RZK_CUDA_TRY(cudaStreamSynchronize(st));
        for (int i = 0; i < nn; ++i) {
            rzk_bvh_node &o = h_nodes[i];
            for (int k = 0; k < 3; ++k) { o.bmin[k] = mn[3 * i + k]; o.bmax[k] = mx[3 * i + k]; }
            o.start = a[i]; o.end = b[i]; o.left = l[i]; o.right = r[i]; o.level = lv[i]; o.pad = 0;
        }
    }
    RZK_CUDA_TRY(cudaStreamSynchronize(st));
    return RZK_OK;
}

rzk_status rzk_morton_codes(rzk_scene *s, uint32_t *h_codes, void *stream) {
    if (!s || !h_codes) return RZK_ERR_INVALID;
    if (s->n_tris) RZK_CUDA_TRY(cudaMemcpyAsync(h_codes, s->d_codes, 4 * (size_t)s->n_tris, cudaMemcpyDeviceToHost, as_stream(stream)));
    RZK_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));
    return RZK_OK;
}

rzk_status rzk_occluded_batch(rzk_scene *s, const float *d_p, const float *d_q, int n, uint8_t *d_out,
                              void *stream) {
    if (!s || n < 0 || (n > 0 && (!d_p || !d_q || !d_out))) return RZK_ERR_INVALID;
    return launch_occluded(s->dev(), d_p, d_q, n, d_out, as_stream(stream));
}

rzk_status rzk_closest_batch(rzk_scene *s, const float *d_o, const float *d_d, int n, float *d_t,
                             rzk_receiver *d_recv, void *stream) {
    if (!s || n < 0 || (n > 0 && (!d_o || !d_d))) return RZK_ERR_INVALID;
    if (d_recv && !aligned16(d_recv)) return RZK_ERR_INVALID;
    return launch_closest(s->dev(), d_o, d_d, n, d_t, d_recv, as_stream(stream));
}

rzk_status rzk_ray_query_batch(rzk_scene *s, const rzk_ray *d_rays, int n, int closest, rzk_ray_hit *d_out,
                               void *stream) {
    if (!s || n < 0 || (closest != 0 && closest != 1) || (n > 0 && (!d_rays || !d_out))) return RZK_ERR_INVALID;
    if (n > 0 && (!aligned16(d_rays) || !aligned16(d_out))) return RZK_ERR_INVALID;
    return launch_ray_query(s->dev(), s->d_perm, d_rays, n, closest, d_out, as_stream(stream));
}

rzk_status rzk_primary(rzk_scene *s, const rzk_camera *cam, rzk_receiver *d_out, void *stream) {
    if (!s || !cam || !d_out || cam->width < 0 || cam->height < 0 || !aligned16(d_out)) return RZK_ERR_INVALID;
    return launch_primary(s->dev(), *cam, d_out, as_stream(stream));
}

rzk_status rzk_camera_setup(const float eye[3], const float lookat[3], const float up[3], float fov_deg,
                            int width, int height, float film_w, float film_h, rzk_camera *o) {
    const float DEGREE_TO_RADIAN = A_PI / 180.0f;
    // Camera::focal_length_from_fov (camera.h:228-230)
    float focal = film_h / (2.0f * tanf(fov_deg / 2 * DEGREE_TO_RADIAN));
    return rzk_camera_setup_focal(eye, lookat, up, focal, width, height, film_w, film_h, o);
}

rzk_status rzk_camera_setup_focal(const float eye[3], const float lookat[3], const float up[3], float focal,
                                  int width, int height, float film_w, float film_h, rzk_camera *o) {
    if (!eye || !lookat || !up || !o || width <= 0 || height <= 0) return RZK_ERR_INVALID;
    memset(o, 0, sizeof(*o));
    V3 e = ld3(eye), l = ld3(lookat), u = ld3(up);
    // Onb::init_from_nv(eye - lookat, up) (camera.cc:25, onb.cc:117-127)
    V3 nn = sub(e, l);
    V3 c = unit(cross(u, nn));
    Onb onb;
    if (isnan3(c)) {
        onb = onb_from_n(nn);
    } else {
        onb.n = unit(nn);
        onb.u = c;
        onb.v = cross(onb.n, onb.u);
    }
    st3(o->eye, e); st3(o->u, onb.u); st3(o->v, onb.v); st3(o->n, onb.n);
    o->focal = focal;
    float W = (float)width, H = (float)height;
    float inv2 = 1.0f / 2.0f;   // Size2::operator/(Float) (size.h:26-29)
    o->cop[0] = W * inv2;
    o->cop[1] = H * inv2;
    o->scale[0] = W / film_w;
    o->scale[1] = H / film_h;
    o->width = width;
    o->height = height;
    return RZK_OK;
}

rzk_status rzk_vpl_generate(rzk_scene *s, uint32_t seed, int n_particles, int max_bounce, rzk_vpl *d_out,
                            int cap, int *d_count, void *stream) {
    if (!s || n_particles < 0 || cap < 0 || (cap > 0 && !d_out) || !aligned16(d_out)) return RZK_ERR_INVALID;
    return launch_vplgen(s, seed, n_particles, max_bounce, d_out, cap, d_count, as_stream(stream));
}

static rzk_status check_gather_args(rzk_context *ctx, rzk_scene *s, const rzk_receiver *recv, int n_recv,
                                    const rzk_vpl *vpls, int n_vpl, int mode) {
    if (!ctx || !s || n_recv < 0 || n_vpl < 0) return RZK_ERR_INVALID;
    if (n_recv > 0 && (!recv || !aligned16(recv))) return RZK_ERR_INVALID;
    if (n_vpl > 0 && (!vpls || !aligned16(vpls))) return RZK_ERR_INVALID;
    if (mode < RZK_CLAMP_NONE || mode > RZK_CLAMP_RADIANCE) return RZK_ERR_INVALID;
    return RZK_OK;
}

int rzk_gather_variants(void) { return gather_variant_count(); }

rzk_status rzk_gather_cfg(rzk_context *ctx, rzk_scene *s, const rzk_receiver *d_recv, int n_recv,
                          int image_width, const rzk_vpl *d_vpls, int n_vpl, int clamp_mode, float tau,
                          float scale, float *d_rgb, int variant, int n_chunks, void *stream) {
    RZK_TRY(check_gather_args(ctx, s, d_recv, n_recv, d_vpls, n_vpl, clamp_mode));
    if ((n_recv > 0 && !d_rgb) || image_width < 0) return RZK_ERR_INVALID;
    return launch_gather(ctx, s->dev(), s->box, d_recv, n_recv, image_width, d_vpls, n_vpl, clamp_mode, tau,
                         scale, d_rgb, variant, n_chunks, as_stream(stream));
}

rzk_status rzk_gather(rzk_context *ctx, rzk_scene *s, const rzk_receiver *d_recv, int n_recv,
                      const rzk_vpl *d_vpls, int n_vpl, int clamp_mode, float tau, float scale,
                      float *d_rgb, void *stream) {
    return rzk_gather_cfg(ctx, s, d_recv, n_recv, 0, d_vpls, n_vpl, clamp_mode, tau, scale, d_rgb, 0, 0,
                          stream);
}

rzk_status rzk_gather_host(rzk_context *ctx, rzk_scene *s, const rzk_receiver *h_recv, int n_recv,
                           int image_width, const rzk_vpl *h_vpls, int n_vpl, int clamp_mode, float tau,
                           float scale, float *h_rgb, void *stream) {
    if (image_width < 0) return RZK_ERR_INVALID;
    RZK_TRY(check_gather_args(ctx, s, h_recv, n_recv, h_vpls, n_vpl, clamp_mode));
    if (n_recv > 0 && !h_rgb) return RZK_ERR_INVALID;
    cudaStream_t st = as_stream(stream);
    size_t rb = sizeof(rzk_receiver) * (size_t)n_recv, vb = sizeof(rzk_vpl) * (size_t)n_vpl,
           ob = sizeof(float) * 3 * (size_t)n_recv;
    size_t need = rb + vb + ob + 512;
    if (need > ctx->stage_bytes) {
        if (ctx->d_stage) cudaFree(ctx->d_stage);
        ctx->d_stage = nullptr;
        ctx->stage_bytes = 0;
        RZK_CUDA_TRY(cudaMalloc(&ctx->d_stage, need));
        ctx->stage_bytes = need;
    }
    char *base = (char *)ctx->d_stage;
    rzk_receiver *d_recv = (rzk_receiver *)base;
    rzk_vpl *d_vpls = (rzk_vpl *)(base + ((rb + 255) & ~(size_t)255));
    float *d_out = (float *)((char *)d_vpls + ((vb + 255) & ~(size_t)255));
    if (rb) RZK_CUDA_TRY(cudaMemcpyAsync(d_recv, h_recv, rb, cudaMemcpyHostToDevice, st));
    if (vb) RZK_CUDA_TRY(cudaMemcpyAsync(d_vpls, h_vpls, vb, cudaMemcpyHostToDevice, st));
    RZK_TRY(launch_gather(ctx, s->dev(), s->box, d_recv, n_recv, image_width, d_vpls, n_vpl, clamp_mode, tau,
                          scale, d_out, 0, 0, st));
    if (ob) RZK_CUDA_TRY(cudaMemcpyAsync(h_rgb, d_out, ob, cudaMemcpyDeviceToHost, st));
    RZK_CUDA_TRY(cudaStreamSynchronize(st));
    return RZK_OK;
}

rzk_status rzk_gather_matrix(rzk_scene *s, const rzk_receiver *d_recv, int n_recv, const rzk_vpl *d_vpls,
                             int n_vpl, int clamp_mode, float tau, float *d_matrix, uint8_t *d_vis,
                             void *stream) {
    if (!s || n_recv < 0 || n_vpl < 0 || (n_recv && n_vpl && !d_matrix)) return RZK_ERR_INVALID;
    if (clamp_mode < RZK_CLAMP_NONE || clamp_mode > RZK_CLAMP_RADIANCE) return RZK_ERR_INVALID;
    return launch_matrix(s->dev(), d_recv, n_recv, d_vpls, n_vpl, clamp_mode, tau, d_matrix, d_vis, 0,
                         as_stream(stream));
}

rzk_status rzk_incident_matrix(rzk_scene *s, const rzk_receiver *d_recv, int n_recv, const rzk_vpl *d_vpls,
                               int n_vpl, int clamp_mode, float tau, float *d_matrix, void *stream) {
    if (!s || n_recv < 0 || n_vpl < 0 || (n_recv && n_vpl && !d_matrix)) return RZK_ERR_INVALID;
    if (clamp_mode < RZK_CLAMP_NONE || clamp_mode > RZK_CLAMP_RADIANCE) return RZK_ERR_INVALID;
    return launch_matrix(s->dev(), d_recv, n_recv, d_vpls, n_vpl, clamp_mode, tau, d_matrix, nullptr, 1,
                         as_stream(stream));
}

rzk_status rzk_mean_contribution(rzk_context *ctx, rzk_scene *s, const rzk_receiver *d_recv, int n_recv,
                                 const rzk_vpl *d_vpls, int n_vpl, uint32_t seed, int n_pairs,
                                 double *h_mean, void *stream) {
    if (!ctx || !s || !h_mean || n_pairs < 0) return RZK_ERR_INVALID;
    return launch_mean(ctx, s->dev(), d_recv, n_recv, d_vpls, n_vpl, seed, n_pairs, h_mean, as_stream(stream));
}

}  // extern "C"
