// rzk_internal.cuh - library-internal types shared by the .cu files of librzk_cuda.so.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

#include "../../include/rzk.h"
#include "rzk_math.cuh"

#define RZK_CUDA_TRY(expr)                                   \
    do {                                                     \
        cudaError_t _e = (expr);                             \
        if (_e != cudaSuccess) {                             \
            rzk::set_last_cuda_error(_e, #expr, __FILE__, __LINE__); \
            return _e == cudaErrorMemoryAllocation ? RZK_ERR_NOMEM : RZK_ERR_CUDA; \
        }                                                    \
    } while (0)
#define RZK_TRY(expr) do { rzk_status _s = (expr); if (_s != RZK_OK) return _s; } while (0)

namespace rzk {

void set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line);

// Device error word bits (written by kernels, read by rzk_context_check).
enum : uint32_t { ERR_TIMEOUT = 1u, ERR_STACK = 2u, ERR_BOUNDS = 4u };

// Code of an unused entry of a 4-wide traversal node.
constexpr int kWideEmpty = 0x7fffffff;

// Area light as the VPL generator samples it (area_light.cc:27-46, quad.cc:73-87).
struct DevLight {
    float4 p0[2], p1[2], p2[2];   // the (one or two) triangles of the light's shape
    float4 n[2];                  // their facet normals; .w = area
    float4 basis_n, basis_u;      // Surface::get_basis: larger triangle's n and tangent
    float4 emit;                  // radiance; .w unused
    float t0_ratio;
    int kind, flags, n_tris;
};

// Everything a kernel needs to trace and shade in one scene (passed by value).
struct DevScene {
    const float4 *nodes;      // 2 x float4 per slot, slot = BFS node index + 1
    const float4 *tri_isect;  // 3 x float4 per sorted triangle (see tri_hit)
    const float4 *tri_shade;  // 2 x float4 per sorted triangle: {n, surf}, {u, -}
    const float4 *wide;       // 8 x float4 per 4-wide traversal node (see rzk_bvh.cu K6)
    const float4 *trav;       // any-hit tree, same packing as nodes (rzk_sah.cu; = nodes without it)
    const int4 *surf;         // per surface {mat, flags, light, -}
    const rzk_material *mats;
    const DevLight *lights;
    const float *light_pdf;
    const float *light_cdf;
    int n_tris, n_nodes, n_mats, n_lights;
    float tmin;
    uint32_t *err;            // device error word (context-owned)
    unsigned long long *rays; // shadow rays traced by the gather kernels (context-owned counter)
};

struct Scene;

struct BatchPlan;   // rzk_batch.cu: a batch of gathers split into launch tables

}  // namespace rzk

struct rzk_context {
    int device = 0;
    uint32_t *d_err = nullptr;             // error word (the first 8 bytes of a 16-byte allocation)
    unsigned long long *d_rays = nullptr;  // shadow rays traced by the gather kernels (its last 8)
    // reusable gather scratch: per-(VPL chunk, receiver) partial sums
    float *d_partial = nullptr;
    size_t partial_bytes = 0;
    // staging for rzk_gather_host
    void *d_stage = nullptr;
    size_t stage_bytes = 0;
    double *d_mean = nullptr;
    // work counter of the persistent gather and its resident grid size per variant
    int *d_work = nullptr;
    // spatially ordered VPL copy of a chunked gather, its sort keys and sort scratch
    void *d_order = nullptr;
    size_t order_bytes = 0;
    int persistent_grid[16] = {0};
};

struct rzk_scene {
    rzk_context *ctx = nullptr;
    int n_tris = 0, n_nodes = 0, n_levels = 0, n_surfs = 0, n_mats = 0, n_lights = 0;
    float tmin = 1e-3f;
    float box[6] = {0, 0, 0, 0, 0, 0};   // Aggregate::box (min xyz, max xyz), incl. the origin
    // original (flattened, input-order) triangles
    float *d_v = nullptr;        // [n][9]
    float *d_tp = nullptr;       // [n][3] tangent reference vertex
    int *d_tri_surf = nullptr;   // [n]
    float *d_tri_n = nullptr;    // [n][3] facet normal
    float *d_tri_u = nullptr;    // [n][3] tangent
    float *d_tri_area = nullptr; // [n]
    float *d_bmin = nullptr, *d_bmax = nullptr;   // [n][3] triangle boxes
    // build products
    uint32_t *d_codes = nullptr, *d_sorted_codes = nullptr;
    int *d_perm = nullptr;
    int *d_start = nullptr, *d_end = nullptr, *d_left = nullptr, *d_right = nullptr,
        *d_level = nullptr;
    float *d_nbmin = nullptr, *d_nbmax = nullptr;  // [nodes][3]
    std::vector<int> level_first, level_last;
    // packed traversal layout
    float4 *d_nodes = nullptr, *d_tri_isect = nullptr, *d_tri_shade = nullptr;
    float4 *d_wide = nullptr;
    int n_wide = 0, n_wide_cap = 0;
    float4 *d_trav = nullptr;    // SAH any-hit tree (rzk_sah.cu)
    int trav_depth = 0;
    size_t trav_bytes = 0;
    bool build_trav = true;
    int4 *d_surf = nullptr;
    rzk_material *d_mats = nullptr;
    rzk::DevLight *d_lights = nullptr;
    float *d_light_pdf = nullptr, *d_light_cdf = nullptr;
    std::vector<int> light_surf;   // host: surface index of each light
    size_t device_bytes = 0;
    // scratch for the build (freed after)
    rzk::DevScene dev() const {
        rzk::DevScene s;
        s.nodes = d_nodes; s.tri_isect = d_tri_isect; s.tri_shade = d_tri_shade; s.wide = d_wide;
        s.trav = d_trav ? d_trav : d_nodes;
        s.surf = d_surf; s.mats = d_mats; s.lights = d_lights; s.light_pdf = d_light_pdf;
        s.light_cdf = d_light_cdf; s.n_tris = n_tris; s.n_nodes = n_nodes; s.n_mats = n_mats;
        s.n_lights = n_lights; s.tmin = tmin; s.err = ctx ? ctx->d_err : nullptr;
        s.rays = ctx ? ctx->d_rays : nullptr;
        return s;
    }
};

namespace rzk {
// rzk_bvh.cu
rzk_status bvh_build(rzk_scene *s, cudaStream_t st);
// rzk_sah.cu
rzk_status build_sah_tree(rzk_scene *s, cudaStream_t st);
// utilities (rzk_bvh.cu)
rzk_status exclusive_scan_i32(const int *d_in, int *d_out, int n, int *d_total, void *d_tmp,
                              size_t tmp_bytes, cudaStream_t st);
size_t exclusive_scan_tmp_bytes(int n);
size_t radix_sort_scratch_bytes(int n);
rzk_status radix_sort_u32(uint32_t *keys, int *vals, int n, int bits, void *scratch, cudaStream_t st);
int exclusive_scan_launches(int n, bool total);   // kernels one exclusive_scan_i32 call launches
int radix_sort_launches(int n, int bits);         // kernels one radix_sort_u32 call launches

// rzk_gather.cu: spatial VPL order of chunked gathers.  Each segment is one gather's VPL
// set; ordering writes every segment's VPLs, stably sorted by the Hilbert-curve index of
// their positions' cells on a 256^3 grid over that gather's scene box, to
// out[begin, begin + n).
constexpr int kOrderSegs = 128;
struct OrderSeg {
    const rzk_vpl *src;
    int begin, n;
    float lo[3], k[3];
};
struct OrderTable {
    OrderSeg seg[kOrderSegs];
    int n_segs, total;
};
void order_table_init(OrderTable &t);
// appends a segment (no device work); false when the table is full
bool order_table_add(OrderTable &t, const rzk_vpl *src, int n, const float *box);
size_t order_scratch_bytes(int total);
int order_launches(const OrderTable &t);
rzk_status order_vpls(const OrderTable &t, void *scratch, rzk_vpl *out, cudaStream_t st);
// rzk_gather.cu: every (receiver, VPL) pair into a column-major [n_vpl][n_recv][3] matrix;
// kind 0 radiance, 1 incident radiance, 2 visible x incident radiance (+ visibility)
rzk_status launch_matrix(const DevScene &s, const rzk_receiver *recv, int n_recv, const rzk_vpl *vpls,
                         int n_vpl, int mode, float tau, float *mat, uint8_t *vis, int kind,
                         cudaStream_t st);
// rzk_gather.cu: kernels one rzk_gather_cfg call launches
int gather_launches(int n_recv, int n_vpl, int n_chunks);
// Chunk ring of the persistent gather on fixed scratch (rzk_gather.cu, used by
// rzk_gather_noalloc): the per-chunk sums of at most `slots` warp tiles at a time.  Tile t writes its chunks to slot t % slots once the slot
// has finished t / slots tiles (`round`); the warp that writes a tile's last chunk (`done`)
// adds the chunks in chunk order, writes the tile's pixels and frees the slot.  The
// counters start at zero (one memset of ring_counter_bytes); the sums need no clearing.
struct ChunkRing {
    int *done;     // [slots] chunks of the slot's current tile written
    int *round;    // [slots] tiles the slot has finished
    float *sums;   // [slots][n_chunks][32 lanes][3]
    int slots;
};
constexpr int kRingSlots = 8192;   // most slots a ring is given (96 MiB at 32 chunks)
size_t ring_counter_bytes(int slots);
size_t ring_bytes(int slots, int n_chunks);
int ring_slots_fitting(size_t bytes, int n_chunks);   // slots whose ring fits in `bytes`
ChunkRing ring_at(void *base, int slots);
// the ring's slot wait on a slot nothing frees, limited to timeout_ms (rzk_debug_ring_wait)
rzk_status launch_ring_wait_probe(rzk_context *ctx, int timeout_ms, int *h_acquired, cudaStream_t st);
// rzk_gather.cu: make the context's scratch (d_partial) at least `bytes` long
rzk_status ensure_scratch(rzk_context *ctx, size_t bytes);
// rzk_batch.cu: plan a batch (validates jobs; no device work), then launch it on a partial
// buffer of batch_plan_partial_floats floats, an ordering buffer of batch_plan_order_bytes
// bytes (16-byte aligned; null when that is 0) and batch_plan_tables work counters;
// grid 0 = the variant's resident grid.
rzk_status batch_plan_create(const rzk_gather_job *jobs, int n_jobs, int chunk_len, int tile_width,
                             BatchPlan **out);
int batch_variant_tile_width(int variant);   // warp tile width (pixels) of a batch variant
void batch_plan_destroy(BatchPlan *p);
size_t batch_plan_partial_floats(const BatchPlan *p);
size_t batch_plan_order_bytes(const BatchPlan *p);
int batch_plan_tables(const BatchPlan *p);
int batch_plan_launches(const BatchPlan *p);   // kernels one batch_plan_launch launches
rzk_status batch_plan_launch(BatchPlan *p, float *partial, void *order, int *work, int variant, int grid,
                             cudaStream_t st);
}  // namespace rzk
