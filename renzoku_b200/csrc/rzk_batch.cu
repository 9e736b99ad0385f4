// rzk_batch.cu - many independent gathers (different scenes, images, VPL sets, clamps) in
// one persistent launch, and the autotuner that picks its tile configuration.
//
// The batch is described once (rzk_batch_create): tables of up to 128 jobs, each with its
// scene, receivers, VPLs, clamp and output, and one partial-sum buffer for all of them.
// rzk_batch_run then issues one memset of the work counters and, per table, the ordering
// of its chunked jobs' VPLs, the persistent kernel and the chunk reduction - no allocation
// and no host synchronisation, so it can be captured in a CUDA graph and replayed.  Work items are (job, 8 x 4 receiver
// tile, VPL chunk), numbered job-major; every warp takes the next item from one atomic
// counter, so small and large jobs share the SMs without a per-launch tail.  Each job's
// image is bit-identical to rzk_gather_cfg with the same chunk length.
#include "rzk_gather_dev.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

namespace rzk {

struct BatchJob {
    DevScene s;
    const rzk_receiver *recv;
    const rzk_vpl *vpls;
    float *partial;
    float *out;
    long long item_begin;   // first work item of this job
    long long out_begin;    // first output float (3 per receiver) of this job in the batch
    int n_recv, img_w, n_vpl, chunk_len, n_chunks, n_wtiles, mode;
    float tau, scale;
};

// Jobs travel in the launch's parameter block (a __grid_constant__ table): the kernel
// reads each job field from the constant bank where it is used, as the single-instance
// kernel reads its arguments, instead of holding a descriptor in registers.  Larger
// batches are split into several launches of at most kJobsPerLaunch jobs.
constexpr int kJobsPerLaunch = 128;
struct JobTable {
    BatchJob jobs[kJobsPerLaunch];
    int n_jobs;
    int n_items;
    long long n_out;
};
static_assert(sizeof(JobTable) <= 32000, "kernel parameter block limit");

namespace {

__device__ __forceinline__ int find_job(const JobTable &t, long long item, bool by_out) {
    int lo = 0, hi = t.n_jobs - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        long long b = by_out ? t.jobs[mid].out_begin : t.jobs[mid].item_begin;
        if (b <= item) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <int WARPS, int TILE, int MINB, int TW = 8>
__global__ void __launch_bounds__(WARPS * 32, MINB) batch_gather_kernel(const __grid_constant__ JobTable t,
                                                                        int *work) {
    __shared__ __align__(128) rzk_vpl tiles[WARPS][2][TILE];
    __shared__ __align__(8) uint64_t bar[WARPS][2];
    __shared__ int stacks[WARPS][STACK_CAP];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    WarpStage<TILE> ws;
    ws.init(tiles[w], bar[w], stacks[w], lane);
    while (true) {
        int item = 0;
        if (lane == 0) item = atomicAdd(work, 1);
        item = __shfl_sync(kFull, item, 0);
        if (item >= t.n_items) break;
        const int j = find_job(t, item, false);
        const BatchJob &jb = t.jobs[j];
        const int local = item - (int)jb.item_begin;
        const int wt = local / jb.n_chunks;   // tile-major, as gather_persistent_kernel
        const int chunk = local - wt * jb.n_chunks;
        if (!gather_item<TILE, TW>(jb.s, jb.recv, jb.n_recv, jb.img_w, jb.vpls, jb.n_vpl, chunk, wt,
                                   jb.chunk_len, jb.mode, jb.tau, ws, lane, PlaneSink{jb.partial, jb.n_recv, chunk}))
            break;
    }
}

__global__ void batch_reduce_kernel(const __grid_constant__ JobTable t) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.n_out) return;
    const int j = find_job(t, i, true);
    const BatchJob &jb = t.jobs[j];
    const long long k = i - jb.out_begin;
    const long long stride = 3LL * jb.n_recv;
    float acc = __ldcs(jb.partial + k);   // read once: evict-first
    for (int c = 1; c < jb.n_chunks; ++c) acc += __ldcs(jb.partial + (size_t)c * stride + k);
    jb.out[k] = acc * jb.scale;
}

// The tile shapes the autotuner searches: warps per CTA (x 32 receivers, one lane per
// shadow ray: the warp is the packet), VPLs per shared-memory tile, resident CTAs per SM
// (the register cap), and the warp tile's width in pixels (8 x 4, 4 x 8, 16 x 2, 32 x 1).
// The traversal stack stays at the reference's 64 entries (256 bytes of shared memory per
// warp, which never limits residency).
struct BatchVariant {
    int warps, tile, minb, tw;
};
const BatchVariant kBatchVariants[] = {{4, 32, 7, 8}, {4, 32, 6, 8}, {2, 32, 1, 8}, {4, 16, 5, 8},
                                       {4, 32, 5, 4}, {4, 32, 5, 16}, {4, 32, 5, 32}};

template <int WARPS, int TILE, int MINB, int TW = 8>
int batch_grid() {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_gather_kernel<WARPS, TILE, MINB, TW>, WARPS * 32,
                                                  0);
    return std::max(1, sms * std::max(1, per_sm));
}

int grid_for(int variant) {
    switch (variant) {
        case 0: return batch_grid<4, 32, 7>();
        case 1: return batch_grid<4, 32, 6>();
        case 2: return batch_grid<2, 32, 1>();
        case 4: return batch_grid<4, 32, 5, 4>();
        case 5: return batch_grid<4, 32, 5, 16>();
        case 6: return batch_grid<4, 32, 5, 32>();
        default: return batch_grid<4, 16, 5>();
    }
}

}  // namespace

// A batch split into launch tables: consecutive jobs go into one launch until it holds
// kJobsPerLaunch jobs or 2^30 work items.
// Jobs with several VPL chunks gather from a spatially ordered copy of their VPLs, exactly as
// rzk_gather_cfg does: per table one ordering pass writes the copies into the plan's
// ordering buffer (laid out [sorted VPLs of every table | sort scratch]).
struct BatchPlan {
    std::vector<JobTable> tables;
    std::vector<OrderTable> orders;          // per table: the ordered jobs' VPL sets
    std::vector<std::vector<int>> ordered;   // per table: job slot of each order segment
    std::vector<size_t> order_base;          // per table: its first VPL in the sorted copy
    size_t sorted_vpls = 0;
    int max_order_total = 0;
    size_t partial_floats = 0;
    float *bound = nullptr;        // partial buffer the tables point into
    void *order_bound = nullptr;   // ordering buffer the ordered jobs point into
};

static size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }

int batch_variant_tile_width(int variant) {
    return variant >= 0 && variant < (int)(sizeof(kBatchVariants) / sizeof(kBatchVariants[0]))
               ? kBatchVariants[variant].tw : 8;
}

rzk_status batch_plan_create(const rzk_gather_job *jobs, int n_jobs, int chunk_len, int tile_width,
                             BatchPlan **out) {
    if (!jobs || n_jobs <= 0 || !out || chunk_len < 0 || (chunk_len % 128) != 0) return RZK_ERR_INVALID;
    *out = nullptr;
    std::vector<BatchJob> h(n_jobs);
    size_t partial = 0;
    for (int i = 0; i < n_jobs; ++i) {
        const rzk_gather_job &g = jobs[i];
        if (!g.scene || g.n_recv <= 0 || g.n_vpl < 0 || g.image_width < 0 || !g.d_recv || !g.d_rgb ||
            (g.n_vpl > 0 && !g.d_vpls) || ((uintptr_t)g.d_recv & 15u) || ((uintptr_t)g.d_vpls & 15u) ||
            g.clamp_mode < RZK_CLAMP_NONE || g.clamp_mode > RZK_CLAMP_RADIANCE)
            return RZK_ERR_INVALID;
        BatchJob &b = h[i];
        b.s = g.scene->dev();
        b.recv = g.d_recv;
        b.vpls = g.d_vpls;
        b.out = g.d_rgb;
        b.n_recv = g.n_recv;
        b.img_w = g.image_width;
        b.n_vpl = g.n_vpl;
        b.mode = g.clamp_mode;
        b.tau = g.tau;
        b.scale = g.scale;
        const long long wtiles = tile_width == 4    ? warp_tiles<4>(b.n_recv, b.img_w)
                                 : tile_width == 16 ? warp_tiles<16>(b.n_recv, b.img_w)
                                 : tile_width == 32 ? warp_tiles<32>(b.n_recv, b.img_w)
                                                    : warp_tiles<8>(b.n_recv, b.img_w);
        b.n_wtiles = (int)wtiles;
        int cl = chunk_len;
        if (cl == 0) {   // the default of rzk_gather: at most 32 chunks of a multiple of 128 VPLs
            int nc = std::max(1, std::min(32, (b.n_vpl + 127) / 128));
            cl = b.n_vpl > 0 ? (b.n_vpl + nc - 1) / nc : 0;
            cl = (cl + 127) / 128 * 128;
        }
        b.chunk_len = cl;
        b.n_chunks = (b.n_vpl > 0 && cl > 0) ? (b.n_vpl + cl - 1) / cl : 1;
        if (b.n_vpl <= 0) b.chunk_len = 0;
        if ((long long)b.n_wtiles * b.n_chunks >= (1LL << 30)) return RZK_ERR_CAPACITY;
        partial += 3ull * b.n_recv * b.n_chunks;
    }
    BatchPlan *p = new BatchPlan();
    p->partial_floats = partial;
    for (int i = 0; i < n_jobs; ++i) {
        long long items = (long long)h[i].n_wtiles * h[i].n_chunks;
        if (p->tables.empty() || p->tables.back().n_jobs == kJobsPerLaunch ||
            p->tables.back().n_items + items >= (1LL << 30)) {
            p->tables.emplace_back();
            JobTable &t = p->tables.back();
            memset(&t, 0, sizeof(t));
            p->orders.emplace_back();
            order_table_init(p->orders.back());
            p->ordered.emplace_back();
        }
        JobTable &t = p->tables.back();
        BatchJob &b = h[i];
        b.item_begin = t.n_items;
        b.out_begin = t.n_out;
        t.n_items += (int)items;
        t.n_out += 3LL * b.n_recv;
        if (b.n_chunks > 1) {   // kJobsPerLaunch == kOrderSegs: the table has room
            order_table_add(p->orders.back(), b.vpls, b.n_vpl, jobs[i].scene->box);
            p->ordered.back().push_back(t.n_jobs);
        }
        t.jobs[t.n_jobs++] = b;
    }
    for (const OrderTable &o : p->orders) {
        p->order_base.push_back(p->sorted_vpls);
        p->sorted_vpls += (size_t)o.total;
        p->max_order_total = std::max(p->max_order_total, o.total);
    }
    *out = p;
    return RZK_OK;
}

void batch_plan_destroy(BatchPlan *p) { delete p; }
size_t batch_plan_partial_floats(const BatchPlan *p) { return p->partial_floats; }
size_t batch_plan_order_bytes(const BatchPlan *p) {
    if (p->sorted_vpls == 0) return 0;
    return up256(sizeof(rzk_vpl) * p->sorted_vpls) + order_scratch_bytes(p->max_order_total);
}
int batch_plan_tables(const BatchPlan *p) { return (int)p->tables.size(); }
int batch_plan_launches(const BatchPlan *p) {
    int n = 0;
    for (const OrderTable &o : p->orders) n += 2 + order_launches(o);
    return n;
}

rzk_status batch_plan_launch(BatchPlan *p, float *partial, void *order, int *work, int variant, int grid,
                             cudaStream_t st) {
    if (p->sorted_vpls > 0 && (!order || ((uintptr_t)order & 15u))) return RZK_ERR_INVALID;
    rzk_vpl *sorted = (rzk_vpl *)order;
    if (p->bound != partial || p->order_bound != order) {
        size_t off = 0;
        for (JobTable &t : p->tables)
            for (int i = 0; i < t.n_jobs; ++i) {
                t.jobs[i].partial = partial + off;
                off += 3ull * t.jobs[i].n_recv * t.jobs[i].n_chunks;
            }
        for (size_t k = 0; k < p->tables.size(); ++k)
            for (int g = 0; g < p->orders[k].n_segs; ++g)
                p->tables[k].jobs[p->ordered[k][g]].vpls = sorted + p->order_base[k] + p->orders[k].seg[g].begin;
        p->bound = partial;
        p->order_bound = order;
    }
    if (grid <= 0) grid = grid_for(variant);
    void *scratch = p->sorted_vpls > 0 ? (char *)order + up256(sizeof(rzk_vpl) * p->sorted_vpls) : nullptr;
    RZK_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int) * p->tables.size(), st));
    for (size_t k = 0; k < p->tables.size(); ++k) {
        const JobTable &t = p->tables[k];
        int *w = work + k;
        if (p->orders[k].total > 0) RZK_TRY(order_vpls(p->orders[k], scratch, sorted + p->order_base[k], st));
        switch (variant) {
            case 0: batch_gather_kernel<4, 32, 7><<<grid, 128, 0, st>>>(t, w); break;
            case 1: batch_gather_kernel<4, 32, 6><<<grid, 128, 0, st>>>(t, w); break;
            case 2: batch_gather_kernel<2, 32, 1><<<grid, 64, 0, st>>>(t, w); break;
            case 4: batch_gather_kernel<4, 32, 5, 4><<<grid, 128, 0, st>>>(t, w); break;
            case 5: batch_gather_kernel<4, 32, 5, 16><<<grid, 128, 0, st>>>(t, w); break;
            case 6: batch_gather_kernel<4, 32, 5, 32><<<grid, 128, 0, st>>>(t, w); break;
            default: batch_gather_kernel<4, 16, 5><<<grid, 128, 0, st>>>(t, w); break;
        }
        RZK_CUDA_TRY(cudaGetLastError());
        batch_reduce_kernel<<<(unsigned)((t.n_out + 255) / 256), 256, 0, st>>>(t);
        RZK_CUDA_TRY(cudaGetLastError());
    }
    return RZK_OK;
}

}  // namespace rzk

struct rzk_batch {
    rzk_context *ctx = nullptr;
    rzk::BatchPlan *plan = nullptr;
    float *d_partial = nullptr;
    void *d_order = nullptr;             // spatially ordered VPL copies and sort scratch
    int *d_work = nullptr;               // one work counter per table
    int n_jobs = 0, variant = 0, grid = 0;
};

using namespace rzk;

extern "C" {

int rzk_batch_variants(void) { return (int)(sizeof(kBatchVariants) / sizeof(kBatchVariants[0])); }

rzk_status rzk_batch_destroy(rzk_batch *b) {
    if (!b) return RZK_ERR_INVALID;
    if (b->d_partial) cudaFree(b->d_partial);
    if (b->d_order) cudaFree(b->d_order);
    if (b->d_work) cudaFree(b->d_work);
    if (b->plan) batch_plan_destroy(b->plan);
    delete b;
    return RZK_OK;
}

rzk_status rzk_batch_create(rzk_context *ctx, const rzk_gather_job *jobs, int n_jobs, int variant, int chunk_len,
                            rzk_batch **out) {
    if (!ctx || !jobs || n_jobs <= 0 || !out || variant < 0 || variant >= rzk_batch_variants()) return RZK_ERR_INVALID;
    if (chunk_len < 0 || (chunk_len % 128) != 0) return RZK_ERR_INVALID;
    *out = nullptr;
    BatchPlan *plan = nullptr;
    rzk_status r = batch_plan_create(jobs, n_jobs, chunk_len, batch_variant_tile_width(variant), &plan);
    if (r != RZK_OK) return r;
    rzk_batch *bt = new rzk_batch();
    bt->ctx = ctx;
    bt->plan = plan;
    bt->n_jobs = n_jobs;
    bt->variant = variant;
    auto fail = [&](cudaError_t e) {
        set_last_cuda_error(e, "batch", __FILE__, __LINE__);
        rzk_batch_destroy(bt);
        return e == cudaErrorMemoryAllocation ? RZK_ERR_NOMEM : RZK_ERR_CUDA;
    };
    cudaError_t e = cudaMalloc((void **)&bt->d_partial, sizeof(float) * std::max<size_t>(plan->partial_floats, 1));
    if (e != cudaSuccess) return fail(e);
    if ((e = cudaMalloc((void **)&bt->d_work, sizeof(int) * plan->tables.size())) != cudaSuccess) return fail(e);
    const size_t ob = batch_plan_order_bytes(plan);
    if (ob > 0 && (e = cudaMalloc(&bt->d_order, ob)) != cudaSuccess) return fail(e);
    bt->grid = grid_for(variant);
    *out = bt;
    return RZK_OK;
}

rzk_status rzk_batch_run(rzk_batch *b, void *stream) {
    if (!b) return RZK_ERR_INVALID;
    return batch_plan_launch(b->plan, b->d_partial, b->d_order, b->d_work, b->variant, b->grid,
                             (cudaStream_t)stream);
}

rzk_status rzk_batch_variant_info(int variant, int32_t *warps, int32_t *vpl_tile, int32_t *ctas_per_sm,
                                  int32_t *tile_width) {
    if (variant < 0 || variant >= rzk_batch_variants()) return RZK_ERR_INVALID;
    const BatchVariant &v = kBatchVariants[variant];
    if (warps) *warps = v.warps;
    if (vpl_tile) *vpl_tile = v.tile;
    if (ctas_per_sm) *ctas_per_sm = v.minb;
    if (tile_width) *tile_width = v.tw;
    return RZK_OK;
}

rzk_status rzk_batch_autotune(rzk_context *ctx, const rzk_gather_job *jobs, int n_jobs, int max_probe_jobs,
                              int *best_variant, int *best_chunk_len, float *best_ms, float *h_probe_ms,
                              void *stream) {
    if (!ctx || !jobs || n_jobs <= 0 || !best_variant || !best_chunk_len) return RZK_ERR_INVALID;
    // probe on an evenly spaced subset of the jobs (all of them if max_probe_jobs <= 0)
    std::vector<rzk_gather_job> probe;
    int k = (max_probe_jobs <= 0 || max_probe_jobs >= n_jobs) ? n_jobs : max_probe_jobs;
    for (int i = 0; i < k; ++i) probe.push_back(jobs[(long long)i * n_jobs / k]);
    const int chunks[] = {0, 512, 1024, 2048};   // 0 = rzk_gather's per-job default
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t a, b;
    RZK_CUDA_TRY(cudaEventCreate(&a));
    RZK_CUDA_TRY(cudaEventCreate(&b));
    float best = 3.4e38f;
    *best_variant = 0;
    *best_chunk_len = 0;
    rzk_status res = RZK_OK;
    for (int v = 0; v < rzk_batch_variants() && res == RZK_OK; ++v) {
        for (int ci = 0; ci < 4; ++ci) {
            const int c = chunks[ci];
            rzk_batch *bt = nullptr;
            res = rzk_batch_create(ctx, probe.data(), (int)probe.size(), v, c, &bt);
            if (res != RZK_OK) break;
            res = rzk_batch_run(bt, stream);   // warm
            float ms = 3.4e38f;
            for (int rep = 0; rep < 2 && res == RZK_OK; ++rep) {   // best of two timed runs
                float t = 0.0f;
                cudaEventRecord(a, st);
                res = rzk_batch_run(bt, stream);
                cudaEventRecord(b, st);
                cudaEventSynchronize(b);
                cudaEventElapsedTime(&t, a, b);
                ms = std::min(ms, t);
            }
            rzk_batch_destroy(bt);
            if (h_probe_ms) h_probe_ms[v * 4 + ci] = ms;
            if (res == RZK_OK && ms < best) {
                best = ms;
                *best_variant = v;
                *best_chunk_len = c;
            }
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (best_ms) *best_ms = best;
    return res;
}

}  // extern "C"
