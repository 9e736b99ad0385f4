// rzk_mrcs.cu - matrix row-column sampling (MatrixRowColumnSampling, mrcs.cc:16-186; Hasan,
// Pellacini and Bala, "Matrix Row-Column Sampling for the Many-Light Problem", SIGGRAPH 2007).
//
// Set-up (rzk_mrcs_create), in the reference's order and from one random stream
// (seed, 7, 0) consumed in its program order:
//   1. one pixel per block_size x block_size stratum (ImageSampler::sample_stratified,
//      image_sampler.cc:8-23): two draws per stratum, row-major over the strata;
//   2. with more than max_columns VPLs, max_columns columns resampled by average power
//      (mrcs.cc:79-94): one draw each, contribution divided by the column's probability
//      and by max_columns;
//   3. the reduced matrix: a primary hit per sampled pixel (Camera::shoot_ray), then
//      gather_point for every (pixel, column) pair (LightTransportMatrix::fill) - the
//      device matrix kernel;
//   4. ClusterBuilder::cluster_by_sampling on it (device distances, host draws that
//      continue the same stream).
// Gathering (rzk_mrcs_gather, MatrixRowColumnSampling::gather_clusters, mrcs.cc:28-41):
// per receiver, the weighted sum over the clusters' representatives in cluster order - a
// tracing pass of warp-packet visibility ballots, then an in-order summing pass.
#include "rzk_gather_dev.cuh"
#include "rzk_cluster.cuh"
#include "rzk_hostutil.h"

#include <algorithm>
#include <chrono>
#include <vector>

namespace rzk {
namespace {

constexpr int kPixBlock = 128;

// Camera::shoot_ray(y, x) and the closest hit for each sampled pixel (x may lie past the
// image's last column, and y past its last row, where a stratum overhangs the image: the
// reference shoots those rays as well).
__global__ void __launch_bounds__(kPixBlock) pixel_receivers_kernel(DevScene s, rzk_camera cam, const int *px,
                                                                     int n, rzk_receiver *out) {
    __shared__ int stack_mem[STACK_CAP * kPixBlock];
    const int k = blockIdx.x * kPixBlock + threadIdx.x;
    if (k >= n) return;
    Stack<kPixBlock> stk;
    stk.init(stack_mem + threadIdx.x);
    const Ray r = camera_ray(cam, px[2 * k + 1], px[2 * k]);
    float t, b, g;
    rzk_receiver *o = out + k;
    const int slot = closest_hit<kPixBlock>(s, r, s.tmin, RAY_TMAX, stk, &t, &b, &g);
    if (slot < 0) { write_miss(o); return; }
    HitGeo h;
    fill_hit(s, r, slot, t, b, g, h);
    write_receiver(h, r, o);
}

// out[c] = vpls[rep[c]]
__global__ void take_reps_kernel(const rzk_vpl *vpls, const int *rep, int n, rzk_vpl *out) {
    constexpr int W = (int)(sizeof(rzk_vpl) / 4);
    const long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= (long long)n * W) return;
    const int c = (int)(w / W), i = (int)(w % W);
    reinterpret_cast<uint32_t *>(out)[w] = reinterpret_cast<const uint32_t *>(vpls + rep[c])[i];
}

// gather_clusters for every receiver, in two passes so that the work splits finely
// without changing any sum.  Tracing: items (warp tile, run of kVisChunk representatives)
// from an atomic counter, each storing one visibility ballot per representative.  Summing:
// one warp per tile adds weight x radiance over the representatives in cluster order for
// the pairs the ballots mark - the pairs and the order of a one-pass gather
// (mrcs.cc:31-39).
constexpr int kVisChunk = 128;

template <int WARPS, int TILE, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) mrcs_vis_kernel(DevScene s, const rzk_receiver *recv,
                                                                    int n_recv, int img_w, const rzk_vpl *reps,
                                                                    int n_reps, int n_wtiles, int *work,
                                                                    uint32_t *masks) {
    __shared__ __align__(128) rzk_vpl tiles[WARPS][2][TILE];
    __shared__ __align__(8) uint64_t bar[WARPS][2];
    __shared__ int stacks[WARPS][STACK_CAP];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    WarpStage<TILE> ws;
    ws.init(tiles[w], bar[w], stacks[w], lane);
    const int nch = (n_reps + kVisChunk - 1) / kVisChunk;
    const long long n_items = (long long)n_wtiles * nch;
    while (true) {
        int item = 0;
        if (lane == 0) item = atomicAdd(work, 1);
        item = __shfl_sync(kFull, item, 0);
        if (item >= n_items) break;
        const int wt = item / nch, c = item - wt * nch;
        const int j0 = c * kVisChunk, j1 = min(n_reps, j0 + kVisChunk);
        if (!visibility_item<TILE>(s, recv, n_recv, img_w, reps, j0, j1, wt, ws, lane,
                                   masks + (long long)wt * n_reps + j0))
            break;
    }
}

constexpr int kShadeBlock = 128;

__global__ void __launch_bounds__(kShadeBlock) mrcs_shade_kernel(DevScene s, const rzk_receiver *recv, int n_recv,
                                                                 int img_w, const rzk_vpl *reps, const float *weights,
                                                                 int n_reps, int n_wtiles, const uint32_t *masks,
                                                                 int mode, float tau, float *sums) {
    const int wt = (int)(((long long)blockIdx.x * kShadeBlock + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (wt >= n_wtiles) return;
    shade_item<true>(s, recv, n_recv, img_w, reps, n_reps, masks + (long long)wt * n_reps, wt, mode, tau, sums,
                     lane, weights);
}

__global__ void scale_kernel(float *x, long long n, float scale) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = x[i] * scale;
}

template <typename T>
struct DBuf {
    T *p = nullptr;
    ~DBuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t n) {
        if (p) cudaFree(p);
        p = nullptr;
        return cudaMalloc((void **)&p, sizeof(T) * std::max<size_t>(n, 1));
    }
};

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace
}  // namespace rzk

struct rzk_mrcs {
    rzk_context *ctx = nullptr;
    rzk_scene *scene = nullptr;
    rzk_mrcs_params prm{};
    int clamp_mode = 0;
    float tau = 0.0f;
    int n_vpl = 0, n_columns = 0, num_clusters = 0, n_clusters = 0;
    std::vector<int32_t> pixels;                 // 2 per sampled pixel (x, y)
    std::vector<int32_t> center, rep;
    std::vector<float> weight;
    rzk::DBuf<rzk_vpl> reps;                     // representatives' records, cluster order
    rzk::DBuf<float> weights;
    int weight_n = 0;                            // clusters with a representative
    rzk::DBuf<int> work;
    rzk::DBuf<uint32_t> masks;                   // visibility ballots of the tracing pass
    size_t mask_words = 0;
    int grid = 0;
    float ms[4] = {0, 0, 0, 0};
};

using namespace rzk;

extern "C" {

rzk_status rzk_mrcs_params_default(rzk_mrcs_params *p) {
    if (!p) return RZK_ERR_INVALID;
    p->block_size = 32;        // MatrixRowColumnSampling::MatrixRowColumnSampling (mrcs.cc:16-20)
    p->cluster_ratio = 0.01f;
    p->max_clusters = 1000;
    p->max_columns = 10000;    // mrcs.cc:79
    p->seed = 2013;
    return RZK_OK;
}

rzk_status rzk_mrcs_destroy(rzk_mrcs *m) {
    if (!m) return RZK_ERR_INVALID;
    delete m;
    return RZK_OK;
}

rzk_status rzk_mrcs_create(rzk_context *ctx, rzk_scene *scene, const rzk_camera *cam, const rzk_vpl *d_vpls,
                           int n_vpl, int clamp_mode, float tau, const rzk_mrcs_params *params, void *stream,
                           rzk_mrcs **out) {
    if (!ctx || !scene || !cam || !params || !out || n_vpl < 0 || (n_vpl > 0 && !d_vpls) ||
        ((uintptr_t)d_vpls & 15u) || clamp_mode < RZK_CLAMP_NONE || clamp_mode > RZK_CLAMP_RADIANCE ||
        cam->width <= 0 || cam->height <= 0 || params->block_size <= 0 || params->max_clusters <= 0 ||
        params->max_columns <= 0 || !(params->cluster_ratio >= 0.0f))
        return RZK_ERR_INVALID;
    *out = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    rzk_mrcs *m = new rzk_mrcs();
    auto fail = [&](rzk_status s) { delete m; return s; };
    m->ctx = ctx;
    m->scene = scene;
    m->prm = *params;
    m->clamp_mode = clamp_mode;
    m->tau = tau;
    m->n_vpl = n_vpl;
    // mrcs.cc:47-52 (float ratio times the VPL count, truncated)
    m->num_clusters = std::max(1, (int)(params->cluster_ratio * (float)n_vpl));
    if (m->num_clusters > params->max_clusters) m->num_clusters = params->max_clusters;

    double t0 = now_ms();
    HostRng g{params->seed, 7u, 0u};
    // 1. stratified pixels (image_sampler.cc:8-23)
    const int bs = params->block_size;
    for (int i = 0; i < cam->height; i += bs)
        for (int j = 0; j < cam->width; j += bs) {
            const float sx = g.next();
            const float sy = g.next();
            m->pixels.push_back((int32_t)((float)j + sx * (float)bs));
            m->pixels.push_back((int32_t)((float)i + sy * (float)bs));
        }
    const int rows = (int)(m->pixels.size() / 2);
    DBuf<int> d_px;
    DBuf<rzk_receiver> d_recv;
    cudaError_t e;
    if ((e = d_px.alloc(2 * (size_t)rows)) != cudaSuccess || (e = d_recv.alloc(rows)) != cudaSuccess)
        return fail(RZK_ERR_NOMEM);
    if ((e = cudaMemcpyAsync(d_px.p, m->pixels.data(), sizeof(int) * 2 * rows, cudaMemcpyHostToDevice, st)) !=
        cudaSuccess) {
        set_last_cuda_error(e, "mrcs pixels", __FILE__, __LINE__);
        return fail(RZK_ERR_CUDA);
    }
    const DevScene ds = scene->dev();
    pixel_receivers_kernel<<<(rows + kPixBlock - 1) / kPixBlock, kPixBlock, 0, st>>>(ds, *cam, d_px.p, rows,
                                                                                     d_recv.p);
    // 2. the columns: every VPL, or max_columns resampled by average power (mrcs.cc:79-94)
    const rzk_vpl *cols_v = d_vpls;
    DBuf<rzk_vpl> d_reduced;
    int cols = n_vpl;
    if (n_vpl > params->max_columns) {
        std::vector<rzk_vpl> hv(n_vpl);
        if ((e = cudaMemcpyAsync(hv.data(), d_vpls, sizeof(rzk_vpl) * n_vpl, cudaMemcpyDeviceToHost, st)) !=
                cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess) {
            set_last_cuda_error(e, "mrcs columns", __FILE__, __LINE__);
            return fail(RZK_ERR_CUDA);
        }
        std::vector<float> power(n_vpl);
        for (int i = 0; i < n_vpl; ++i)   // Rgb::avg (rgb.h:43)
            power[i] = (hv[i].contrib[0] + hv[i].contrib[1] + hv[i].contrib[2]) / 3.0f;
        DPdf pdf;
        pdf.set(power.data(), n_vpl);
        cols = params->max_columns;
        std::vector<rzk_vpl> red(cols);
        for (int i = 0; i < cols; ++i) {
            int k = -1;
            float pk = 0.0f;
            pdf.sample(g.next(), k, pk);
            red[i] = hv[k >= 0 ? k : 0];
            for (int c = 0; c < 3; ++c)
                red[i].contrib[c] = k >= 0 ? hv[k].contrib[c] / pk / (float)cols : 0.0f;
        }
        if ((e = d_reduced.alloc(cols)) != cudaSuccess) return fail(RZK_ERR_NOMEM);
        if ((e = cudaMemcpyAsync(d_reduced.p, red.data(), sizeof(rzk_vpl) * cols, cudaMemcpyHostToDevice, st)) !=
            cudaSuccess) {
            set_last_cuda_error(e, "mrcs columns", __FILE__, __LINE__);
            return fail(RZK_ERR_CUDA);
        }
        cols_v = d_reduced.p;
    }
    m->n_columns = cols;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) {
        set_last_cuda_error(e, "mrcs rows", __FILE__, __LINE__);
        return fail(RZK_ERR_CUDA);
    }
    double t1 = now_ms();
    // 3. the reduced matrix (LightTransportMatrix::fill), column-major [cols][rows][3]
    DBuf<float> d_mat;
    if ((e = d_mat.alloc(3 * (size_t)rows * std::max(cols, 1))) != cudaSuccess) return fail(RZK_ERR_NOMEM);
    rzk_status r = launch_matrix(ds, d_recv.p, rows, cols_v, cols, clamp_mode, tau, d_mat.p, nullptr, 0, st);
    if (r != RZK_OK) return fail(r);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) {
        set_last_cuda_error(e, "mrcs matrix", __FILE__, __LINE__);
        return fail(RZK_ERR_CUDA);
    }
    double t2 = now_ms();
    // 4. clustering (cluster_builder.cc:82-273), the stream continuing
    const int cap = std::max(m->num_clusters, cols);
    std::vector<int32_t> center(cap), rep(cap), assign(std::max(cols, 1));
    std::vector<float> weight(cap);
    int n = 0;
    r = cluster_by_sampling(d_mat.p, rows, cols, m->num_clusters, g, &n, center.data(), rep.data(), weight.data(),
                            assign.data(), st);
    if (r != RZK_OK) return fail(r);
    double t3 = now_ms();
    // the clusters that can gather: representative >= 0 (the "too few VPLs" case of
    // cluster_builder.cc:90-101 leaves every representative at -1)
    std::vector<int32_t> take;
    for (int c = 0; c < n; ++c) {
        m->center.push_back(center[c]);
        m->rep.push_back(rep[c]);
        m->weight.push_back(weight[c]);
        if (rep[c] >= 0) take.push_back(c);
    }
    m->n_clusters = n;
    const int nt = (int)take.size();
    std::vector<int32_t> rep_idx(nt);
    std::vector<float> w(nt);
    for (int t = 0; t < nt; ++t) {
        rep_idx[t] = rep[take[t]];
        w[t] = weight[take[t]];
    }
    DBuf<int> d_rep;
    if ((e = m->reps.alloc(nt)) != cudaSuccess || (e = m->weights.alloc(nt)) != cudaSuccess ||
        (e = d_rep.alloc(nt)) != cudaSuccess || (e = m->work.alloc(1)) != cudaSuccess)
        return fail(RZK_ERR_NOMEM);
    if (nt > 0) {
        if ((e = cudaMemcpyAsync(d_rep.p, rep_idx.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, st)) !=
                cudaSuccess ||
            (e = cudaMemcpyAsync(m->weights.p, w.data(), sizeof(float) * nt, cudaMemcpyHostToDevice, st)) !=
                cudaSuccess) {
            set_last_cuda_error(e, "mrcs representatives", __FILE__, __LINE__);
            return fail(RZK_ERR_CUDA);
        }
        const long long words = (long long)nt * (long long)(sizeof(rzk_vpl) / 4);
        take_reps_kernel<<<(unsigned)((words + 255) / 256), 256, 0, st>>>(cols_v, d_rep.p, nt, m->reps.p);
    }
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        set_last_cuda_error(e, "mrcs representatives", __FILE__, __LINE__);
        return fail(RZK_ERR_CUDA);
    }
    m->weight_n = nt;
    double t4 = now_ms();
    m->ms[0] = (float)(t1 - t0);
    m->ms[1] = (float)(t2 - t1);
    m->ms[2] = (float)(t3 - t2);
    m->ms[3] = (float)(t4 - t3);
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mrcs_vis_kernel<4, 32, 5>, 128, 0);
    m->grid = std::max(1, sms * std::max(1, per_sm));
    *out = m;
    return RZK_OK;
}

rzk_status rzk_mrcs_info(const rzk_mrcs *m, int *n_rows, int *n_columns, int *num_clusters, int *n_clusters,
                         float *stage_ms) {
    if (!m) return RZK_ERR_INVALID;
    if (n_rows) *n_rows = (int)(m->pixels.size() / 2);
    if (n_columns) *n_columns = m->n_columns;
    if (num_clusters) *num_clusters = m->num_clusters;
    if (n_clusters) *n_clusters = m->n_clusters;
    if (stage_ms)
        for (int i = 0; i < 4; ++i) stage_ms[i] = m->ms[i];
    return RZK_OK;
}

rzk_status rzk_mrcs_clusters(const rzk_mrcs *m, int32_t *h_pixels, int32_t *h_center, int32_t *h_rep,
                             float *h_weight) {
    if (!m) return RZK_ERR_INVALID;
    if (h_pixels) std::copy(m->pixels.begin(), m->pixels.end(), h_pixels);
    if (h_center) std::copy(m->center.begin(), m->center.end(), h_center);
    if (h_rep) std::copy(m->rep.begin(), m->rep.end(), h_rep);
    if (h_weight) std::copy(m->weight.begin(), m->weight.end(), h_weight);
    return RZK_OK;
}

rzk_status rzk_mrcs_gather(rzk_mrcs *m, const rzk_receiver *d_recv, int n_recv, int image_width, float scale,
                           float *d_rgb, void *stream) {
    if (!m || n_recv < 0 || image_width < 0 || (n_recv > 0 && (!d_recv || !d_rgb)) || ((uintptr_t)d_recv & 15u))
        return RZK_ERR_INVALID;
    if (n_recv == 0) return RZK_OK;
    cudaStream_t st = (cudaStream_t)stream;
    long long wtiles;
    if (image_width > 0) {
        const long long img_h = ((long long)n_recv + image_width - 1) / image_width;
        wtiles = (long long)((image_width + 7) / 8) * ((img_h + 3) / 4);
    } else {
        wtiles = ((long long)n_recv + 31) / 32;
    }
    const int nr = m->weight_n;
    const long long nch = (nr + kVisChunk - 1) / kVisChunk;
    if (wtiles * std::max<long long>(nch, 1) >= (1LL << 31)) return RZK_ERR_CAPACITY;
    const size_t words = (size_t)wtiles * (size_t)nr;
    if (words > m->mask_words) {   // grows with the image: the first gather of a size allocates
        RZK_CUDA_TRY(m->masks.alloc(words));
        m->mask_words = words;
    }
    const DevScene ds = m->scene->dev();
    if (nr > 0) {
        RZK_CUDA_TRY(cudaMemsetAsync(m->work.p, 0, sizeof(int), st));
        mrcs_vis_kernel<4, 32, 5><<<m->grid, 128, 0, st>>>(ds, d_recv, n_recv, image_width, m->reps.p, nr,
                                                           (int)wtiles, m->work.p, m->masks.p);
        RZK_CUDA_TRY(cudaGetLastError());
    }
    const long long threads = 32LL * wtiles;
    mrcs_shade_kernel<<<(unsigned)((threads + kShadeBlock - 1) / kShadeBlock), kShadeBlock, 0, st>>>(
        ds, d_recv, n_recv, image_width, m->reps.p, m->weights.p, nr, (int)wtiles, m->masks.p, m->clamp_mode,
        m->tau, d_rgb);
    RZK_CUDA_TRY(cudaGetLastError());
    const long long n3 = 3LL * n_recv;
    scale_kernel<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(d_rgb, n3, scale);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

}  // extern "C"
