// rzk_cluster.cu - light-transport-matrix statistics and column clustering on the device.
//
//   LightTransportMatrix::generate_alphas_for_clustering (light_transport_matrix.cc:72-106)
//   LightTransportMatrix::get_column_norms                (light_transport_matrix.cc:118-130)
//   ClusterBuilder::cluster_by_sampling                   (cluster_builder.cc:82-273)
//
// Matrix layout: column-major MatrixC<Rgb> (matrix_c.h:177-184), [cols][rows][3] floats,
// as rzk_gather_matrix writes it.  Every reduction the reference forms is a plain loop in
// float; here each is one thread's loop in the same order (and the library is built
// without FMA contraction), so alphas, norms, distances and the argmin are bit-identical.
// The column-to-cluster distances |‖K_j‖‖m_i‖ − m_i·K_j| are a cols x clusters x 3·rows
// contraction: a shared-memory tiled product in which every output accumulates over the
// 3·rows index in increasing order.  The reference's random draws (centre sampling and
// one representative per cluster) are sequential and stay on the host, drawing from the
// counter-based stream (seed, 1, 0) in the reference's order.
#include "rzk_internal.cuh"
#include "rzk_hostutil.h"
#include "rzk_cluster.cuh"

#include <algorithm>
#include <vector>

namespace rzk {

namespace {

// Per column j: the magnitude-matrix norm (Rmag = |R_ij|, then sqrt Σ Rmag²), the
// get_column_norms norm (sqrt Σ (r² + g² + b²)) and magnitude() of the flattened column
// (sqrt Σ over r, g, b in order), each in row order.
__global__ void colstats_kernel(const float *mat, int rows, int cols, float *rmag_norm, float *col_norm,
                                float *flat_norm) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cols) return;
    const float *c = mat + (size_t)j * rows * 3;
    float s_mag = 0.0f, s_cn = 0.0f, s_flat = 0.0f;
    for (int i = 0; i < rows; ++i) {
        float r = c[3 * i], g = c[3 * i + 1], b = c[3 * i + 2];
        float m = sqrtf(r * r + g * g + b * b);   // MatrixC<Rgb>::flatten_magnitude (matrix_c.cc:49-58)
        s_mag += m * m;
        s_cn += r * r + g * g + b * b;
        s_flat += r * r;
        s_flat += g * g;
        s_flat += b * b;
    }
    if (rmag_norm) rmag_norm[j] = sqrtf(s_mag);
    if (col_norm) col_norm[j] = sqrtf(s_cn);
    if (flat_norm) flat_norm[j] = sqrtf(s_flat);
}

// u = R * 1 (MatrixC::row_sum, matrix_c.h:236-245): per row i, over columns in order.
__global__ void rowsum_kernel(const float *mat, int rows, int cols, float *u) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    float acc = 0.0f;
    for (int j = 0; j < cols; ++j) {
        const float *e = mat + ((size_t)j * rows + i) * 3;
        acc += sqrtf(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
    }
    u[i] = acc;
}

// c = column_norms.row_sum (one value, columns in order).
__global__ void sum_kernel(const float *x, int n, float *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float acc = 0.0f;
    for (int j = 0; j < n; ++j) acc += x[j];
    *out = acc;
}

// alpha_j = ‖R_j‖ c - (Rᵀ u)_j with Rᵀu summed over rows in order (MatrixC::mul).
__global__ void alpha_kernel(const float *mat, int rows, int cols, const float *u, const float *rmag_norm,
                             const float *c0, float *alphas) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cols) return;
    const float *c = mat + (size_t)j * rows * 3;
    float v = 0.0f;
    for (int i = 0; i < rows; ++i) {
        float m = sqrtf(c[3 * i] * c[3 * i] + c[3 * i + 1] * c[3 * i + 1] + c[3 * i + 2] * c[3 * i + 2]);
        v += m * u[i];
    }
    alphas[j] = rmag_norm[j] * (*c0) - v;
}

// K = selected columns, each scaled by its cluster weight (cluster_builder.cc:176-190).
__global__ void gather_centers_kernel(const float *mat, int rows, const int *centers, const float *w,
                                      int count, float *K) {
    size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t n3 = 3 * (size_t)rows;
    if (e >= n3 * count) return;
    int c = (int)(e / n3);
    size_t k = e - (size_t)c * n3;
    K[e] = mat[(size_t)centers[c] * n3 + k] * w[c];
}

// D[i][j] = |kn_j * nm_i - Σ_e R[i][e] K[j][e]|, e in increasing order per output.
constexpr int TI = 64, TJ = 64, TE = 16;
__global__ void __launch_bounds__(256) distance_kernel(const float *R, const float *K, int n3, int cols,
                                                       int count, const float *kn, const float *nm, float *D) {
    __shared__ float As[TE][TI + 1];
    __shared__ float Bs[TE][TJ + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int i0 = blockIdx.x * TI, j0 = blockIdx.y * TJ;
    float acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = 0.0f;
    for (int e0 = 0; e0 < n3; e0 += TE) {
        for (int t = threadIdx.x; t < TI * TE; t += 256) {
            int ii = t / TE, ee = t % TE;
            int i = i0 + ii, e = e0 + ee;
            As[ee][ii] = (i < cols && e < n3) ? R[(size_t)i * n3 + e] : 0.0f;
            int j = j0 + ii;
            Bs[ee][ii] = (j < count && e < n3) ? K[(size_t)j * n3 + e] : 0.0f;
        }
        __syncthreads();
        const int emax = min(TE, n3 - e0);
        for (int ee = 0; ee < emax; ++ee) {
            float av[4], bv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) av[a] = As[ee][ty * 4 + a];
#pragma unroll
            for (int b = 0; b < 4; ++b) bv[b] = Bs[ee][tx * 4 + b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] += av[a] * bv[b];
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        int i = i0 + ty * 4 + a;
        if (i >= cols) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            int j = j0 + tx * 4 + b;
            if (j < count) D[(size_t)i * count + j] = fabsf(kn[j] * nm[i] - acc[a][b]);
        }
    }
}

// Nearest cluster of each column: strict < over clusters in order (lowest index wins).
__global__ void argmin_kernel(const float *D, int cols, int count, int *owner) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cols) return;
    const float *d = D + (size_t)i * count;
    int best = -1;
    float bd = 3.402823466e+38f;   // FLT_MAX
    for (int j = 0; j < count; ++j) {
        float x = d[j];
        if (x < bd) { best = j; bd = x; }
    }
    owner[i] = best;
}

template <class T>
struct DevBuf {
    T *p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t n) { return cudaMalloc((void **)&p, sizeof(T) * (n > 0 ? n : 1)); }
};

}  // namespace

rzk_status ltm_alphas(const float *mat, int rows, int cols, float *alphas, float *col_norms, cudaStream_t st) {
    if (cols <= 0) return RZK_OK;
    DevBuf<float> rmag, u, c0;
    RZK_CUDA_TRY(rmag.alloc(cols));
    RZK_CUDA_TRY(u.alloc(rows));
    RZK_CUDA_TRY(c0.alloc(1));
    colstats_kernel<<<(cols + 127) / 128, 128, 0, st>>>(mat, rows, cols, rmag.p, col_norms, nullptr);
    rowsum_kernel<<<(rows + 127) / 128, 128, 0, st>>>(mat, rows, cols, u.p);
    sum_kernel<<<1, 32, 0, st>>>(rmag.p, cols, c0.p);
    alpha_kernel<<<(cols + 127) / 128, 128, 0, st>>>(mat, rows, cols, u.p, rmag.p, c0.p, alphas);
    RZK_CUDA_TRY(cudaGetLastError());
    RZK_CUDA_TRY(cudaStreamSynchronize(st));
    return RZK_OK;
}

rzk_status cluster_by_sampling(const float *mat, int rows, int cols, int num_clusters, uint32_t seed,
                               int *h_n, int32_t *h_center, int32_t *h_rep, float *h_weight,
                               int32_t *h_assign, cudaStream_t st, float *h_mags) {
    HostRng g{seed, 1u, 0u};
    return cluster_by_sampling(mat, rows, cols, num_clusters, g, h_n, h_center, h_rep, h_weight, h_assign, st,
                               h_mags);
}

rzk_status cluster_by_sampling(const float *mat, int rows, int cols, int num_clusters, HostRng &g, int *h_n,
                               int32_t *h_center, int32_t *h_rep, float *h_weight, int32_t *h_assign,
                               cudaStream_t st, float *h_mags) {
    for (int j = 0; j < cols; ++j) h_assign[j] = -1;
    if (cols < num_clusters) {   // cluster_builder.cc:90-101
        for (int i = 0; i < cols; ++i) { h_center[i] = i; h_weight[i] = 1.0f; h_rep[i] = -1; }
        *h_n = cols;
        return RZK_OK;
    }
    DevBuf<float> alphas;
    RZK_CUDA_TRY(alphas.alloc(cols));
    rzk_status e = ltm_alphas(mat, rows, cols, alphas.p, nullptr, st);
    if (e != RZK_OK) return e;
    std::vector<float> a(cols);
    RZK_CUDA_TRY(cudaMemcpyAsync(a.data(), alphas.p, sizeof(float) * cols, cudaMemcpyDeviceToHost, st));
    RZK_CUDA_TRY(cudaStreamSynchronize(st));
    // centre sampling (cluster_builder.cc:110-156)
    DPdf pa;
    pa.set(a.data(), cols);
    std::vector<int> cen;
    std::vector<float> w;
    std::vector<int> slot(cols, -1);
    // The reference draws until it holds num_clusters distinct centres, which never ends
    // when fewer columns than that can be drawn at all (zero alpha); the target is capped
    // at the drawable count, and a draw budget bounds a pathological distribution.
    int drawable = 0;
    for (int i = 0; i < cols; ++i) drawable += pa.pdf[i] > 0.0f;
    const int target = std::min(num_clusters, drawable);
    long long draws = 0;
    const long long max_draws = 100000000LL;
    while ((int)cen.size() < target && draws++ < max_draws) {
        int k;
        float pk;
        pa.sample(g.next(), k, pk);
        if (pk == 0.0f) continue;
        if (slot[k] < 0) {
            slot[k] = (int)cen.size();
            cen.push_back(k);
            w.push_back(1.0f / pk);
        } else {
            w[slot[k]] += 1.0f / pk;
        }
    }
    const int count = (int)cen.size();
    if (count == 0) {   // nothing can be drawn: no cluster, no assignment
        *h_n = 0;
        if (h_mags) std::fill(h_mags, h_mags + cols, 0.0f);
        return RZK_OK;
    }
    const size_t n3 = 3 * (size_t)rows;
    DevBuf<int> d_cen, d_owner;
    DevBuf<float> d_w, K, kn, nm, D;
    RZK_CUDA_TRY(d_cen.alloc(count));
    RZK_CUDA_TRY(d_w.alloc(count));
    RZK_CUDA_TRY(K.alloc(n3 * count));
    RZK_CUDA_TRY(kn.alloc(count));
    RZK_CUDA_TRY(nm.alloc(cols));
    RZK_CUDA_TRY(d_owner.alloc(cols));
    RZK_CUDA_TRY(D.alloc((size_t)cols * count));
    RZK_CUDA_TRY(cudaMemcpyAsync(d_cen.p, cen.data(), sizeof(int) * count, cudaMemcpyHostToDevice, st));
    RZK_CUDA_TRY(cudaMemcpyAsync(d_w.p, w.data(), sizeof(float) * count, cudaMemcpyHostToDevice, st));
    size_t tot = n3 * count;
    gather_centers_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(mat, rows, d_cen.p, d_w.p, count, K.p);
    colstats_kernel<<<(count + 127) / 128, 128, 0, st>>>(K.p, rows, count, nullptr, kn.p, nullptr);
    colstats_kernel<<<(cols + 127) / 128, 128, 0, st>>>(mat, rows, cols, nullptr, nullptr, nm.p);
    dim3 grid((cols + TI - 1) / TI, (count + TJ - 1) / TJ);
    distance_kernel<<<grid, 256, 0, st>>>(mat, K.p, (int)n3, cols, count, kn.p, nm.p, D.p);
    argmin_kernel<<<(cols + 127) / 128, 128, 0, st>>>(D.p, cols, count, d_owner.p);
    RZK_CUDA_TRY(cudaGetLastError());
    std::vector<int> owner(cols);
    std::vector<float> mags(cols);
    RZK_CUDA_TRY(cudaMemcpyAsync(owner.data(), d_owner.p, sizeof(int) * cols, cudaMemcpyDeviceToHost, st));
    RZK_CUDA_TRY(cudaMemcpyAsync(mags.data(), nm.p, sizeof(float) * cols, cudaMemcpyDeviceToHost, st));
    RZK_CUDA_TRY(cudaStreamSynchronize(st));
    if (h_mags) std::copy(mags.begin(), mags.end(), h_mags);
    // members in column order, pdf over magnitudes, representative (cluster_builder.cc:228-272)
    std::vector<std::vector<int>> members(count);
    for (int i = 0; i < cols; ++i)
        if (owner[i] >= 0) members[owner[i]].push_back(i);
    std::vector<int> rep(count);
    std::vector<float> wf(count);
    for (int c = 0; c < count; ++c) {
        std::vector<float> mm(members[c].size());
        for (size_t t = 0; t < mm.size(); ++t) mm[t] = mags[members[c][t]];
        DPdf pc;
        pc.set(mm.data(), (int)mm.size());
        int j;
        float pj;
        pc.sample(g.next(), j, pj);
        if (j < 0) {
            rep[c] = members[c].empty() ? -1 : members[c][members[c].size() / 2];
            wf[c] = 0.0f;
        } else {
            rep[c] = members[c][j];
            wf[c] = 1.0f / pj;
        }
    }
    int n = 0;
    std::vector<int> map(count, -1);
    for (int c = 0; c < count; ++c) {
        if (rep[c] < 0) continue;
        map[c] = n;
        h_center[n] = cen[c];
        h_rep[n] = rep[c];
        h_weight[n] = wf[c];
        n++;
    }
    for (int i = 0; i < cols; ++i) h_assign[i] = owner[i] >= 0 ? map[owner[i]] : -1;
    *h_n = n;
    return RZK_OK;
}

}  // namespace rzk

extern "C" {

rzk_status rzk_ltm_alphas(const float *d_matrix, int rows, int cols, float *d_alphas, float *d_col_norms,
                          void *stream) {
    if (rows < 0 || cols < 0 || (cols > 0 && (!d_matrix || !d_alphas))) return RZK_ERR_INVALID;
    return rzk::ltm_alphas(d_matrix, rows, cols, d_alphas, d_col_norms, (cudaStream_t)stream);
}

rzk_status rzk_cluster_by_sampling(const float *d_matrix, int rows, int cols, int num_clusters, uint32_t seed,
                                   int *h_n_clusters, int32_t *h_center, int32_t *h_representative,
                                   float *h_weight, int32_t *h_assign, void *stream) {
    if (rows < 0 || cols < 0 || num_clusters <= 0 || !h_n_clusters || !h_center || !h_representative ||
        !h_weight || (cols > 0 && (!d_matrix || !h_assign)))
        return RZK_ERR_INVALID;
    return rzk::cluster_by_sampling(d_matrix, rows, cols, num_clusters, seed, h_n_clusters, h_center,
                                    h_representative, h_weight, h_assign, (cudaStream_t)stream);
}

}  // extern "C"
