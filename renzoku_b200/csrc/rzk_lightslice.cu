// rzk_lightslice.cu - LightSlice (lightslice.cc, kdtree_n.h): the shading points sliced by a
// 6-D kd-tree, the reduced transport matrix of the slice representatives, the global VPL
// clustering refined per slice, Jensen's per-slice luminance maps, and the clustered gather.
//
// Where the work is:
//   device  6-D points of every shading point, the one-bounce VPL filter, the reduced matrix
//           (one shadow ray + incident radiance per (slice, VPL)), the global clustering
//           (rzk_cluster.cu), the slice lookup of every pixel and the gather over each
//           slice's cluster representatives (the per-frame cost);
//   host    the kd-tree build (its quickselect pivots are drawn sequentially, as in the
//           reference), the per-slice heap refinement (std::priority_queue / std::sort tie
//           order is part of the result), the per-cluster totals and the maps; slices are
//           refined in parallel threads, each from its own counter-based stream.
// Random streams (seed, stream, path): kd-tree + slice representatives (seed, 4, 0), global
// clustering (seed, 1, 0), refinement of slice s (seed, 5, s).
#include "rzk_gather_dev.cuh"
#include "rzk_guide.cuh"
#include "rzk_hostutil.h"
#include "rzk_cluster.cuh"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <queue>
#include <thread>
#include <utility>
#include <vector>

namespace rzk {
namespace {

constexpr float kPlaneBias = -1e-3f;              // KdTreeN::PLANE_BIAS (kdtree_n.h:196)
constexpr float kPi = 3.14159265358979f;          // common.h:38-41
constexpr float kTwoPi = 6.28318530717959f;
constexpr float kZeroEps = 1e-6f;                 // ZERO_EPSILON (common.h:55)

// LightSlice::generate_slices (lightslice.cc:261-275): a point per pixel hit with a material.
__global__ void points_kernel(const rzk_receiver *recv, int n, const rzk_material *mats, float diag,
                              float *pts, int *flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    RecvRegs r = load_receiver(recv + i);
    const int f = r.mat >= 0;
    flag[i] = f;
    if (f) {
        rzk_material m = load_material(mats + r.mat);
        map_vec6(r.p, r.ns, &m, r.wo, diag, pts + 6 * (size_t)i);
    }
}

__global__ void compact_points_kernel(const float *pts, const int *flag, const int *pos, int n, float *cpts,
                                      int *cpix) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !flag[i]) return;
    const int k = pos[i];
    for (int d = 0; d < 6; ++d) cpts[6 * (size_t)k + d] = pts[6 * (size_t)i + d];
    cpix[k] = i;
}

// LightSlice::initialize keeps the VPLs of bounce <= 1 in order (lightslice.cc:606-613).
__global__ void vpl_flag_kernel(const rzk_vpl *v, int n, int *flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = v[i].bounce <= 1;
}

__global__ void vpl_compact_kernel(const rzk_vpl *v, const int *flag, const int *pos, int n, rzk_vpl *out,
                                   int *orig) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !flag[i]) return;
    out[pos[i]] = v[i];
    orig[pos[i]] = i;
}

__global__ void gather_recv_kernel(const rzk_receiver *recv, const int *idx, int n, rzk_receiver *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = recv[idx[i]];
}

// KdTreeN::find_cluster (kdtree_n.h:486-518) on the tree's upper part: x = axis, or
// -1 - slice on a clustered node; y, z = children; w = plane bits.
__device__ __forceinline__ int find_slice(const int4 *kd, int n_kd, const float *p) {
    int idx = 0;
    for (int step = 0; step < n_kd && idx >= 0; ++step) {
        const int4 nd = kd[idx];
        if (nd.x < 0) return -1 - nd.x;
        const float dist = p[nd.x] - __int_as_float(nd.w) + kPlaneBias;
        idx = dist <= 0.0f ? nd.y : nd.z;
    }
    return -1;
}

__global__ void slice_of_kernel(const rzk_receiver *recv, int n, const rzk_material *mats, float diag,
                                const int4 *kd, int n_kd, int *slice, int *count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    RecvRegs r = load_receiver(recv + i);
    int s = -1;
    if (r.mat >= 0) {
        rzk_material m = load_material(mats + r.mat);
        float p[6];
        map_vec6(r.p, r.ns, &m, r.wo, diag, p);
        s = find_slice(kd, n_kd, p);
        if (s >= 0 && count) atomicAdd(count + s, 1);
    }
    slice[i] = s;
}

__device__ __forceinline__ uint32_t spread_bits(uint32_t v) {   // 16-bit -> even bits
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

// Sort keys that group the pixels by slice and, within a slice, along a Morton curve of
// (x, y) when the receivers are an image of width `img_w` (else in pixel order), so that a
// warp's 32 pixels form a compact patch; pixels without a slice go last.
__global__ void bin_keys_kernel(const int *slice, int n, int img_w, int mbits, uint32_t *keys, int *vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = slice[i];
    uint32_t k = 0xffffffffu;
    if (s >= 0) {
        uint32_t m = 0;
        if (img_w > 0) {
            const uint32_t y = (uint32_t)(i / img_w), x = (uint32_t)(i - (int)y * img_w);
            m = spread_bits(x) | (spread_bits(y) << 1);
        }
        k = ((uint32_t)s << mbits) | m;
    }
    keys[i] = k;
    vals[i] = i;
}

// LightSlice::gather_clusters (lightslice.cc:1315-1345) for the pixels of every slice:
// work item = (slice, 32 consecutive pixels of its bin); the slice's cluster
// representatives stream through the warp's VPL tiles, each radiance scaled by its
// cluster weight, summed in cluster order.  A pixel's sum does not depend on where its
// bin placed it.
struct SliceTables {
    const int *tile_off;      // [n_slices + 1] first work item of the slice at each position
    const int *order;         // [n_slices] slice at each position: most representatives first
    const int *pix_off;       // [n_slices] first binned pixel
    const int *pix_cnt;       // [n_slices]
    const int *rep_off;       // [n_slices] first representative
    const int *rep_cnt;       // [n_slices]
    const rzk_vpl *reps;      // representatives' records, slice-major
    const float *weights;     // cluster weights, same order
    int n_slices, n_items;
};

// The clustered gather runs in two passes so that its work splits finely without changing
// any sum.  Tracing: items (slice position, 32-pixel tile, run of kVisChunk
// representatives) - small and many, so the persistent warps finish together - each storing
// one visibility ballot per representative.  Summing: one warp per tile adds
// weight x radiance over its slice's representatives in cluster order for the pairs the
// ballots mark, which are exactly the pairs (and the order) of a one-pass gather.
constexpr int kVisChunk = 128;

struct VisTables {
    const int *vis_off;          // [n_slices + 1] first tracing item of the slice at each position
    const long long *mask_off;   // [n_slices] first visibility word of the slice at each position
    uint32_t *masks;             // per slice: [tile][representative]
    int n_items;
};

template <int WARPS, int TILE, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) cluster_vis_kernel(DevScene s, const rzk_receiver *recv,
                                                                       SliceTables t, VisTables v, int *work) {
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
        if (item >= v.n_items) break;
        int lo = 0, hi = t.n_slices - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (v.vis_off[mid] <= item) lo = mid; else hi = mid - 1;
        }
        const int sl = t.order[lo];
        const int nc = t.rep_cnt[sl];
        const int nch = (nc + kVisChunk - 1) / kVisChunk;
        const int local = item - v.vis_off[lo];
        const int wt = local / nch, c = local - wt * nch;
        const int j0 = c * kVisChunk, j1 = min(nc, j0 + kVisChunk);
        const int po = t.pix_off[sl], nr = t.pix_cnt[sl], ro = t.rep_off[sl];
        uint32_t *m = v.masks + v.mask_off[lo] + (long long)wt * nc + j0;
        if (!visibility_item<TILE>(s, recv + po, nr, 0, t.reps + ro, j0, j1, wt, ws, lane, m)) break;
    }
}

constexpr int kShadeBlock = 128;

__global__ void __launch_bounds__(kShadeBlock) cluster_shade_kernel(DevScene s, const rzk_receiver *recv,
                                                                    SliceTables t, VisTables v, int mode, float tau,
                                                                    float *sums) {
    const int item = (int)(((long long)blockIdx.x * kShadeBlock + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (item >= t.n_items) return;
    int lo = 0, hi = t.n_slices - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (t.tile_off[mid] <= item) lo = mid; else hi = mid - 1;
    }
    const int sl = t.order[lo];
    const int wt = item - t.tile_off[lo];
    const int po = t.pix_off[sl], nr = t.pix_cnt[sl], ro = t.rep_off[sl], nc = t.rep_cnt[sl];
    shade_item<true>(s, recv + po, nr, 0, t.reps + ro, nc, v.masks + v.mask_off[lo] + (long long)wt * nc, wt, mode,
                     tau, sums + 3 * (size_t)po, lane, t.weights + ro);
}

__global__ void scatter_kernel(const float *sums, const int *pix, int n, float scale, float *out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int p = pix[k];
    out[3 * (size_t)p] = sums[3 * (size_t)k] * scale;
    out[3 * (size_t)p + 1] = sums[3 * (size_t)k + 1] * scale;
    out[3 * (size_t)p + 2] = sums[3 * (size_t)k + 2] * scale;
}

// ---------------------------------------------------------------------------------------
// host: KdTreeN<6> with clustering (kdtree_n.h:192-361, 400-430, 486-572)

struct P6 {
    float p[6];
    int index;
    int cluster;
};

struct BoxN {
    float mn[6], mx[6];
    BoxN() {
        for (int i = 0; i < 6; ++i) { mn[i] = FLT_MAX; mx[i] = -FLT_MAX; }
    }
    void merge(const float *p) {   // std::min / std::max (boundingbox_n.h:88-93)
        for (int i = 0; i < 6; ++i) {
            mn[i] = std::min(mn[i], p[i]);
            mx[i] = std::max(mx[i], p[i]);
        }
    }
    int longest_axis() const {     // boundingbox_n.h:74-86
        int index = 0;
        float longest = 0.0f;
        for (int i = 0; i < 6; ++i) {
            float a = std::fabs(mx[i] - mn[i]);
            if (a > longest) { index = i; longest = a; }
        }
        return index;
    }
    float min_sq_dist(const float *p) const {   // boundingbox_n.h:95-106
        float sum = 0.0f;
        for (int i = 0; i < 6; ++i) {
            float c = std::min(std::max(p[i], mn[i]), mx[i]);
            float d = c - p[i];
            sum += d * d;
        }
        return sum;
    }
};

struct KdNode {
    int left = -1, right = -1;
    float plane = FLT_MAX;
    int axis = 127;
    bool clustered = false;
    int median = 0;
};

class KdSlicer {
public:
    std::vector<P6> data;                       // median-sorted points (the tree's data)
    std::vector<KdNode> nodes;
    std::vector<std::pair<int, int>> clusters;  // slices: [start, end] into data
    std::vector<BoxN> boxes;                    // per slice, for the nearest-slice search

    void build(std::vector<P6> pts, int max_cluster_size, HostRng &rd) {
        const int n = (int)pts.size();
        data = std::move(pts);
        nodes.clear();
        clusters.clear();
        boxes.clear();
        if (n <= 0) return;
        std::vector<P6> median(data);
        nodes.reserve(2 * (size_t)n);
        nodes.emplace_back();
        cluster_rec(max_cluster_size, 0, data.data(), 0, n - 1, rd, median.data());
    }

    int find_cluster(const float *p) const {
        if (nodes.empty()) return -1;
        int idx = 0;
        while (idx >= 0 && idx < (int)nodes.size()) {
            const KdNode &nd = nodes[idx];
            if (nd.clustered) return data[nd.median].cluster;
            if (nd.axis > 5) return -1;
            const float dist = p[nd.axis] - nd.plane + kPlaneBias;
            idx = dist <= 0.0f ? nd.left : nd.right;
        }
        return -1;
    }

    // furthest first, as the reference pops its max-heap
    void find_nearest_cluster(const float *p, int k, std::vector<int> &out) const {
        out.clear();
        if (nodes.empty()) return;
        struct Less {
            const std::vector<BoxN> *b;
            const float *p;
            bool operator()(int a, int c) const { return (*b)[a].min_sq_dist(p) < (*b)[c].min_sq_dist(p); }
        };
        std::priority_queue<int, std::vector<int>, Less> heap(Less{&boxes, p});
        nearest_rec(0, p, k, heap);
        while (!heap.empty()) {
            out.push_back(heap.top());
            heap.pop();
        }
    }

private:
    // quick_select_k (kdtree_n.h:208-256), iterative form of the same recursion
    static void quick_select(HostRng &rd, int axis, int k, P6 *in, int start, int end, P6 *out) {
        while (start <= end) {
            const int p = start + (int)(rd.next() * (float)(end - start + 1));
            const float v = in[p].p[axis];
            int pos = start;
            for (int i = start; i <= end; ++i)
                if (in[i].p[axis] < v) out[pos++] = in[i];
            const int equal_start = pos;
            for (int i = start; i <= end; ++i)
                if (in[i].p[axis] == v) out[pos++] = in[i];
            const int equal_end = pos - 1;
            for (int i = start; i <= end; ++i)
                if (!(in[i].p[axis] < v) && !(in[i].p[axis] == v)) out[pos++] = in[i];
            if (k >= equal_start && k <= equal_end) {
                for (int i = start; i <= end; ++i) in[i] = out[i];
                return;
            } else if (k < equal_start) {
                for (int i = equal_start; i <= end; ++i) in[i] = out[i];
                end = equal_start - 1;
            } else {
                for (int i = start; i <= equal_end; ++i) in[i] = out[i];
                start = equal_end + 1;
            }
            std::swap(in, out);
        }
    }

    int new_node() {
        nodes.emplace_back();
        return (int)nodes.size() - 1;
    }

    // KdTreeN::cluster_kdtree (kdtree_n.h:299-361)
    void cluster_rec(int max_cluster_size, int index, P6 *d, int start, int end, HostRng &rd, P6 *med) {
        if (start >= end) return;
        if (end - start + 1 <= max_cluster_size && d[start].cluster < 0 && !nodes[index].clustered) {
            const int c = (int)clusters.size();
            for (int i = start; i <= end; ++i) {
                d[i].cluster = c;
                med[i].cluster = c;
            }
            clusters.emplace_back(start, end);
            BoxN bb;
            for (int i = start; i <= end; ++i) bb.merge(d[i].p);
            boxes.push_back(bb);
            nodes[index].clustered = true;
        }
        BoxN bb;
        for (int i = start; i <= end; ++i) bb.merge(d[i].p);
        const int axis = bb.longest_axis();
        nodes[index].axis = axis;
        const int median = (end + start) / 2;
        quick_select(rd, axis, median, d, start, end, med);
        nodes[index].plane = med[median].p[axis];
        nodes[index].median = median;
        const bool clustered = nodes[index].clustered;
        if (start <= median) {
            const int l = new_node();
            nodes[index].left = l;
            nodes[l].clustered = clustered;
            cluster_rec(max_cluster_size, l, med, start, median, rd, d);
        }
        if (median + 1 <= end) {
            const int r = new_node();
            nodes[index].right = r;
            nodes[r].clustered = clustered;
            cluster_rec(max_cluster_size, r, med, median + 1, end, rd, d);
        }
    }

    template <class Heap>
    void nearest_rec(int index, const float *p, int k, Heap &heap) const {   // kdtree_n.h:522-556
        const KdNode &nd = nodes[index];
        if (nd.clustered) {
            const int c = data[nd.median].cluster;
            if ((int)heap.size() < k) {
                heap.push(c);
            } else {
                const int f = heap.top();
                if (boxes[c].min_sq_dist(p) < boxes[f].min_sq_dist(p)) {
                    heap.pop();
                    heap.push(c);
                }
            }
            return;
        }
        const float dist = p[nd.axis] - nd.plane + kPlaneBias;
        const int first = dist <= 0.0f ? nd.left : nd.right;
        const int second = dist <= 0.0f ? nd.right : nd.left;
        if (first >= 0) nearest_rec(first, p, k, heap);
        if (second >= 0 && !heap.empty()) {
            const int f = heap.top();
            if ((int)heap.size() < k || boxes[f].min_sq_dist(p) > dist * dist) nearest_rec(second, p, k, heap);
        }
    }
};

// ---------------------------------------------------------------------------------------
// host: per-slice refinement (lightslice.cc:789-1060)

struct HostCluster {
    std::vector<int> idx;       // columns (one-bounce VPL indices), in the reference's order
    DPdf pdf;
    int rep = -1;
    float weight = 0.0f;
    float inc[3] = {0.0f, 0.0f, 0.0f};   // total incident radiance (= total outgoing)
    float wi[3] = {0.0f, 0.0f, 0.0f};    // direction to the representative
    bool upper = false;
};

struct Scratch {
    std::vector<float> f, norms, u, v, ab, pick;
    std::vector<std::pair<int, float>> line;
};

struct Refiner {
    const float *R;            // reduced matrix, column-major [cols][rows][3]
    const uint8_t *V;          // visibility [cols][rows]
    int rows, cols;
    const float *norms_R;      // get_column_norms of R
    // flatten(subcol(subrow(R, rows_sel), cols_sel)) into sc.f, column-major (3 n_rows) x m
    void flat(const std::vector<int> &rsel, const int *csel, int m, Scratch &sc) const {
        const int nr3 = 3 * (int)rsel.size();
        sc.f.resize((size_t)nr3 * m);
        for (int j = 0; j < m; ++j) {
            const float *col = R + (size_t)csel[j] * rows * 3;
            float *o = sc.f.data() + (size_t)j * nr3;
            for (size_t i = 0; i < rsel.size(); ++i) {
                const float *x = col + 3 * (size_t)rsel[i];
                o[3 * i] = x[0];
                o[3 * i + 1] = x[1];
                o[3 * i + 2] = x[2];
            }
        }
    }
    // MatrixC<Float>::get_column_norm (matrix_c.cc:90-103) + compute_distance
    // (lightslice.cc:333-355) on sc.f
    static float cost(int nr3, int m, Scratch &sc) {
        const float *f = sc.f.data();
        sc.norms.resize(m);
        for (int j = 0; j < m; ++j) {
            float mag = 0.0f;
            for (int r = 0; r < nr3; ++r) mag += f[(size_t)j * nr3 + r] * f[(size_t)j * nr3 + r];
            sc.norms[j] = std::sqrt(mag);
        }
        sc.u.assign(nr3, 0.0f);
        for (int j = 0; j < m; ++j)
            for (int r = 0; r < nr3; ++r) sc.u[r] += f[(size_t)j * nr3 + r];
        sc.v.assign(m, 0.0f);
        for (int j = 0; j < m; ++j) {
            float acc = 0.0f;
            for (int r = 0; r < nr3; ++r) acc += f[(size_t)j * nr3 + r] * sc.u[r];
            sc.v[j] = acc;
        }
        float c = 0.0f;
        for (int j = 0; j < m; ++j) c += sc.norms[j];
        float cost = 0.0f;
        for (int j = 0; j < m; ++j) cost += sc.norms[j] * c - sc.v[j];
        return cost;
    }
    void set_pdf(HostCluster &cl, Scratch &sc) const {   // pick(norms_R, indices) -> pdf
        sc.pick.resize(cl.idx.size());
        for (size_t t = 0; t < cl.idx.size(); ++t) sc.pick[t] = norms_R[cl.idx[t]];
        cl.pdf.set(sc.pick.data(), (int)sc.pick.size());
    }
    static void choose_rep(HostRng &rd, HostCluster &cl) {   // lightslice.cc:383-397
        int j;
        float pj;
        cl.pdf.sample(rd.next(), j, pj);
        if (j < 0) {
            cl.rep = cl.idx[cl.idx.size() / 2];
            cl.weight = 0.0f;
        } else {
            cl.rep = cl.idx[j];
            cl.weight = 1.0f / pj;
        }
    }
    // split_cluster (lightslice.cc:403-475) on sc.f (the cluster's columns)
    static void split(HostRng &rd, const HostCluster &cl, int nr3, Scratch &sc, std::vector<int> &i1,
                      std::vector<int> &i2) {
        i1.clear();
        i2.clear();
        const int m = (int)cl.idx.size();
        if (m == 1) { i1.push_back(cl.idx[0]); return; }
        if (m == 2) { i1.push_back(cl.idx[0]); i2.push_back(cl.idx[1]); return; }
        int i, j;
        float pi, pj;
        cl.pdf.sample(rd.next(), i, pi);
        cl.pdf.sample(rd.next(), j, pj);
        auto half = [&]() {
            i1.assign(cl.idx.begin(), cl.idx.begin() + m / 2);
            i2.assign(cl.idx.begin() + m / 2, cl.idx.end());
        };
        if (i < 0 || j < 0) { half(); return; }
        const float *f = sc.f.data();
        const float *a = f + (size_t)i * nr3, *b = f + (size_t)j * nr3;
        sc.ab.resize(nr3);
        for (int r = 0; r < nr3; ++r) sc.ab[r] = a[r] - b[r];
        sc.line.clear();
        for (int k = 0; k < m; ++k) {
            if (k == i || k == j) continue;
            const float *c = f + (size_t)k * nr3;
            float t = 0.0f;
            for (int r = 0; r < nr3; ++r) t += (a[r] - c[r]) * sc.ab[r];
            sc.line.emplace_back(k, t);
        }
        std::sort(sc.line.begin(), sc.line.end(),
                  [](const std::pair<int, float> &x, const std::pair<int, float> &y) { return x.second < y.second; });
        float max_dist = 0.0f;
        int max_k = -1;
        for (int k = 1; k < (int)sc.line.size(); ++k) {
            float d = sc.line[k].second - sc.line[k - 1].second;
            if (d > max_dist) { max_dist = d; max_k = k; }
        }
        if (max_k == -1) { half(); return; }
        i1.push_back(cl.idx[i]);
        i2.push_back(cl.idx[j]);
        for (int k = 0; k < max_k; ++k) i1.push_back(cl.idx[sc.line[k].first]);
        for (int k = max_k; k < (int)sc.line.size(); ++k) i2.push_back(cl.idx[sc.line[k].first]);
    }

    // the heap refinement of one slice (lightslice.cc:858-935)
    void refine(const std::vector<int> &nb, const std::vector<HostCluster> &global, int max_clusters,
                HostRng &rd, std::vector<HostCluster> &cl, Scratch &sc) const {
        cl = global;
        const int nr3 = 3 * (int)nb.size();
        struct CC {
            int index;
            float cost;
        };
        struct CCLess {
            bool operator()(const CC &a, const CC &b) const { return a.cost < b.cost; }
        };
        std::priority_queue<CC, std::vector<CC>, CCLess> heap;
        for (int c = 0; c < (int)cl.size(); ++c) {
            flat(nb, cl[c].idx.data(), (int)cl[c].idx.size(), sc);
            heap.push(CC{c, cost(nr3, (int)cl[c].idx.size(), sc)});
        }
        std::vector<int> i1, i2;
        while (!heap.empty() && (int)cl.size() < max_clusters) {
            const CC cc = heap.top();
            if (cl[cc.index].idx.size() <= 1) break;
            flat(nb, cl[cc.index].idx.data(), (int)cl[cc.index].idx.size(), sc);
            split(rd, cl[cc.index], nr3, sc, i1, i2);
            flat(nb, i1.data(), (int)i1.size(), sc);
            const float cost1 = cost(nr3, (int)i1.size(), sc);
            cl[cc.index].idx = i1;
            set_pdf(cl[cc.index], sc);
            choose_rep(rd, cl[cc.index]);
            HostCluster c2;
            flat(nb, i2.data(), (int)i2.size(), sc);
            const float cost2 = cost(nr3, (int)i2.size(), sc);
            c2.idx = i2;
            set_pdf(c2, sc);
            choose_rep(rd, c2);
            const int new_index = (int)cl.size();
            heap.pop();
            heap.push(CC{cc.index, cost1});
            heap.push(CC{new_index, cost2});
            cl.push_back(std::move(c2));
        }
    }
};

// direction_to_square (concentric_mapping.h:100-108): uniform hemisphere -> disk -> square
void direction_to_square(const float *w, float &sx, float &sy) {
    const float r2 = 1.0f - w[2];
    const float dx = w[0] / std::sqrt(2.0f - r2);
    const float dy = w[1] / std::sqrt(2.0f - r2);
    const float r = std::sqrt(dx * dx + dy * dy);
    float phi = std::atan2(dy, dx);
    if (phi < -kPi / 4) phi += kTwoPi;
    float a, b;
    if (phi < kPi / 4) {
        a = r;
        b = phi * a / (kPi / 4);
    } else if (phi < 3 * kPi / 4) {
        b = r;
        a = -(phi - kPi / 2) * b / (kPi / 4);
    } else if (phi < 5 * kPi / 4) {
        a = -r;
        b = (phi - kPi) * a / (kPi / 4);
    } else {
        b = -r;
        a = -(phi - 3 * kPi / 2) * b / (kPi / 4);
    }
    sx = a * 0.5f + 0.5f;
    sy = b * 0.5f + 0.5f;
}

template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    ~DBuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t count) {
        if (p) cudaFree(p);
        p = nullptr;
        n = count;
        return cudaMalloc((void **)&p, sizeof(T) * (count > 0 ? count : 1));
    }
};

}  // namespace
}  // namespace rzk

using namespace rzk;

struct rzk_lightslice {
    rzk_context *ctx = nullptr;
    rzk_scene *scene = nullptr;
    rzk_lightslice_params prm{};
    int width = 0, height = 0, n_points = 0, n_vpl1 = 0, n_global = 0;
    float diag = 0.0f;
    double ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    KdSlicer kd;
    std::vector<int> rep_point;                 // per slice: data position of its representative
    std::vector<std::vector<int>> neighbors;    // per slice: nearest slices, furthest first
    std::vector<std::vector<HostCluster>> clusters;
    std::vector<float> cluster_pdf;             // per slice per cluster, concatenated
    std::vector<uint8_t> valid;
    std::vector<float> sum_vpl;
    std::vector<float> maps;                    // [slice][res][res] luminance
    std::vector<float> map_cdf_col;             // [slice][res][res]
    std::vector<float> map_row_pdf, map_row_cdf;   // [slice][res]
    std::vector<float> map_total;               // [slice]
    // Metropolis sampler: per slice its visible clusters' directions on the unit square of the
    // slice's sampling record and their radiance weight x R(slice, representative) (the
    // points of the slice's KdTree2, lightslice.cc:1182-1217), and the cluster distribution's
    // CDF and directions (the chain's first state)
    std::vector<int> m_off;                     // [slice + 1] point offsets
    std::vector<float> m_pt;                    // [point][2], a slice's points ordered by grid cell
    std::vector<float> m_rad;                   // [point][4]: r, g, b, 0
    std::vector<int> m_cell;                    // [slice][grid^2 + 1]: first point of each cell
    int m_grid = 1;                             // cells per side, each at least density_radius wide
    std::vector<int> c_off;                     // [slice + 1] cluster offsets
    std::vector<float> c_cdf;                   // [cluster]
    std::vector<float> c_wi;                    // [cluster][3]
    std::vector<int> vpl1_orig;                 // one-bounce VPL -> input VPL index
    // the global clustering as cluster_by_sampling returned it: per cluster its
    // representative column and weight, per column its cluster
    std::vector<int32_t> global_rep, global_assign;
    std::vector<float> global_weight;
    std::vector<rzk_receiver> rep_recv;         // per slice
    std::vector<int4> h_kd;                     // upper tree for the device lookup
    bool on_device = false;                     // false: built from host inputs, no gather
    // device
    DBuf<rzk_vpl> d_vpl1;
    DBuf<float> d_R;
    DBuf<uint8_t> d_V;
    DBuf<int4> d_kd;
    int n_kd = 0;
    DBuf<rzk_vpl> d_reps;
    DBuf<float> d_weights;
    DBuf<int> d_rep_off, d_rep_cnt;
    // device copy of the sampling state for the guided path tracer (built on first use)
    bool guide_ready = false;
    DBuf<float> g_box, g_rep, g_uvn, g_prob, g_row_cdf, g_col_cdf, g_total;
    DBuf<uint8_t> g_valid;
    DBuf<int> g_m_off, g_m_cell, g_c_off;
    DBuf<float> g_m_pt, g_m_rad, g_c_cdf, g_c_wi, g_sum;
    // per-gather scratch (grown on demand)
    DBuf<int> d_slice, d_count, d_off, d_cursor, d_pix, d_tile_off, d_order, d_vis_off, d_work;
    DBuf<long long> d_mask_off;
    DBuf<uint32_t> d_masks;   // visibility ballots of the tracing pass
    DBuf<uint32_t> d_keys;
    DBuf<unsigned char> d_sort;
    DBuf<rzk_receiver> d_perm;
    DBuf<float> d_sums;
};

namespace {

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

rzk_status fail_cuda(cudaError_t e, const char *what) {
    set_last_cuda_error(e, what, __FILE__, __LINE__);
    return e == cudaErrorMemoryAllocation ? RZK_ERR_NOMEM : RZK_ERR_CUDA;
}

#define LS_TRY(expr)                                                   \
    do {                                                               \
        cudaError_t e_ = (expr);                                       \
        if (e_ != cudaSuccess) return fail_cuda(e_, #expr);            \
    } while (0)

// stable compaction positions of flagged items; returns the count
rzk_status compact_positions(const int *d_flag, int n, DBuf<int> &pos, int &count, cudaStream_t st) {
    LS_TRY(pos.alloc(n));
    DBuf<int> total;
    LS_TRY(total.alloc(1));
    size_t tb = exclusive_scan_tmp_bytes(n);
    DBuf<unsigned char> tmp;
    LS_TRY(tmp.alloc(tb));
    rzk_status r = exclusive_scan_i32(d_flag, pos.p, n, total.p, tmp.p, tb, st);
    if (r != RZK_OK) return r;
    LS_TRY(cudaMemcpyAsync(&count, total.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    LS_TRY(cudaStreamSynchronize(st));
    return RZK_OK;
}

// phase A: the kd-tree over the points, one representative and one colour draw per slice
// (lightslice.cc:252-303), the nearest slices of every representative, the device lookup tree
void slice_points(rzk_lightslice *L, const float *h_pts, const int *h_pix, int n_pts) {
    const rzk_lightslice_params &P = L->prm;
    L->n_points = n_pts;
    HostRng rd{P.seed, 4u, 0u};
    {
        std::vector<P6> node(n_pts);
        for (int i = 0; i < n_pts; ++i) {
            std::memcpy(node[i].p, h_pts + 6 * (size_t)i, 6 * sizeof(float));
            node[i].index = h_pix[i];
            node[i].cluster = -1;
        }
        L->kd.build(std::move(node), P.max_slice_size, rd);
    }
    const int ns = (int)L->kd.clusters.size();
    L->rep_point.resize(ns);
    for (int s = 0; s < ns; ++s) {
        const int a = L->kd.clusters[s].first, b = L->kd.clusters[s].second;
        int rep = (int)((float)a + rd.next() * (float)(b - a + 1));
        L->rep_point[s] = std::min(rep, n_pts - 1);
        (void)rd.next();   // Rgb::from_hsv(rd() * 360, ...) slice colour
    }
    L->neighbors.assign(ns, {});
    for (int s = 0; s < ns; ++s)
        L->kd.find_nearest_cluster(L->kd.data[L->rep_point[s]].p, P.num_neighbor_slices, L->neighbors[s]);
    // the upper tree for the device lookup: nodes down to the clustered ones
    std::vector<int> remap(L->kd.nodes.size(), -1);
    std::vector<int> stack{0}, order;
    while (!stack.empty()) {
        int i = stack.back();
        stack.pop_back();
        remap[i] = (int)order.size();
        order.push_back(i);
        const KdNode &nd = L->kd.nodes[i];
        if (nd.clustered) continue;
        if (nd.right >= 0) stack.push_back(nd.right);
        if (nd.left >= 0) stack.push_back(nd.left);
    }
    L->h_kd.resize(order.size());
    for (size_t k = 0; k < order.size(); ++k) {
        const KdNode &nd = L->kd.nodes[order[k]];
        if (nd.clustered) {
            L->h_kd[k] = make_int4(-1 - L->kd.data[nd.median].cluster, -1, -1, 0);
        } else {
            int bits;
            std::memcpy(&bits, &nd.plane, 4);
            L->h_kd[k] = make_int4(nd.axis, nd.left >= 0 ? remap[nd.left] : -1, nd.right >= 0 ? remap[nd.right] : -1,
                                   bits);
        }
    }
    L->n_kd = (int)L->h_kd.size();
}

// orders slice s's Metropolis points by the grid cell they fall in (row-major, stable) and
// appends the slice's cell offsets, so that a density query reads only the cells within
// density_radius of it
void bin_points(rzk_lightslice *L, int s) {
    const int G = L->m_grid, b = L->m_off[s], e = L->m_off[s + 1];
    std::vector<int> cell(e - b), count(G * G + 1, 0);
    for (int i = b; i < e; ++i) {
        const int cx = std::min(G - 1, std::max(0, (int)(L->m_pt[2 * (size_t)i] * G)));
        const int cy = std::min(G - 1, std::max(0, (int)(L->m_pt[2 * (size_t)i + 1] * G)));
        cell[i - b] = cy * G + cx;
        count[cell[i - b] + 1]++;
    }
    for (int c = 0; c < G * G; ++c) count[c + 1] += count[c];
    std::vector<float> pt(2 * (size_t)(e - b)), rad(4 * (size_t)(e - b));
    std::vector<int> cursor(count.begin(), count.end() - 1);
    for (int i = b; i < e; ++i) {
        const int to = cursor[cell[i - b]]++;
        std::copy(&L->m_pt[2 * (size_t)i], &L->m_pt[2 * (size_t)i] + 2, &pt[2 * (size_t)to]);
        std::copy(&L->m_rad[4 * (size_t)i], &L->m_rad[4 * (size_t)i] + 4, &rad[4 * (size_t)to]);
    }
    std::copy(pt.begin(), pt.end(), L->m_pt.begin() + 2 * (size_t)b);
    std::copy(rad.begin(), rad.end(), L->m_rad.begin() + 4 * (size_t)b);
    for (int c = 0; c <= G * G; ++c) L->m_cell.push_back(b + count[c]);
}

// phase D: per-slice refinement, totals and cluster distribution (in parallel over slices),
// validity and Jensen's maps.  hR / hV: the reduced matrix and visibility, column-major
// [n1][ns]; global: the clusters of ClusterBuilder::cluster_by_sampling.
void refine_slices(rzk_lightslice *L, const float *hR, const uint8_t *hV, int n1, const rzk_vpl *h_vpl1,
                   const std::vector<HostCluster> &global) {
    const rzk_lightslice_params &P = L->prm;
    const int ns = (int)L->kd.clusters.size();
    L->n_vpl1 = n1;
    L->n_global = (int)global.size();
    double t0 = now_ms();
    // LightTransportMatrix::get_column_norms (light_transport_matrix.cc:114-130)
    std::vector<float> norms_R(n1);
    for (int c = 0; c < n1; ++c) {
        float mag = 0.0f;
        for (int r = 0; r < ns; ++r) {
            const float *x = hR + 3 * ((size_t)c * ns + r);
            mag += x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
        }
        norms_R[c] = std::sqrt(mag);
    }
    L->clusters.assign(ns, {});
    std::vector<std::vector<float>> cpdf(ns);
    Refiner rf{hR, hV, ns, n1, norms_R.data()};
    const int max_sc = P.max_slice_clusters;
    std::atomic<int> next{0};
    auto worker = [&]() {
        Scratch scr;
        while (true) {
            const int s = next.fetch_add(1);
            if (s >= ns) break;
            HostRng srd{P.seed, 5u, (uint32_t)s};
            std::vector<HostCluster> &cl = L->clusters[s];
            rf.refine(L->neighbors[s], global, max_sc, srd, cl, scr);
            // totals, direction to the representative, upper hemisphere (lightslice.cc:957-1010):
            // visibility x incident radiance is the reduced matrix entry itself
            const rzk_receiver &rv = L->rep_recv[s];
            const V3 rp = ld3(rv.p), rn = ld3(rv.ns);
            for (HostCluster &c : cl) {
                float inc[3] = {0.0f, 0.0f, 0.0f};
                for (int k : c.idx) {
                    const float *x = hR + 3 * ((size_t)k * ns + s);
                    inc[0] += x[0];
                    inc[1] += x[1];
                    inc[2] += x[2];
                    if (k == c.rep) {
                        V3 wi = unit(sub(ld3(h_vpl1[k].p), rp));
                        c.wi[0] = wi.x; c.wi[1] = wi.y; c.wi[2] = wi.z;
                        const bool nonblack = x[0] != 0.0f || x[1] != 0.0f || x[2] != 0.0f;
                        c.upper = hV[(size_t)k * ns + s] && dot(rn, wi) > kZeroEps && nonblack;
                    }
                }
                c.inc[0] = inc[0]; c.inc[1] = inc[1]; c.inc[2] = inc[2];
            }
            // cluster distribution from the neighbours' rows (lightslice.cc:1117-1174)
            std::vector<float> &cn = cpdf[s];
            cn.resize(cl.size());
            for (size_t c = 0; c < cl.size(); ++c) {
                float mag = 0.0f;
                const float *col = hR + 3 * (size_t)cl[c].rep * ns;
                for (int row : L->neighbors[s]) {
                    const float *x = col + 3 * (size_t)row;
                    mag += x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
                }
                float nrm = std::sqrt(mag);
                nrm *= cl[c].weight;
                if (!cl[c].upper) nrm = 0.0f;
                cn[c] = nrm;
            }
        }
    };
    int nt = P.n_threads > 0 ? P.n_threads : (int)std::max(1u, std::thread::hardware_concurrency());
    nt = std::max(1, std::min(nt, ns));
    {
        std::vector<std::thread> th;
        for (int i = 1; i < nt; ++i) th.emplace_back(worker);
        worker();
        for (auto &t : th) t.join();
    }
    L->cluster_pdf.clear();
    L->c_off.assign(1, 0);
    L->c_cdf.clear();
    L->c_wi.clear();
    for (int s = 0; s < ns; ++s) {
        DPdf d;
        d.set(cpdf[s].data(), (int)cpdf[s].size());
        L->cluster_pdf.insert(L->cluster_pdf.end(), d.pdf.begin(), d.pdf.end());
        L->c_cdf.insert(L->c_cdf.end(), d.cdf.begin(), d.cdf.end());
        for (const HostCluster &c : L->clusters[s]) L->c_wi.insert(L->c_wi.end(), c.wi, c.wi + 3);
        L->c_off.push_back((int)L->c_cdf.size());
    }
    L->ms[4] = now_ms() - t0;

    // validity (estimate_sum, lightslice.cc:1520-1551) and Jensen's maps (lightslice.cc:2058-2151)
    t0 = now_ms();
    const int res = P.map_resolution;
    L->valid.assign(ns, 0);
    L->sum_vpl.assign(ns, 0.0f);
    L->maps.assign((size_t)ns * res * res, 0.0f);
    L->map_cdf_col.assign((size_t)ns * res * res, 0.0f);
    L->map_row_pdf.assign((size_t)ns * res, 0.0f);
    L->map_row_cdf.assign((size_t)ns * res, 0.0f);
    L->map_total.assign(ns, 0.0f);
    L->m_off.assign(1, 0);
    L->m_pt.clear();
    L->m_rad.clear();
    L->m_cell.clear();
    L->m_grid = std::max(1, std::min(64, (int)(1.0f / P.density_radius)));
    for (int s = 0; s < ns; ++s) {
        const std::vector<HostCluster> &cl = L->clusters[s];
        float tot[3] = {0.0f, 0.0f, 0.0f};
        for (const HostCluster &c : cl) {
            if (!c.upper) continue;
            const float k = P.density_radius * P.density_radius * kPi * c.weight;
            const float *x = hR + 3 * ((size_t)c.rep * ns + s);
            tot[0] += k * x[0];
            tot[1] += k * x[1];
            tot[2] += k * x[2];
        }
        const float sum = std::sqrt(tot[0] * tot[0] + tot[1] * tot[1] + tot[2] * tot[2]) * kTwoPi;
        L->sum_vpl[s] = sum;
        L->valid[s] = sum > 0.0f;
        float *map = &L->maps[(size_t)s * res * res];
        if (L->valid[s]) {
            const rzk_receiver &rv = L->rep_recv[s];
            float msum = 0.0f;
            for (const HostCluster &c : cl) {
                if (!c.upper) continue;
                const float lw[3] = {rv.u[0] * c.wi[0] + rv.u[1] * c.wi[1] + rv.u[2] * c.wi[2],
                                     rv.v[0] * c.wi[0] + rv.v[1] * c.wi[1] + rv.v[2] * c.wi[2],
                                     rv.n[0] * c.wi[0] + rv.n[1] * c.wi[1] + rv.n[2] * c.wi[2]};
                if (lw[2] <= 0.0f) continue;
                const float *x = hR + 3 * ((size_t)c.rep * ns + s);
                const float rr = c.weight * x[0], rg = c.weight * x[1], rb = c.weight * x[2];
                float sx, sy;
                direction_to_square(lw, sx, sy);
                int ix = (int)(sx * res), iy = (int)(sy * res);
                if (ix >= res) ix = res - 1;
                if (iy >= res) iy = res - 1;
                if (ix < 0) ix = 0;
                if (iy < 0) iy = 0;
                const float lum = std::sqrt(rr * rr + rg * rg + rb * rb);
                map[(size_t)iy * res + ix] += lum;
                msum += lum;
                L->m_pt.push_back(sx);
                L->m_pt.push_back(sy);
                L->m_rad.insert(L->m_rad.end(), {rr, rg, rb, 0.0f});
            }
            for (int j = 0; j < res; ++j)
                for (int i = 0; i < res; ++i) map[(size_t)i * res + j] += P.map_epsilon * msum;
        }
        L->m_off.push_back((int)(L->m_pt.size() / 2));
        bin_points(L, s);
        // DiscretePdf2D::set_distribution (pdf.cc:195-229)
        std::vector<float> row_sum(res);
        float total = 0.0f;
        for (int i = 0; i < res; ++i) {
            row_sum[i] = 0.0f;
            for (int j = 0; j < res; ++j) row_sum[i] += map[(size_t)i * res + j];
            total += row_sum[i];
            float acc = 0.0f;
            for (int j = 0; j < res; ++j) {
                acc += map[(size_t)i * res + j];
                L->map_cdf_col[((size_t)s * res + i) * res + j] = acc / row_sum[i];
            }
        }
        DPdf rows;
        rows.set(row_sum.data(), res);
        std::copy(rows.pdf.begin(), rows.pdf.end(), L->map_row_pdf.begin() + (size_t)s * res);
        std::copy(rows.cdf.begin(), rows.cdf.end(), L->map_row_cdf.begin() + (size_t)s * res);
        L->map_total[s] = total;
    }
    L->ms[5] = now_ms() - t0;
}

// global clusters from cluster_by_sampling's output: members in column order, the
// distribution over the column magnitudes
std::vector<HostCluster> make_global(int n1, int ng, const int32_t *rep, const float *w, const int32_t *assign,
                                     const float *mags) {
    std::vector<HostCluster> g(ng);
    for (int i = 0; i < n1; ++i)
        if (assign[i] >= 0 && assign[i] < ng) g[assign[i]].idx.push_back(i);
    for (int c = 0; c < ng; ++c) {
        std::vector<float> mm(g[c].idx.size());
        for (size_t t = 0; t < mm.size(); ++t) mm[t] = mags[g[c].idx[t]];
        g[c].pdf.set(mm.data(), (int)mm.size());
        g[c].rep = rep[c];
        g[c].weight = w[c];
    }
    return g;
}

rzk_status build(rzk_lightslice *L, const rzk_receiver *d_recv, const rzk_vpl *d_vpls, int n_vpl,
                 cudaStream_t st) {
    rzk_scene *sc = L->scene;
    const rzk_lightslice_params &P = L->prm;
    const int n_pix = L->width * L->height;
    const float *bx = sc->box;
    {   // BoundingBox::diagonal (boundingbox.h:109-111) of the aggregate box
        float dx = bx[3] - bx[0], dy = bx[4] - bx[1], dz = bx[5] - bx[2];
        L->diag = std::sqrt(dx * dx + dy * dy + dz * dz);
    }
    double t0 = now_ms();
    // points of the shading points with a material, in pixel order
    DBuf<float> pts, cpts;
    DBuf<int> flag, pos, cpix;
    LS_TRY(pts.alloc(6 * (size_t)n_pix));
    LS_TRY(flag.alloc(n_pix));
    points_kernel<<<(n_pix + 255) / 256, 256, 0, st>>>(d_recv, n_pix, sc->d_mats, L->diag, pts.p, flag.p);
    LS_TRY(cudaGetLastError());
    int n_pts = 0;
    rzk_status r = compact_positions(flag.p, n_pix, pos, n_pts, st);
    if (r != RZK_OK) return r;
    LS_TRY(cpts.alloc(6 * (size_t)std::max(n_pts, 1)));
    LS_TRY(cpix.alloc(std::max(n_pts, 1)));
    compact_points_kernel<<<(n_pix + 255) / 256, 256, 0, st>>>(pts.p, flag.p, pos.p, n_pix, cpts.p, cpix.p);
    LS_TRY(cudaGetLastError());
    std::vector<float> h_pts(6 * (size_t)n_pts);
    std::vector<int> h_pix(n_pts);
    if (n_pts > 0) {
        LS_TRY(cudaMemcpyAsync(h_pts.data(), cpts.p, sizeof(float) * h_pts.size(), cudaMemcpyDeviceToHost, st));
        LS_TRY(cudaMemcpyAsync(h_pix.data(), cpix.p, sizeof(int) * n_pts, cudaMemcpyDeviceToHost, st));
    }
    // VPLs of bounce <= 1
    DBuf<int> vflag, vpos, vorig;
    LS_TRY(vflag.alloc(std::max(n_vpl, 1)));
    int n1 = 0;
    if (n_vpl > 0) {
        vpl_flag_kernel<<<(n_vpl + 255) / 256, 256, 0, st>>>(d_vpls, n_vpl, vflag.p);
        LS_TRY(cudaGetLastError());
        r = compact_positions(vflag.p, n_vpl, vpos, n1, st);
        if (r != RZK_OK) return r;
    }
    LS_TRY(L->d_vpl1.alloc(std::max(n1, 1)));
    LS_TRY(vorig.alloc(std::max(n1, 1)));
    if (n1 > 0) {
        vpl_compact_kernel<<<(n_vpl + 255) / 256, 256, 0, st>>>(d_vpls, vflag.p, vpos.p, n_vpl, L->d_vpl1.p,
                                                                vorig.p);
        LS_TRY(cudaGetLastError());
    }
    std::vector<rzk_vpl> h_vpl1(n1);
    L->vpl1_orig.resize(n1);
    if (n1 > 0) {
        LS_TRY(cudaMemcpyAsync(h_vpl1.data(), L->d_vpl1.p, sizeof(rzk_vpl) * n1, cudaMemcpyDeviceToHost, st));
        LS_TRY(cudaMemcpyAsync(L->vpl1_orig.data(), vorig.p, sizeof(int) * n1, cudaMemcpyDeviceToHost, st));
    }
    LS_TRY(cudaStreamSynchronize(st));
    if (n_pts < 2 || n1 <= 0) return RZK_ERR_INVALID;   // nothing to slice or to cluster
    L->ms[0] = now_ms() - t0;

    t0 = now_ms();
    slice_points(L, h_pts.data(), h_pix.data(), n_pts);
    const int ns = (int)L->kd.clusters.size();
    LS_TRY(L->d_kd.alloc(L->h_kd.size()));
    LS_TRY(cudaMemcpyAsync(L->d_kd.p, L->h_kd.data(), sizeof(int4) * L->h_kd.size(), cudaMemcpyHostToDevice, st));
    L->ms[1] = now_ms() - t0;

    // the reduced matrix: slice representatives x one-bounce VPLs (lightslice.cc:698-748)
    t0 = now_ms();
    std::vector<int> rep_pix(ns);
    for (int s = 0; s < ns; ++s) rep_pix[s] = L->kd.data[L->rep_point[s]].index;
    DBuf<int> d_rep_pix;
    DBuf<rzk_receiver> d_rows;
    LS_TRY(d_rep_pix.alloc(ns));
    LS_TRY(d_rows.alloc(ns));
    LS_TRY(cudaMemcpyAsync(d_rep_pix.p, rep_pix.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st));
    gather_recv_kernel<<<(ns + 127) / 128, 128, 0, st>>>(d_recv, d_rep_pix.p, ns, d_rows.p);
    LS_TRY(cudaGetLastError());
    LS_TRY(L->d_R.alloc(3 * (size_t)ns * n1));
    LS_TRY(L->d_V.alloc((size_t)ns * n1));
    r = launch_matrix(sc->dev(), d_rows.p, ns, L->d_vpl1.p, n1, P.incident_clamp_mode, P.incident_tau, L->d_R.p,
                      L->d_V.p, 2, st);
    if (r != RZK_OK) return r;
    std::vector<float> hR(3 * (size_t)ns * n1);
    std::vector<uint8_t> hV((size_t)ns * n1);
    L->rep_recv.resize(ns);
    LS_TRY(cudaMemcpyAsync(hR.data(), L->d_R.p, sizeof(float) * hR.size(), cudaMemcpyDeviceToHost, st));
    LS_TRY(cudaMemcpyAsync(hV.data(), L->d_V.p, hV.size(), cudaMemcpyDeviceToHost, st));
    LS_TRY(cudaMemcpyAsync(L->rep_recv.data(), d_rows.p, sizeof(rzk_receiver) * ns, cudaMemcpyDeviceToHost, st));
    LS_TRY(cudaStreamSynchronize(st));
    L->ms[2] = now_ms() - t0;

    // global clustering of the columns (ClusterBuilder::cluster_by_sampling)
    t0 = now_ms();
    std::vector<HostCluster> global;
    {
        const int cap = std::max(P.num_clusters, n1);
        std::vector<int32_t> cen(cap), rep(cap), assign(n1);
        std::vector<float> w(cap), mags(n1, 1.0f);
        int ng = 0;
        r = cluster_by_sampling(L->d_R.p, ns, n1, P.num_clusters, P.seed, &ng, cen.data(), rep.data(), w.data(),
                                assign.data(), st, mags.data());
        if (r != RZK_OK) return r;
        if (n1 < P.num_clusters) {   // one column per cluster (cluster_builder.cc:90-101)
            ng = n1;
            for (int i = 0; i < n1; ++i) { assign[i] = i; rep[i] = i; w[i] = 1.0f; }
        }
        global = make_global(n1, ng, rep.data(), w.data(), assign.data(), mags.data());
        L->global_rep.assign(rep.begin(), rep.begin() + ng);
        L->global_weight.assign(w.begin(), w.begin() + ng);
        L->global_assign = assign;
    }
    L->ms[3] = now_ms() - t0;

    refine_slices(L, hR.data(), hV.data(), n1, h_vpl1.data(), global);

    // the gather's tables: every slice's representatives and weights, slice-major
    t0 = now_ms();
    std::vector<rzk_vpl> reps;
    std::vector<float> wts;
    std::vector<int> roff(ns), rcnt(ns);
    for (int s = 0; s < ns; ++s) {
        roff[s] = (int)reps.size();
        rcnt[s] = (int)L->clusters[s].size();
        for (const HostCluster &c : L->clusters[s]) {
            reps.push_back(h_vpl1[c.rep]);
            wts.push_back(c.weight);
        }
    }
    LS_TRY(L->d_reps.alloc(reps.size()));
    LS_TRY(L->d_weights.alloc(wts.size()));
    LS_TRY(L->d_rep_off.alloc(ns));
    LS_TRY(L->d_rep_cnt.alloc(ns));
    LS_TRY(cudaMemcpyAsync(L->d_reps.p, reps.data(), sizeof(rzk_vpl) * reps.size(), cudaMemcpyHostToDevice, st));
    LS_TRY(cudaMemcpyAsync(L->d_weights.p, wts.data(), sizeof(float) * wts.size(), cudaMemcpyHostToDevice, st));
    LS_TRY(cudaMemcpyAsync(L->d_rep_off.p, roff.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st));
    LS_TRY(cudaMemcpyAsync(L->d_rep_cnt.p, rcnt.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st));
    LS_TRY(cudaStreamSynchronize(st));
    L->ms[6] = now_ms() - t0;
    L->on_device = true;
    return RZK_OK;
}

// Resident grid of the persistent tracing kernel on the current device, computed once per
// device (std::call_once: concurrent first calls from several host threads wait for the one
// computation).
cudaError_t cluster_vis_grid(int *blocks) {
    struct Grid {
        std::once_flag once;
        int blocks = 0;
        cudaError_t err = cudaSuccess;
    };
    constexpr int kMaxDevices = 64;
    static Grid per_device[kMaxDevices];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    Grid &g = per_device[dev];
    std::call_once(g.once, [&g, dev] {
        int sms = 0, per_sm = 0;
        g.err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (g.err == cudaSuccess)
            g.err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cluster_vis_kernel<4, 32, 7>, 128, 0);
        g.blocks = std::max(1, sms * std::max(1, per_sm));
    });
    *blocks = g.blocks;
    return g.err;
}

}  // namespace

rzk_status rzk::guide_tables(rzk_lightslice *L, GuideDev *out, cudaStream_t st) {
    if (!L || !L->on_device || !out) return RZK_ERR_INVALID;
    const int ns = (int)L->kd.clusters.size(), res = L->prm.map_resolution;
    if (!L->guide_ready) {
        std::vector<float> box(12 * (size_t)ns), rep(3 * (size_t)ns), uvn(9 * (size_t)ns);
        std::vector<float> prob((size_t)ns * res * res);
        for (int s = 0; s < ns; ++s) {
            for (int d = 0; d < 6; ++d) {
                box[12 * (size_t)s + d] = L->kd.boxes[s].mn[d];
                box[12 * (size_t)s + 6 + d] = L->kd.boxes[s].mx[d];
            }
            for (int d = 0; d < 3; ++d) rep[3 * (size_t)s + d] = L->kd.data[L->rep_point[s]].p[d];
            const rzk_receiver &rv = L->rep_recv[s];
            for (int d = 0; d < 3; ++d) {
                uvn[9 * (size_t)s + d] = rv.u[d];
                uvn[9 * (size_t)s + 3 + d] = rv.v[d];
                uvn[9 * (size_t)s + 6 + d] = rv.n[d];
            }
            // DiscretePdf2D::probability (pdf.cc:188-193)
            for (int k = 0; k < res * res; ++k)
                prob[(size_t)s * res * res + k] = L->maps[(size_t)s * res * res + k] / L->map_total[s];
        }
        LS_TRY(L->g_box.alloc(box.size()));
        LS_TRY(L->g_rep.alloc(rep.size()));
        LS_TRY(L->g_uvn.alloc(uvn.size()));
        LS_TRY(L->g_prob.alloc(prob.size()));
        LS_TRY(L->g_row_cdf.alloc(L->map_row_cdf.size()));
        LS_TRY(L->g_col_cdf.alloc(L->map_cdf_col.size()));
        LS_TRY(L->g_total.alloc(ns));
        LS_TRY(L->g_valid.alloc(ns));
        LS_TRY(cudaMemcpyAsync(L->g_box.p, box.data(), sizeof(float) * box.size(), cudaMemcpyHostToDevice, st));
        LS_TRY(cudaMemcpyAsync(L->g_rep.p, rep.data(), sizeof(float) * rep.size(), cudaMemcpyHostToDevice, st));
        LS_TRY(cudaMemcpyAsync(L->g_uvn.p, uvn.data(), sizeof(float) * uvn.size(), cudaMemcpyHostToDevice, st));
        LS_TRY(cudaMemcpyAsync(L->g_prob.p, prob.data(), sizeof(float) * prob.size(), cudaMemcpyHostToDevice, st));
        LS_TRY(cudaMemcpyAsync(L->g_row_cdf.p, L->map_row_cdf.data(), sizeof(float) * L->map_row_cdf.size(),
                               cudaMemcpyHostToDevice, st));
        LS_TRY(cudaMemcpyAsync(L->g_col_cdf.p, L->map_cdf_col.data(), sizeof(float) * L->map_cdf_col.size(),
                               cudaMemcpyHostToDevice, st));
        LS_TRY(cudaMemcpyAsync(L->g_total.p, L->map_total.data(), sizeof(float) * ns, cudaMemcpyHostToDevice, st));
        LS_TRY(cudaMemcpyAsync(L->g_valid.p, L->valid.data(), ns, cudaMemcpyHostToDevice, st));
        // Metropolis tables (one element at least, so that every pointer is valid)
        auto up_i = [&](DBuf<int> &d, const std::vector<int> &h) -> rzk_status {
            LS_TRY(d.alloc(std::max<size_t>(1, h.size())));
            if (!h.empty()) LS_TRY(cudaMemcpyAsync(d.p, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, st));
            return RZK_OK;
        };
        auto up_f = [&](DBuf<float> &d, const std::vector<float> &h) -> rzk_status {
            LS_TRY(d.alloc(std::max<size_t>(1, h.size())));
            if (!h.empty()) LS_TRY(cudaMemcpyAsync(d.p, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice, st));
            return RZK_OK;
        };
        rzk_status r;
        if ((r = up_i(L->g_m_off, L->m_off)) != RZK_OK) return r;
        if ((r = up_i(L->g_m_cell, L->m_cell)) != RZK_OK) return r;
        if ((r = up_i(L->g_c_off, L->c_off)) != RZK_OK) return r;
        if ((r = up_f(L->g_m_pt, L->m_pt)) != RZK_OK) return r;
        if ((r = up_f(L->g_m_rad, L->m_rad)) != RZK_OK) return r;
        if ((r = up_f(L->g_c_cdf, L->c_cdf)) != RZK_OK) return r;
        if ((r = up_f(L->g_c_wi, L->c_wi)) != RZK_OK) return r;
        if ((r = up_f(L->g_sum, L->sum_vpl)) != RZK_OK) return r;
        LS_TRY(cudaStreamSynchronize(st));
        L->guide_ready = true;
    }
    GuideDev &G = *out;
    G.kd = L->d_kd.p;
    G.box = L->g_box.p;
    G.rep_pos = L->g_rep.p;
    G.rec_uvn = L->g_uvn.p;
    G.rec_valid = L->g_valid.p;
    G.prob = L->g_prob.p;
    G.row_cdf = L->g_row_cdf.p;
    G.col_cdf = L->g_col_cdf.p;
    G.total = L->g_total.p;
    G.m_off = L->g_m_off.p;
    G.m_cell = L->g_m_cell.p;
    G.m_grid = L->m_grid;
    G.m_pt = reinterpret_cast<const float2 *>(L->g_m_pt.p);
    G.m_rad = reinterpret_cast<const float4 *>(L->g_m_rad.p);
    G.sum_f = L->g_sum.p;
    G.c_off = L->g_c_off.p;
    G.c_cdf = L->g_c_cdf.p;
    G.c_wi = L->g_c_wi.p;
    G.density_radius = L->prm.density_radius;
    G.pool = nullptr;
    G.pool_n = 0;
    G.n_kd = L->n_kd;
    G.n_slices = ns;
    G.res = res;
    G.view_cos = std::cos(kPi * 0.25f);   // view_similarity_cosine_max (lightslice.cc:70)
    G.diag = L->diag;
    return RZK_OK;
}

extern "C" {

rzk_status rzk_lightslice_params_default(rzk_lightslice_params *p) {
    if (!p) return RZK_ERR_INVALID;
    // LightSlice::LightSlice (lightslice.cc:23-85)
    p->num_clusters = 600;
    p->max_slice_size = 256;
    p->num_neighbor_slices = 16;
    p->max_slice_clusters = 1200;
    p->map_resolution = 32;
    p->map_epsilon = 1e-3f;
    p->density_radius = 0.1f;
    p->incident_clamp_mode = RZK_CLAMP_NONE;
    p->incident_tau = 0.0f;
    p->seed = 2013u;
    p->n_threads = 0;
    return RZK_OK;
}

rzk_status rzk_lightslice_create(rzk_context *ctx, rzk_scene *scene, const rzk_receiver *d_recv, int width,
                                 int height, const rzk_vpl *d_vpls, int n_vpl, const rzk_lightslice_params *params,
                                 rzk_lightslice **out, void *stream) {
    if (!ctx || !scene || !d_recv || width <= 0 || height <= 0 || n_vpl < 0 || (n_vpl > 0 && !d_vpls) || !params ||
        !out)
        return RZK_ERR_INVALID;
    const rzk_lightslice_params &P = *params;
    if (P.num_clusters <= 0 || P.max_slice_size < 2 || P.num_neighbor_slices <= 0 || P.max_slice_clusters <= 0 ||
        P.map_resolution <= 0 || P.map_resolution > 1024 || P.incident_clamp_mode < RZK_CLAMP_NONE ||
        P.incident_clamp_mode > RZK_CLAMP_RADIANCE || ((uintptr_t)d_vpls & 15u))
        return RZK_ERR_INVALID;
    *out = nullptr;
    rzk_lightslice *L = new rzk_lightslice();
    L->ctx = ctx;
    L->scene = scene;
    L->prm = P;
    L->width = width;
    L->height = height;
    rzk_status r = build(L, d_recv, d_vpls, n_vpl, (cudaStream_t)stream);
    if (r != RZK_OK) {
        delete L;
        return r;
    }
    *out = L;
    return RZK_OK;
}

rzk_status rzk_lightslice_host_slice(const rzk_lightslice_params *params, const float *h_points,
                                     const int32_t *h_pixel, int n_points, rzk_lightslice **out) {
    if (!params || !h_points || !h_pixel || n_points < 2 || !out || params->max_slice_size < 2 ||
        params->num_neighbor_slices <= 0)
        return RZK_ERR_INVALID;
    rzk_lightslice *L = new rzk_lightslice();
    L->prm = *params;
    slice_points(L, h_points, h_pixel, n_points);
    *out = L;
    return RZK_OK;
}

rzk_status rzk_lightslice_host_refine(rzk_lightslice *L, const float *h_R, const uint8_t *h_V, int n_vpl_used,
                                      const rzk_vpl *h_vpls_used, const rzk_receiver *h_rep_recv,
                                      int n_global, const int32_t *h_global_rep, const float *h_global_weight,
                                      const int32_t *h_assign, const float *h_mags) {
    if (!L || !h_R || !h_V || n_vpl_used <= 0 || !h_vpls_used || !h_rep_recv || n_global <= 0 || !h_global_rep ||
        !h_global_weight || !h_assign || !h_mags || L->prm.map_resolution <= 0)
        return RZK_ERR_INVALID;
    const int ns = (int)L->kd.clusters.size();
    L->rep_recv.assign(h_rep_recv, h_rep_recv + ns);
    std::vector<HostCluster> g = make_global(n_vpl_used, n_global, h_global_rep, h_global_weight, h_assign, h_mags);
    refine_slices(L, h_R, h_V, n_vpl_used, h_vpls_used, g);
    return RZK_OK;
}

rzk_status rzk_lightslice_host_find(const rzk_lightslice *L, const float *h_points, int n, int32_t *h_slice) {
    if (!L || n < 0 || (n > 0 && (!h_points || !h_slice))) return RZK_ERR_INVALID;
    for (int i = 0; i < n; ++i) h_slice[i] = L->kd.find_cluster(h_points + 6 * (size_t)i);
    return RZK_OK;
}

rzk_status rzk_lightslice_destroy(rzk_lightslice *L) {
    if (!L) return RZK_ERR_INVALID;
    delete L;
    return RZK_OK;
}

rzk_status rzk_lightslice_info(const rzk_lightslice *L, int32_t *n_points, int32_t *n_slices, int32_t *n_vpl_used,
                               int32_t *n_global_clusters, int32_t *n_slice_clusters, double *h_ms) {
    if (!L) return RZK_ERR_INVALID;
    if (n_points) *n_points = L->n_points;
    if (n_slices) *n_slices = (int32_t)L->kd.clusters.size();
    if (n_vpl_used) *n_vpl_used = L->n_vpl1;
    if (n_global_clusters) *n_global_clusters = L->n_global;
    if (n_slice_clusters) {
        int64_t t = 0;
        for (const auto &c : L->clusters) t += (int64_t)c.size();
        *n_slice_clusters = (int32_t)t;
    }
    if (h_ms) for (int i = 0; i < 8; ++i) h_ms[i] = L->ms[i];
    return RZK_OK;
}

rzk_status rzk_lightslice_global(const rzk_lightslice *L, int32_t *h_rep, float *h_weight, int32_t *h_assign) {
    if (!L || !L->on_device) return RZK_ERR_INVALID;
    if (h_rep) std::copy(L->global_rep.begin(), L->global_rep.end(), h_rep);
    if (h_weight) std::copy(L->global_weight.begin(), L->global_weight.end(), h_weight);
    if (h_assign) std::copy(L->global_assign.begin(), L->global_assign.end(), h_assign);
    return RZK_OK;
}

rzk_status rzk_lightslice_slices(const rzk_lightslice *L, int32_t *h_point_pixel, int32_t *h_start, int32_t *h_end,
                                 int32_t *h_rep, int32_t *h_neighbors) {
    if (!L) return RZK_ERR_INVALID;
    const int ns = (int)L->kd.clusters.size();
    if (h_point_pixel)
        for (int i = 0; i < L->n_points; ++i) h_point_pixel[i] = L->kd.data[i].index;
    for (int s = 0; s < ns; ++s) {
        if (h_start) h_start[s] = L->kd.clusters[s].first;
        if (h_end) h_end[s] = L->kd.clusters[s].second;
        if (h_rep) h_rep[s] = L->rep_point[s];
        if (h_neighbors) {
            const int k = L->prm.num_neighbor_slices;
            for (int t = 0; t < k; ++t)
                h_neighbors[(size_t)s * k + t] = t < (int)L->neighbors[s].size() ? L->neighbors[s][t] : -1;
        }
    }
    return RZK_OK;
}

rzk_status rzk_lightslice_clusters(const rzk_lightslice *L, int32_t *h_count, int32_t *h_rep, float *h_weight,
                                   uint8_t *h_upper, float *h_wi, float *h_incident, float *h_pdf,
                                   int32_t *h_size, int32_t *h_members) {
    if (!L) return RZK_ERR_INVALID;
    size_t k = 0, m = 0;
    for (size_t s = 0; s < L->clusters.size(); ++s) {
        if (h_count) h_count[s] = (int32_t)L->clusters[s].size();
        for (const HostCluster &c : L->clusters[s]) {
            if (h_rep) h_rep[k] = c.rep;
            if (h_weight) h_weight[k] = c.weight;
            if (h_upper) h_upper[k] = c.upper ? 1 : 0;
            if (h_wi) for (int d = 0; d < 3; ++d) h_wi[3 * k + d] = c.wi[d];
            if (h_incident) for (int d = 0; d < 3; ++d) h_incident[3 * k + d] = c.inc[d];
            if (h_pdf) h_pdf[k] = L->cluster_pdf[k];
            if (h_size) h_size[k] = (int32_t)c.idx.size();
            if (h_members) for (int x : c.idx) h_members[m++] = x;
            ++k;
        }
    }
    return RZK_OK;
}

rzk_status rzk_lightslice_maps(const rzk_lightslice *L, float *h_maps, uint8_t *h_valid, float *h_sum,
                               float *h_row_cdf, float *h_col_cdf) {
    if (!L) return RZK_ERR_INVALID;
    if (h_maps) std::copy(L->maps.begin(), L->maps.end(), h_maps);
    if (h_valid) std::copy(L->valid.begin(), L->valid.end(), h_valid);
    if (h_sum) std::copy(L->sum_vpl.begin(), L->sum_vpl.end(), h_sum);
    if (h_row_cdf) std::copy(L->map_row_cdf.begin(), L->map_row_cdf.end(), h_row_cdf);
    if (h_col_cdf) std::copy(L->map_cdf_col.begin(), L->map_cdf_col.end(), h_col_cdf);
    return RZK_OK;
}

rzk_status rzk_lightslice_matrix(const rzk_lightslice *L, float *d_R, uint8_t *d_V, int32_t *h_vpl_index,
                                 void *stream) {
    if (!L || !L->on_device) return RZK_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)L->kd.clusters.size() * L->n_vpl1;
    if (d_R) RZK_CUDA_TRY(cudaMemcpyAsync(d_R, L->d_R.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, st));
    if (d_V) RZK_CUDA_TRY(cudaMemcpyAsync(d_V, L->d_V.p, n, cudaMemcpyDeviceToDevice, st));
    if (h_vpl_index) std::copy(L->vpl1_orig.begin(), L->vpl1_orig.end(), h_vpl_index);
    return RZK_OK;
}

rzk_status rzk_lightslice_find_slice(rzk_lightslice *L, const rzk_receiver *d_recv, int n_recv, int32_t *d_slice,
                                     void *stream) {
    if (!L || !L->on_device || n_recv < 0 || (n_recv > 0 && (!d_recv || !d_slice))) return RZK_ERR_INVALID;
    if (n_recv == 0) return RZK_OK;
    slice_of_kernel<<<(n_recv + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        d_recv, n_recv, L->scene->d_mats, L->diag, L->d_kd.p, L->n_kd, d_slice, nullptr);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

rzk_status rzk_lightslice_gather(rzk_lightslice *L, const rzk_receiver *d_recv, int n_recv, int clamp_mode,
                                 float tau, float scale, float *d_rgb, void *stream) {
    if (!L || !L->on_device || n_recv < 0 || (n_recv > 0 && (!d_recv || !d_rgb)) || clamp_mode < RZK_CLAMP_NONE ||
        clamp_mode > RZK_CLAMP_RADIANCE || ((uintptr_t)d_recv & 15u))
        return RZK_ERR_INVALID;
    if (n_recv == 0) return RZK_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const int ns = (int)L->kd.clusters.size();
    if (L->d_slice.n < (size_t)n_recv) {
        LS_TRY(L->d_slice.alloc(n_recv));
        LS_TRY(L->d_pix.alloc(n_recv));
        LS_TRY(L->d_perm.alloc(n_recv));
        LS_TRY(L->d_sums.alloc(3 * (size_t)n_recv));
        LS_TRY(L->d_keys.alloc(n_recv));
        LS_TRY(L->d_sort.alloc(radix_sort_scratch_bytes(n_recv)));
    }
    if (L->d_count.n < (size_t)ns + 1) {
        LS_TRY(L->d_count.alloc(ns + 1));
        LS_TRY(L->d_off.alloc(ns + 1));
        LS_TRY(L->d_cursor.alloc(ns + 1));
        LS_TRY(L->d_tile_off.alloc(ns + 1));
        LS_TRY(L->d_order.alloc(ns + 1));
        LS_TRY(L->d_vis_off.alloc(ns + 1));
        LS_TRY(L->d_mask_off.alloc(ns + 1));
        LS_TRY(L->d_work.alloc(1));
    }
    // slice of every pixel and the bin sizes
    LS_TRY(cudaMemsetAsync(L->d_count.p, 0, sizeof(int) * (ns + 1), st));
    slice_of_kernel<<<(n_recv + 255) / 256, 256, 0, st>>>(d_recv, n_recv, L->scene->d_mats, L->diag, L->d_kd.p,
                                                          L->n_kd, L->d_slice.p, L->d_count.p);
    LS_TRY(cudaGetLastError());
    std::vector<int> cnt(ns);
    LS_TRY(cudaMemcpyAsync(cnt.data(), L->d_count.p, sizeof(int) * ns, cudaMemcpyDeviceToHost, st));
    LS_TRY(cudaStreamSynchronize(st));
    std::vector<int> off(ns + 1), toff(ns + 1), order(ns);
    off[0] = 0;
    for (int s = 0; s < ns; ++s) off[s + 1] = off[s] + cnt[s];
    // Work items are handed out in order of decreasing cost: the tiles of the slices with
    // the most representatives first (a tile costs its 32 pixels x the slice's
    // representatives), so that the last items to start are short ones.  Every pixel still
    // adds its slice's representatives in cluster order; only which warp takes which tile,
    // and when, changes.
    for (int s = 0; s < ns; ++s) order[s] = s;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return L->clusters[a].size() > L->clusters[b].size(); });
    toff[0] = 0;
    for (int p = 0; p < ns; ++p) toff[p + 1] = toff[p] + (cnt[order[p]] + 31) / 32;
    std::vector<int> voff(ns + 1);
    std::vector<long long> moff(ns + 1);
    voff[0] = 0;
    moff[0] = 0;
    for (int p = 0; p < ns; ++p) {
        const long long tiles = (cnt[order[p]] + 31) / 32, nc = (long long)L->clusters[order[p]].size();
        const long long items = voff[p] + tiles * ((nc + kVisChunk - 1) / kVisChunk);
        if (items >= (1LL << 31)) return RZK_ERR_CAPACITY;
        voff[p + 1] = (int)items;
        moff[p + 1] = moff[p] + tiles * nc;
    }
    if ((size_t)moff[ns] > L->d_masks.n) LS_TRY(L->d_masks.alloc((size_t)moff[ns]));
    const int binned = off[ns];
    LS_TRY(cudaMemcpyAsync(L->d_off.p, off.data(), sizeof(int) * (ns + 1), cudaMemcpyHostToDevice, st));
    LS_TRY(cudaMemcpyAsync(L->d_tile_off.p, toff.data(), sizeof(int) * (ns + 1), cudaMemcpyHostToDevice, st));
    LS_TRY(cudaMemcpyAsync(L->d_order.p, order.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st));
    LS_TRY(cudaMemcpyAsync(L->d_vis_off.p, voff.data(), sizeof(int) * (ns + 1), cudaMemcpyHostToDevice, st));
    LS_TRY(cudaMemcpyAsync(L->d_mask_off.p, moff.data(), sizeof(long long) * (ns + 1), cudaMemcpyHostToDevice, st));
    // bins: a stable sort of the pixels by (slice, Morton code) - see bin_keys_kernel
    int sbits = 1;
    while ((1 << sbits) < ns + 1) ++sbits;
    int img_w = 0, mbits = 0;
    if (n_recv == L->width * L->height && L->width > 0) {
        int side = std::max(L->width, L->height), b = 0;
        while ((1 << b) < side) ++b;
        if (sbits + 2 * b <= 32) { img_w = L->width; mbits = 2 * b; }
    }
    if (sbits + mbits > 32) return RZK_ERR_CAPACITY;
    bin_keys_kernel<<<(n_recv + 255) / 256, 256, 0, st>>>(L->d_slice.p, n_recv, img_w, mbits, L->d_keys.p,
                                                          L->d_pix.p);
    LS_TRY(cudaGetLastError());
    {
        // pixels without a slice carry all-ones keys: include the slice bits' top value
        rzk_status rs = radix_sort_u32(L->d_keys.p, L->d_pix.p, n_recv, 32, L->d_sort.p, st);
        if (rs != RZK_OK) return rs;
    }
    LS_TRY(cudaMemsetAsync(d_rgb, 0, sizeof(float) * 3 * (size_t)n_recv, st));
    if (binned > 0) {
        gather_recv_kernel<<<(binned + 255) / 256, 256, 0, st>>>(d_recv, L->d_pix.p, binned, L->d_perm.p);
        SliceTables t;
        t.tile_off = L->d_tile_off.p;
        t.order = L->d_order.p;
        t.pix_off = L->d_off.p;
        t.pix_cnt = L->d_count.p;
        t.rep_off = L->d_rep_off.p;
        t.rep_cnt = L->d_rep_cnt.p;
        t.reps = L->d_reps.p;
        t.weights = L->d_weights.p;
        t.n_slices = ns;
        t.n_items = toff[ns];
        VisTables v;
        v.vis_off = L->d_vis_off.p;
        v.mask_off = L->d_mask_off.p;
        v.masks = L->d_masks.p;
        v.n_items = voff[ns];
        LS_TRY(cudaMemsetAsync(L->d_work.p, 0, sizeof(int), st));
        int grid = 0;
        LS_TRY(cluster_vis_grid(&grid));
        const DevScene ds = L->scene->dev();
        if (v.n_items > 0)
            cluster_vis_kernel<4, 32, 7><<<grid, 128, 0, st>>>(ds, L->d_perm.p, t, v, L->d_work.p);
        LS_TRY(cudaGetLastError());
        const long long threads = 32LL * t.n_items;
        cluster_shade_kernel<<<(unsigned)((threads + kShadeBlock - 1) / kShadeBlock), kShadeBlock, 0, st>>>(
            ds, L->d_perm.p, t, v, clamp_mode, tau, L->d_sums.p);
        LS_TRY(cudaGetLastError());
        scatter_kernel<<<(binned + 255) / 256, 256, 0, st>>>(L->d_sums.p, L->d_pix.p, binned, scale, d_rgb);
        LS_TRY(cudaGetLastError());
    }
    return RZK_OK;
}

}  // extern "C"
