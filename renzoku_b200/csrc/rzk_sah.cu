// rzk_sah.cu - a surface-area-heuristic tree over the scene's triangles for any-hit
// (shadow-ray) traversal.
//
// The any-hit answer is "some triangle whose own box passes the slab test and whose
// triangle test passes": every inner box is the exact min/max of the boxes below it and the
// rounded slab test is monotone in the bounds, so which tree leads to a triangle never
// changes whether it is tested under its own box.  Any tree with one triangle per leaf,
// leaf box = the triangle's box (the reference's leaf box, aggregate_bvh.cc:183-209) and
// inner box = the exact union of its children therefore returns the reference's visibility
// bit for bit; a tree with less overlap than the Morton LBVH simply reaches the answer in
// fewer steps.  Closest-hit queries keep the reference tree, whose visit order decides ties.
//
// Built on the host with binned SAH (32 bins on the centroid axis of largest extent; a
// median split past depth 32 or when the centroids coincide), nodes numbered depth-first
// with siblings adjacent, packed like the reference tree (two float4 per node slot).
#include "rzk_internal.cuh"

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <vector>

namespace rzk {
namespace {

struct Box {
    float mn[3], mx[3];
    void reset() {
        for (int i = 0; i < 3; ++i) { mn[i] = FLT_MAX; mx[i] = -FLT_MAX; }
    }
    void grow(const Box &b) {
        for (int i = 0; i < 3; ++i) {
            mn[i] = std::min(mn[i], b.mn[i]);
            mx[i] = std::max(mx[i], b.mx[i]);
        }
    }
    float area() const {
        float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
        if (dx < 0.0f) return 0.0f;
        return dx * dy + dy * dz + dz * dx;
    }
};

struct Builder {
    const std::vector<Box> &box;     // per sorted triangle slot
    std::vector<float> cen;          // 3 per slot
    std::vector<int> idx;            // slots, partitioned in place
    std::vector<float4> out;         // 2 float4 per node slot; slot = node + 1
    int next = 1;                    // next free node index (root = 0)
    int max_depth = 0;

    explicit Builder(const std::vector<Box> &b) : box(b) {}

    static float bits(int a) {
        float f;
        std::memcpy(&f, &a, sizeof(f));
        return f;
    }
    void write(int node, const Box &b, int a) {
        out[2 * (node + 1)] = make_float4(b.mn[0], b.mn[1], b.mn[2], bits(a));
        out[2 * (node + 1) + 1] = make_float4(b.mx[0], b.mx[1], b.mx[2], bits(0));
    }

    // returns the node's box; the node's record is written here
    Box build(int node, int begin, int end, int depth) {
        max_depth = std::max(max_depth, depth);
        Box nb;
        nb.reset();
        for (int i = begin; i < end; ++i) nb.grow(box[idx[i]]);
        if (end - begin == 1) {
            write(node, nb, -1 - idx[begin]);
            return nb;
        }
        float cmn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, cmx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int i = begin; i < end; ++i)
            for (int d = 0; d < 3; ++d) {
                cmn[d] = std::min(cmn[d], cen[3 * idx[i] + d]);
                cmx[d] = std::max(cmx[d], cen[3 * idx[i] + d]);
            }
        int axis = 0;
        for (int d = 1; d < 3; ++d)
            if (cmx[d] - cmn[d] > cmx[axis] - cmn[axis]) axis = d;
        int mid = -1;
        const float ext = cmx[axis] - cmn[axis];
        if (ext > 0.0f && depth < 32) {
            constexpr int B = 32;
            Box bb[B];
            int cnt[B] = {0};
            for (int b = 0; b < B; ++b) bb[b].reset();
            const float k = B / ext;
            auto bin_of = [&](int s) {
                int b = (int)((cen[3 * s + axis] - cmn[axis]) * k);
                return std::min(std::max(b, 0), B - 1);
            };
            for (int i = begin; i < end; ++i) {
                const int b = bin_of(idx[i]);
                cnt[b]++;
                bb[b].grow(box[idx[i]]);
            }
            float right_area[B];
            int right_cnt[B];
            Box acc;
            acc.reset();
            int c = 0;
            for (int b = B - 1; b > 0; --b) {
                acc.grow(bb[b]);
                c += cnt[b];
                right_area[b] = acc.area();
                right_cnt[b] = c;
            }
            acc.reset();
            c = 0;
            float best = FLT_MAX;
            int best_b = -1;
            for (int b = 0; b < B - 1; ++b) {
                acc.grow(bb[b]);
                c += cnt[b];
                if (c == 0 || right_cnt[b + 1] == 0) continue;
                const float cost = c * acc.area() + right_cnt[b + 1] * right_area[b + 1];
                if (cost < best) { best = cost; best_b = b; }
            }
            if (best_b >= 0) {
                int *first = idx.data() + begin, *last = idx.data() + end;
                int *m = std::partition(first, last, [&](int s) { return bin_of(s) <= best_b; });
                mid = (int)(m - idx.data());
                if (mid == begin || mid == end) mid = -1;
            }
        }
        if (mid < 0) {   // coincident centroids or too deep: median by centroid
            mid = (begin + end) / 2;
            std::nth_element(idx.begin() + begin, idx.begin() + mid, idx.begin() + end,
                             [&](int x, int y) { return cen[3 * x + axis] < cen[3 * y + axis]; });
        }
        const int left = next;
        next += 2;
        build(left, begin, mid, depth + 1);
        build(left + 1, mid, end, depth + 1);
        write(node, nb, left);
        return nb;
    }
};

}  // namespace

rzk_status build_sah_tree(rzk_scene *s, cudaStream_t st) {
    const int n = s->n_tris;
    if (n <= 0) return RZK_OK;
    std::vector<float> bmin(3 * (size_t)n), bmax(3 * (size_t)n);
    std::vector<int> perm(n);
    RZK_CUDA_TRY(cudaMemcpyAsync(bmin.data(), s->d_bmin, sizeof(float) * bmin.size(), cudaMemcpyDeviceToHost, st));
    RZK_CUDA_TRY(cudaMemcpyAsync(bmax.data(), s->d_bmax, sizeof(float) * bmax.size(), cudaMemcpyDeviceToHost, st));
    RZK_CUDA_TRY(cudaMemcpyAsync(perm.data(), s->d_perm, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    RZK_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<Box> box(n);
    for (int slot = 0; slot < n; ++slot) {
        const int t = perm[slot];
        for (int d = 0; d < 3; ++d) {
            box[slot].mn[d] = bmin[3 * (size_t)t + d];
            box[slot].mx[d] = bmax[3 * (size_t)t + d];
        }
    }
    Builder b(box);
    b.cen.resize(3 * (size_t)n);
    for (int slot = 0; slot < n; ++slot)
        for (int d = 0; d < 3; ++d) b.cen[3 * (size_t)slot + d] = 0.5f * (box[slot].mn[d] + box[slot].mx[d]);
    b.idx.resize(n);
    for (int i = 0; i < n; ++i) b.idx[i] = i;
    const int n_nodes = 2 * n - 1;
    b.out.assign(2 * ((size_t)n_nodes + 1), make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    b.build(0, 0, n, 0);
    if (b.max_depth >= STACK_CAP - 2) return RZK_ERR_STACK;
    if (s->d_trav) {
        cudaFree(s->d_trav);
        s->device_bytes -= s->trav_bytes;
    }
    s->d_trav = nullptr;
    s->trav_bytes = sizeof(float4) * b.out.size();
    RZK_CUDA_TRY(cudaMalloc((void **)&s->d_trav, s->trav_bytes));
    RZK_CUDA_TRY(cudaMemcpyAsync(s->d_trav, b.out.data(), sizeof(float4) * b.out.size(), cudaMemcpyHostToDevice, st));
    RZK_CUDA_TRY(cudaStreamSynchronize(st));
    s->trav_depth = b.max_depth;
    s->device_bytes += s->trav_bytes;
    return RZK_OK;
}

}  // namespace rzk
