// rzk_bvh.cu - device-resident Morton LBVH build, bit-identical to AggregateBvh::build
// (aggregate_bvh.cc:48-240, morton.h:16-120).
//
//   K0 tri_setup      facet normal, tangent, area, box of each triangle (triangle.cc:7-22)
//   K1 morton         scene box incl. the origin, centroid codes (morton.h:28-46, 98-102)
//   K2 radix sort     stable LSD sort of (code, index): the reference's qsort is a stable
//                     merge sort on glibc, so equal codes keep input order
//   K3 level split    BFS levels; children of a level are numbered by an exclusive scan
//                     of the internal-node flags, which reproduces the reference queue
//                     order (aggregate_bvh.cc:116-181)
//   K4 refit          reverse-level box merge (aggregate_bvh.cc:183-209)
//   K5 pack           32-byte node records (two children adjacent -> one 64-byte load)
//                     and 48-byte triangle records for the traversal kernels
#include "rzk_internal.cuh"

#include <algorithm>
#include <cstring>

namespace rzk {

namespace {

constexpr int kScanBlock = 1024;           // threads per scan block
constexpr int kScanItems = 2 * kScanBlock; // items per scan block

__global__ void scan_blocks_kernel(const int *in, int *out, int *block_sums, int n) {
    __shared__ int sh[kScanItems];
    int base = blockIdx.x * kScanItems;
    int t = threadIdx.x;
    int i0 = base + 2 * t, i1 = i0 + 1;
    sh[2 * t] = i0 < n ? in[i0] : 0;
    sh[2 * t + 1] = i1 < n ? in[i1] : 0;
    // Blelloch up-sweep / down-sweep over kScanItems elements
    int offset = 1;
    for (int d = kScanItems >> 1; d > 0; d >>= 1) {
        __syncthreads();
        if (t < d) {
            int ai = offset * (2 * t + 1) - 1, bi = offset * (2 * t + 2) - 1;
            sh[bi] += sh[ai];
        }
        offset <<= 1;
    }
    __syncthreads();
    if (t == 0) {
        if (block_sums) block_sums[blockIdx.x] = sh[kScanItems - 1];
        sh[kScanItems - 1] = 0;
    }
    for (int d = 1; d < kScanItems; d <<= 1) {
        offset >>= 1;
        __syncthreads();
        if (t < d) {
            int ai = offset * (2 * t + 1) - 1, bi = offset * (2 * t + 2) - 1;
            int tmp = sh[ai];
            sh[ai] = sh[bi];
            sh[bi] += tmp;
        }
    }
    __syncthreads();
    if (i0 < n) out[i0] = sh[2 * t];
    if (i1 < n) out[i1] = sh[2 * t + 1];
}

__global__ void scan_add_kernel(int *out, const int *block_offsets, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += block_offsets[i / kScanItems];
}

__global__ void scan_total_kernel(const int *in, const int *out, int n, int *total) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *total = n > 0 ? out[n - 1] + in[n - 1] : 0;
}

}  // namespace

size_t exclusive_scan_tmp_bytes(int n) {
    size_t bytes = 0;
    while (n > kScanItems) {
        int nb = (n + kScanItems - 1) / kScanItems;
        bytes += 2 * sizeof(int) * (size_t)nb + 256;
        n = nb;
    }
    return bytes + 256;
}

// Exclusive prefix sum of n ints; *d_total (device) receives the sum when non-null.
rzk_status exclusive_scan_i32(const int *d_in, int *d_out, int n, int *d_total, void *d_tmp,
                              size_t tmp_bytes, cudaStream_t st) {
    if (n <= 0) {
        if (d_total) RZK_CUDA_TRY(cudaMemsetAsync(d_total, 0, sizeof(int), st));
        return RZK_OK;
    }
    if (tmp_bytes < exclusive_scan_tmp_bytes(n)) return RZK_ERR_CAPACITY;
    int nb = (n + kScanItems - 1) / kScanItems;
    if (nb == 1) {
        scan_blocks_kernel<<<1, kScanBlock, 0, st>>>(d_in, d_out, nullptr, n);
    } else {
        char *tmp = (char *)d_tmp;
        int *sums = (int *)tmp;
        int *offs = sums + nb;
        size_t used = 2 * sizeof(int) * (size_t)nb + 256;
        scan_blocks_kernel<<<nb, kScanBlock, 0, st>>>(d_in, d_out, sums, n);
        rzk_status s = exclusive_scan_i32(sums, offs, nb, nullptr, tmp + used, tmp_bytes - used, st);
        if (s != RZK_OK) return s;
        scan_add_kernel<<<(n + 255) / 256, 256, 0, st>>>(d_out, offs, n);
    }
    if (d_total) scan_total_kernel<<<1, 32, 0, st>>>(d_in, d_out, n, d_total);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

namespace {

// K0: per-triangle geometry in input order (triangle.cc:7-22, quad.cc:20-22).
__global__ void tri_setup_kernel(const float *v, const float *tp, int n, float *tri_n,
                                 float *tri_u, float *tri_area, float *bmin, float *bmax) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3 p0 = ld3(v + 9 * i), p1 = ld3(v + 9 * i + 3), p2 = ld3(v + 9 * i + 6);
    V3 p01 = sub(p0, p1), p02 = sub(p0, p2);
    tri_area[i] = len(cross(p01, p02)) * 0.5f;
    st3(tri_u + 3 * i, unit(sub(p0, ld3(tp + 3 * i))));
    st3(tri_n + 3 * i, unit(cross(p01, p02)));
    st3(bmin + 3 * i, vmin(vmin(p0, p1), p2));
    st3(bmax + 3 * i, vmax(vmax(p0, p1), p2));
}

// Scene box: min / max over every triangle box and the origin (aggregate_bvh.cc:59-73,
// boundingbox.h:100-103).  min / max are exact; a zero result is +0 as in the reference,
// whose running box starts at +0 and keeps it on ties.
__device__ __forceinline__ float canon0(float x) { return x == 0.0f ? 0.0f : x; }

__global__ void box_reduce_kernel(const float *bmin, const float *bmax, int n, float *partial) {
    __shared__ float sh[6][256];
    V3 mn = mk(0.0f, 0.0f, 0.0f), mx = mk(0.0f, 0.0f, 0.0f);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        mn = vmin(mn, ld3(bmin + 3 * i));
        mx = vmax(mx, ld3(bmax + 3 * i));
    }
    int t = threadIdx.x;
    sh[0][t] = mn.x; sh[1][t] = mn.y; sh[2][t] = mn.z;
    sh[3][t] = mx.x; sh[4][t] = mx.y; sh[5][t] = mx.z;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (t < s) {
            for (int k = 0; k < 3; ++k) sh[k][t] = smin(sh[k][t], sh[k][t + s]);
            for (int k = 3; k < 6; ++k) sh[k][t] = smax(sh[k][t], sh[k][t + s]);
        }
        __syncthreads();
    }
    if (t < 6) partial[blockIdx.x * 6 + t] = sh[t][0];
}

__global__ void box_final_kernel(const float *partial, int nb, float *box6) {
    if (threadIdx.x != 0) return;
    V3 mn = mk(0.0f, 0.0f, 0.0f), mx = mk(0.0f, 0.0f, 0.0f);
    for (int b = 0; b < nb; ++b) {
        mn = vmin(mn, ld3(partial + 6 * b));
        mx = vmax(mx, ld3(partial + 6 * b + 3));
    }
    box6[0] = canon0(mn.x); box6[1] = canon0(mn.y); box6[2] = canon0(mn.z);
    box6[3] = canon0(mx.x); box6[4] = canon0(mx.y); box6[5] = canon0(mx.z);
}

__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {   // morton.h:28-35
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

// K1 (morton.h:37-46, 98-102)
__global__ void morton_kernel(const float *bmin, const float *bmax, int n, const float *box6,
                              uint32_t *codes, int *idx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3 smn = ld3(box6), smx = ld3(box6 + 3);
    V3 c = scl(add(ld3(bmin + 3 * i), ld3(bmax + 3 * i)), 0.5f);
    c = dvv(sub(c, smn), sub(smx, smn));
    float x = smin(smax(c.x * 1024.0f, 0.0f), 1023.0f);
    float y = smin(smax(c.y * 1024.0f, 0.0f), 1023.0f);
    float z = smin(smax(c.z * 1024.0f, 0.0f), 1023.0f);
    codes[i] = expand_bits((uint32_t)x) * 4 + expand_bits((uint32_t)y) * 2 + expand_bits((uint32_t)z);
    idx[i] = i;
}

// K2: stable LSD radix sort, 8-bit digits.
constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;                       // items per thread per tile
constexpr int kSortTile = kSortThreads * kSortItems;

__global__ void radix_hist_kernel(const uint32_t *keys, int n, int shift, int *hist, int nblocks) {
    __shared__ int cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    int base = blockIdx.x * kSortTile;
    for (int k = 0; k < kSortItems; ++k) {
        int i = base + k * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & 255u], 1);
    }
    __syncthreads();
    hist[threadIdx.x * nblocks + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void radix_scatter_kernel(const uint32_t *keys_in, const int *vals_in, int n, int shift,
                                     const int *offsets, int nblocks, uint32_t *keys_out,
                                     int *vals_out) {
    __shared__ int base[256];
    __shared__ int run[256];
    __shared__ int wcnt[kSortThreads / 32][257];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    base[t] = offsets[t * nblocks + blockIdx.x];
    run[t] = 0;
    const int tile = blockIdx.x * kSortTile;
    for (int k = 0; k < kSortItems; ++k) {
        for (int w = 0; w < kSortThreads / 32; ++w) wcnt[w][t] = 0;
        __syncthreads();
        int i = tile + k * kSortThreads + t;
        bool valid = i < n;
        uint32_t key = valid ? keys_in[i] : 0u;
        int d = valid ? (int)((key >> shift) & 255u) : 256;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        int rank = __popc(peers & ((1u << lane) - 1u));
        if (valid && rank == 0) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            int before = 0;
            for (int w = 0; w < warp; ++w) before += wcnt[w][d];
            int pos = base[d] + run[d] + before + rank;
            keys_out[pos] = key;
            vals_out[pos] = vals_in[i];
        }
        __syncthreads();
        int tot = 0;
        for (int w = 0; w < kSortThreads / 32; ++w) tot += wcnt[w][t];
        run[t] += tot;
        __syncthreads();
    }
}

// morton.h:16-26 (__clz of the reference is a software count; same value)
__device__ __forceinline__ int clz32(uint32_t v) { return __clz(v); }

// morton.h:48-88
__device__ int find_split(const uint32_t *c, int first, int last) {
    uint32_t fc = c[first], lc = c[last];
    if (fc == lc) return (first + last) >> 1;
    int common = clz32(fc ^ lc);
    int split = first, step = last - first;
    do {
        step = (step + 1) >> 1;
        int ns = split + step;
        if (ns < last) {
            if (clz32(fc ^ c[ns]) > common) split = ns;
        }
    } while (step > 1);
    return split;
}

// K3a: split every node of a level; flag the internal ones.
__global__ void level_split_kernel(const uint32_t *codes, int first, int count, int level,
                                   const int *start, const int *end, int *split, int *flag,
                                   int *lvl) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    int i = first + k;
    lvl[i] = level;
    int s = start[i], e = end[i];
    if (s == e) {
        flag[k] = 0;
        split[k] = -1;
    } else {
        flag[k] = 1;
        split[k] = find_split(codes, s, e);
    }
}

// K3b: children of the internal node with rank r in this level sit at last + 2r, last+2r+1.
__global__ void level_link_kernel(int first, int count, int last, const int *split,
                                  const int *flag, const int *rank, int *start, int *end,
                                  int *left, int *right) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    int i = first + k;
    if (!flag[k]) {
        left[i] = -1;
        right[i] = -1;
        return;
    }
    int c = last + 2 * rank[k];
    int sp = split[k];
    left[i] = c;
    right[i] = c + 1;
    start[c] = start[i];
    end[c] = sp;
    start[c + 1] = sp + 1;
    end[c + 1] = end[i];
}

// K4 (aggregate_bvh.cc:183-209)
__global__ void refit_kernel(int first, int count, const int *start, const int *left,
                             const int *right, const int *perm, const float *tbmin,
                             const float *tbmax, float *nbmin, float *nbmax) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    int i = first + k;
    int l = left[i], r = right[i];
    V3 mn, mx;
    if (l < 0) {
        if (r < 0) {
            int t = perm[start[i]];
            mn = ld3(tbmin + 3 * t);
            mx = ld3(tbmax + 3 * t);
        } else {
            mn = ld3(nbmin + 3 * r);
            mx = ld3(nbmax + 3 * r);
        }
    } else {
        mn = ld3(nbmin + 3 * l);
        mx = ld3(nbmax + 3 * l);
        if (r >= 0) {
            mn = vmin(mn, ld3(nbmin + 3 * r));
            mx = vmax(mx, ld3(nbmax + 3 * r));
        }
    }
    st3(nbmin + 3 * i, mn);
    st3(nbmax + 3 * i, mx);
}

// K5: node records.  Slot s = node + 1 holds {bmin, a}, {bmax, b} where for an inner node
// a = left child (right = a + 1) and for a leaf a = -1 - sorted triangle slot.
__global__ void pack_nodes_kernel(int n_nodes, const int *start, const int *left, const int *right,
                                  const float *nbmin, const float *nbmax, float4 *nodes) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    int a = left[i] >= 0 ? left[i] : -1 - start[i];
    int b = right[i];
    nodes[2 * (i + 1)] = make_float4(nbmin[3 * i], nbmin[3 * i + 1], nbmin[3 * i + 2], __int_as_float(a));
    nodes[2 * (i + 1) + 1] = make_float4(nbmax[3 * i], nbmax[3 * i + 1], nbmax[3 * i + 2], __int_as_float(b));
}

__global__ void pack_tris_kernel(int n, const int *perm, const float *v, const float *tri_n,
                                 const float *tri_u, const int *tri_surf, float4 *isect,
                                 float4 *shade) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int t = perm[s];
    V3 p0 = ld3(v + 9 * t), p1 = ld3(v + 9 * t + 3), p2 = ld3(v + 9 * t + 6);
    V3 a = sub(p0, p1), b = sub(p0, p2);
    isect[3 * s] = make_float4(p0.x, p0.y, p0.z, a.x);
    isect[3 * s + 1] = make_float4(a.y, a.z, b.x, b.y);
    isect[3 * s + 2] = make_float4(b.z, 0.0f, 0.0f, 0.0f);
    shade[2 * s] = make_float4(tri_n[3 * t], tri_n[3 * t + 1], tri_n[3 * t + 2], __int_as_float(tri_surf[t]));
    shade[2 * s + 1] = make_float4(tri_u[3 * t], tri_u[3 * t + 1], tri_u[3 * t + 2], 0.0f);
}

// K6: 4-wide traversal nodes collapsed from the reference tree.  Every inner node on an
// even BFS level becomes a node whose entries are its children where they are leaves and
// its grandchildren otherwise; grandchildren inner nodes are again on an even level.  The
// entries keep the reference's exact boxes, so a triangle is reached through this tree
// under exactly the same slab tests as through the binary one (every box contains the
// boxes below it and the rounded slab test is monotone in the bounds).
// Record: 8 x float4, entry k = {bmin.xyz, code}, {bmax.xyz, 0}; code = node index,
// -1 - sorted triangle slot for a leaf, or kWideEmpty.
__global__ void wide_flag_kernel(int n_nodes, const int *left, const int *level, int *flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    flag[i] = (left[i] >= 0 && (level[i] & 1) == 0) ? 1 : 0;
}

__device__ __forceinline__ void wide_entry(float4 *dst, int node, int code, const float *nbmin,
                                           const float *nbmax) {
    dst[0] = make_float4(nbmin[3 * node], nbmin[3 * node + 1], nbmin[3 * node + 2], __int_as_float(code));
    dst[1] = make_float4(nbmax[3 * node], nbmax[3 * node + 1], nbmax[3 * node + 2], 0.0f);
}

__global__ void wide_fill_kernel(int n_nodes, const int *start, const int *left, const int *right,
                                 const int *flag, const int *idx, const float *nbmin, const float *nbmax,
                                 float4 *wide) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes || !flag[i]) return;
    float4 *rec = wide + 8 * (size_t)idx[i];
    int k = 0;
    const int kids[2] = {left[i], right[i]};
    for (int a = 0; a < 2; ++a) {
        int c = kids[a];
        if (left[c] < 0) {
            wide_entry(rec + 2 * k++, c, -1 - start[c], nbmin, nbmax);
        } else {
            const int g2[2] = {left[c], right[c]};
            for (int b = 0; b < 2; ++b) {
                int g = g2[b];
                int code = left[g] < 0 ? -1 - start[g] : idx[g];
                wide_entry(rec + 2 * k++, g, code, nbmin, nbmax);
            }
        }
    }
    for (; k < 4; ++k) {
        rec[2 * k] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(kWideEmpty));
        rec[2 * k + 1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

template <class T>
rzk_status dalloc(T **p, size_t count, size_t *acc) {
    if (*p) return RZK_OK;
    size_t bytes = sizeof(T) * (count > 0 ? count : 1);
    RZK_CUDA_TRY(cudaMalloc((void **)p, bytes));
    if (acc) *acc += bytes;
    return RZK_OK;
}

}  // namespace


rzk_status bvh_build(rzk_scene *s, cudaStream_t st) {
    const int n = s->n_tris;
    s->n_nodes = 0;
    s->n_levels = 0;
    s->level_first.clear();
    s->level_last.clear();
    if (n <= 0) return RZK_OK;
    const int cap = 2 * n;
    size_t *acc = &s->device_bytes;
    RZK_TRY(dalloc(&s->d_tri_n, 3 * (size_t)n, acc));
    RZK_TRY(dalloc(&s->d_tri_u, 3 * (size_t)n, acc));
    RZK_TRY(dalloc(&s->d_tri_area, (size_t)n, acc));
    RZK_TRY(dalloc(&s->d_bmin, 3 * (size_t)n, acc));
    RZK_TRY(dalloc(&s->d_bmax, 3 * (size_t)n, acc));
    RZK_TRY(dalloc(&s->d_codes, (size_t)n, acc));
    RZK_TRY(dalloc(&s->d_sorted_codes, (size_t)n, acc));
    RZK_TRY(dalloc(&s->d_perm, (size_t)n, acc));
    RZK_TRY(dalloc(&s->d_start, (size_t)cap, acc));
    RZK_TRY(dalloc(&s->d_end, (size_t)cap, acc));
    RZK_TRY(dalloc(&s->d_left, (size_t)cap, acc));
    RZK_TRY(dalloc(&s->d_right, (size_t)cap, acc));
    RZK_TRY(dalloc(&s->d_level, (size_t)cap, acc));
    RZK_TRY(dalloc(&s->d_nbmin, 3 * (size_t)cap, acc));
    RZK_TRY(dalloc(&s->d_nbmax, 3 * (size_t)cap, acc));
    RZK_TRY(dalloc(&s->d_nodes, 2 * (size_t)(cap + 1), acc));
    RZK_TRY(dalloc(&s->d_tri_isect, 3 * (size_t)n, acc));
    RZK_TRY(dalloc(&s->d_tri_shade, 2 * (size_t)n, acc));

    // build-only scratch
    const int nblocks_sort = (n + kSortTile - 1) / kSortTile;
    const int hist_n = 256 * nblocks_sort;
    size_t scan_bytes = std::max(exclusive_scan_tmp_bytes(hist_n), exclusive_scan_tmp_bytes(cap));
    size_t scratch_bytes = 0;
    auto carve = [&](size_t bytes) { size_t off = scratch_bytes; scratch_bytes += (bytes + 255) & ~(size_t)255; return off; };
    size_t o_keys2 = carve(sizeof(uint32_t) * (size_t)n);
    size_t o_vals2 = carve(sizeof(int) * (size_t)n);
    size_t o_hist = carve(sizeof(int) * (size_t)hist_n);
    size_t o_offs = carve(sizeof(int) * (size_t)hist_n);
    size_t o_split = carve(sizeof(int) * (size_t)n);
    size_t o_flag = carve(sizeof(int) * (size_t)cap);
    size_t o_rank = carve(sizeof(int) * (size_t)cap);
    size_t o_box = carve(sizeof(float) * 6 * 1024 + 64);
    size_t o_total = carve(64);
    size_t o_scan = carve(scan_bytes);
    char *scratch = nullptr;
    RZK_CUDA_TRY(cudaMalloc((void **)&scratch, scratch_bytes));
    struct Free { char *p; ~Free() { if (p) cudaFree(p); } } guard{scratch};
    uint32_t *keys2 = (uint32_t *)(scratch + o_keys2);
    int *vals2 = (int *)(scratch + o_vals2);
    int *hist = (int *)(scratch + o_hist);
    int *offs = (int *)(scratch + o_offs);
    int *split = (int *)(scratch + o_split);
    int *flag = (int *)(scratch + o_flag);
    int *rank = (int *)(scratch + o_rank);
    float *box = (float *)(scratch + o_box);
    int *total = (int *)(scratch + o_total);
    void *scan_tmp = scratch + o_scan;

    const int TB = 256;
    const int grid = (n + TB - 1) / TB;
    tri_setup_kernel<<<grid, TB, 0, st>>>(s->d_v, s->d_tp, n, s->d_tri_n, s->d_tri_u,
                                          s->d_tri_area, s->d_bmin, s->d_bmax);
    int rb = std::min(1024, grid);
    box_reduce_kernel<<<rb, 256, 0, st>>>(s->d_bmin, s->d_bmax, n, box + 6);
    box_final_kernel<<<1, 32, 0, st>>>(box + 6, rb, box);
    RZK_CUDA_TRY(cudaMemcpyAsync(s->box, box, sizeof(float) * 6, cudaMemcpyDeviceToHost, st));
    morton_kernel<<<grid, TB, 0, st>>>(s->d_bmin, s->d_bmax, n, box, s->d_codes, s->d_perm);
    RZK_CUDA_TRY(cudaGetLastError());

    // K2: four 8-bit passes; the data ends in d_sorted_codes / d_perm after an even count
    RZK_CUDA_TRY(cudaMemcpyAsync(s->d_sorted_codes, s->d_codes, sizeof(uint32_t) * n,
                                 cudaMemcpyDeviceToDevice, st));
    uint32_t *ka = s->d_sorted_codes, *kb = keys2;
    int *va = s->d_perm, *vb = vals2;
    for (int pass = 0; pass < 4; ++pass) {
        int shift = 8 * pass;
        radix_hist_kernel<<<nblocks_sort, kSortThreads, 0, st>>>(ka, n, shift, hist, nblocks_sort);
        RZK_TRY(exclusive_scan_i32(hist, offs, hist_n, nullptr, scan_tmp, scan_bytes, st));
        radix_scatter_kernel<<<nblocks_sort, kSortThreads, 0, st>>>(ka, va, n, shift, offs,
                                                                    nblocks_sort, kb, vb);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    RZK_CUDA_TRY(cudaGetLastError());

    // K3: BFS levels; the host needs each level's size to size the next launch
    int first = 0, last = 1, level = 0;
    RZK_CUDA_TRY(cudaMemsetAsync(s->d_start, 0, sizeof(int), st));
    int nm1 = n - 1;
    RZK_CUDA_TRY(cudaMemcpyAsync(s->d_end, &nm1, sizeof(int), cudaMemcpyHostToDevice, st));
    int n_nodes = 1;
    int h_total = 0;
    for (;;) {
        int count = last - first;
        s->level_first.push_back(first);
        s->level_last.push_back(last);
        int g = (count + TB - 1) / TB;
        level_split_kernel<<<g, TB, 0, st>>>(s->d_sorted_codes, first, count, level, s->d_start,
                                             s->d_end, split, flag, s->d_level);
        RZK_TRY(exclusive_scan_i32(flag, rank, count, total, scan_tmp, scan_bytes, st));
        level_link_kernel<<<g, TB, 0, st>>>(first, count, last, split, flag, rank, s->d_start,
                                            s->d_end, s->d_left, s->d_right);
        RZK_CUDA_TRY(cudaMemcpyAsync(&h_total, total, sizeof(int), cudaMemcpyDeviceToHost, st));
        RZK_CUDA_TRY(cudaStreamSynchronize(st));
        if (h_total == 0) break;
        first = last;
        last = last + 2 * h_total;
        n_nodes += 2 * h_total;
        level++;
        if (last > cap) return RZK_ERR_CAPACITY;
    }
    s->n_nodes = n_nodes;
    s->n_levels = (int)s->level_first.size();

    // K4: bottom-up boxes
    for (int l = s->n_levels - 1; l >= 0; --l) {
        int f = s->level_first[l], c = s->level_last[l] - f;
        refit_kernel<<<(c + TB - 1) / TB, TB, 0, st>>>(f, c, s->d_start, s->d_left, s->d_right,
                                                        s->d_perm, s->d_bmin, s->d_bmax,
                                                        s->d_nbmin, s->d_nbmax);
    }
    // K5: packed layouts
    RZK_CUDA_TRY(cudaMemsetAsync(s->d_nodes, 0, 2 * sizeof(float4), st));
    pack_nodes_kernel<<<(n_nodes + TB - 1) / TB, TB, 0, st>>>(n_nodes, s->d_start, s->d_left,
                                                              s->d_right, s->d_nbmin, s->d_nbmax,
                                                              s->d_nodes);
    pack_tris_kernel<<<grid, TB, 0, st>>>(n, s->d_perm, s->d_v, s->d_tri_n, s->d_tri_u,
                                          s->d_tri_surf, s->d_tri_isect, s->d_tri_shade);
    RZK_CUDA_TRY(cudaGetLastError());
    // K6: 4-wide traversal nodes
    {
        const int gn = (n_nodes + TB - 1) / TB;
        wide_flag_kernel<<<gn, TB, 0, st>>>(n_nodes, s->d_left, s->d_level, flag);
        RZK_TRY(exclusive_scan_i32(flag, rank, n_nodes, total, scan_tmp, scan_bytes, st));
        int n_wide = 0;
        RZK_CUDA_TRY(cudaMemcpyAsync(&n_wide, total, sizeof(int), cudaMemcpyDeviceToHost, st));
        RZK_CUDA_TRY(cudaStreamSynchronize(st));
        if (!s->d_wide || s->n_wide_cap < n_wide) {
            if (s->d_wide) cudaFree(s->d_wide);
            s->d_wide = nullptr;
            RZK_CUDA_TRY(cudaMalloc((void **)&s->d_wide, 8 * sizeof(float4) * (size_t)std::max(1, n_wide)));
            s->device_bytes += 8 * sizeof(float4) * (size_t)std::max(1, n_wide);
            s->n_wide_cap = n_wide;
        }
        s->n_wide = n_wide;
        wide_fill_kernel<<<gn, TB, 0, st>>>(n_nodes, s->d_start, s->d_left, s->d_right, flag, rank,
                                            s->d_nbmin, s->d_nbmax, s->d_wide);
        RZK_CUDA_TRY(cudaGetLastError());
    }
    RZK_CUDA_TRY(cudaStreamSynchronize(st));
    // the any-hit traversal tree (rzk_sah.cu); without it any-hit walks the reference tree
    if (s->build_trav) {
        rzk_status r = build_sah_tree(s, st);
        if (r == RZK_ERR_STACK) {   // too deep for the traversal stack: walk the reference tree
            if (s->d_trav) cudaFree(s->d_trav);
            s->d_trav = nullptr;
            s->device_bytes -= s->trav_bytes;
            s->trav_bytes = 0;
        } else if (r != RZK_OK) {
            return r;
        }
    }
    return RZK_OK;
}

// Stable LSD radix sort of (key, value) pairs on the low `bits` bits of the keys, with the
// K2 kernels.  keys/vals hold the input; the sorted pairs end in keys/vals (an even number
// of 8-bit passes) or are copied back there.  scratch: radix_sort_scratch_bytes(n) bytes.
size_t radix_sort_scratch_bytes(int n) {
    const int nblocks = (n + kSortTile - 1) / kSortTile;
    const int hist_n = 256 * std::max(nblocks, 1);
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    return up(sizeof(uint32_t) * (size_t)std::max(n, 1)) + up(sizeof(int) * (size_t)std::max(n, 1)) +
           2 * up(sizeof(int) * (size_t)hist_n) + up(exclusive_scan_tmp_bytes(hist_n));
}

int exclusive_scan_launches(int n, bool total) {
    if (n <= 0) return 0;
    const int nb = (n + kScanItems - 1) / kScanItems;
    const int k = nb == 1 ? 1 : 2 + exclusive_scan_launches(nb, false);
    return k + (total ? 1 : 0);
}

int radix_sort_launches(int n, int bits) {
    if (n <= 1) return 0;
    const int nblocks = (n + kSortTile - 1) / kSortTile;
    const int passes = std::max(1, (bits + 7) / 8);
    return passes * (2 + exclusive_scan_launches(256 * nblocks, false));
}

rzk_status radix_sort_u32(uint32_t *keys, int *vals, int n, int bits, void *scratch, cudaStream_t st) {
    if (n <= 1) return RZK_OK;
    const int nblocks = (n + kSortTile - 1) / kSortTile;
    const int hist_n = 256 * nblocks;
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    char *p = (char *)scratch;
    uint32_t *k2 = (uint32_t *)p;
    p += up(sizeof(uint32_t) * (size_t)n);
    int *v2 = (int *)p;
    p += up(sizeof(int) * (size_t)n);
    int *hist = (int *)p;
    p += up(sizeof(int) * (size_t)hist_n);
    int *offs = (int *)p;
    p += up(sizeof(int) * (size_t)hist_n);
    void *scan_tmp = p;
    const size_t scan_bytes = exclusive_scan_tmp_bytes(hist_n);
    uint32_t *ka = keys, *kb = k2;
    int *va = vals, *vb = v2;
    const int passes = std::max(1, (bits + 7) / 8);
    for (int pass = 0; pass < passes; ++pass) {
        const int shift = 8 * pass;
        radix_hist_kernel<<<nblocks, kSortThreads, 0, st>>>(ka, n, shift, hist, nblocks);
        RZK_TRY(exclusive_scan_i32(hist, offs, hist_n, nullptr, scan_tmp, scan_bytes, st));
        radix_scatter_kernel<<<nblocks, kSortThreads, 0, st>>>(ka, va, n, shift, offs, nblocks, kb, vb);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    RZK_CUDA_TRY(cudaGetLastError());
    if (ka != keys) {
        RZK_CUDA_TRY(cudaMemcpyAsync(keys, ka, sizeof(uint32_t) * (size_t)n, cudaMemcpyDeviceToDevice, st));
        RZK_CUDA_TRY(cudaMemcpyAsync(vals, va, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, st));
    }
    return RZK_OK;
}

}  // namespace rzk
