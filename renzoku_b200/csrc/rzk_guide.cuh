// rzk_guide.cuh - LightSlice's direction sampler on the device: choosing the slice whose
// sampling record serves a receiver, and drawing / evaluating directions from that slice's
// Jensen map (lightslice.cc:1569-1707, 1930-2056, 2313-2377; kdtree_n.h:522-572).
#ifndef RZK_GUIDE_CUH_
#define RZK_GUIDE_CUH_

#include "rzk_sample.cuh"

struct rzk_lightslice;

namespace rzk {

// Device copy of a LightSlice's sampling state.
struct GuideDev {
    const int4 *kd;           // upper kd-tree: x = axis or -1 - slice, y/z children, w = plane bits
    const float *box;         // [slice][12]: 6-D box min, then max (the slice's data box)
    const float *rep_pos;     // [slice][3]: position of the slice representative
    const float *rec_uvn;     // [slice][9]: sampling record basis u, v, n
    const uint8_t *rec_valid; // [slice]: sampling record valid (VPL sum > 0)
    const float *prob;        // [slice][res][res]: DiscretePdf2D::probability
    const float *row_cdf;     // [slice][res]
    const float *col_cdf;     // [slice][res][res]
    const float *total;       // [slice]: DiscretePdf2D dist_total
    // Metropolis sampler (lightslice.cc:1427-1517, 1709-1928)
    const int *m_off;         // [slice + 1]: the slice's points
    const int *m_cell;        // [slice][m_grid^2 + 1]: first point of each cell (row-major)
    int m_grid;               // cells per side of the unit square
    const float2 *m_pt;       // per point: visible cluster direction on the record's unit square
    const float4 *m_rad;      // per point: cluster weight x R(slice, representative)
    const float *sum_f;       // [slice]: SamplingRecord sum_f = sum_vpl (estimate_sum)
    const int *c_off;         // [slice + 1]: the slice's clusters
    const float *c_cdf;       // per cluster: the slice's cluster distribution (CDF)
    const float *c_wi;        // per cluster [3]: direction to its representative
    const float4 *pool;       // [slice][pool_n]: chain states (direction, density)
    int pool_n;
    float density_radius;
    int n_kd, n_slices, res;
    float view_cos;           // cos(pi / 4) as the host computes it (view_similarity_cosine_max)
    float diag;               // scene box diagonal (map_vec6)
};

// Builds (once) and returns the device tables of `ls`.
rzk_status guide_tables(rzk_lightslice *ls, GuideDev *out, cudaStream_t st);

constexpr float kGuidePlaneBias = -1e-3f;   // KdTreeN::PLANE_BIAS
constexpr int kGuideStack = 64;

__device__ __forceinline__ float guide_box_dist(const GuideDev &G, int c, const float *p) {
    const float *b = G.box + 12 * (size_t)c;
    float sum = 0.0f;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        float x = smin(smax(p[i], b[i]), b[6 + i]);   // std::min(std::max(p, lo), hi)
        float d = x - p[i];
        sum += d * d;
    }
    return sum;
}

// A max-heap of cluster indices ordered by box distance, with libstdc++'s push_heap /
// pop_heap steps, so that equal distances leave the same elements as the reference's
// std::priority_queue.
template <int K>
struct SliceHeap {
    float d[K];
    int c[K];
    int size;
    __device__ __forceinline__ void sift_up(int hole, float vd, int vc) {
        int parent = (hole - 1) / 2;
        while (hole > 0 && d[parent] < vd) {
            d[hole] = d[parent];
            c[hole] = c[parent];
            hole = parent;
            parent = (hole - 1) / 2;
        }
        d[hole] = vd;
        c[hole] = vc;
    }
    __device__ __forceinline__ void push(float vd, int vc) {
        sift_up(size, vd, vc);
        size++;
    }
    __device__ __forceinline__ void pop() {
        const int len = size - 1;
        if (len > 0) {
            const float vd = d[len];
            const int vc = c[len];
            int hole = 0, second = 0;
            while (second < (len - 1) / 2) {
                second = 2 * (second + 1);
                if (d[second] < d[second - 1]) second--;
                d[hole] = d[second];
                c[hole] = c[second];
                hole = second;
            }
            if ((len & 1) == 0 && second == (len - 2) / 2) {
                second = 2 * (second + 1);
                d[hole] = d[second - 1];
                c[hole] = c[second - 1];
                hole = second - 1;
            }
            sift_up(hole, vd, vc);
        }
        size = len;
    }
};

// KdTreeN::find_nearest_cluster (kdtree_n.h:522-572): the k nearest slices by 6-D box
// distance, furthest first; the recursion is replayed with an explicit stack.  Returns the
// count, or -1 if the stack bound was hit.
template <int K>
__device__ int guide_nearest(const GuideDev &G, const float *p, int *out) {
    SliceHeap<K> h;
    h.size = 0;
    int node[kGuideStack], second[kGuideStack];
    float split[kGuideStack];
    int top = 0;
    node[0] = 0;
    second[0] = -2;   // -2: not entered yet
    while (top >= 0) {
        const int n = node[top];
        if (second[top] == -2) {
            const int4 nd = G.kd[n];
            if (nd.x < 0) {
                const int c = -1 - nd.x;
                const float dc = guide_box_dist(G, c, p);
                if (h.size < K) {
                    h.push(dc, c);
                } else if (dc < h.d[0]) {
                    h.pop();
                    h.push(dc, c);
                }
                --top;
                continue;
            }
            const float dist = p[nd.x] - __int_as_float(nd.w) + kGuidePlaneBias;
            const int first = dist <= 0.0f ? nd.y : nd.z;
            second[top] = dist <= 0.0f ? nd.z : nd.y;
            split[top] = dist;
            if (first >= 0) {
                if (top + 1 >= kGuideStack) return -1;
                ++top;
                node[top] = first;
                second[top] = -2;
            }
            continue;
        }
        // back from the first child
        const int s2 = second[top];
        const float dist = split[top];
        --top;
        if (s2 >= 0 && h.size > 0 && (h.size < K || h.d[0] > dist * dist)) {
            ++top;
            node[top] = s2;
            second[top] = -2;
        }
    }
    int k = 0;
    while (h.size > 0) {
        out[k++] = h.c[0];
        h.pop();
    }
    return k;
}

struct GuideRecv {
    V3 p, ns, wo;
    Onb uvn;
    int mat;
};

// map_vec6 (lightslice.cc:148-190): position, and the reflection direction (glossy) or the
// normal (diffuse) scaled by diagonal / 16.
__host__ __device__ inline void map_vec6(V3 p, V3 n, const rzk_material *m, V3 wo, float diag, float *out) {
    const float weight = 1.0f / 16.0f * diag;
    V3 d = n;
    if (m && (m->type == RZK_BSDF_PHONG || m->type == RZK_BSDF_WARD)) {
        // ISpecular::get_gloss_exponential (phong.h:49-51, ward.h:38-40)
        const float g = m->type == RZK_BSDF_PHONG ? m->p0 : smax(1.0f / m->p0, 1.0f / m->p1);
        V3 wr = sub(scl(n, 2.0f * dot(wo, n)), wo);
        const float gs = smin(4.0f, smax(1.0f, g / 1000.0f));
        d = scl(wr, gs);
    }
    out[0] = p.x; out[1] = p.y; out[2] = p.z;
    out[3] = d.x * weight; out[4] = d.y * weight; out[5] = d.z * weight;
}

__device__ __forceinline__ void map6(const GuideRecv &r, const rzk_material &m, float diag, float *out) {
    map_vec6(r.p, r.ns, &m, r.wo, diag, out);
}

__device__ __forceinline__ Onb guide_rec_onb(const GuideDev &G, int s) {
    const float *u = G.rec_uvn + 9 * (size_t)s;
    Onb o;
    o.u = mk(u[0], u[1], u[2]);
    o.v = mk(u[3], u[4], u[5]);
    o.n = mk(u[6], u[7], u[8]);
    return o;
}

// LightSlice::is_view_similar (lightslice.cc:87-121), same_local_wi
__device__ __forceinline__ bool guide_view_similar(const GuideDev &G, const Onb &a, const Onb &b) {
    if (dot(a.n, b.n) < G.view_cos) return false;
    if (dot(a.u, b.u) < G.view_cos) return false;
    return true;
}

template <int K>
__device__ __forceinline__ int guide_pick(const GuideDev &G, const GuideRecv &r, const float *p6) {
    int idx[K];
    const int n = guide_nearest<K>(G, p6, idx);
    float min_dist = 3.402823466e38f;
    int best = -1;
    for (int i = 0; i < n; ++i) {
        const int s = idx[i];
        if (G.rec_valid[s] && guide_view_similar(G, guide_rec_onb(G, s), r.uvn)) {
            const float *q = G.rep_pos + 3 * (size_t)s;
            const float d = len(sub(mk(q[0], q[1], q[2]), r.p));
            if (d < min_dist) {
                min_dist = d;
                best = s;
            }
        }
    }
    return best;
}

// the slice of multi_slice_sample / multi_slice_pdf: the nearest valid, view-similar slice
// among the nearest one, else among the 32 nearest; -1 if none
__device__ __forceinline__ int guide_slice(const GuideDev &G, const GuideRecv &r, const float *p6) {
    int s = guide_pick<1>(G, r, p6);
    if (s < 0) s = guide_pick<32>(G, r, p6);
    return s;
}

// concentric_mapping.h:13-98
__device__ __forceinline__ void guide_square_to_disk(float sx, float sy, float &u, float &v) {
    float phi, r;
    const float a = 2.0f * sx - 1.0f;
    const float b = 2.0f * sy - 1.0f;
    if (a > -b) {
        if (a > b) { r = a; phi = (A_PI / 4) * (b / a); }
        else { r = b; phi = (A_PI / 4) * (2 - (a / b)); }
    } else {
        if (a < b) { r = -a; phi = (A_PI / 4) * (4 + (b / a)); }
        else {
            r = -b;
            if (b != 0.0f) phi = (A_PI / 4) * (6 - (a / b));
            else phi = 0.0f;
        }
    }
    u = r * cosf(phi);
    v = r * sinf(phi);
}

__device__ __forceinline__ V3 guide_square_to_direction(float sx, float sy) {
    float dx, dy;
    guide_square_to_disk(sx, sy, dx, dy);
    const float r2 = dx * dx + dy * dy;
    return mk(dx * sqrtf(2.0f - r2), dy * sqrtf(2.0f - r2), 1.0f - r2);
}

__device__ __forceinline__ void guide_direction_to_square(V3 w, float &sx, float &sy) {
    const float r2 = 1.0f - w.z;
    const float dx = w.x / sqrtf(2.0f - r2);
    const float dy = w.y / sqrtf(2.0f - r2);
    const float r = sqrtf(dx * dx + dy * dy);
    float phi = atan2f(dy, dx);
    if (phi < -A_PI / 4) phi += TWO_PI;
    float a, b;
    if (phi < A_PI / 4) { a = r; b = phi * a / (A_PI / 4); }
    else if (phi < 3 * A_PI / 4) { b = r; a = -(phi - A_PI / 2) * b / (A_PI / 4); }
    else if (phi < 5 * A_PI / 4) { a = -r; b = (phi - A_PI) * a / (A_PI / 4); }
    else { b = -r; a = -(phi - 3 * A_PI / 2) * b / (A_PI / 4); }
    sx = a * 0.5f + 0.5f;
    sy = b * 0.5f + 0.5f;
}

// Onb::spherical_to_world (onb.cc:157-164)
__device__ __forceinline__ V3 guide_spherical(const Onb &o, float theta, float phi) {
    const float st = sinf(theta), ct = cosf(theta), sp = sinf(phi), cp = cosf(phi);
    return l2w(o, mk(st * cp, st * sp, ct));
}

// LightSlice::pdf_map (lightslice.cc:2350-2377)
__device__ __forceinline__ float guide_pdf_map(const GuideDev &G, int s, V3 dir) {
    const Onb rec = guide_rec_onb(G, s);
    const V3 lw = w2l(rec, dir);
    if (lw.z <= 0.0f) return 0.0f;
    if (!(G.total[s] > 0.0f)) return INV_2PI;
    float sx, sy;
    guide_direction_to_square(lw, sx, sy);
    const int res = G.res;
    int col = (int)(sx * res), row = (int)(sy * res);
    if (col >= res) col = res - 1;
    if (row >= res) row = res - 1;
    float pdf_k = 0.0f;
    if (row >= 0 && col >= 0) pdf_k = G.prob[((size_t)s * res + row) * res + col];
    const int num_pixels = res * res;
    const float pdf_unit_square = num_pixels * pdf_k;
    const float pdf_unit_disk = pdf_unit_square * INV_PI;
    return pdf_unit_disk * 0.5f;
}

// LightSlice::multi_slice_pdf (lightslice.cc:1930-2056) with JENSEN maps; `s` is
// guide_slice(G, r, p6) (a function of the receiver alone, so callers compute it once)
__device__ __forceinline__ float guide_pdf_at(const GuideDev &G, const GuideRecv &r, int s, V3 wi) {
    if (r.mat < 0) return 0.0f;
    if (dot(r.ns, wi) <= 0.0f) return 0.0f;
    if (s < 0) return INV_2PI;
    const V3 dir = l2w(guide_rec_onb(G, s), w2l(r.uvn, wi));
    return guide_pdf_map(G, s, dir);
}

__device__ __forceinline__ float guide_pdf(const GuideDev &G, const GuideRecv &r, const float *p6, V3 wi) {
    if (r.mat < 0 || dot(r.ns, wi) <= 0.0f) return 0.0f;
    return guide_pdf_at(G, r, guide_slice(G, r, p6), wi);
}

// LightSlice::multi_slice_sample (lightslice.cc:1569-1707) with sample_map
// (lightslice.cc:2313-2348); returns the receiver's BRDF for the drawn direction.  `s` is
// guide_slice(G, r, p6).
__device__ __forceinline__ Rgb guide_sample_at(const GuideDev &G, const GuideRecv &r, const rzk_material &m,
                                               int s, Rng &g, V3 &wi, float &pdf) {
    if (r.mat < 0) {
        wi = mk(0.0f, 0.0f, 0.0f);
        pdf = 0.0f;
        return crgb(0.0f, 0.0f, 0.0f);
    }
    if (s < 0) {   // no usable record: uniform hemisphere at the receiver
        const float sx = g.uniform(), sy = g.uniform();
        const float phi = TWO_PI * sx;
        const float theta = acosf(sy);
        wi = unit(guide_spherical(r.uvn, theta, phi));
        pdf = INV_2PI;
        return brdf_eval(m, r.uvn, r.wo, wi);
    }
    const Onb rec = guide_rec_onb(G, s);
    V3 ws;
    if (!(G.total[s] > 0.0f)) {
        const float sx = g.uniform(), sy = g.uniform();
        const float phi = TWO_PI * sx;
        const float theta = acosf(sy);
        ws = unit(guide_spherical(rec, theta, phi));
    } else {
        const int res = G.res;
        const float u0 = g.uniform(), u1 = g.uniform();   // Vec2::random: x then y
        int row = -1, col = -1;
        const float *rc = G.row_cdf + (size_t)s * res;
        for (int i = 0; i < res; ++i)
            if (u0 < rc[i]) { row = i; break; }
        if (row >= 0) {
            const float *cc = G.col_cdf + ((size_t)s * res + row) * res;
            for (int j = 0; j < res; ++j)
                if (u1 < cc[j]) { col = j; break; }
        }
        if (row < 0 || col < 0) {
            ws = mk(0.0f, 0.0f, 0.0f);
        } else {
            const float jx = g.uniform(), jy = g.uniform();
            const float sx = (col + jx) / res, sy = (row + jy) / res;
            ws = l2w(rec, guide_square_to_direction(sx, sy));
        }
    }
    wi = l2w(r.uvn, w2l(rec, ws));   // same local direction at the receiver
    pdf = guide_pdf_at(G, r, s, wi);
    return brdf_eval(m, r.uvn, r.wo, wi);
}

// LightSlice::eval_incoming_radiance with FIXED_RADIUS (lightslice.cc:1427-1517): the
// radiance of the slice's points strictly within density_radius of x on the unit square
// (KdTree2::find_nearest with a radius, kdtree_2.cc:203-234, finds exactly these), its
// luminance (Rgb::luminance, the norm, rgb.h:57) plus density_epsilon_ratio (1e-2) x sum_vpl
// The cells a query at (x, y) reads: rows [*y0, *y1], columns [*x0, *x1] of the grid, padded
// by a little so that rounding of (x +- r) * grid never drops a cell holding a point within r
// (the distance test decides membership).
__device__ __forceinline__ void guide_cells(const GuideDev &G, float x, float y, int &x0, int &x1, int &y0,
                                            int &y1) {
    const float r = G.density_radius, n = (float)G.m_grid;
    x0 = max(0, (int)floorf((x - r) * n - 1e-3f));
    x1 = min(G.m_grid - 1, (int)floorf((x + r) * n + 1e-3f));
    y0 = max(0, (int)floorf((y - r) * n - 1e-3f));
    y1 = min(G.m_grid - 1, (int)floorf((y + r) * n + 1e-3f));
}

__device__ __forceinline__ float guide_density(const GuideDev &G, int s, float x, float y) {
    const float r2 = G.density_radius * G.density_radius;
    float sr = 0.0f, sg = 0.0f, sb = 0.0f;
    int x0, x1, y0, y1;
    guide_cells(G, x, y, x0, x1, y0, y1);
    const int *cell = G.m_cell + (size_t)s * (G.m_grid * G.m_grid + 1);
    for (int cy = y0; cy <= y1; ++cy) {
        for (int i = cell[cy * G.m_grid + x0], e = cell[cy * G.m_grid + x1 + 1]; i < e; ++i) {
            const float2 q = G.m_pt[i];
            const float dx = q.x - x, dy = q.y - y;
            if (dx * dx + dy * dy < r2) {
                const float4 c = G.m_rad[i];
                sr += c.x;
                sg += c.y;
                sb += c.z;
            }
        }
    }
    return 1e-2f * G.sum_f[s] + sqrtf(sr * sr + sg * sg + sb * sb);
}

// LightSlice::metropolis_get_pdf (lightslice.cc:1913-1928) at a world direction
__device__ __forceinline__ float guide_metro_pdf_map(const GuideDev &G, int s, V3 dir) {
    const V3 lw = w2l(guide_rec_onb(G, s), dir);
    if (lw.z <= 0.0f) return 0.0f;
    const float sum = G.sum_f[s];
    if (!(sum > 0.0f)) return 0.0f;
    float sx, sy;
    guide_direction_to_square(lw, sx, sy);
    return guide_density(G, s, sx, sy) / sum;
}

// LightSlice::multi_slice_pdf (lightslice.cc:1930-2056) with the METROPOLIS sampler
__device__ __forceinline__ float guide_metro_pdf_at(const GuideDev &G, const GuideRecv &r, int s, V3 wi) {
    if (r.mat < 0) return 0.0f;
    if (dot(r.ns, wi) <= 0.0f) return 0.0f;
    if (s < 0) return INV_2PI;
    const V3 dir = l2w(guide_rec_onb(G, s), w2l(r.uvn, wi));
    return guide_metro_pdf_map(G, s, dir);
}

// LightSlice::multi_slice_sample (lightslice.cc:1569-1707) with metropolis_fetch_cached_sample
// (lightslice.cc:1709-1761): a state of the slice's chain, drawn uniformly from the pool the
// chain kernel filled (the reference hands out its 1,024-state caches in shuffled order);
// the pdf is the density over sum_f, not the chain's.  Returns the receiver's BRDF.
__device__ __forceinline__ Rgb guide_metro_sample_at(const GuideDev &G, const GuideRecv &r, const rzk_material &m,
                                                     int s, Rng &g, V3 &wi, float &pdf) {
    if (r.mat < 0) {
        wi = mk(0.0f, 0.0f, 0.0f);
        pdf = 0.0f;
        return crgb(0.0f, 0.0f, 0.0f);
    }
    if (s < 0) {   // no usable record: uniform hemisphere at the receiver
        const float sx = g.uniform(), sy = g.uniform();
        const float phi = TWO_PI * sx;
        const float theta = acosf(sy);
        wi = unit(guide_spherical(r.uvn, theta, phi));
        pdf = INV_2PI;
        return brdf_eval(m, r.uvn, r.wo, wi);
    }
    int k = (int)(g.uniform() * G.pool_n);
    if (k >= G.pool_n) k = G.pool_n - 1;
    const float4 st = G.pool[(size_t)s * G.pool_n + k];
    const V3 ws = mk(st.x, st.y, st.z);
    wi = l2w(r.uvn, w2l(guide_rec_onb(G, s), ws));   // same local direction at the receiver
    pdf = guide_metro_pdf_at(G, r, s, wi);
    return brdf_eval(m, r.uvn, r.wo, wi);
}

}  // namespace rzk

#endif  // RZK_GUIDE_CUH_
