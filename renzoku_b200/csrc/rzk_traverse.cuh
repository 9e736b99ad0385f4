// rzk_traverse.cuh - BVH traversal on the packed layout (device functions).
//
// Node slot s = BFS index + 1 holds two float4: {bmin.xyz, a}, {bmax.xyz, b}.  For an
// inner node a is its left child (the right child is a + 1, so both children are one
// contiguous, 64-byte-aligned 64-byte record); for a leaf a = -1 - sorted triangle slot.
// The stack holds these `a` codes, so popping an inner node costs a single 64-byte load
// that yields both child boxes and both children's own codes.
//
// Closest hit visits nodes in exactly the reference's order (aggregate_bvh.cc:402-448):
// pop, leaf -> triangle test that shrinks tmax, inner -> test left box then right box
// with the current tmax, push the ones that pass (right is popped first); the loops here
// go straight on to the entry that would be popped next instead of pushing and popping it.  Any-hit
// (aggregate_bvh.cc:452-478) returns whether any reachable triangle passes; its answer
// does not depend on visit order, so leaf children are tested as soon as their box
// passes instead of being pushed.  Both keep the reference's 64-entry stack, which drops
// pushes when full (holding one entry fewer per level than the reference's, it fills
// later); a drop sets ERR_STACK in the scene's error word.
#pragma once

#include "rzk_internal.cuh"

namespace rzk {

// Per-thread stack: STRIDE = 1 for a private array, STRIDE = block size for a stack
// interleaved in shared memory (entry k of thread t at [k * STRIDE + t]).
template <int STRIDE>
struct Stack {
    int *base;
    int top;
    __device__ __forceinline__ void init(int *b) { base = b; top = -1; }
    __device__ __forceinline__ bool empty() const { return top < 0; }
    __device__ __forceinline__ int pop() { return base[(top--) * STRIDE]; }
    __device__ __forceinline__ bool push(int v) {
        if (top < STACK_CAP - 1) { base[(++top) * STRIDE] = v; return true; }
        return false;
    }
};

struct TraceStats {
    uint32_t inner, leaf;
    __device__ __forceinline__ void reset() { inner = 0; leaf = 0; }
};

__device__ __forceinline__ void load_tri(const DevScene &s, int slot, float4 &a, float4 &b, float4 &c) {
    const float4 *p = s.tri_isect + 3 * slot;
    a = __ldg(p); b = __ldg(p + 1); c = __ldg(p + 2);
}

// TRAV: walk the any-hit tree (DevScene::trav) instead of the reference tree; the answer is
// the same (see rzk_sah.cu), only the visit order differs.
template <int STRIDE, bool STATS, bool TRAV = false>
__device__ __forceinline__ bool any_hit(const DevScene &s, const Ray &r, float tmin, float tmax,
                                        Stack<STRIDE> &stk, TraceStats *ts = nullptr) {
    if (s.n_nodes == 0) return false;
    const float4 *tree = TRAV ? s.trav : s.nodes;
    float4 lo = __ldg(tree + 2), hi = __ldg(tree + 3);
    if (!box_hit(lo, hi, r, tmin, tmax)) return false;
    int a = __float_as_int(lo.w);
    float4 ta, tb, tc;
    if (a < 0) {
        if (STATS) ts->leaf++;
        load_tri(s, -1 - a, ta, tb, tc);
        return tri_hit<false>(ta, tb, tc, r, tmin, tmax, nullptr, nullptr, nullptr);
    }
    // the loop continues into the child it would pop next (the right one where both are
    // entered) and pushes only the other: the visit order of pushing both, without a stack
    // store and load on each step's dependency chain
    stk.top = -1;
    int c = a;
    bool overflow = false;
    for (;;) {
        if (STATS) ts->inner++;
        const float4 *p = tree + 2 * (c + 1);
        float4 l0 = __ldg(p), l1 = __ldg(p + 1), r0 = __ldg(p + 2), r1 = __ldg(p + 3);
        bool hl = box_hit(l0, l1, r, tmin, tmax);
        bool hr = box_hit(r0, r1, r, tmin, tmax);
        int al = __float_as_int(l0.w), ar = __float_as_int(r0.w);
        if (hl && al < 0) {
            if (STATS) ts->leaf++;
            load_tri(s, -1 - al, ta, tb, tc);
            if (tri_hit<false>(ta, tb, tc, r, tmin, tmax, nullptr, nullptr, nullptr)) return true;
        }
        if (hr && ar < 0) {
            if (STATS) ts->leaf++;
            load_tri(s, -1 - ar, ta, tb, tc);
            if (tri_hit<false>(ta, tb, tc, r, tmin, tmax, nullptr, nullptr, nullptr)) return true;
        }
        const bool gl = hl && al >= 0, gr = hr && ar >= 0;
        if (gr) {
            if (gl && !stk.push(al)) overflow = true;
            c = ar;
        } else if (gl) {
            c = al;
        } else {
            if (stk.empty()) break;
            c = stk.pop();
        }
    }
    if (overflow && s.err) atomicOr(s.err, ERR_STACK);
    return false;
}

// Returns the sorted triangle slot of the closest hit or -1.
template <int STRIDE>
__device__ __forceinline__ int closest_hit(const DevScene &s, const Ray &r, float tmin, float tmax,
                                           Stack<STRIDE> &stk, float *t_out, float *beta_out,
                                           float *gamma_out) {
    if (s.n_nodes == 0) return -1;
    float4 lo = __ldg(s.nodes + 2), hi = __ldg(s.nodes + 3);
    if (!box_hit(lo, hi, r, tmin, tmax)) return -1;
    int best = -1;
    float bt = RAY_TMAX, bb = 0.0f, bg = 0.0f;
    bool overflow = false;
    // as any_hit: the loop continues into the entry it would pop next (the right child
    // where both boxes pass, each tested with the tmax of that moment) and pushes only the
    // other, so the nodes are visited in the reference's order
    stk.top = -1;
    int c = __float_as_int(lo.w);
    for (;;) {
        if (c < 0) {
            float4 ta, tb, tc;
            load_tri(s, -1 - c, ta, tb, tc);
            float t, b, g;
            if (tri_hit<true>(ta, tb, tc, r, tmin, tmax, &t, &b, &g)) {
                tmax = t;
                bt = t; bb = b; bg = g;
                best = -1 - c;
            }
            if (stk.empty()) break;
            c = stk.pop();
            continue;
        }
        const float4 *p = s.nodes + 2 * (c + 1);
        float4 l0 = __ldg(p), l1 = __ldg(p + 1), r0 = __ldg(p + 2), r1 = __ldg(p + 3);
        const bool hl = box_hit(l0, l1, r, tmin, tmax);
        const bool hr = box_hit(r0, r1, r, tmin, tmax);
        if (hr) {
            if (hl && !stk.push(__float_as_int(l0.w))) overflow = true;
            c = __float_as_int(r0.w);
        } else if (hl) {
            c = __float_as_int(l0.w);
        } else {
            if (stk.empty()) break;
            c = stk.pop();
        }
    }
    if (overflow && s.err) atomicOr(s.err, ERR_STACK);
    if (best >= 0) { *t_out = bt; *beta_out = bb; *gamma_out = bg; }
    return best;
}

struct HitGeo {
    V3 p, ng, ns;
    Onb uvn;
    int mat, light;
    float t;
};

// Triangle::fill_hit_record (triangle.cc:277-296) + Surface::fill_hit_record
// (surface.cc:62-96) + the hit point r.org() + t * r.dir().
__device__ __forceinline__ void fill_hit(const DevScene &s, const Ray &r, int slot, float t,
                                         float beta, float gamma, HitGeo &h) {
    float4 s0 = __ldg(s.tri_shade + 2 * slot), s1 = __ldg(s.tri_shade + 2 * slot + 1);
    V3 n = mk(s0.x, s0.y, s0.z), u = mk(s1.x, s1.y, s1.z);
    int4 sf = __ldg(s.surf + __float_as_int(s0.w));
    V3 normal = n;
    V3 dn = sub(n, n);
    V3 shading = unit(add(add(n, scl(dn, beta)), scl(dn, gamma)));
    if (sf.y & RZK_SURF_FLIPPED) { normal = neg(normal); shading = neg(shading); }
    if ((sf.y & RZK_SURF_TWO_SIDED) && dot(shading, r.d) > 0.0f) {
        if (sf.x >= 0) { shading = neg(shading); normal = neg(normal); }
    }
    h.uvn = onb_from_nu(shading, u);
    h.p = add(r.o, scl(r.d, t));
    h.ng = normal;
    h.ns = shading;
    h.mat = sf.x;
    h.light = sf.z;
    h.t = t;
}

__device__ __forceinline__ void write_receiver(const HitGeo &h, const Ray &r, rzk_receiver *o) {
    float w[24];
    st3(w + 0, h.p); st3(w + 3, h.ng); st3(w + 6, h.ns); st3(w + 9, neg(r.d));
    st3(w + 12, h.uvn.u); st3(w + 15, h.uvn.v); st3(w + 18, h.uvn.n);
    w[21] = __int_as_float(h.mat); w[22] = __int_as_float(h.light); w[23] = __int_as_float(1);
    float4 *dst = reinterpret_cast<float4 *>(o);
#pragma unroll
    for (int k = 0; k < 6; ++k) dst[k] = make_float4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
}

__device__ __forceinline__ void write_miss(rzk_receiver *o) {
    float4 *dst = reinterpret_cast<float4 *>(o);
    float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int k = 0; k < 5; ++k) dst[k] = z;
    dst[5] = make_float4(0.0f, __int_as_float(-1), __int_as_float(-1), __int_as_float(0));
}

// Camera::shoot_ray (camera.cc:52-65) followed by the Ray constructor.
__device__ __forceinline__ Ray camera_ray(const rzk_camera &c, int i, int j) {
    float H = (float)c.height;
    float px = (float)j + 0.5f;
    float py = H - 1 - (float)i + 0.5f;
    float fx = (px - c.cop[0]) / c.scale[0];
    float fy = (py - c.cop[1]) / c.scale[1];
    Onb o{ld3(c.u), ld3(c.v), ld3(c.n)};
    V3 dir = unit(l2w(o, mk(fx, fy, -c.focal)));
    return make_ray(ld3(c.eye), dir);
}

}  // namespace rzk
