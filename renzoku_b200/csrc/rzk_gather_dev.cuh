// rzk_gather_dev.cuh - device building blocks of the gather kernels (rzk_gather.cu,
// rzk_batch.cu): bulk-copy / mbarrier helpers, receiver and material loads, the exact-zero
// pair test, the pair's radiance, the warp-packet any-hit and one persistent work item.
#pragma once

#include "rzk_traverse.cuh"

namespace rzk {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Bounded wait on a bulk-copy barrier: gives up after ~2^24 polls and reports it.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t *err) {
    for (uint32_t it = 0; it < (1u << 24); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicOr(err, ERR_TIMEOUT);
    return false;
}

struct RecvRegs {
    V3 p, ng, ns, wo;
    Onb uvn;
    int mat;
};

__device__ __forceinline__ RecvRegs load_receiver(const rzk_receiver *r) {
    const float4 *q = reinterpret_cast<const float4 *>(r);
    float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3), e = __ldg(q + 4),
           f = __ldg(q + 5);
    RecvRegs o;
    o.p = mk(a.x, a.y, a.z);
    o.ng = mk(a.w, b.x, b.y);
    o.ns = mk(b.z, b.w, c.x);
    o.wo = mk(c.y, c.z, c.w);
    o.uvn.u = mk(d.x, d.y, d.z);
    o.uvn.v = mk(d.w, e.x, e.y);
    o.uvn.n = mk(e.z, e.w, f.x);
    o.mat = __float_as_int(f.y);
    return o;
}

// r with its tangent basis vectors u, v read again from the receiver record
__device__ __forceinline__ RecvRegs reload_basis(RecvRegs r, const rzk_receiver *rec) {
    const float4 *q = reinterpret_cast<const float4 *>(rec);
    const float4 d = __ldg(q + 3), e = __ldg(q + 4);
    r.uvn.u = mk(d.x, d.y, d.z);
    r.uvn.v = mk(d.w, e.x, e.y);
    return r;
}

__device__ __forceinline__ rzk_material load_material(const rzk_material *m) {
    const float4 *q = reinterpret_cast<const float4 *>(m);
    float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
    rzk_material o;
    o.type = __float_as_int(a.x);
    o.kd[0] = a.y; o.kd[1] = a.z; o.kd[2] = a.w;
    o.ks[0] = b.x; o.ks[1] = b.y; o.ks[2] = b.z;
    o.p0 = b.w; o.p1 = c.x;
    o.pad[0] = o.pad[1] = o.pad[2] = 0.0f;
    return o;
}

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ bool finite3(Rgb c) {
    return isfinite(c.r) && isfinite(c.g) && isfinite(c.b);
}

// Receiver index of a lane: a TW x (32 / TW) pixel tile of a row-major image of width
// img_w (8 x 4 by default; the autotuner also tries 4 x 8, 16 x 2 and 32 x 1), or 32
// consecutive receivers when img_w == 0.  -1 outside the receiver range.
template <int TW = 8>
__device__ __forceinline__ int lane_receiver(int gwarp, int lane, int n_recv, int img_w) {
    static_assert(TW == 4 || TW == 8 || TW == 16 || TW == 32, "warp tile width");
    constexpr int TH = 32 / TW;
    if (img_w <= 0) {
        int ri = gwarp * 32 + lane;
        return ri < n_recv ? ri : -1;
    }
    int tiles_x = (img_w + TW - 1) / TW;
    int x = (gwarp % tiles_x) * TW + (lane % TW);
    int y = (gwarp / tiles_x) * TH + (lane / TW);
    if (x >= img_w) return -1;
    long long ri = (long long)y * img_w + x;
    return ri < n_recv ? (int)ri : -1;
}

struct PairGeo {
    V3 q;
    float G;
    V3 wi;
    Rgb power;
};

// The VPL-only facts the per-pair tests use: its power is finite (all three components),
// and it was reached from behind its surface (a BRDF VPL whose stored incident direction
// makes a cosine <= ZERO_EPSILON with its normal: its BRDF's early-out then fires for every
// receiver).  The gathers form them once per VPL, one VPL per lane, instead of in every
// lane for every VPL.
__device__ __forceinline__ bool vpl_power_finite(const rzk_vpl &l) {
    return isfinite(l.contrib[0]) && isfinite(l.contrib[1]) && isfinite(l.contrib[2]);
}
__device__ __forceinline__ bool vpl_from_behind(const rzk_vpl &l) {
    return l.mat >= 0 && dot(ld3(l.wi), ld3(l.nn)) <= ZERO_EPSILON;
}

// Geometry of a pair and the exact-zero test of its term: returns false when either
// BRDF's early-out makes the term exactly zero (G and the power finite).  `fin` and
// `behind` are vpl_power_finite(l) and vpl_from_behind(l).
__device__ __forceinline__ bool pair_survives(const RecvRegs &r, const rzk_vpl &l, PairGeo &pg, bool fin,
                                              bool behind) {
    pg.q = ld3(l.p);
    pg.G = form_factor_abs(r.p, r.ns, pg.q, ld3(l.n));
    pg.wi = unit(sub(pg.q, r.p));
    pg.power = crgb(l.contrib[0], l.contrib[1], l.contrib[2]);
    if (isfinite(pg.G) && fin) {
        if (dot(pg.wi, r.uvn.n) <= ZERO_EPSILON || dot(r.wo, r.uvn.n) <= ZERO_EPSILON) return false;
        if (behind) return false;
        if (l.mat >= 0 && dot(neg(pg.wi), ld3(l.nn)) <= ZERO_EPSILON) return false;
    }
    return true;
}

__device__ __forceinline__ bool pair_survives(const RecvRegs &r, const rzk_vpl &l, PairGeo &pg) {
    return pair_survives(r, l, pg, vpl_power_finite(l), vpl_from_behind(l));
}

// A cheaper first test that implies pair_survives' "exactly zero" answer: no division or
// square root.  It returns true only where G and the power are certainly finite and one of
// the BRDF early-outs certainly fires: the receiver sees its surface from behind or the VPL
// was reached from behind its surface (the same dot products pair_survives tests, exactly),
// or the VPL lies behind the receiver's surface / the receiver behind the VPL's, judged on
// the unnormalised direction d = q - p with a margin: dot(d, n) <= -4e-6 |d| puts the
// rounded dot(unit(d), n) below -2e-6, under ZERO_EPSILON whatever the rounding of either
// product (each within ~1e-6 of exact for unit normals).  Pairs it passes go through
// pair_survives, so the set of surviving pairs is unchanged.  `fin` and `behind` as for
// pair_survives.
__device__ __forceinline__ bool pair_clearly_zero(const RecvRegs &r, const rzk_vpl &l, bool fin, bool behind) {
    const V3 d = sub(ld3(l.p), r.p);
    const float dd = dot(d, d);
    if (!(dd >= 1e-18f && dd <= 1e30f)) return false;
    if (!fin) return false;
    // G = |d1 d2| / dd^2 finite: d1 d2 finite and at most 1e30 dd^2
    const float g = dot(r.ns, d) * dot(ld3(l.n), d);
    if (!(fabsf(g) <= dd * dd * 1e30f)) return false;
    if (dot(r.wo, r.uvn.n) <= ZERO_EPSILON) return true;
    const float m2 = 1.6e-11f * dd;   // (4e-6)^2 |d|^2
    const float a = dot(d, r.uvn.n);
    if (a < 0.0f && a * a >= m2) return true;
    if (behind) return true;
    if (l.mat >= 0) {
        const float b = dot(d, ld3(l.nn));
        if (b > 0.0f && b * b >= m2) return true;
    }
    return false;
}

__device__ __forceinline__ bool pair_clearly_zero(const RecvRegs &r, const rzk_vpl &l) {
    return pair_clearly_zero(r, l, vpl_power_finite(l), vpl_from_behind(l));
}

__device__ __forceinline__ Rgb pair_radiance(const DevScene &s, const RecvRegs &r, const rzk_material &rm,
                                             const rzk_vpl &l, const PairGeo &pg, int mode, float tau) {
    Rgb sb = brdf_eval(rm, r.uvn, r.wo, pg.wi);
    Rgb lb;
    if (l.mat >= 0) {
        rzk_material lm = load_material(s.mats + l.mat);
        Onb lu{ld3(l.u), ld3(l.v), ld3(l.nn)};
        lb = brdf_eval(lm, lu, ld3(l.wi), neg(pg.wi));
    } else {
        lb = crgb(1.0f, 1.0f, 1.0f);
    }
    return radiance_terms(pg.power, sb, lb, pg.G, mode, tau);
}

// Packet any-hit, nearer child first by lane majority.  Returns whether this lane's
// segment is unoccluded (lanes with act == false return false).
// `cache` and `cache2` (per lane) name the any-hit-tree leaves whose triangles last
// occluded this lane's receiver (most recent first), or -1.  They are tried first, then the
// leaves cached by five neighbouring lanes: a triangle whose own box and triangle tests pass
// occludes the segment whichever way it was found, so a hit there is the traversal's
// answer; the leaf of any triangle found becomes the lane's `cache`, the previous one its
// `cache2`.
__device__ __forceinline__ bool packet_visible_near(const DevScene &s, const Ray &ray, float tmax, bool act,
                                                    int *stk, int &cache, int &cache2) {
    if (s.n_nodes == 0) return act;
    const float4 lo = __ldg(s.trav + 2), hi = __ldg(s.trav + 3);
    float t_root = 0.0f;
    bool alive = act && box_hit_fast(lo, hi, ray, s.tmin, tmax, t_root);
    if (!__any_sync(kFull, alive)) return act;
    const int a = __float_as_int(lo.w);
    if (a < 0) {
        if (alive) {
            float4 ta, tb, tc;
            load_tri(s, -1 - a, ta, tb, tc);
            if (tri_hit<false>(ta, tb, tc, ray, s.tmin, tmax, nullptr, nullptr, nullptr)) return false;
        }
        return act;
    }
    bool occluded = false;
    if (alive && cache >= 0) {
        const float4 *pc = s.trav + 2 * (cache + 1);
        const float4 c0 = __ldg(pc), c1 = __ldg(pc + 1);
        float tc0 = 0.0f;
        if (box_hit_fast(c0, c1, ray, s.tmin, tmax, tc0)) {
            float4 ta, tb, tc;
            load_tri(s, -1 - __float_as_int(c0.w), ta, tb, tc);
            if (tri_hit<false>(ta, tb, tc, ray, s.tmin, tmax, nullptr, nullptr, nullptr)) occluded = true;
        }
    }
    if (alive && !occluded && cache2 >= 0 && cache2 != cache) {   // the one before it
        const float4 *pc = s.trav + 2 * (cache2 + 1);
        const float4 c0 = __ldg(pc), c1 = __ldg(pc + 1);
        float tc0 = 0.0f;
        if (box_hit_fast(c0, c1, ray, s.tmin, tmax, tc0)) {
            float4 ta, tb, tc;
            load_tri(s, -1 - __float_as_int(c0.w), ta, tb, tc);
            if (tri_hit<false>(ta, tb, tc, ray, s.tmin, tmax, nullptr, nullptr, nullptr)) {
                occluded = true;
                const int t = cache;
                cache = cache2;
                cache2 = t;
            }
        }
    }
    // Then the leaves cached by the lanes at xor distances 1, 8, 2, 16 and 4: in an 8 x 4
    // pixel tile those are the neighbouring pixels, whose shadow rays toward the same VPL
    // run almost parallel and are often blocked by the same triangle.  The same rule
    // applies (own box and triangle tests), so the answer is still exact; a lane blocked by
    // a neighbour's leaf adopts it.  Every lane takes part in each shuffle.
    constexpr int kNeighbours[5] = {1, 8, 2, 16, 4};
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        const int other = __shfl_xor_sync(kFull, cache, kNeighbours[q]);
        if (alive && !occluded && other >= 0 && other != cache) {
            const float4 *pc = s.trav + 2 * (other + 1);
            const float4 c0 = __ldg(pc), c1 = __ldg(pc + 1);
            float tc0 = 0.0f;
            if (box_hit_fast(c0, c1, ray, s.tmin, tmax, tc0)) {
                float4 ta, tb, tc;
                load_tri(s, -1 - __float_as_int(c0.w), ta, tb, tc);
                if (tri_hit<false>(ta, tb, tc, ray, s.tmin, tmax, nullptr, nullptr, nullptr)) {
                    occluded = true;
                    cache2 = cache;
                    cache = other;
                }
            }
        }
    }
    // every lane takes part in the vote (the cache tests above are per lane)
    alive = alive && !occluded;
    if (!__any_sync(kFull, alive)) return act && !occluded;
    // lanes whose root test failed cannot reach any triangle below it: they stay visible.
    // The warp descends straight into the child it visits next (the nearer one where both
    // are entered) and pushes only the other: the visit order of a push-both stack, without
    // a shared-memory store and load on the step's dependency chain.
    int top = -1;
    int c = a;
    bool overflow = false;
    for (;;) {
        const float4 *pn = s.trav + 2 * (c + 1);
        const float4 l0 = __ldg(pn), l1 = __ldg(pn + 1), r0 = __ldg(pn + 2), r1 = __ldg(pn + 3);
        const int al = __float_as_int(l0.w), ar = __float_as_int(r0.w);
        float tl = 0.0f, tr = 0.0f;
        bool hl = alive && box_hit_fast(l0, l1, ray, s.tmin, tmax, tl);
        bool hr = alive && box_hit_fast(r0, r1, ray, s.tmin, tmax, tr);
        if (al < 0 && hl && !occluded) {
            float4 ta, tb, tc;
            load_tri(s, -1 - al, ta, tb, tc);
            if (tri_hit<false>(ta, tb, tc, ray, s.tmin, tmax, nullptr, nullptr, nullptr)) {
                occluded = true;
                if (cache != c) { cache2 = cache; cache = c; }
            }
        }
        if (ar < 0 && hr && !occluded) {
            float4 ta, tb, tc;
            load_tri(s, -1 - ar, ta, tb, tc);
            if (tri_hit<false>(ta, tb, tc, ray, s.tmin, tmax, nullptr, nullptr, nullptr)) {
                occluded = true;
                if (cache != c + 1) { cache2 = cache; cache = c + 1; }
            }
        }
        alive = alive && !occluded;
        const bool pl = al >= 0 && __any_sync(kFull, hl && alive);
        const bool pr = ar >= 0 && __any_sync(kFull, hr && alive);
        if (!__any_sync(kFull, alive)) break;
        if (pl && pr) {
            // visit the child most live lanes enter first; the other waits on the stack
            unsigned left_first = __ballot_sync(kFull, alive && hl && hr && tl <= tr);
            unsigned right_first = __ballot_sync(kFull, alive && hl && hr && tr < tl);
            const int first = __popc(left_first) >= __popc(right_first) ? al : ar;
            if (top < STACK_CAP - 1) stk[++top] = first == al ? ar : al; else overflow = true;
            c = first;
        } else if (pl) {
            c = al;
        } else if (pr) {
            c = ar;
        } else {
            if (top < 0) break;
            c = stk[top--];
        }
    }
    if (overflow && s.err) atomicOr(s.err, ERR_STACK);
    return act && !occluded;
}


// Per-warp staging state of the persistent gathers: the warp's two VPL tiles, their
// barriers (with the number of completed phases of each) and its packet stack.
template <int TILE>
struct WarpStage {
    rzk_vpl (*tl)[TILE];
    uint64_t *mb;
    int *stk;
    uint32_t uses[2];
    __device__ __forceinline__ void init(rzk_vpl (*tiles)[TILE], uint64_t *bar, int *stack, int lane) {
        tl = tiles;
        mb = bar;
        stk = stack;
        uses[0] = uses[1] = 0u;
        if (lane == 0) {
            mbar_init(&mb[0], 1);
            mbar_init(&mb[1], 1);
            fence_barrier_init();
        }
        __syncwarp();
    }
};

// Warp tiles of an image (TW x (32 / TW) pixels each), or of 32 consecutive receivers
// without an image width.
template <int TW = 8>
__host__ __device__ __forceinline__ long long warp_tiles(long long n_recv, int img_w) {
    if (img_w <= 0) return (n_recv + 31) / 32;
    const long long img_h = (n_recv + img_w - 1) / img_w;
    return (long long)((img_w + TW - 1) / TW) * ((img_h + 32 / TW - 1) / (32 / TW));
}

// One work item of the persistent gathers: the 32 receivers of warp tile `wt` against VPL
// chunk `chunk`.  Each lane hands `sink(ri, sum, ok)` its receiver's index (-1 for none)
// and the sum of its terms over the chunk's VPLs in VPL order (zero without a receiver);
// ok is false, and the sum incomplete, if a bounded wait gave up (reported in the error
// word), and the item then returns false.  The tile shape changes which receivers share a
// packet, never a receiver's sum.
template <int TILE, int TW = 8, class Sink>
__device__ __forceinline__ bool gather_item(const DevScene &s, const rzk_receiver *recv, int n_recv, int img_w,
                                            const rzk_vpl *vpls, int n_vpl, int chunk, int wt, int chunk_len,
                                            int mode, float tau, WarpStage<TILE> &ws, int lane, Sink &&sink) {
    const int ri = lane_receiver<TW>(wt, lane, n_recv, img_w);
    const int j0 = chunk * chunk_len;
    const int j1 = min(n_vpl, j0 + chunk_len);
    const int n_tiles = (j1 - j0 + TILE - 1) / TILE;

    RecvRegs r;
    r.p = mk(0.0f, 0.0f, 0.0f);   // lanes without a receiver still form (unused) rays
    bool active = false;
    if (ri >= 0) {
        r = load_receiver(recv + ri);
        active = r.mat >= 0;
    }
    // a tile of inactive lanes, or an empty chunk, contributes nothing: no VPL stream (an
    // empty chunk must not arm a barrier phase that no wait consumes)
    if (n_tiles <= 0 || !__any_sync(kFull, active)) {
        sink(ri, crgb(0.0f, 0.0f, 0.0f), true);
        return true;
    }
    Rgb sum = crgb(0.0f, 0.0f, 0.0f);
    unsigned long long n_rays = 0;         // shadow rays of this item (lane 0's count)
    int occ_cache = -1, occ_cache2 = -1;   // this lane's last two occluders (any-hit tree leaves)
    if (lane == 0) {
        int cnt = min(TILE, j1 - j0);
        fence_proxy_async();
        mbar_expect_tx(&ws.mb[0], cnt * (uint32_t)sizeof(rzk_vpl));
        bulk_g2s(&ws.tl[0][0], vpls + j0, cnt * (uint32_t)sizeof(rzk_vpl), &ws.mb[0]);
    }
    for (int k = 0; k < n_tiles; ++k) {
        const int buf = k & 1;
        if (lane == 0 && k + 1 < n_tiles) {
            int jn = j0 + (k + 1) * TILE;
            int cnt = min(TILE, j1 - jn);
            fence_proxy_async();
            mbar_expect_tx(&ws.mb[buf ^ 1], cnt * (uint32_t)sizeof(rzk_vpl));
            bulk_g2s(&ws.tl[buf ^ 1][0], vpls + jn, cnt * (uint32_t)sizeof(rzk_vpl), &ws.mb[buf ^ 1]);
        }
        bool ok = mbar_wait_bounded(&ws.mb[buf], ws.uses[buf] & 1u, lane == 0 ? s.err : nullptr);
        ws.uses[buf]++;
        if (__any_sync(kFull, !ok)) {
            sink(ri, sum, false);
            return false;
        }
        const rzk_vpl *tile = ws.tl[buf];
        const int cnt = min(TILE, j1 - (j0 + k * TILE));
        // the VPL-only facts of the tile's VPLs, one VPL per lane
        static_assert(TILE <= 32, "one VPL per lane");
        const rzk_vpl &mine = tile[lane < cnt ? lane : 0];
        const unsigned fin_mask = __ballot_sync(kFull, lane < cnt && vpl_power_finite(mine));
        const unsigned behind_mask = __ballot_sync(kFull, lane < cnt && vpl_from_behind(mine));
        for (int v = 0; v < cnt; ++v) {
            const rzk_vpl &l = tile[v];
            const bool fin = (fin_mask >> v) & 1u, behind = (behind_mask >> v) & 1u;
            if (!__any_sync(kFull, active && !pair_clearly_zero(r, l, fin, behind))) continue;
            PairGeo pg;
            bool act = active && pair_survives(r, l, pg, fin, behind);
            const unsigned am = __ballot_sync(kFull, act);
            if (!am) continue;
            n_rays += (unsigned)__popc(am);
            Ray ray = make_ray(r.p, sub(pg.q, r.p));
            float tmax = len(sub(pg.q, r.p)) - s.tmin;
            if (packet_visible_near(s, ray, tmax, act, ws.stk, occ_cache, occ_cache2)) {
                // the pair's geometry (recomputed: the same operations on the same values),
                // the material and the receiver's tangent basis are read or formed again here
                // rather than held in registers through the traversal
                PairGeo pv;
                pair_survives(r, l, pv, fin, behind);
                sum = cadd(sum, pair_radiance(s, reload_basis(r, recv + ri), load_material(s.mats + r.mat), l, pv,
                                              mode, tau));
            }
        }
        __syncwarp();
    }
    if (lane == 0 && s.rays && n_rays) atomicAdd(s.rays, n_rays);
    sink(ri, sum, true);
    return true;
}

// Sink of gather_item writing an item's partial sums to chunk `chunk`'s plane of `partial`
// (planes of n_recv x 3 floats); nothing is written for an item whose wait gave up.
struct PlaneSink {
    float *partial;
    int n_recv, chunk;
    __device__ __forceinline__ void operator()(int ri, Rgb sum, bool ok) const {
        if (ok && ri >= 0) {
            // partial sums are read once by the chunk reduction: streaming stores keep them
            // from displacing the traversal working set in L2
            float *o = partial + 3 * ((size_t)chunk * n_recv + ri);
            __stcs(o, sum.r); __stcs(o + 1, sum.g); __stcs(o + 2, sum.b);
        }
    }
};

// Visibility half of gather_item, for gathers split into a tracing pass and a summing
// pass: the 32 receivers of warp tile `wt` (img_w as in lane_receiver) against VPLs [j0, j1); masks[j - j0] = ballot of
// the lanes whose pair's term is not exactly zero (pair_survives) and whose shadow segment
// is unoccluded - exactly the pairs gather_item adds.  Returns false if a bounded wait gave
// up (reported in the error word).
template <int TILE>
__device__ __forceinline__ bool visibility_item(const DevScene &s, const rzk_receiver *recv, int n_recv, int img_w,
                                                const rzk_vpl *vpls, int j0, int j1, int wt, WarpStage<TILE> &ws,
                                                int lane, uint32_t *masks) {
    const int ri = lane_receiver(wt, lane, n_recv, img_w);
    const int n_tiles = (j1 - j0 + TILE - 1) / TILE;
    RecvRegs r;
    r.p = mk(0.0f, 0.0f, 0.0f);
    bool active = false;
    if (ri >= 0) {
        r = load_receiver(recv + ri);
        active = r.mat >= 0;
    }
    if (n_tiles <= 0 || !__any_sync(kFull, active)) {
        for (int j = j0 + lane; j < j1; j += 32) masks[j - j0] = 0u;
        return true;
    }
    int occ_cache = -1, occ_cache2 = -1;
    unsigned long long n_rays = 0;
    if (lane == 0) {
        int cnt = min(TILE, j1 - j0);
        fence_proxy_async();
        mbar_expect_tx(&ws.mb[0], cnt * (uint32_t)sizeof(rzk_vpl));
        bulk_g2s(&ws.tl[0][0], vpls + j0, cnt * (uint32_t)sizeof(rzk_vpl), &ws.mb[0]);
    }
    for (int k = 0; k < n_tiles; ++k) {
        const int buf = k & 1;
        if (lane == 0 && k + 1 < n_tiles) {
            int jn = j0 + (k + 1) * TILE;
            int cnt = min(TILE, j1 - jn);
            fence_proxy_async();
            mbar_expect_tx(&ws.mb[buf ^ 1], cnt * (uint32_t)sizeof(rzk_vpl));
            bulk_g2s(&ws.tl[buf ^ 1][0], vpls + jn, cnt * (uint32_t)sizeof(rzk_vpl), &ws.mb[buf ^ 1]);
        }
        bool ok = mbar_wait_bounded(&ws.mb[buf], ws.uses[buf] & 1u, lane == 0 ? s.err : nullptr);
        ws.uses[buf]++;
        if (__any_sync(kFull, !ok)) return false;
        const rzk_vpl *tile = ws.tl[buf];
        const int cnt = min(TILE, j1 - (j0 + k * TILE));
        // the VPL-only facts of the tile's VPLs, one VPL per lane (as in gather_item)
        static_assert(TILE <= 32, "one VPL per lane");
        const rzk_vpl &mine = tile[lane < cnt ? lane : 0];
        const unsigned fin_mask = __ballot_sync(kFull, lane < cnt && vpl_power_finite(mine));
        const unsigned behind_mask = __ballot_sync(kFull, lane < cnt && vpl_from_behind(mine));
        for (int v = 0; v < cnt; ++v) {
            const rzk_vpl &l = tile[v];
            const bool fin = (fin_mask >> v) & 1u, behind = (behind_mask >> v) & 1u;
            PairGeo pg;
            bool act = active && !pair_clearly_zero(r, l, fin, behind) && pair_survives(r, l, pg, fin, behind);
            unsigned vis = 0u;
            const unsigned am = __ballot_sync(kFull, act);
            n_rays += (unsigned)__popc(am);
            if (am) {
                Ray ray = make_ray(r.p, sub(pg.q, r.p));
                float tmax = len(sub(pg.q, r.p)) - s.tmin;
                vis = __ballot_sync(kFull, packet_visible_near(s, ray, tmax, act, ws.stk, occ_cache, occ_cache2));
            }
            if (lane == 0) masks[k * TILE + v] = vis;
        }
        __syncwarp();
    }
    if (lane == 0 && s.rays && n_rays) atomicAdd(s.rays, n_rays);
    return true;
}

// Summing half: the 32 receivers of warp tile `wt` add, in VPL order, the terms of the
// pairs that `masks` (one word per VPL, from visibility_item) marks - the same values in
// the same order as gather_item with one chunk, so the sums are bit-identical to it.
// WEIGHTED: VPL j's radiance is multiplied by weights[j] before it is added (a cluster
// representative standing for its cluster).  Writes partial[3 * ri ...].
template <bool WEIGHTED>
__device__ __forceinline__ void shade_item(const DevScene &s, const rzk_receiver *recv, int n_recv, int img_w,
                                           const rzk_vpl *vpls, int n_vpl, const uint32_t *masks, int wt, int mode,
                                           float tau, float *partial, int lane, const float *weights) {
    const int ri = lane_receiver(wt, lane, n_recv, img_w);
    if (ri < 0) return;
    RecvRegs r = load_receiver(recv + ri);
    Rgb sum = crgb(0.0f, 0.0f, 0.0f);
    if (r.mat >= 0) {
        const rzk_material rm = load_material(s.mats + r.mat);
        const unsigned bit = 1u << lane;
        for (int j = 0; j < n_vpl; ++j) {
            if (!(masks[j] & bit)) continue;
            const rzk_vpl &l = vpls[j];
            PairGeo pg;
            pair_survives(r, l, pg);
            Rgb L = pair_radiance(s, r, rm, l, pg, mode, tau);
            if (WEIGHTED) {
                const float w = weights[j];
                L = crgb(w * L.r, w * L.g, w * L.b);
            }
            sum = cadd(sum, L);
        }
    }
    float *o = partial + 3 * (size_t)ri;
    o[0] = sum.r; o[1] = sum.g; o[2] = sum.b;
}

}  // namespace rzk
