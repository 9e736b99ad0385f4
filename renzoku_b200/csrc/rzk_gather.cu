// rzk_gather.cu - the VPL gather: per (shading point, VPL) pair, shadow-ray visibility
// through the LBVH, geometry term, both BRDFs and the clamp
// (VirtualPointLight::gather_point, vpl.cc:661-688), summed per shading point.
//
// Layout: a CTA owns BLOCK consecutive receivers (one per thread, loaded once into
// registers) and one contiguous chunk of VPLs (with several chunks, of the VPLs sorted
// along a Hilbert curve through their positions).  The chunk streams through shared memory
// in TILE-VPL tiles, double-buffered, each tile one bulk copy (cp.async.bulk, no
// multicast) completing on an mbarrier.  Every thread walks the tile in VPL order; the
// shading term is evaluated first and the shadow ray is traced only when it is non-zero
// (a zero term contributes zero whatever the visibility, so the sum is unchanged).
// Per-thread sums are written per chunk and a second kernel adds the chunks in chunk
// order, so the image does not depend on scheduling; with one chunk the summation order
// is exactly the reference's (VPL order, single precision).
#include "rzk_gather_dev.cuh"

#include <algorithm>
#include <mutex>

namespace rzk {

namespace {

// The shading part of gather_point after its visibility test (vpl.cc:676-687);
// pn is the receiver's shading normal (LocalGeometry::n, local_geometry.h:52-56).
__device__ __forceinline__ Rgb shade(const DevScene &s, const RecvRegs &r, const rzk_material &rm,
                                     const rzk_vpl &l, int mode, float tau, V3 &q) {
    q = ld3(l.p);
    float G = form_factor_abs(r.p, r.ns, q, ld3(l.n));
    V3 wi = unit(sub(q, r.p));
    Rgb sb = brdf_eval(rm, r.uvn, r.wo, wi);
    Rgb lb;
    if (l.mat >= 0) {
        rzk_material lm = load_material(s.mats + l.mat);
        Onb lu{ld3(l.u), ld3(l.v), ld3(l.nn)};
        lb = brdf_eval(lm, lu, ld3(l.wi), neg(wi));
    } else {
        lb = crgb(1.0f, 1.0f, 1.0f);
    }
    return radiance_terms(crgb(l.contrib[0], l.contrib[1], l.contrib[2]), sb, lb, G, mode, tau);
}

template <int BLOCK, int TILE>
__global__ void __launch_bounds__(BLOCK) gather_kernel(DevScene s, const rzk_receiver *recv, int n_recv,
                                                       const rzk_vpl *vpls, int n_vpl, int chunk_len,
                                                       int mode, float tau, float *partial) {
    __shared__ __align__(128) rzk_vpl tile[2][TILE];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int stack_mem[STACK_CAP * BLOCK];
    __shared__ int abort_flag;

    const int t = threadIdx.x;
    const int ri = blockIdx.x * BLOCK + t;
    const int chunk = blockIdx.y;
    const int j0 = chunk * chunk_len;
    const int j1 = min(n_vpl, j0 + chunk_len);
    const int n_tiles = j1 > j0 ? (j1 - j0 + TILE - 1) / TILE : 0;

    RecvRegs r;
    bool active = false;
    rzk_material rm;
    if (ri < n_recv) {
        r = load_receiver(recv + ri);
        active = r.mat >= 0;
        if (active) rm = load_material(s.mats + r.mat);
    }
    Stack<BLOCK> stk;
    stk.init(stack_mem + t);

    if (t == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        abort_flag = 0;
        fence_barrier_init();
    }
    __syncthreads();
    if (t == 0 && n_tiles > 0) {
        int cnt = min(TILE, j1 - j0);
        mbar_expect_tx(&bar[0], cnt * (uint32_t)sizeof(rzk_vpl));
        bulk_g2s(&tile[0][0], vpls + j0, cnt * (uint32_t)sizeof(rzk_vpl), &bar[0]);
    }

    Rgb sum = crgb(0.0f, 0.0f, 0.0f);
    for (int k = 0; k < n_tiles; ++k) {
        const int buf = k & 1;
        if (t == 0 && k + 1 < n_tiles) {
            int jn = j0 + (k + 1) * TILE;
            int cnt = min(TILE, j1 - jn);
            fence_proxy_async();
            mbar_expect_tx(&bar[buf ^ 1], cnt * (uint32_t)sizeof(rzk_vpl));
            bulk_g2s(&tile[buf ^ 1][0], vpls + jn, cnt * (uint32_t)sizeof(rzk_vpl), &bar[buf ^ 1]);
        }
        if (!mbar_wait_bounded(&bar[buf], (k >> 1) & 1, s.err)) abort_flag = 1;
        const int cnt = min(TILE, j1 - (j0 + k * TILE));
        if (active && !abort_flag) {
            for (int v = 0; v < cnt; ++v) {
                const rzk_vpl &l = tile[buf][v];
                V3 q;
                Rgb L = shade(s, r, rm, l, mode, tau, q);
                if (cblack(L)) continue;
                Ray ray = make_ray(r.p, sub(q, r.p));
                float tmax = len(sub(q, r.p)) - s.tmin;
                if (any_hit<BLOCK, false>(s, ray, s.tmin, tmax, stk)) continue;
                sum = cadd(sum, L);
            }
        }
        __syncthreads();
        if (abort_flag) break;
    }
    if (ri < n_recv) {
        float *o = partial + 3 * ((size_t)chunk * n_recv + ri);
        o[0] = sum.r; o[1] = sum.g; o[2] = sum.b;
    }
}

// ---------------------------------------------------------------------------------
// Warp-packet gather.
//
// A warp owns 32 receivers (an 8 x 4 pixel tile of an image, or 32 consecutive
// receivers) and streams its VPL chunk through its own double-buffered shared-memory
// tiles: one cp.async.bulk per tile issued by lane 0, completing on the warp's mbarrier,
// no block-wide barrier.  For each VPL every lane evaluates its pair's shading term; the
// lanes with a non-zero term then trace their shadow rays together as a packet: one
// warp-uniform stack in shared memory, each inner-node visit one broadcast 64-byte load
// of both children, a child pushed when the box test passes for any lane still
// unoccluded (ballot).  Each lane tests a leaf's triangle only where its own test of that
// leaf's box passed, so its answer is exactly the reference's any-hit answer: a
// triangle is reached iff its own box passes, because every inner box is the exact
// min / max of the boxes below it and the rounded slab test is monotone in the box
// bounds.  Rays of one warp toward one VPL are coherent (about 20-26 of the 32 lanes
// trace together, and the union of their paths is 4-15% longer than the longest single
// path on the 300k-triangle scene), so the packet costs about what the slowest lane
// costs alone, with one node fetch per step instead of one per lane.
// Each lane adds its visible terms in VPL order: the sum is formed in the reference's
// order.
// ---------------------------------------------------------------------------------
// shade() with the BRDFs' own early-outs hoisted: where either BRDF returns black
// (lambertian.cc:63-66, phong.cc:74-77, ward.cc:104-109: the same dot products, the
// products commute exactly) and G and the power are finite, the pair's term is exactly
// zero, so the BRDF values and the clamp need not be formed.
__device__ __forceinline__ Rgb shade_cull(const DevScene &s, const RecvRegs &r, const rzk_material &rm,
                                          const rzk_vpl &l, int mode, float tau) {
    V3 q = ld3(l.p);
    float G = form_factor_abs(r.p, r.ns, q, ld3(l.n));
    V3 wi = unit(sub(q, r.p));
    Rgb power = crgb(l.contrib[0], l.contrib[1], l.contrib[2]);
    if (isfinite(G) && finite3(power)) {
        if (dot(wi, r.uvn.n) <= ZERO_EPSILON || dot(r.wo, r.uvn.n) <= ZERO_EPSILON)
            return crgb(0.0f, 0.0f, 0.0f);
        if (l.mat >= 0) {
            V3 lnn = ld3(l.nn);
            if (dot(neg(wi), lnn) <= ZERO_EPSILON || dot(ld3(l.wi), lnn) <= ZERO_EPSILON)
                return crgb(0.0f, 0.0f, 0.0f);
        }
    }
    Rgb sb = brdf_eval(rm, r.uvn, r.wo, wi);
    Rgb lb;
    if (l.mat >= 0) {
        rzk_material lm = load_material(s.mats + l.mat);
        Onb lu{ld3(l.u), ld3(l.v), ld3(l.nn)};
        lb = brdf_eval(lm, lu, ld3(l.wi), neg(wi));
    } else {
        lb = crgb(1.0f, 1.0f, 1.0f);
    }
    return radiance_terms(power, sb, lb, G, mode, tau);
}

// Packet any-hit for the lanes in `act`; returns the lanes that stay unoccluded.
__device__ __forceinline__ bool packet_visible(const DevScene &s, const Ray &ray, float tmax, bool act,
                                               int *stk) {
    if (s.n_nodes == 0) return act;
    const float4 lo = __ldg(s.nodes + 2), hi = __ldg(s.nodes + 3);
    bool hit_root = act && box_hit(lo, hi, ray, s.tmin, tmax);
    if (!__any_sync(kFull, hit_root)) return act;
    const int a = __float_as_int(lo.w);
    if (a < 0) {
        if (hit_root) {
            float4 ta, tb, tc;
            load_tri(s, -1 - a, ta, tb, tc);
            if (tri_hit<false>(ta, tb, tc, ray, s.tmin, tmax, nullptr, nullptr, nullptr)) act = false;
        }
        return act;
    }
    // lanes whose root test failed cannot reach any triangle below it: they stay visible
    bool alive = hit_root;
    bool occluded = false;
    int top = 0;
    stk[0] = a;
    bool overflow = false;
    while (top >= 0) {
        const int c = stk[top--];
        const float4 *pn = s.nodes + 2 * (c + 1);
        const float4 l0 = __ldg(pn), l1 = __ldg(pn + 1), r0 = __ldg(pn + 2), r1 = __ldg(pn + 3);
        const int al = __float_as_int(l0.w), ar = __float_as_int(r0.w);
        bool hl = alive && box_hit(l0, l1, ray, s.tmin, tmax);
        bool hr = alive && box_hit(r0, r1, ray, s.tmin, tmax);
        if (al < 0 && hl) {
            float4 ta, tb, tc;
            load_tri(s, -1 - al, ta, tb, tc);
            if (tri_hit<false>(ta, tb, tc, ray, s.tmin, tmax, nullptr, nullptr, nullptr)) occluded = true;
        }
        if (ar < 0 && hr && !occluded) {
            float4 ta, tb, tc;
            load_tri(s, -1 - ar, ta, tb, tc);
            if (tri_hit<false>(ta, tb, tc, ray, s.tmin, tmax, nullptr, nullptr, nullptr)) occluded = true;
        }
        alive = alive && !occluded;
        // push order as the reference: left first, so the right child is visited next
        if (al >= 0 && __any_sync(kFull, hl && alive)) {
            if (top < STACK_CAP - 1) stk[++top] = al; else overflow = true;
        }
        if (ar >= 0 && __any_sync(kFull, hr && alive)) {
            if (top < STACK_CAP - 1) stk[++top] = ar; else overflow = true;
        }
        if (!__any_sync(kFull, alive)) break;
    }
    if (overflow && s.err) atomicOr(s.err, ERR_STACK);
    return act && !occluded;
}

// Packet any-hit over the 4-wide tree: per step one broadcast 128-byte node load, four
// independent box tests per lane, leaf triangles tested where the lane's own leaf-box
// test passed, inner entries pushed when any unoccluded lane passed them.
__device__ __forceinline__ bool packet_visible_wide(const DevScene &s, const Ray &ray, float tmax, bool act,
                                                    int *stk) {
    if (s.n_nodes == 0) return act;
    const float4 lo = __ldg(s.nodes + 2), hi = __ldg(s.nodes + 3);
    bool alive = act && box_hit(lo, hi, ray, s.tmin, tmax);
    if (!__any_sync(kFull, alive)) return act;
    const int a = __float_as_int(lo.w);
    if (a < 0) {
        if (alive) {
            float4 ta, tb, tc;
            load_tri(s, -1 - a, ta, tb, tc);
            if (tri_hit<false>(ta, tb, tc, ray, s.tmin, tmax, nullptr, nullptr, nullptr)) act = false;
        }
        return act;
    }
    // lanes whose root test failed cannot reach any triangle below it: they stay visible
    bool occluded = false;
    int top = 0;
    stk[0] = 0;
    bool overflow = false;
    while (top >= 0) {
        const float4 *pn = s.wide + 8 * stk[top--];
        float4 e0[4], e1[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) { e0[k] = __ldg(pn + 2 * k); e1[k] = __ldg(pn + 2 * k + 1); }
        bool h[4];
        int code[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            code[k] = __float_as_int(e0[k].w);
            h[k] = alive && code[k] != kWideEmpty && box_hit(e0[k], e1[k], ray, s.tmin, tmax);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (code[k] < 0 && h[k] && !occluded) {
                float4 ta, tb, tc;
                load_tri(s, -1 - code[k], ta, tb, tc);
                if (tri_hit<false>(ta, tb, tc, ray, s.tmin, tmax, nullptr, nullptr, nullptr)) occluded = true;
            }
        }
        alive = alive && !occluded;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (code[k] >= 0 && code[k] != kWideEmpty && __any_sync(kFull, h[k] && alive)) {
                if (top < STACK_CAP - 1) stk[++top] = code[k]; else overflow = true;
            }
        }
        if (!__any_sync(kFull, alive)) break;
    }
    if (overflow && s.err) atomicOr(s.err, ERR_STACK);
    return act && !occluded;
}

template <int WARPS, int TILE, bool WIDE>
__global__ void __launch_bounds__(WARPS * 32) gather_packet_kernel(DevScene s, const rzk_receiver *recv,
                                                                   int n_recv, int img_w,
                                                                   const rzk_vpl *vpls, int n_vpl,
                                                                   int chunk_len, int mode, float tau,
                                                                   float *partial) {
    __shared__ __align__(128) rzk_vpl tiles[WARPS][2][TILE];
    __shared__ __align__(8) uint64_t bar[WARPS][2];
    __shared__ int stacks[WARPS][STACK_CAP];

    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int ri = lane_receiver(blockIdx.x * WARPS + w, lane, n_recv, img_w);
    const int chunk = blockIdx.y;
    const int j0 = chunk * chunk_len;
    const int j1 = min(n_vpl, j0 + chunk_len);
    const int n_tiles = j1 > j0 ? (j1 - j0 + TILE - 1) / TILE : 0;

    RecvRegs r;
    r.p = mk(0.0f, 0.0f, 0.0f);   // lanes without a receiver still form (unused) rays
    bool active = false;
    rzk_material rm;
    if (ri >= 0) {
        r = load_receiver(recv + ri);
        active = r.mat >= 0;
        if (active) rm = load_material(s.mats + r.mat);
    }
    uint64_t *mb = bar[w];
    rzk_vpl(*tl)[TILE] = tiles[w];
    int *stk = stacks[w];

    if (lane == 0) {
        mbar_init(&mb[0], 1);
        mbar_init(&mb[1], 1);
        fence_barrier_init();
        if (n_tiles > 0) {
            int cnt = min(TILE, j1 - j0);
            mbar_expect_tx(&mb[0], cnt * (uint32_t)sizeof(rzk_vpl));
            bulk_g2s(&tl[0][0], vpls + j0, cnt * (uint32_t)sizeof(rzk_vpl), &mb[0]);
        }
    }
    __syncwarp();

    Rgb sum = crgb(0.0f, 0.0f, 0.0f);
    for (int k = 0; k < n_tiles; ++k) {
        const int buf = k & 1;
        if (lane == 0 && k + 1 < n_tiles) {
            int jn = j0 + (k + 1) * TILE;
            int cnt = min(TILE, j1 - jn);
            fence_proxy_async();
            mbar_expect_tx(&mb[buf ^ 1], cnt * (uint32_t)sizeof(rzk_vpl));
            bulk_g2s(&tl[buf ^ 1][0], vpls + jn, cnt * (uint32_t)sizeof(rzk_vpl), &mb[buf ^ 1]);
        }
        bool ok = mbar_wait_bounded(&mb[buf], (k >> 1) & 1, lane == 0 ? s.err : nullptr);
        if (__any_sync(kFull, !ok)) break;
        const rzk_vpl *tile = tl[buf];
        const int cnt = min(TILE, j1 - (j0 + k * TILE));
        for (int v = 0; v < cnt; ++v) {
            const rzk_vpl &l = tile[v];
            Rgb L = crgb(0.0f, 0.0f, 0.0f);
            bool act = false;
            if (active) {
                L = shade_cull(s, r, rm, l, mode, tau);
                act = !cblack(L);
            }
            if (!__any_sync(kFull, act)) continue;
            V3 q = ld3(l.p);
            Ray ray = make_ray(r.p, sub(q, r.p));
            float tmax = len(sub(q, r.p)) - s.tmin;
            bool vis = WIDE ? packet_visible_wide(s, ray, tmax, act, stk) : packet_visible(s, ray, tmax, act, stk);
            if (vis) sum = cadd(sum, L);
        }
        __syncwarp();
    }
    if (ri >= 0) {
        float *o = partial + 3 * ((size_t)chunk * n_recv + ri);
        o[0] = sum.r; o[1] = sum.g; o[2] = sum.b;
    }
}

// ---------------------------------------------------------------------------------
// Persistent warp-packet gather (the production kernel).
//
// One resident grid (SMs x resident CTAs); every warp repeatedly takes the next work
// item - an 8 x 4 receiver tile x a chunk of VPLs - from a global counter, so no SM idles
// while another still holds long work (the tail of a fixed grid cost about 40% of the
// issue slots).  Per VPL the lanes first apply only the BRDFs' early-outs (the exact zero
// tests of lambertian.cc:63-66, phong.cc:74-77, ward.cc:104-109); the surviving lanes
// trace their shadow rays as a packet, nearer child first by majority; the full BRDF
// values and the clamp are evaluated only for the lanes that stay visible (about 80% of
// traced shadow rays are occluded on the scaled scene).  Each lane adds its terms in VPL
// order; the chunk sums are added in chunk order by reduce_chunks_kernel after the launch
// or, on fixed scratch, inside it through the chunk ring (RingSink).
// ---------------------------------------------------------------------------------

// Bounded wait of lane 0 until a ring slot has finished `rnd` tiles (its previous tile has
// been summed and the slot freed); limit_ns of the GPU's global timer at most (4 s in the
// gather), then ERR_TIMEOUT.  Warp-uniform result.
__device__ __forceinline__ bool ring_acquire(const ChunkRing &ring, int slot, int rnd, uint32_t *err, int lane,
                                             unsigned long long limit_ns = 4000000000ull) {
    int ok = 1;
    if (lane == 0) {
        const volatile int *r = ring.round + slot;
        if (*r != rnd) {
            uint64_t t0, t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
            for (uint32_t it = 0; *r != rnd; ++it) {
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                if (t - t0 > limit_ns || it > (1u << 26)) {
                    if (err) atomicOr(err, ERR_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(200);
            }
        }
        __threadfence();   // acquire: the previous tile's reads of the slot came first
    }
    return __shfl_sync(kFull, ok, 0) != 0;
}

// One warp runs the ring's slot wait on a slot that nothing frees (round 0, waiting for
// round 1): the wait must give up after limit_ns, set ERR_TIMEOUT and return, leaving the
// context usable.  *acquired = 1 if the wait (wrongly) succeeded.
__global__ void ring_wait_probe_kernel(ChunkRing ring, uint32_t *err, unsigned long long limit_ns, int *acquired) {
    const int lane = threadIdx.x & 31;
    const bool ok = ring_acquire(ring, 0, 1, err, lane, limit_ns);
    if (lane == 0) *acquired = ok ? 1 : 0;
}

// Sink of gather_item adding an item's sums to the chunk ring (ChunkRing): waits until the
// slot's previous tile has been summed, writes the chunk's entry, counts it, and - in the
// warp that writes the tile's last chunk - adds the tile's chunks in chunk order (the order
// and operations of reduce_chunks_kernel, so the image is the same bit for bit), scales and
// writes the pixels, then frees the slot.  `stop` is set when the slot wait gives up.
struct RingSink {
    ChunkRing ring;
    int wt, chunk, n_chunks, lane;
    float scale;
    float *out;
    uint32_t *err;
    bool *stop;
    __device__ __forceinline__ void operator()(int ri, Rgb sum, bool ok) const {
        if (!ok) sum = crgb(0.0f, 0.0f, 0.0f);   // reported in the error word; the tile still completes
        // the slot's previous tile (wt - slots) had every item handed out before this one,
        // to warps that are running; they wait only on still earlier tiles, so the wait ends
        const int slot = wt % ring.slots;
        const int rnd = wt / ring.slots;
        if (!ring_acquire(ring, slot, rnd, err, lane)) {
            *stop = true;
            return;
        }
        // streaming (evict-first) stores: the sums are read once, by the tile's last warp,
        // and must not displace the traversal working set from L2
        float *e = ring.sums + ((size_t)slot * n_chunks + chunk) * 96 + 3 * lane;
        __stcs(e, sum.r); __stcs(e + 1, sum.g); __stcs(e + 2, sum.b);
        __threadfence();   // release this chunk's sums before it is counted
        __syncwarp();
        int prev = 0;
        if (lane == 0) prev = atomicAdd(ring.done + slot, 1);
        prev = __shfl_sync(kFull, prev, 0);
        if (prev != n_chunks - 1) return;
        // the tile's last chunk; read past L1 (this SM may hold older lines of the slot)
        __threadfence();
        const float *b = ring.sums + (size_t)slot * n_chunks * 96 + 3 * lane;
        float ar = __ldcg(b), ag = __ldcg(b + 1), ab = __ldcg(b + 2);
        for (int c = 1; c < n_chunks; ++c) {
            const float *bc = b + (size_t)c * 96;
            ar += __ldcg(bc);
            ag += __ldcg(bc + 1);
            ab += __ldcg(bc + 2);
        }
        if (ri >= 0) {
            out[3 * (size_t)ri] = ar * scale;
            out[3 * (size_t)ri + 1] = ag * scale;
            out[3 * (size_t)ri + 2] = ab * scale;
        }
        __syncwarp();   // every lane's reads of the slot precede its release
        if (lane == 0) {
            ring.done[slot] = 0;
            __threadfence();
            atomicExch(ring.round + slot, rnd + 1);
        }
    }
};

// RING = false: each item writes its chunk's plane of `partial` (n_chunks planes of n_recv x
// 3 floats) and reduce_chunks_kernel adds the planes afterwards; RING = true: the chunk
// ring (RingSink) sums each tile inside the launch and writes `out` (scaled by `scale`).
template <int WARPS, int TILE, int MINB, int TW = 8, bool RING = false>
__global__ void __launch_bounds__(WARPS * 32, MINB) gather_persistent_kernel(
    DevScene s, const rzk_receiver *recv, int n_recv, int img_w, const rzk_vpl *vpls, int n_vpl,
    int chunk_len, int n_chunks, int n_wtiles, int *work, int mode, float tau, float *partial, float scale,
    ChunkRing ring, float *out) {
    __shared__ __align__(128) rzk_vpl tiles[WARPS][2][TILE];
    __shared__ __align__(8) uint64_t bar[WARPS][2];
    __shared__ int stacks[WARPS][STACK_CAP];

    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    WarpStage<TILE> ws;
    ws.init(tiles[w], bar[w], stacks[w], lane);
    const long long n_items = (long long)n_wtiles * n_chunks;
    while (true) {
        int item = 0;
        if (lane == 0) item = atomicAdd(work, 1);
        item = __shfl_sync(kFull, item, 0);
        if (item >= n_items) break;
        // tile-major: the warps in flight work on a few hundred neighbouring tiles (a compact
        // band of ray origins) against every chunk; a tile's items are all handed out before
        // any item of a later tile, which is what ends the ring's waits
        const int wt = item / n_chunks;
        const int chunk = item - wt * n_chunks;
        if constexpr (RING) {
            bool stop = false;
            const bool ok = gather_item<TILE, TW>(s, recv, n_recv, img_w, vpls, n_vpl, chunk, wt, chunk_len, mode,
                                                  tau, ws, lane,
                                                  RingSink{ring, wt, chunk, n_chunks, lane, scale, out, s.err, &stop});
            if (!ok || stop) break;
        } else {
            if (!gather_item<TILE, TW>(s, recv, n_recv, img_w, vpls, n_vpl, chunk, wt, chunk_len, mode, tau, ws,
                                       lane, PlaneSink{partial, n_recv, chunk}))
                break;
        }
    }
}

__global__ void reduce_chunks_kernel(const float *partial, int n_recv, int n_chunks, float scale,
                                     float *out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * n_recv) return;
    float acc = __ldcs(partial + i);   // read once: evict-first
    for (int c = 1; c < n_chunks; ++c) acc += __ldcs(partial + (size_t)c * 3 * n_recv + i);
    out[i] = acc * scale;
}

// LightTransportMatrix::fill: every pair, visibility always traced.  kind 0: radiance
// (gather_point, lights skipped); kind 1: incident radiance without visibility; kind 2:
// (float)visible x incident radiance, the reduced matrix of LightSlice
// (lightslice.cc:721-737), with the visibility written as well.
constexpr int kMatBlock = 128;
__global__ void __launch_bounds__(kMatBlock) matrix_kernel(DevScene s, const rzk_receiver *recv,
                                                           int n_recv, const rzk_vpl *vpls, int n_vpl,
                                                           int mode, float tau, float *mat,
                                                           uint8_t *vis, int kind) {
    __shared__ int stack_mem[STACK_CAP * kMatBlock];
    const int ri = blockIdx.x * kMatBlock + threadIdx.x;
    if (ri >= n_recv) return;
    Stack<kMatBlock> stk;
    stk.init(stack_mem + threadIdx.x);
    RecvRegs r = load_receiver(recv + ri);
    for (int j = blockIdx.y; j < n_vpl; j += gridDim.y) {
    rzk_vpl l = vpls[j];
    Rgb L = crgb(0.0f, 0.0f, 0.0f);
    bool visible = false;
    if (kind >= 1) {
        // VirtualPointLight::incident_radiance (vpl.cc:411-440): geometric normal, no
        // visibility, surface BRDF white.
        V3 q = ld3(l.p);
        float G = form_factor_abs(r.p, r.ng, q, ld3(l.n));
        V3 wi = unit(sub(q, r.p));
        Rgb lb = crgb(1.0f, 1.0f, 1.0f);
        if (l.mat >= 0) {
            rzk_material lm = load_material(s.mats + l.mat);
            Onb lu{ld3(l.u), ld3(l.v), ld3(l.nn)};
            lb = brdf_eval(lm, lu, ld3(l.wi), neg(wi));
        }
        L = radiance_terms(crgb(l.contrib[0], l.contrib[1], l.contrib[2]), crgb(1.0f, 1.0f, 1.0f),
                           lb, G, mode, tau);
        if (kind == 2) {
            Ray ray = make_ray(r.p, sub(q, r.p));
            float tmax = len(sub(q, r.p)) - s.tmin;
            visible = !any_hit<kMatBlock, false, true>(s, ray, s.tmin, tmax, stk);
            const float vf = visible ? 1.0f : 0.0f;
            L = crgb(vf * L.r, vf * L.g, vf * L.b);
        }
    } else if (r.mat >= 0) {
        V3 q = ld3(l.p);
        Ray ray = make_ray(r.p, sub(q, r.p));
        float tmax = len(sub(q, r.p)) - s.tmin;
        if (!any_hit<kMatBlock, false, true>(s, ray, s.tmin, tmax, stk)) {
            visible = true;
            rzk_material rm = load_material(s.mats + r.mat);
            L = shade(s, r, rm, l, mode, tau, q);
        }
    }
    size_t k = (size_t)j * n_recv + ri;
    mat[3 * k] = L.r; mat[3 * k + 1] = L.g; mat[3 * k + 2] = L.b;
    if (vis) vis[k] = visible ? 1 : 0;
    }
}

// Seeded pairs for the "0.1 x mean contribution" clamp base; block partials in double.
constexpr int kMeanBlock = 128;
__global__ void __launch_bounds__(kMeanBlock) mean_kernel(DevScene s, const rzk_receiver *recv,
                                                          int n_recv, const rzk_vpl *vpls, int n_vpl,
                                                          uint32_t seed, int n_pairs, double *block_sums) {
    __shared__ int stack_mem[STACK_CAP * kMeanBlock];
    __shared__ double red[kMeanBlock];
    const int k = blockIdx.x * kMeanBlock + threadIdx.x;
    double val = 0.0;
    if (k < n_pairs) {
        uint4 blk = philox4x32_10(make_uint4(0u, (uint32_t)k, 3u, 0x52454e5au), seed, 0x4b5a4f52u);
        int ri = (int)(blk.x % (uint32_t)n_recv);
        int vi = (int)(blk.y % (uint32_t)n_vpl);
        RecvRegs r = load_receiver(recv + ri);
        if (r.mat >= 0) {
            Stack<kMeanBlock> stk;
            stk.init(stack_mem + threadIdx.x);
            rzk_vpl l = vpls[vi];
            V3 q = ld3(l.p);
            Ray ray = make_ray(r.p, sub(q, r.p));
            float tmax = len(sub(q, r.p)) - s.tmin;
            if (!any_hit<kMeanBlock, false, true>(s, ray, s.tmin, tmax, stk)) {
                rzk_material rm = load_material(s.mats + r.mat);
                Rgb L = shade(s, r, rm, l, RZK_CLAMP_NONE, 0.0f, q);
                val = (double)cval(L);
            }
        }
    }
    red[threadIdx.x] = val;
    __syncthreads();
    for (int w = kMeanBlock / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) block_sums[blockIdx.x] = red[0];
}

__global__ void mean_final_kernel(const double *block_sums, int nb, int n_pairs, double *out) {
    if (threadIdx.x != 0) return;
    double acc = 0.0;
    for (int b = 0; b < nb; ++b) acc += block_sums[b];
    *out = n_pairs > 0 ? acc / n_pairs : 0.0;
}

// 8 bits spread to every third bit (bit i -> bit 3i).
__device__ __forceinline__ uint32_t spread3(uint32_t x) {
    x &= 0xffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

// segment holding concatenated position i (segments in order of begin)
__device__ __forceinline__ int order_seg_of(const OrderTable &t, int i) {
    int lo = 0, hi = t.n_segs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (t.seg[mid].begin <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// 24-bit index of cell (x, y, z) of a 256^3 grid along a 3-D Hilbert curve: J. Skilling's
// transform of the axes to the curve's transposed index ("Programming the Hilbert curve",
// AIP Conf. Proc. 707, 2004) - undo the excess work level by level, then Gray-encode -
// followed by interleaving the transposed words, first axis most significant.
__device__ __forceinline__ uint32_t hilbert3_8(uint32_t x, uint32_t y, uint32_t z) {
    uint32_t a[3] = {x, y, z};
    for (uint32_t q = 128u; q > 1u; q >>= 1) {
        const uint32_t p = q - 1u;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (a[d] & q) {
                a[0] ^= p;
            } else {
                const uint32_t s = (a[0] ^ a[d]) & p;
                a[0] ^= s;
                a[d] ^= s;
            }
        }
    }
    a[1] ^= a[0];
    a[2] ^= a[1];
    uint32_t flip = 0;
    for (uint32_t q = 128u; q > 1u; q >>= 1)
        if (a[2] & q) flip ^= q - 1u;
    a[0] ^= flip;
    a[1] ^= flip;
    a[2] ^= flip;
    return (spread3(a[0]) << 2) | (spread3(a[1]) << 1) | spread3(a[2]);
}

// Key of concatenated VPL i: its segment in the top bits, below them the Hilbert index of
// its position's cell on a 256^3 grid over the segment's box (positions outside the box
// clamp to the border cells, NaN to cell 0).
__global__ void order_keys_kernel(const __grid_constant__ OrderTable t, uint32_t *keys, int *idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.total) return;
    const int sg = order_seg_of(t, i);
    const OrderSeg &g = t.seg[sg];
    const rzk_vpl &v = g.src[i - g.begin];
    auto cell = [](float x) { return (uint32_t)fminf(fmaxf(x, 0.0f), 255.0f); };
    const uint32_t x = cell((v.p[0] - g.lo[0]) * g.k[0]);
    const uint32_t y = cell((v.p[1] - g.lo[1]) * g.k[1]);
    const uint32_t z = cell((v.p[2] - g.lo[2]) * g.k[2]);
    keys[i] = ((uint32_t)sg << 24) | hilbert3_8(x, y, z);
    idx[i] = i;
}

// out[j] = concatenated VPL idx[j], one 4-byte word per thread (coalesced writes; each
// record's 96 bytes are read by 24 consecutive threads).
__global__ void order_permute_kernel(const __grid_constant__ OrderTable t, const int *idx, rzk_vpl *out) {
    constexpr int W = (int)(sizeof(rzk_vpl) / 4);
    const long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= (long long)t.total * W) return;
    const int j = (int)(w / W), c = (int)(w % W);
    const int i = idx[j];
    const OrderSeg &g = t.seg[order_seg_of(t, i)];
    reinterpret_cast<uint32_t *>(out)[w] = reinterpret_cast<const uint32_t *>(g.src + (i - g.begin))[c];
}

}  // namespace

// Spatial order of a chunked gather's VPLs.  With several chunks the image is a sum of
// per-chunk sums anyway, so which VPLs share a chunk changes only the float summation
// order; chunks of nearby VPLs make the consecutive shadow rays of a warp end near one
// another, so they walk the same tree nodes (L1 hits) and the per-lane occluder cache hits
// more often.  One stable radix sort orders all segments of a table at once (segment in
// the top key bits, ties keep push order).
static_assert(sizeof(OrderTable) <= 32000, "kernel parameter block limit");

void order_table_init(OrderTable &t) {
    t.n_segs = 0;
    t.total = 0;
}

bool order_table_add(OrderTable &t, const rzk_vpl *src, int n, const float *box) {
    if (t.n_segs == kOrderSegs) return false;
    OrderSeg &g = t.seg[t.n_segs++];
    g.src = src;
    g.begin = t.total;
    g.n = n;
    for (int d = 0; d < 3; ++d) {
        const float ext = box[3 + d] - box[d];
        g.lo[d] = box[d];
        g.k[d] = ext > 0.0f ? 256.0f / ext : 0.0f;
    }
    t.total += n;
    return true;
}

static int order_bits(const OrderTable &t) {
    int b = 0;
    while ((1 << b) < t.n_segs) ++b;
    return 24 + b;
}

static size_t order_up(size_t b) { return (b + 255) & ~(size_t)255; }

size_t order_scratch_bytes(int total) {
    return 2 * order_up(sizeof(uint32_t) * (size_t)total) + radix_sort_scratch_bytes(total);
}

int order_launches(const OrderTable &t) {
    return t.total > 0 ? 2 + radix_sort_launches(t.total, order_bits(t)) : 0;
}

rzk_status order_vpls(const OrderTable &t, void *scratch, rzk_vpl *out, cudaStream_t st) {
    if (t.total <= 0) return RZK_OK;
    char *p = (char *)scratch;
    uint32_t *keys = (uint32_t *)p;
    int *idx = (int *)(p + order_up(sizeof(uint32_t) * (size_t)t.total));
    void *sort = p + 2 * order_up(sizeof(uint32_t) * (size_t)t.total);
    order_keys_kernel<<<(t.total + 255) / 256, 256, 0, st>>>(t, keys, idx);
    RZK_CUDA_TRY(cudaGetLastError());
    RZK_TRY(radix_sort_u32(keys, idx, t.total, order_bits(t), sort, st));
    const long long words = (long long)t.total * (long long)(sizeof(rzk_vpl) / 4);
    order_permute_kernel<<<(unsigned)((words + 255) / 256), 256, 0, st>>>(t, idx, out);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

// Orders one gather's VPLs into the context's buffer: [sorted VPLs | sort scratch].
static rzk_status order_gather_vpls(rzk_context *ctx, const float *box, const rzk_vpl *vpls, int n_vpl,
                                    const rzk_vpl **sorted, cudaStream_t st) {
    const size_t vb = order_up(sizeof(rzk_vpl) * (size_t)n_vpl);
    const size_t need = vb + order_scratch_bytes(n_vpl);
    if (need > ctx->order_bytes) {
        if (ctx->d_order) cudaFree(ctx->d_order);
        ctx->d_order = nullptr;
        ctx->order_bytes = 0;
        RZK_CUDA_TRY(cudaMalloc(&ctx->d_order, need));
        ctx->order_bytes = need;
    }
    OrderTable t;
    order_table_init(t);
    order_table_add(t, vpls, n_vpl, box);
    rzk_vpl *out = (rzk_vpl *)ctx->d_order;
    RZK_TRY(order_vpls(t, (char *)ctx->d_order + vb, out, st));
    *sorted = out;
    return RZK_OK;
}

// Tile configurations compiled in; the autotuner picks one per workload.
//   kind 3: persistent warp-packet kernel (the production path)      variants 0-3, 8-10
//           (0 and 3 cap registers for 7 and 6 resident 4-warp CTAs per SM; 0 is the
//           default, fastest on the scaled scene; 8-10 are the kernel at 5 CTAs per SM
//           with warp tiles of 4 x 8, 16 x 2 and 32 x 1 pixels instead of 8 x 4)
//   kind 1: warp-packet kernel, one CTA per receiver block            variants 4-5
//   kind 2: warp-packet kernel on the 4-wide tree                     variant 6
//   kind 0: per-thread block-lockstep kernel (first implementation)   variant 7
struct GatherVariant {
    int kind, warps_or_block, tile, tw;
};
static const GatherVariant kVariants[] = {
    {3, 4, 32, 8}, {3, 2, 32, 8}, {3, 4, 32, 8}, {3, 4, 32, 8}, {1, 4, 32, 8}, {1, 2, 32, 8}, {2, 4, 32, 8},
    {0, 128, 64, 8}, {3, 4, 32, 4}, {3, 4, 32, 16}, {3, 4, 32, 32}};

int gather_variant_count() { return (int)(sizeof(kVariants) / sizeof(kVariants[0])); }

template <int WARPS, int TILE, int MINB, int TW = 8>
static int persistent_grid(rzk_context *ctx, int variant) {
    if (ctx->persistent_grid[variant] == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gather_persistent_kernel<WARPS, TILE, MINB, TW>,
                                                      WARPS * 32, 0);
        ctx->persistent_grid[variant] = std::max(1, sms * std::max(1, per_sm));
    }
    return ctx->persistent_grid[variant];
}

// Chunk count and length of a gather (n_chunks <= 0: automatic).  Chunk boundaries are
// multiples of 128 VPLs whatever the variant's tile, so every variant sums the same VPLs in
// the same order for a given n_chunks.
static void resolve_chunks(int n_vpl, int &n_chunks, int &chunk_len) {
    const int max_chunks = std::max(1, (n_vpl + 127) / 128);
    if (n_chunks <= 0) n_chunks = std::min(32, max_chunks);   // ~1k-VPL chunks at 32k VPLs
    n_chunks = std::min(std::min(n_chunks, max_chunks), 65535);
    if (n_vpl <= 0) n_chunks = 1;
    chunk_len = n_vpl > 0 ? (n_vpl + n_chunks - 1) / n_chunks : 0;
    chunk_len = (chunk_len + 127) / 128 * 128;
    if (chunk_len > 0) n_chunks = (n_vpl + chunk_len - 1) / chunk_len;
}

int gather_launches(int n_recv, int n_vpl, int n_chunks) {
    if (n_recv <= 0) return 0;
    int chunk_len = 0;
    resolve_chunks(n_vpl, n_chunks, chunk_len);
    int k = 2;   // gather + chunk reduction
    if (n_chunks > 1) {
        OrderTable t;
        order_table_init(t);
        const float box[6] = {0, 0, 0, 1, 1, 1};
        order_table_add(t, nullptr, n_vpl, box);
        k += order_launches(t);
    }
    return k;
}

rzk_status launch_gather(rzk_context *ctx, const DevScene &s, const float *box, const rzk_receiver *recv,
                         int n_recv, int img_w, const rzk_vpl *vpls, int n_vpl, int mode, float tau,
                         float scale, float *out, int variant, int n_chunks, cudaStream_t st) {
    if (n_recv <= 0) return RZK_OK;
    if (variant < 0 || variant >= gather_variant_count()) variant = 0;
    const GatherVariant gv = kVariants[variant];
    if (gv.kind == 0) img_w = 0;
    const long long wtiles = gv.tw == 4    ? warp_tiles<4>(n_recv, img_w)
                             : gv.tw == 16 ? warp_tiles<16>(n_recv, img_w)
                             : gv.tw == 32 ? warp_tiles<32>(n_recv, img_w)
                                           : warp_tiles<8>(n_recv, img_w);
    int chunk_len = 0;
    resolve_chunks(n_vpl, n_chunks, chunk_len);
    // one plane of partial sums per chunk, added by reduce_chunks_kernel (the chunk ring that
    // rzk_gather_noalloc sums in measured 1.3% slower here, where memory is not short)
    const size_t need = sizeof(float) * 3 * (size_t)n_recv * n_chunks;
    if (need > ctx->partial_bytes) {
        if (ctx->d_partial) cudaFree(ctx->d_partial);
        ctx->d_partial = nullptr;
        ctx->partial_bytes = 0;
        RZK_CUDA_TRY(cudaMalloc((void **)&ctx->d_partial, need));
        ctx->partial_bytes = need;
    }
    if (!ctx->d_work) RZK_CUDA_TRY(cudaMalloc((void **)&ctx->d_work, 64));
    float *part = ctx->d_partial;
    if (n_chunks > 1) RZK_TRY(order_gather_vpls(ctx, box, vpls, n_vpl, &vpls, st));
    if (gv.kind == 3) {
        RZK_CUDA_TRY(cudaMemsetAsync(ctx->d_work, 0, sizeof(int), st));
        const int wt = (int)wtiles;
        const ChunkRing nr{};
        switch (variant) {
            case 2: gather_persistent_kernel<4, 32, 1><<<persistent_grid<4, 32, 1>(ctx, 2), 128, 0, st>>>(s, recv, n_recv, img_w, vpls, n_vpl, chunk_len, n_chunks, wt, ctx->d_work, mode, tau, part, scale, nr, out); break;
            case 1: gather_persistent_kernel<2, 32, 1><<<persistent_grid<2, 32, 1>(ctx, 1), 64, 0, st>>>(s, recv, n_recv, img_w, vpls, n_vpl, chunk_len, n_chunks, wt, ctx->d_work, mode, tau, part, scale, nr, out); break;
            case 0: gather_persistent_kernel<4, 32, 7><<<persistent_grid<4, 32, 7>(ctx, 0), 128, 0, st>>>(s, recv, n_recv, img_w, vpls, n_vpl, chunk_len, n_chunks, wt, ctx->d_work, mode, tau, part, scale, nr, out); break;
            case 8: gather_persistent_kernel<4, 32, 5, 4><<<persistent_grid<4, 32, 5, 4>(ctx, 8), 128, 0, st>>>(s, recv, n_recv, img_w, vpls, n_vpl, chunk_len, n_chunks, wt, ctx->d_work, mode, tau, part, scale, nr, out); break;
            case 9: gather_persistent_kernel<4, 32, 5, 16><<<persistent_grid<4, 32, 5, 16>(ctx, 9), 128, 0, st>>>(s, recv, n_recv, img_w, vpls, n_vpl, chunk_len, n_chunks, wt, ctx->d_work, mode, tau, part, scale, nr, out); break;
            case 10: gather_persistent_kernel<4, 32, 5, 32><<<persistent_grid<4, 32, 5, 32>(ctx, 10), 128, 0, st>>>(s, recv, n_recv, img_w, vpls, n_vpl, chunk_len, n_chunks, wt, ctx->d_work, mode, tau, part, scale, nr, out); break;
            default: gather_persistent_kernel<4, 32, 6><<<persistent_grid<4, 32, 6>(ctx, 3), 128, 0, st>>>(s, recv, n_recv, img_w, vpls, n_vpl, chunk_len, n_chunks, wt, ctx->d_work, mode, tau, part, scale, nr, out); break;
        }
    } else {
        int rb = gv.kind == 0 ? (n_recv + gv.warps_or_block - 1) / gv.warps_or_block
                              : (int)((wtiles + gv.warps_or_block - 1) / gv.warps_or_block);
        dim3 grid(rb, n_chunks);
        switch (variant) {
            case 4: gather_packet_kernel<4, 32, false><<<grid, 128, 0, st>>>(s, recv, n_recv, img_w, vpls, n_vpl, chunk_len, mode, tau, part); break;
            case 5: gather_packet_kernel<2, 32, false><<<grid, 64, 0, st>>>(s, recv, n_recv, img_w, vpls, n_vpl, chunk_len, mode, tau, part); break;
            case 6: gather_packet_kernel<4, 32, true><<<grid, 128, 0, st>>>(s, recv, n_recv, img_w, vpls, n_vpl, chunk_len, mode, tau, part); break;
            default: gather_kernel<128, 64><<<grid, 128, 0, st>>>(s, recv, n_recv, vpls, n_vpl, chunk_len, mode, tau, part); break;
        }
    }
    RZK_CUDA_TRY(cudaGetLastError());
    reduce_chunks_kernel<<<(3 * n_recv + 255) / 256, 256, 0, st>>>(part, n_recv, n_chunks, scale, out);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

// Grows the context's scratch (cudaFree / cudaMalloc synchronise with work still using it).
rzk_status ensure_scratch(rzk_context *ctx, size_t bytes) {
    if (bytes <= ctx->partial_bytes) return RZK_OK;
    if (ctx->d_partial) cudaFree(ctx->d_partial);
    ctx->d_partial = nullptr;
    ctx->partial_bytes = 0;
    RZK_CUDA_TRY(cudaMalloc((void **)&ctx->d_partial, bytes));
    ctx->partial_bytes = bytes;
    return RZK_OK;
}

rzk_status launch_matrix(const DevScene &s, const rzk_receiver *recv, int n_recv, const rzk_vpl *vpls,
                         int n_vpl, int mode, float tau, float *mat, uint8_t *vis, int kind,
                         cudaStream_t st) {
    if (n_recv <= 0 || n_vpl <= 0) return RZK_OK;
    dim3 grid((n_recv + kMatBlock - 1) / kMatBlock, std::min(n_vpl, 65535));
    matrix_kernel<<<grid, kMatBlock, 0, st>>>(s, recv, n_recv, vpls, n_vpl, mode, tau, mat, vis, kind);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

rzk_status launch_mean(rzk_context *ctx, const DevScene &s, const rzk_receiver *recv, int n_recv,
                       const rzk_vpl *vpls, int n_vpl, uint32_t seed, int n_pairs, double *h_mean,
                       cudaStream_t st) {
    if (n_pairs <= 0 || n_recv <= 0 || n_vpl <= 0) { *h_mean = 0.0; return RZK_OK; }
    int nb = (n_pairs + kMeanBlock - 1) / kMeanBlock;
    double *buf = nullptr;
    RZK_CUDA_TRY(cudaMalloc((void **)&buf, sizeof(double) * (nb + 1)));
    mean_kernel<<<nb, kMeanBlock, 0, st>>>(s, recv, n_recv, vpls, n_vpl, seed, n_pairs, buf + 1);
    mean_final_kernel<<<1, 32, 0, st>>>(buf + 1, nb, n_pairs, buf);
    cudaError_t e = cudaMemcpyAsync(h_mean, buf, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(buf);
    if (e != cudaSuccess) { set_last_cuda_error(e, "mean", __FILE__, __LINE__); return RZK_ERR_CUDA; }
    (void)ctx;
    return RZK_OK;
}

// The persistent gather (4 warps, 32-VPL tiles, 7 CTAs per SM, 8 x 4 warp tiles) on
// caller-provided scratch: a chunk ring in `ring_mem` with as many tile slots as its
// `ring_mem_bytes` hold (up to kRingSlots; RZK_ERR_CAPACITY when not one fits) and the work
// counter `work`, both zeroed on `st` first.  n_chunks as resolved by the caller (chunk
// boundaries on multiples of 128 VPLs).  Used by the allocation-free entry point
// (rzk_noalloc.cu).
rzk_status launch_gather_scratch(const DevScene &s, const rzk_receiver *recv, int n_recv, int img_w,
                                 const rzk_vpl *vpls, int n_vpl, int mode, float tau, float scale,
                                 float *out, int n_chunks, void *ring_mem, size_t ring_mem_bytes, int *work,
                                 cudaStream_t st) {
    if (n_recv <= 0) return RZK_OK;
    const long long wtiles = warp_tiles<8>(n_recv, img_w);
    if (n_vpl <= 0) n_chunks = 1;
    int chunk_len = n_vpl > 0 ? (n_vpl + n_chunks - 1) / n_chunks : 0;
    chunk_len = (chunk_len + 127) / 128 * 128;
    if (chunk_len > 0) n_chunks = (n_vpl + chunk_len - 1) / chunk_len;
    const int slots = (int)std::min<long long>(wtiles, ring_slots_fitting(ring_mem_bytes, n_chunks));
    if (slots < 1) return RZK_ERR_CAPACITY;
    // resident grid per device, computed once per device (std::call_once: concurrent first
    // calls from several host threads wait for the one computation)
    struct Grid {
        std::once_flag once;
        int blocks = 0;
        cudaError_t err = cudaSuccess;
    };
    static Grid grid_per_device[64];
    int dev = 0;
    RZK_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return RZK_ERR_UNSUPPORTED;
    Grid &g = grid_per_device[dev];
    std::call_once(g.once, [&g, dev] {
        int sms = 0, per_sm = 0;
        g.err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (g.err == cudaSuccess)
            g.err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gather_persistent_kernel<4, 32, 7, 8, true>,
                                                                  128, 0);
        g.blocks = std::max(1, sms * std::max(1, per_sm));
    });
    RZK_CUDA_TRY(g.err);
    RZK_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int), st));
    RZK_CUDA_TRY(cudaMemsetAsync(ring_mem, 0, ring_counter_bytes(slots), st));
    gather_persistent_kernel<4, 32, 7, 8, true><<<g.blocks, 128, 0, st>>>(
        s, recv, n_recv, img_w, vpls, n_vpl, chunk_len, n_chunks, (int)wtiles, work, mode, tau, nullptr, scale,
        ring_at(ring_mem, slots), out);
    RZK_CUDA_TRY(cudaGetLastError());
    return RZK_OK;
}

rzk_status launch_ring_wait_probe(rzk_context *ctx, int timeout_ms, int *h_acquired, cudaStream_t st) {
    RZK_TRY(ensure_scratch(ctx, ring_bytes(1, 1)));
    char *base = (char *)ctx->d_partial;
    int *acquired = (int *)(base + 64);   // inside the counters' 256 bytes, past the two counters
    RZK_CUDA_TRY(cudaMemsetAsync(base, 0, ring_counter_bytes(1), st));
    ring_wait_probe_kernel<<<1, 32, 0, st>>>(ring_at(base, 1), ctx->d_err, 1000000ull * (unsigned long long)timeout_ms,
                                             acquired);
    RZK_CUDA_TRY(cudaGetLastError());
    RZK_CUDA_TRY(cudaMemcpyAsync(h_acquired, acquired, sizeof(int), cudaMemcpyDeviceToHost, st));
    RZK_CUDA_TRY(cudaStreamSynchronize(st));
    return RZK_OK;
}

// Chunk ring layout: [done: slots ints | round: slots ints](256-byte aligned) then the
// sums, slots x n_chunks x 32 lanes x 3 floats.
size_t ring_counter_bytes(int slots) { return ((size_t)2 * sizeof(int) * slots + 255) & ~(size_t)255; }

size_t ring_bytes(int slots, int n_chunks) {
    return ring_counter_bytes(slots) + sizeof(float) * 96 * (size_t)n_chunks * slots;
}

int ring_slots_fitting(size_t bytes, int n_chunks) {
    const size_t per = sizeof(float) * 96 * (size_t)std::max(1, n_chunks) + 2 * sizeof(int);
    long long k = (long long)std::min<size_t>(bytes / per, (size_t)kRingSlots);
    while (k > 0 && ring_bytes((int)k, n_chunks) > bytes) --k;
    return (int)k;
}

ChunkRing ring_at(void *base, int slots) {
    ChunkRing r;
    r.done = (int *)base;
    r.round = r.done + slots;
    r.sums = (float *)((char *)base + ring_counter_bytes(slots));
    r.slots = slots;
    return r;
}

}  // namespace rzk
