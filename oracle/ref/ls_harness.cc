/*
 * ls_harness.cc - TEST INFRASTRUCTURE ONLY.
 *
 * Drives the reference's LightSlice code (lightslice.cc, kdtree_n.h, cluster_builder.cc,
 * matrix_c.cc, cone.cc, pdf.cc), compiled here from the reference sources, so that tests
 * can pin the B200 LightSlice stages against it.  lightslice.cc is included into this
 * translation unit (through the shims of ls_pre.h) because the functions the refinement
 * is made of (split_cluster, compute_distance, choose_representative, pick, map_vec6) are
 * static in it; LightSlice's members (its header alone) are opened with an access macro so
 * that the harness can set the state that LightSlice::initialize would have built.
 *
 * What runs here is reference code: LightSlice::generate_slices (the 6-D points, the
 * KdTreeN<6> cluster build and the representative draws), KdTreeN::find_cluster and
 * find_nearest_cluster, the per-slice refinement's building blocks, Cone::merge_direction,
 * LightSlice::estimate_sum, LightSlice::build_map with DiscretePdf2D, and
 * LightSlice::gather_clusters.  Restated from lightslice.cc (their bodies live in
 * LightSlice::initialize, which also traces the reduced matrix and runs the global
 * clustering from one global random stream): the reduced-matrix loop
 * (lightslice.cc:721-742), the per-slice refinement loop (lightslice.cc:838-1010), the
 * cluster-norm cache (lightslice.cc:1117-1174) and the point loop of generate_slices
 * (lightslice.cc:261-275, for the points in pixel order).  The per-slice loop draws slice
 * s from the counter-based stream (seed, 5, s), as the B200 implementation does, so that
 * slices can be refined independently; everything else in the loop is the reference's.
 */
#include <algorithm>
#include <any>
#include <array>
#include <bitset>
#include <cfloat>
#include <chrono>
#include <condition_variable>
#include <random>
#include <tuple>
#include <unordered_map>
#include <unordered_set>
#include <optional>
#include <variant>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <exception>
#include <fstream>
#include <functional>
#include <iostream>
#include <iterator>
#include <limits>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <queue>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "ref_common.h"
#include "ls_pre.h"
#include "cluster.h"
#include "kdtree_n.h"
#include "light_transport_matrix.h"
#include "kdtree_2.h"
#include "image.h"
#include "events.h"
// only LightSlice's own members are opened; every other class keeps its declared access
// (and so its layout rules) as the other translation units see it
#define private public
#define protected public
#include "lightslice.h"
#undef private
#undef protected
#include "lightslice.cc"
#include "first_bounce.h"

using namespace rref;

namespace {

struct RefLs {
    RefScene *s = nullptr;
    LightSlice *ls = nullptr;
    BrdfPointLights vpls1;
    HarnessEval ev;
    int k = 16;
    int sampler = 0;          // 0 JENSEN, 1 METROPOLIS
    bool metro_ready = false;
};

Receiver rep_receiver(RefLs *h, int s) {
    LightSlice *ls = h->ls;
    Size2 img = ls->scene->get_image_size();
    int pixel_index = ls->node_data[ls->slices[s].representative].index;
    int y = pixel_index / (int)img.width;
    int x = pixel_index % (int)img.width;
    Ray ray = ls->scene->get_camera()->shoot_ray(y, x);
    HitRecord rec;
    ls->scene->get_aggregate()->hit(ray, ls->scene->get_tmin(), ls->scene->get_max_tmax(), ls->scene->get_tick(),
                                    rec);
    return Receiver(ray, rec);
}

}  // namespace

extern "C" {

/* LightSlice::generate_slices on the harness scene with the stream (seed, 4, 0). */
void *rref_ls_create(void *scene, int max_slice_size, int num_neighbors, uint32_t seed) {
    RefLs *h = new RefLs();
    h->s = (RefScene *)scene;
    h->k = num_neighbors;
    h->ls = new LightSlice();
    LightSlice *ls = h->ls;
    ls->scene = h->s->scene;
    ls->scene_bb_diag = h->s->scene->get_bounding_box().diagonal();
    ls->max_slice_size = max_slice_size;
    ls->num_neighbor_slices = num_neighbors;
    h->ev.s = h->s;
    ls->evaluator = &h->ev;
    rref_rng_stream(seed, 4u, 0u);
    ls->generate_slices();
    return h;
}

int rref_ls_num_points(void *hp) {
    RefLs *h = (RefLs *)hp;
    Size2 img = h->ls->scene->get_image_size();
    int n = 0;
    Camera *camera = h->ls->scene->get_camera();
    Aggregate *agg = h->ls->scene->get_aggregate();
    for (int i = 0; i < (int)img.height; ++i)
        for (int j = 0; j < (int)img.width; ++j) {
            Ray r = camera->shoot_ray(i, j);
            HitRecord rec;
            if (agg->hit(r, h->ls->scene->get_tmin(), h->ls->scene->get_max_tmax(), h->ls->scene->get_tick(), rec) &&
                rec.material)
                ++n;
        }
    return n;
}

int rref_ls_num_slices(void *hp) { return (int)((RefLs *)hp)->ls->slices.size(); }

/* The 6-D points in pixel order (the loop of generate_slices, lightslice.cc:261-275). */
void rref_ls_points(void *hp, float *pts, int32_t *pix) {
    RefLs *h = (RefLs *)hp;
    LightSlice *ls = h->ls;
    Size2 img = ls->scene->get_image_size();
    Camera *camera = ls->scene->get_camera();
    Aggregate *agg = ls->scene->get_aggregate();
    int n = 0;
    for (int i = 0; i < (int)img.height; ++i)
        for (int j = 0; j < (int)img.width; ++j) {
            Ray r = camera->shoot_ray(i, j);
            HitRecord rec;
            if (agg->hit(r, ls->scene->get_tmin(), ls->scene->get_max_tmax(), ls->scene->get_tick(), rec) &&
                rec.material) {
                Receiver recv(r, rec);
                Vec6 p = map_vec6(recv.p, recv.shading_n, recv.m, recv.wo, ls->scene_bb_diag);
                for (int d = 0; d < 6; ++d) pts[6 * n + d] = p.p[d];
                pix[n] = i * (int)img.width + j;
                ++n;
            }
        }
}

/* Tree order of the points (their pixels), slices and representatives. */
void rref_ls_slices(void *hp, int32_t *point_pixel, int32_t *start, int32_t *end, int32_t *rep) {
    RefLs *h = (RefLs *)hp;
    LightSlice *ls = h->ls;
    int n = rref_ls_num_points(hp);
    for (int i = 0; i < n; ++i) point_pixel[i] = ls->node_data[i].index;
    for (size_t s = 0; s < ls->slices.size(); ++s) {
        start[s] = ls->slices[s].start;
        end[s] = ls->slices[s].end;
        rep[s] = ls->slices[s].representative;
    }
}

/* KdTreeN::find_nearest_cluster from every representative: k per slice, -1 padded. */
void rref_ls_neighbors(void *hp, int32_t *out) {
    RefLs *h = (RefLs *)hp;
    LightSlice *ls = h->ls;
    vector<int> idx;
    for (size_t s = 0; s < ls->slices.size(); ++s) {
        ls->kdtree->find_nearest_cluster(ls->node_data[ls->slices[s].representative].p, h->k, idx);
        for (int t = 0; t < h->k; ++t) out[s * h->k + t] = t < (int)idx.size() ? idx[t] : -1;
    }
}

/* KdTreeN::find_cluster for 6-D points. */
void rref_ls_find(void *hp, const float *pts, int n, int32_t *out) {
    RefLs *h = (RefLs *)hp;
    for (int i = 0; i < n; ++i) {
        Vec6 p;
        for (int d = 0; d < 6; ++d) p.p[d] = pts[6 * i + d];
        int c = -1;
        h->ls->kdtree->find_cluster(p, c);
        out[i] = c;
    }
}

/* The reduced matrix (lightslice.cc:698-748, restated): the VPLs of bounce <= 1 (returned
 * count), R = visible x incident radiance and V, column-major [n1][slices]; the
 * representatives' receivers. */
int rref_ls_reduced_matrix(void *hp, const rzk_vpl *vpls, int n_vpl, int inc_mode, float inc_tau, float *R,
                           uint8_t *V, rzk_receiver *rep_recv) {
    RefLs *h = (RefLs *)hp;
    LightSlice *ls = h->ls;
    h->ev.inc_mode = inc_mode;
    h->ev.inc_tau = inc_tau;
    h->vpls1.clear();
    for (int i = 0; i < n_vpl; ++i)
        if (vpls[i].bounce <= 1) h->vpls1.push_back(to_vpl(h->s, vpls[i]));
    const int ns = (int)ls->slices.size(), n1 = (int)h->vpls1.size();
    Aggregate *agg = ls->scene->get_aggregate();
    Float tmin = ls->scene->get_tmin(), tick = ls->scene->get_tick();
    for (int s = 0; s < ns; ++s) {
        Receiver recv = rep_receiver(h, s);
        Size2 img = ls->scene->get_image_size();
        int pixel_index = ls->node_data[ls->slices[s].representative].index;
        Ray ray = ls->scene->get_camera()->shoot_ray(pixel_index / (int)img.width, pixel_index % (int)img.width);
        HitRecord rec;
        agg->hit(ray, tmin, ls->scene->get_max_tmax(), tick, rec);
        fill_receiver(ray, rec, rep_recv[s], h->s);
        for (int k = 0; k < n1; ++k) {
            bool visible = (agg->hit(recv.p, h->vpls1[k].org(), tmin, tick) == false);
            Rgb radiance = (Float)visible * h->ev.incident_radiance(ls->scene, recv, h->vpls1[k]);
            put3(R + 3 * ((size_t)k * ns + s), radiance);
            V[(size_t)k * ns + s] = visible ? 1 : 0;
        }
    }
    return n1;
}

/* The one-bounce VPLs of the LightSlice without tracing the reduced matrix (for callers
 * that pass a reduced matrix computed elsewhere to rref_ls_refine); returns their count. */
int rref_ls_set_vpls(void *hp, const rzk_vpl *vpls, int n_vpl) {
    RefLs *h = (RefLs *)hp;
    h->vpls1.clear();
    for (int i = 0; i < n_vpl; ++i)
        if (vpls[i].bounce <= 1) h->vpls1.push_back(to_vpl(h->s, vpls[i]));
    return (int)h->vpls1.size();
}

/* Per-slice refinement and maps from the given reduced matrix and global clusters. */
void rref_ls_refine(void *hp, const float *R, const uint8_t *V, int n1, int n_global, const int32_t *g_rep,
                    const float *g_weight, const int32_t *assign, const float *mags, int max_slice_clusters,
                    uint32_t seed, int res, float eps, float density_radius) {
    RefLs *h = (RefLs *)hp;
    LightSlice *ls = h->ls;
    const int ns = (int)ls->slices.size();
    ls->max_slice_clusters = max_slice_clusters;
    ls->luminance_map_resolution = res;
    ls->luminance_map_epsilon = eps;
    ls->density_radius = density_radius;
    ls->all_vpls = &h->vpls1;
    ls->R.resize(ns, n1);
    MatrixC<Rgb> &matR = ls->R.get_matrix();
    ls->matV.resize(ns, n1);
    for (int k = 0; k < n1; ++k)
        for (int s = 0; s < ns; ++s) {
            const float *x = R + 3 * ((size_t)k * ns + s);
            matR(s, k) = Rgb(x[0], x[1], x[2]);
            ls->matV(s, k) = (Float)V[(size_t)k * ns + s];
        }
    // the global clusters as ClusterBuilder::cluster_by_sampling leaves them
    Clusters &mrcs = ls->mrcs_clusters;
    mrcs.assign(n_global, Cluster());
    for (int i = 0; i < n1; ++i)
        if (assign[i] >= 0) mrcs[assign[i]].indices.push_back(i);
    for (int c = 0; c < n_global; ++c) {
        vector<Float> m(mrcs[c].indices.size());
        for (size_t t = 0; t < m.size(); ++t) m[t] = mags[mrcs[c].indices[t]];
        mrcs[c].pdf.set_distribution(m);
        mrcs[c].representative = g_rep[c];
        mrcs[c].weight = g_weight[c];
    }
    BrdfPointLights &vpls = h->vpls1;
    Random &rd = *ls->scene->get_random();
    int max_cols = 0;
    for (size_t i = 0; i < mrcs.size(); ++i) max_cols = std::max(max_cols, (int)mrcs[i].indices.size());
    vector<int> slice_indices;
    MatrixC<Rgb> matL, matC;
    MatrixC<Float> matCf, matCfTrans;
    ls->matrix_clusters.clear();
    ls->matrix_clusters.resize(ns);
    vector<Float> norms, temp_col, temp_row, norms_R;
    vector<int> indices1, indices2;
    ls->R.get_column_norms(norms_R);
    for (int s = 0; s < ns; ++s) {
        rref_rng_stream(seed, 5u, (uint32_t)s);
        Vec6 &p = ls->node_data[ls->slices[s].representative].p;
        ls->kdtree->find_nearest_cluster(p, ls->num_neighbor_slices, slice_indices);
        matR.subrow(slice_indices, matL);
        Clusters &slice_clusters = ls->matrix_clusters[s];
        slice_clusters.assign(mrcs.begin(), mrcs.end());
        ClusterCostHeap heap;
        for (int c = 0; c < (int)slice_clusters.size(); ++c) {
            matL.subcol(slice_clusters[c].indices, matC);
            matC.flatten(matCf);
            matCf.get_column_norm(norms);
            matCf.transpose(matCfTrans);
            Float cost = compute_distance(matCf, norms, matCfTrans, temp_col, temp_row);
            heap.push(ClusterCost(c, cost));
        }
        while (heap.size() > 0 && (int)slice_clusters.size() < ls->max_slice_clusters) {
            ClusterCost cc = heap.top();
            if (slice_clusters[cc.index].indices.size() <= 1) break;
            matL.subcol(slice_clusters[cc.index].indices, matC);
            matC.flatten(matCf);
            split_cluster(rd, slice_clusters[cc.index], matCf, indices1, indices2);
            Cluster &cluster1 = slice_clusters[cc.index];
            matL.subcol(indices1, matC);
            matC.flatten(matCf);
            matCf.get_column_norm(norms);
            matCf.transpose(matCfTrans);
            Float cost1 = compute_distance(matCf, norms, matCfTrans, temp_col, temp_row);
            cluster1.indices.assign(indices1.begin(), indices1.end());
            pick(norms_R, indices1, norms);
            cluster1.pdf.set_distribution(norms);
            choose_representative(rd, cluster1);
            Cluster cluster2;
            matL.subcol(indices2, matC);
            matC.flatten(matCf);
            matCf.get_column_norm(norms);
            matCf.transpose(matCfTrans);
            Float cost2 = compute_distance(matCf, norms, matCfTrans, temp_col, temp_row);
            cluster2.indices.assign(indices2.begin(), indices2.end());
            pick(norms_R, indices2, norms);
            cluster2.pdf.set_distribution(norms);
            choose_representative(rd, cluster2);
            int new_index = (int)slice_clusters.size();
            ClusterCost cc1(cc.index, cost1);
            ClusterCost cc2(new_index, cost2);
            heap.pop();
            heap.push(cc1);
            heap.push(cc2);
            slice_clusters.push_back(cluster2);
        }
        Receiver recv = rep_receiver(h, s);
        for (int c = 0; c < (int)slice_clusters.size(); ++c) {
            Cluster &cluster = slice_clusters[c];
            Rgb incident, outgoing;
            for (size_t i = 0; i < cluster.indices.size(); ++i) {
                BrdfPointLight &vpl = vpls[cluster.indices[i]];
                Float visibility = ls->matV(s, cluster.indices[i]);
                Rgb incident_power = h->ev.incident_radiance(ls->scene, recv, vpl);
                incident += visibility * incident_power;
                outgoing += matR(s, cluster.indices[i]);
                Vec3 wi = unit_vector(vpl.org() - recv.p);
                if (visibility > 0.0f && dot(recv.shading_n, wi) > ZERO_EPSILON && incident_power != DefaultRgb::black)
                    cluster.bc.merge_direction(wi);
                if (cluster.indices[i] == cluster.representative) {
                    cluster.slice_wi = wi;
                    if (visibility > 0.0f && dot(recv.shading_n, wi) > ZERO_EPSILON &&
                        incident_power != DefaultRgb::black)
                        cluster.is_upper_hemisphere = true;
                }
            }
            if (cluster.bc.half_angle() > HALF_PI) cluster.bc.set_half_angle(HALF_PI);
            cluster.total_incident_radiance = incident;
            cluster.total_outgoing_radiance = outgoing;
        }
    }
    // cluster norms for the slice distributions (lightslice.cc:1117-1174)
    vector<int> reps;
    for (int s = 0; s < ns; ++s) {
        Vec6 &p = ls->node_data[ls->slices[s].representative].p;
        ls->kdtree->find_nearest_cluster(p, ls->num_neighbor_slices, slice_indices);
        matR.subrow(slice_indices, matL);
        reps.resize(ls->matrix_clusters[s].size());
        for (size_t c = 0; c < reps.size(); ++c) reps[c] = ls->matrix_clusters[s][c].representative;
        matL.subcol(reps, matC);
        vector<Float> cluster_norm;
        matC.get_column_norm(cluster_norm);
        for (size_t c = 0; c < reps.size(); ++c) {
            cluster_norm[c] *= ls->matrix_clusters[s][c].weight;
            if (ls->matrix_clusters[s][c].is_upper_hemisphere == false) cluster_norm[c] = 0.0f;
        }
        ls->slices[s].cluster_pdf.set_distribution(cluster_norm);
    }
    // validity from estimate_sum, then build_map (the records made valid first)
    ls->sampling_records.resize(ns);
    for (int s = 0; s < ns; ++s) {
        Receiver recv = rep_receiver(h, s);
        ls->sampling_records[s].uvn = recv.shading_uvn;
        ls->sampling_records[s].is_valid = true;
        Float sum = ls->estimate_sum(s);
        ls->sampling_records[s].sum_vpl = sum;
        ls->sampling_records[s].is_valid = sum > 0.0f;
        ls->build_map(s);
    }
}

int rref_ls_num_slice_clusters(void *hp) {
    RefLs *h = (RefLs *)hp;
    int n = 0;
    for (auto &c : h->ls->matrix_clusters) n += (int)c.size();
    return n;
}

void rref_ls_clusters(void *hp, int32_t *count, int32_t *rep, float *weight, uint8_t *upper, float *wi,
                      float *incident, float *pdf, int32_t *size, int32_t *members, float *cone) {
    RefLs *h = (RefLs *)hp;
    LightSlice *ls = h->ls;
    size_t k = 0, m = 0;
    for (size_t s = 0; s < ls->matrix_clusters.size(); ++s) {
        count[s] = (int32_t)ls->matrix_clusters[s].size();
        for (size_t c = 0; c < ls->matrix_clusters[s].size(); ++c) {
            const Cluster &cl = ls->matrix_clusters[s][c];
            rep[k] = cl.representative;
            weight[k] = cl.weight;
            upper[k] = cl.is_upper_hemisphere ? 1 : 0;
            put3(wi + 3 * k, cl.slice_wi);
            put3(incident + 3 * k, cl.total_incident_radiance);
            pdf[k] = ls->slices[s].cluster_pdf.probability((int)c);
            size[k] = (int32_t)cl.indices.size();
            for (int x : cl.indices) members[m++] = x;
            if (cone) {
                put3(cone + 4 * k, cl.bc.normal());
                cone[4 * k + 3] = cl.bc.half_angle();
            }
            ++k;
        }
    }
}

/* Maps, validity, VPL sums and DiscretePdf2D::probability of every cell. */
void rref_ls_maps(void *hp, float *maps, uint8_t *valid, float *sum, float *prob) {
    RefLs *h = (RefLs *)hp;
    LightSlice *ls = h->ls;
    const int res = ls->luminance_map_resolution;
    for (size_t s = 0; s < ls->slices.size(); ++s) {
        const ImageFloat &map = ls->slices[s].luminance_map;
        const DiscretePdf2D &d = ls->slices[s].luminance_map_pdf;
        for (int y = 0; y < res; ++y)
            for (int x = 0; x < res; ++x) {
                maps[(s * res + y) * res + x] = map(y, x);
                prob[(s * res + y) * res + x] = d.probability(y, x);
            }
        valid[s] = ls->sampling_records[s].is_valid ? 1 : 0;
        sum[s] = ls->sampling_records[s].sum_vpl;
    }
}

/* VirtualPointLight::trace_wellington with METRO_RANDOM (vpl.cc:934-1040), restated (it
 * is a VirtualPointLight member) around the reference's FirstBounce::radiance,
 * ShadingGeometry, Material and LightSlice::sample / pdf; plus the Russian roulette
 * extension at vertices deeper than rr_depth (0 = off). */
static Rgb ref_trace(RefLs *h, const Receiver &r, int bounce, int max_bounce, int rr_depth, float rr_prob,
                     bool direct) {
    Scene *scene = h->ls->scene;
    Aggregate *agg = scene->get_aggregate();
    Random &rd = *scene->get_random();
    Float tmin = scene->get_tmin(), max_tmax = scene->get_max_tmax(), tick = scene->get_tick();
    if (bounce > max_bounce) return DefaultRgb::black;
    if (r.light) {
        if (bounce == 1 && direct) {
            Rgb Le;
            r.light->query(r.p, r.shading_n, r.wo, Le);
            return Le;
        }
        return DefaultRgb::black;
    }
    LocalGeometry dg(r);
    ShadingGeometry sg(r);
    HitRecord rec;
    Vec3 wi;
    Float pdf_wi;
    Rgb radiance, brdf;
    bool is_brdf_sampling = rd() < 0.5f;
    if (bounce > 1 || (bounce == 1 && direct)) radiance = FirstBounce::radiance(scene, r, NULL);
    if (bounce >= max_bounce) return radiance;
    bool rr = false;
    if (rr_depth > 0 && bounce > rr_depth) {
        if (rd() >= rr_prob) return radiance;
        rr = true;
    }
    if (is_brdf_sampling) brdf = sg.sample(rd, wi, pdf_wi);
    else brdf = h->ls->sample(rd, r, wi, pdf_wi);
    if (pdf_wi > 0.0f) {
        Ray ray(r.p, wi);
        if (agg->hit(ray, tmin, max_tmax, tick, rec)) {
            if (rec.light) return radiance;
            Receiver recv(ray, rec);
            Rgb Li = ref_trace(h, recv, bounce + 1, max_bounce, rr_depth, rr_prob, direct);
            Float pdf_wi_other;
            if (is_brdf_sampling) pdf_wi_other = h->ls->pdf(r, wi);
            else pdf_wi_other = r.m->pdf(dg, r.wo, wi);
            Float weight = pdf_wi / (pdf_wi + pdf_wi_other);
            Rgb term = weight * Li * brdf * sg.cosine(wi) / pdf_wi * 2;
            if (rr) term = term / rr_prob;
            radiance += term;
        }
    }
    return radiance;
}

/* The METROPOLIS sampler's set-up, as LightSlice::initialize runs it after the maps
 * (lightslice.cc:1180-1262, restated here around the reference's types): a KdTree2 per slice
 * over its visible clusters' directions on the unit square of its sampling record, and each
 * record's chain reset with sum_f = sum_vpl (FIXED_RADIUS).  Runs once. */
static void metro_prepare(RefLs *h) {
    if (h->metro_ready) return;
    LightSlice *ls = h->ls;
    for (int s = 0; s < (int)ls->matrix_clusters.size(); ++s) {
        const int slice = s;
        int n = 0;
        for (size_t c = 0; c < ls->matrix_clusters[slice].size(); ++c)
            if (ls->matrix_clusters[slice][c].is_upper_hemisphere) n++;
        ls->slices[s].tree_node_data = new NodeData2[n];
        NodeData2 *data = ls->slices[s].tree_node_data;
        n = 0;
        if (!ls->sampling_records[slice].is_valid) continue;
        for (size_t c = 0; c < ls->matrix_clusters[slice].size(); ++c) {
            if (!ls->matrix_clusters[slice][c].is_upper_hemisphere) continue;
            Vec3 local_wi = ls->sampling_records[s].uvn.world_to_local(ls->matrix_clusters[slice][c].slice_wi);
            if (local_wi.z() <= 0.0f) continue;
            data[n].p = direction_to_square(local_wi);
            data[n].index = slice * ls->max_slice_clusters + (int)c;
            n++;
        }
        ls->slices[s].kdtree = new KdTree2(data, n, ls->scene);
    }
    for (int s = 0; s < (int)ls->matrix_clusters.size(); ++s) {
        LightSlice::SamplingRecord &record = ls->sampling_records[s];
        record.start = true;
        record.w = Vec3(0.0f);
        record.f = 0.0f;
        record.sum_f = record.sum_vpl;
    }
    h->metro_ready = true;
}

/* LightSlice::eval_incoming_radiance(slice[i], xy[i]) (FIXED_RADIUS). */
void rref_ls_density(void *hp, const int32_t *slice, const float *xy, int n, float *out) {
    RefLs *h = (RefLs *)hp;
    metro_prepare(h);
    for (int i = 0; i < n; ++i) {
        Vec2 x(xy[2 * i], xy[2 * i + 1]);
        out[i] = h->ls->eval_incoming_radiance(slice[i], x);
    }
}

/* Selects the direction sampler of rref_ls_guided: 0 JENSEN, 1 METROPOLIS (whose chains
 * then start afresh). */
void rref_ls_set_sampler(void *hp, int sampler) {
    RefLs *h = (RefLs *)hp;
    h->sampler = sampler;
    if (sampler == 1) {
        if (h->metro_ready) {
            for (size_t s = 0; s < h->ls->sampling_records.size(); ++s) {
                h->ls->sampling_records[s].start = true;
                h->ls->slices[s].sample_remains = 0;
            }
        }
        metro_prepare(h);
    }
}

/* Guided path tracing of the given pixels (VirtualPointLight::guided_path_trace,
 * vpl.cc:907-932, pixel-centre rays): sample s of pixel k from the stream
 * (seed, 6, k * spp + s); out[(i * spp + s) * 3] for the i-th listed pixel. */
void rref_ls_guided(void *hp, const int32_t *pixels, int n, int spp, int max_bounce, int rr_depth, float rr_prob,
                    int direct, uint32_t seed, float *out) {
    RefLs *h = (RefLs *)hp;
    LightSlice *ls = h->ls;
    ls->sampling_type = h->sampler == 1 ? LightSlice::LocalSampler::METROPOLIS : LightSlice::LocalSampler::JENSEN;
    Scene *scene = ls->scene;
    Size2 img = scene->get_image_size();
    for (int i = 0; i < n; ++i) {
        const int k = pixels[i];
        for (int smp = 0; smp < spp; ++smp) {
            rref_rng_stream(seed, 6u, (uint32_t)(k * spp + smp));
            Ray r = scene->get_camera()->shoot_ray(k / (int)img.width, k % (int)img.width);
            HitRecord rec;
            Rgb L;
            if (scene->get_aggregate()->hit(r, scene->get_tmin(), scene->get_max_tmax(), scene->get_tick(), rec)) {
                Receiver recv(r, rec);
                L = ref_trace(h, recv, 1, max_bounce, rr_depth, rr_prob, direct != 0);
            }
            put3(out + 3 * ((size_t)i * spp + smp), L);
        }
    }
}

/* LightSlice::gather_clusters for receivers (unscaled). */
void rref_ls_gather(void *hp, const rzk_receiver *recv, int n, int mode, float tau, float *out) {
    RefLs *h = (RefLs *)hp;
    h->ev.mode = mode;
    h->ev.tau = tau;
    for (int i = 0; i < n; ++i) {
        Receiver r = to_receiver(h->s, recv[i]);
        Rgb L = h->ls->gather_clusters(r, &h->ev);
        put3(out + 3 * i, L);
    }
}

/* The same on n_threads host threads over the receivers (gather_clusters only reads the
 * LightSlice state, the scene and the evaluator's clamp settings). */
void rref_ls_gather_mt(void *hp, const rzk_receiver *recv, int n, int mode, float tau, float *out, int n_threads) {
    RefLs *h = (RefLs *)hp;
    h->ev.mode = mode;
    h->ev.tau = tau;
    if (n_threads < 1) n_threads = 1;
    auto work = [&](int t) {
        const int i0 = (int)((long long)n * t / n_threads), i1 = (int)((long long)n * (t + 1) / n_threads);
        for (int i = i0; i < i1; ++i) {
            Receiver r = to_receiver(h->s, recv[i]);
            Rgb L = h->ls->gather_clusters(r, &h->ev);
            put3(out + 3 * i, L);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < n_threads; ++t) th.emplace_back(work, t);
    work(0);
    for (auto &x : th) x.join();
}

}  // extern "C"
