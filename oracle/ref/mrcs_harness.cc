/*
 * mrcs_harness.cc - TEST INFRASTRUCTURE ONLY.
 *
 * Runs the reference's MatrixRowColumnSampling (mrcs.cc, with image_sampler.cc,
 * light_transport_matrix.cc, cluster_builder.cc and pdf.cc), compiled here from the
 * reference sources, so that tests can pin the B200 MRCS set-up and gather against it.
 * Everything below the entry point is reference code: MatrixRowColumnSampling::initialize
 * (stratified pixels, column resampling, LightTransportMatrix::fill,
 * ClusterBuilder::cluster_by_sampling) and gather_clusters.  The scene's Random is the
 * counter-based stream of rng_shim.c, set to (seed, 7, 0) before initialize, which is
 * the stream the B200 set-up consumes in the same program order.  The evaluator is the
 * harness's restatement of VirtualPointLight::radiance (ref_common.h).
 */
#include "ref_common.h"
#include "cluster.h"
#include "mrcs.h"

using namespace rref;

namespace {

/* Exposes the clusters MatrixRowColumnSampling keeps. */
class MrcsProbe : public MatrixRowColumnSampling {
public:
    const Clusters &clusters() const { return all_clusters; }
};

}  // namespace

extern "C" {

/* MatrixRowColumnSampling with the given parameters (max_columns is the reference's fixed
 * 10000) initialised on the VPLs, then gather_clusters for every receiver into out_rgb
 * (unscaled).  Writes up to `cap` clusters (centre, representative, weight) and returns
 * the number of clusters. */
int rref_mrcs(void *h, const rzk_vpl *vpls, int n_vpl, int clamp_mode, float tau, uint32_t seed, int block_size,
              float cluster_ratio, int max_clusters, const rzk_receiver *recv, int n_recv, float *out_rgb,
              int32_t *center, int32_t *rep, float *weight, int cap) {
    RefScene *s = (RefScene *)h;
    BrdfPointLights pls;
    pls.reserve(n_vpl);
    for (int j = 0; j < n_vpl; ++j) pls.push_back(to_vpl(s, vpls[j]));
    HarnessEval ev;
    ev.s = s;
    ev.mode = clamp_mode;
    ev.tau = tau;
    MrcsProbe m;
    m.set_block_size(block_size);
    m.set_cluster_ratio(cluster_ratio);
    m.set_max_clusters(max_clusters);
    rref_rng_stream(seed, 7u, 0u);
    m.initialize(s->scene, &ev, pls);
    for (int i = 0; i < n_recv; ++i) {
        Receiver rc = to_receiver(s, recv[i]);
        put3(out_rgb + 3 * i, m.gather_clusters(rc, &ev));
    }
    const Clusters &cl = m.clusters();
    for (size_t c = 0; c < cl.size() && (int)c < cap; ++c) {
        center[c] = cl[c].center;
        rep[c] = cl[c].representative;
        weight[c] = cl[c].weight;
    }
    return (int)cl.size();
}

}  // extern "C"
