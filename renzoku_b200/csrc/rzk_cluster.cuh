// rzk_cluster.cuh - the transport-matrix clustering entry points shared with LightSlice.
#ifndef RZK_CLUSTER_CUH_
#define RZK_CLUSTER_CUH_

#include "rzk_internal.cuh"
#include "rzk_hostutil.h"

namespace rzk {

// LightTransportMatrix::generate_alphas_for_clustering / get_column_norms on the device.
rzk_status ltm_alphas(const float *mat, int rows, int cols, float *alphas, float *col_norms, cudaStream_t st);

// ClusterBuilder::cluster_by_sampling; h_mags (optional, cols floats) receives the column
// magnitudes whose per-cluster distribution picks the representatives.
rzk_status cluster_by_sampling(const float *mat, int rows, int cols, int num_clusters, uint32_t seed,
                               int *h_n, int32_t *h_center, int32_t *h_rep, float *h_weight,
                               int32_t *h_assign, cudaStream_t st, float *h_mags = nullptr);
// The same, drawing from a stream the caller has already advanced (the reference draws
// the clustering from the scene's one stream after whatever came before it).
rzk_status cluster_by_sampling(const float *mat, int rows, int cols, int num_clusters, HostRng &g, int *h_n,
                               int32_t *h_center, int32_t *h_rep, float *h_weight, int32_t *h_assign,
                               cudaStream_t st, float *h_mags = nullptr);

}  // namespace rzk

#endif  // RZK_CLUSTER_CUH_
