"""Clustering oracle (LightTransportMatrix alphas, ClusterBuilder::cluster_by_sampling)
against the reference's own code: the golden fixture and, where the reference harness is
built, a fresh seeded case."""
import hashlib
import os

import numpy as np
import pytest

from renzoku_b200 import scenegen as sg

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "clustering_small.npz")


@pytest.fixture(scope="module")
def mat(oracle_built):
    from cluster_inputs import small_matrix
    return small_matrix()


def test_alphas_and_clusters_match_golden(mat):
    from oracle import Oracle
    g = np.load(GOLDEN)
    assert hashlib.sha256(mat.tobytes()).hexdigest() == str(g["matrix_sha"])
    a, n = Oracle.ltm_alphas(mat)
    assert np.array_equal(a, g["alphas"]) and np.array_equal(n, g["norms"])
    c, r, w, asg = Oracle.cluster_by_sampling(mat, int(g["num_clusters"]), int(g["seed"]))
    for x, y in ((c, g["center"]), (r, g["rep"]), (w, g["weight"]), (asg, g["assign"])):
        assert np.array_equal(x, y)


def test_clusters_match_reference_harness(mat):
    from oracle import Oracle, RefHarness
    if not RefHarness.available():
        pytest.skip("reference harness not built")
    ref = RefHarness(sg.room_objects(120, 24, 24, seed_geo=31, seed_mat=32))
    for k, seed in ((25, 3), (200, 4)):
        got = Oracle.cluster_by_sampling(mat, k, seed)
        exp = ref.cluster_by_sampling(mat, k, seed)
        for x, y in zip(got, exp):
            assert np.array_equal(x, y), (k, seed)
    # fewer columns than clusters: one cluster per column, no representative
    got = Oracle.cluster_by_sampling(mat[:10], 20, 5)
    exp = ref.cluster_by_sampling(mat[:10], 20, 5)
    for x, y in zip(got, exp):
        assert np.array_equal(x, y)
