"""GPU clustering (rzk_ltm_alphas, rzk_cluster_by_sampling) against the reference's
golden outputs and the oracle: bit-identical alphas, norms, centres, representatives,
weights and assignments."""
import os

import numpy as np
import pytest

from renzoku_b200 import scenegen as sg

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "clustering_small.npz")


def test_gpu_clustering_matches_reference_golden(ctx, oracle_built):
    import torch
    from cluster_inputs import small_matrix
    from renzoku_b200 import rzk
    g = np.load(GOLDEN)
    mat = torch.from_numpy(small_matrix()).cuda()
    cb = rzk.ClusterBuilderCuda()
    a, n = cb.alphas(mat)
    assert np.array_equal(a.cpu().numpy(), g["alphas"])
    assert np.array_equal(n.cpu().numpy(), g["norms"])
    c, r, w, asg = cb.cluster_by_sampling(mat, int(g["num_clusters"]), int(g["seed"]))
    for x, y in ((c, g["center"]), (r, g["rep"]), (w, g["weight"]), (asg, g["assign"])):
        assert np.array_equal(x, y)


def test_gpu_fill_and_clustering_scaled(ctx, oracle_built):
    """Matrix filled on the GPU (LightTransportMatrix::fill) for 256 shading points x 4,096
    VPLs of the scaled scene, then clustered on the GPU and by the oracle from the same
    matrix."""
    import torch
    from oracle import Oracle
    from renzoku_b200 import rzk
    sc = sg.room_objects(2000, 128, 128)
    agg = rzk.AggregateCuda(ctx, sc)
    recv_all = rzk.records_from_device(agg.primary(rzk.Camera(sc.camera)), sg.RECEIVER_DTYPE)
    rng = np.random.default_rng(11)
    rows = recv_all[np.sort(rng.choice(recv_all.shape[0], 256, replace=False))].copy()
    vt, n = rzk.VplGeneratorCuda(agg).spawn(12, 3000, 4)
    vt = vt[: 4096 * 96] if n >= 4096 else vt
    ncols = vt.numel() // 96
    ev = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 0.05)
    mat, vis = ev.fill(rzk.records_to_device(rows), rows.shape[0], vt, ncols)
    o = Oracle(sc)
    vpls = rzk.records_from_device(vt, sg.VPL_DTYPE)
    ref_rgb, ref_vis = o.gather_pairs(rows, vpls, rzk.CLAMP_RADIANCE, 0.05)
    assert np.array_equal(vis.cpu().numpy(), ref_vis)
    assert np.allclose(mat.cpu().numpy(), ref_rgb, rtol=1e-4, atol=1e-8)
    cb = rzk.ClusterBuilderCuda()
    m_np = mat.cpu().numpy()
    a_gpu, _ = cb.alphas(mat)
    a_ref, _ = Oracle.ltm_alphas(m_np)
    assert np.array_equal(a_gpu.cpu().numpy(), a_ref)
    got = cb.cluster_by_sampling(mat, 300, 21)
    exp = Oracle.cluster_by_sampling(m_np, 300, 21)
    for x, y in zip(got, exp):
        assert np.array_equal(x, y)
    assert len(got[0]) > 100
