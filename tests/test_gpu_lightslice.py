"""LightSlice on the device against the reference's LightSlice code.

On an all-Lambertian scene every stage is bit-exact: the 6-D points and slicing, the
reduced matrix (visibility x incident radiance), the refined clusters and maps, the slice
lookup of every pixel and the clustered gather.  On the mixed-material scene the incident
radiance of glossy VPLs goes through CUDA's powf / expf, so the stages after the reduced
matrix are compared on the device's own matrix: the clusters stay bit-exact (their incident
totals, which the reference recomputes on the host, within 1e-5), and the gather (glossy
BRDFs at both ends) matches to a relative L2 error below 1e-5.
"""
import numpy as np
import pytest

from renzoku_b200 import scenegen as sg

pytestmark = pytest.mark.gpu
SEED = 2013


def _run(ctx, sc, slice_size, k, n_clusters, max_sc, n_particles):
    import torch
    from oracle import RefHarness
    from renzoku_b200 import rzk
    agg = rzk.AggregateCuda(ctx, sc)
    cam = rzk.Camera(sc.camera)
    recv = agg.primary(cam)
    vt, n = rzk.VplGeneratorCuda(agg).spawn(SEED, n_particles, 3)
    params = rzk.lightslice_params(max_slice_size=slice_size, num_neighbor_slices=k, num_clusters=n_clusters,
                                   max_slice_clusters=max_sc, seed=SEED, n_threads=4)
    ls = rzk.LightSliceCuda.create(agg, recv, cam.width, cam.height, vt, n, params)
    torch.cuda.synchronize()
    ctx.check()
    ref = RefHarness(sc)
    rls = ref.lightslice(slice_size, k, SEED)
    vpls = rzk.records_from_device(vt, sg.VPL_DTYPE)
    return agg, cam, recv, vpls, ls, ref, rls


def _refine_ref_on(rls, ref, ls, R, V):
    from oracle import column_magnitudes
    _, g_rep, g_w, assign = ref.cluster_by_sampling(R, ls.params.num_clusters, SEED)
    rls.refine(R, V, g_rep, g_w, assign, column_magnitudes(R), ls.params.max_slice_clusters, SEED,
               res=ls.params.map_resolution, eps=ls.params.map_epsilon, density_radius=ls.params.density_radius)


def test_lightslice_lambertian_bit_exact(ctx, oracle_built):
    from oracle import RefHarness
    from renzoku_b200 import rzk
    if not RefHarness.available():
        pytest.skip("reference harness not built")
    sc = sg.room_boxes(48, 48)
    agg, cam, recv, vpls, ls, ref, rls = _run(ctx, sc, 64, 8, 40, 80, 400)
    a, b = ls.slices(), rls.slices()
    for key in ("point_pixel", "start", "end", "rep", "neighbors"):
        assert np.array_equal(a[key], b[key]), key
    R_ref, V_ref, _ = rls.reduced_matrix(vpls)
    R, V, idx = ls.matrix()
    assert np.array_equal(R.cpu().numpy(), R_ref)
    assert np.array_equal(V.cpu().numpy(), V_ref)
    assert np.array_equal(idx, np.nonzero(vpls["bounce"] <= 1)[0])
    _refine_ref_on(rls, ref, ls, R_ref, V_ref)
    ca, cb = ls.clusters(), rls.clusters()
    for key in ("count", "size", "members", "rep", "weight", "upper", "wi", "incident", "pdf"):
        assert np.array_equal(ca[key], cb[key]), key
    ma, mb = ls.maps(), rls.maps()
    for key in ("valid", "sum", "maps"):
        assert np.array_equal(ma[key], mb[key]), key
    # slice of every pixel, and the clustered gather
    recv_np = rzk.records_from_device(recv, sg.RECEIVER_DTYPE)
    pts_ref, pix_ref = rls.points()
    sl = ls.find_slice(recv, cam.n_pixels).cpu().numpy()
    want = np.full(cam.n_pixels, -1, np.int32)
    want[pix_ref] = rls.find(pts_ref)
    assert np.array_equal(sl, want)
    out = ls.gather(recv, cam.n_pixels, rzk.CLAMP_NONE, 0.0, scale=1.0).cpu().numpy()
    exp = rls.gather(recv_np, rzk.CLAMP_NONE, 0.0)
    assert np.array_equal(out, exp)
    assert out.sum() > 0
    ctx.check()


def test_lightslice_mixed_materials(ctx, oracle_built):
    from oracle import RefHarness
    from renzoku_b200 import rzk
    if not RefHarness.available():
        pytest.skip("reference harness not built")
    sc = sg.room_objects(60, 40, 40)
    agg, cam, recv, vpls, ls, ref, rls = _run(ctx, sc, 48, 6, 30, 60, 400)
    a, b = ls.slices(), rls.slices()
    for key in ("point_pixel", "start", "end", "rep", "neighbors"):
        assert np.array_equal(a[key], b[key]), key
    R_ref, V_ref, _ = rls.reduced_matrix(vpls)
    R, V, _ = ls.matrix()
    R, V = R.cpu().numpy(), V.cpu().numpy()
    assert np.array_equal(V, V_ref)
    assert np.allclose(R, R_ref, rtol=1e-5, atol=1e-12)
    _refine_ref_on(rls, ref, ls, R, V)
    ca, cb = ls.clusters(), rls.clusters()
    for key in ("count", "size", "members", "rep", "weight", "upper", "wi", "pdf"):
        assert np.array_equal(ca[key], cb[key]), key
    # the reference recomputes each member's incident radiance with the host's powf / expf
    assert np.allclose(ca["incident"], cb["incident"], rtol=1e-5, atol=1e-12)
    recv_np = rzk.records_from_device(recv, sg.RECEIVER_DTYPE)
    for mode, tau in ((rzk.CLAMP_NONE, 0.0), (rzk.CLAMP_FORM_FACTOR, 1e-3)):
        out = ls.gather(recv, cam.n_pixels, mode, tau, scale=1.0).cpu().numpy()
        exp = rls.gather(recv_np, mode, tau)
        rel = np.linalg.norm(out - exp) / max(np.linalg.norm(exp), 1e-30)
        assert rel < 1e-5, (mode, rel)
    ctx.check()


def test_lightslice_rejects_bad_arguments(ctx):
    import ctypes
    from renzoku_b200 import rzk
    lib = rzk.load()
    h = ctypes.c_void_p()
    p = rzk.lightslice_params(max_slice_size=1)
    assert lib.rzk_lightslice_create(ctx.h, None, None, 4, 4, None, 0, ctypes.byref(p), ctypes.byref(h),
                                     None) == rzk.ERR_INVALID
    pts = np.zeros((8, 6), np.float32)
    pix = np.arange(8, dtype=np.int32)
    assert lib.rzk_lightslice_host_slice(ctypes.byref(p), pts.ctypes.data, pix.ctypes.data, 8,
                                         ctypes.byref(h)) == rzk.ERR_INVALID
    ok = rzk.LightSliceCuda.from_host(rzk.lightslice_params(max_slice_size=4), pts, pix)
    # an object built from host inputs has no device tables
    assert lib.rzk_lightslice_gather(ok.h, None, 0, 0, 0.0, 1.0, None, None) == rzk.ERR_INVALID
