"""Parity at the benchmark configurations' own sizes, against the reference's code compiled
in oracle/_ref and the double-precision oracle, on the same inputs.

* Plain gather of the Cornell-style room (256 x 256 shading points x 4,096 VPLs, 36
  triangles): the whole image.  With one VPL chunk the device sums every pixel's terms in
  the reference's order, so the image is bit-identical to the reference's gather (an
  all-Lambertian scene: no transcendental on the path); in the default chunking (runs of
  Hilbert-ordered VPLs) it is within relative L2 1e-3 of it, and both are stated against
  the FP64 oracle.  The device's own shadow-ray count equals the oracle's.
* LightSlice on the scaled scene (512 x 512, 32,768 VPLs, ~300k triangles, 60/25/15 %
  Lambertian / Phong / Ward): slices, reduced matrix, global clusters, refined clusters and
  Jensen maps against the reference's stages, each stage fed the device's previous stage
  (the reduced matrix carries CUDA's powf / expf, so later stages compare on one input),
  and the clustered gather on sampled pixels.
* Guided path tracing on the ~1M-triangle sphere scene (1024 x 1024, 16 spp, max bounce 8,
  Russian roulette beyond depth 3): the LightSlice state against the reference's, then the
  paths of seeded pixels against the reference's tracer drawing the same streams.
"""
import numpy as np
import pytest

from renzoku_b200 import scenegen as sg

pytestmark = pytest.mark.gpu
SEED = 2013
VPL_SEED = 2015


def _rel(a, b):
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def _spawn(agg, n_vpl, particles, max_bounce=3):
    from renzoku_b200 import rzk
    while True:
        vt, made = rzk.VplGeneratorCuda(agg).spawn(VPL_SEED, particles, max_bounce)
        if made >= n_vpl:
            break
        particles *= 2
    vt = vt[: n_vpl * 96].contiguous()
    vpls = rzk.records_from_device(vt, sg.VPL_DTYPE)
    return vt, vpls, int(vpls["path"][-1]) + 1


def _tau(ev, recv_t, n_recv, vt, n_vpl):
    return float(np.float32(0.1 * ev.mean_contribution(recv_t, n_recv, vt, n_vpl, seed=VPL_SEED, n_pairs=65536)))


def test_config1_full_image_matches_reference(ctx, oracle_built):
    from oracle import Oracle, RefHarness
    from renzoku_b200 import rzk
    if not RefHarness.available():
        pytest.skip("reference harness not built")
    sc = sg.room_boxes(256, 256)
    agg = rzk.AggregateCuda(ctx, sc)
    cam = rzk.Camera(sc.camera)
    recv_t = agg.primary(cam)
    recv = rzk.records_from_device(recv_t, sg.RECEIVER_DTYPE)
    ref = RefHarness(sc)
    assert recv.tobytes() == ref.primary().tobytes()
    n_vpl = 4096
    vt, vpls, emitted = _spawn(agg, n_vpl, 3000)
    ev = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 1.0)
    tau = _tau(ev, recv_t, cam.n_pixels, vt, n_vpl)
    ev.clamp_threshold = tau
    scale = 1.0 / emitted
    ctx.rays(reset=True)
    one = ev.gather(recv_t, cam.n_pixels, vt, n_vpl, scale=scale, n_chunks=1, image_width=256).cpu().numpy()
    rays = ctx.rays(reset=True)
    chunked = ev.gather(recv_t, cam.n_pixels, vt, n_vpl, scale=scale, image_width=256).cpu().numpy()
    ctx.check()
    hit = recv["mat"] >= 0
    want = np.zeros((cam.n_pixels, 3), np.float32)
    want[hit] = ref.gather_mt(recv[hit].copy(), vpls, rzk.CLAMP_RADIANCE, tau, scale)
    assert want.sum() > 0 and hit.sum() > 0.5 * cam.n_pixels
    # one chunk: the reference's summation order, bit for bit, every pixel
    assert np.array_equal(one, want), np.abs(one - want).max()
    assert not one[~hit].any() and not chunked[~hit].any()
    # default chunking: the float sum in another order
    o = Oracle(sc)
    _, f64, cnt = o.gather(recv[hit].copy(), vpls, rzk.CLAMP_RADIANCE, tau, scale, f64=True, threads=8)
    # the device's own shadow-ray count: the pairs whose term is not exactly zero (on this
    # all-Lambertian scene the oracle's culling rule selects the same pairs)
    print(f"PARITY config1: shadow rays device {rays} oracle {cnt['rays']} of {cnt['pairs']} pairs")
    assert rays == cnt["rays"]
    r32, r64, r64_ref = _rel(chunked[hit], want[hit]), _rel(chunked[hit], f64), _rel(want[hit], f64)
    print(f"PARITY config1: chunked vs reference rel-L2 {r32:.3e}; vs FP64 {r64:.3e}; reference vs FP64 {r64_ref:.3e}")
    assert r32 <= 1e-3 and r64 <= 1e-3
    assert np.all(np.abs(chunked[hit] - want[hit]) <= 1e-3 * np.abs(want[hit]) + 1e-6)


def test_config2_lightslice_matches_reference(ctx, oracle_built):
    from oracle import RefHarness, column_magnitudes
    from renzoku_b200 import rzk
    if not RefHarness.available():
        pytest.skip("reference harness not built")
    import torch
    sc = sg.room_objects(2000, 512, 512)
    agg = rzk.AggregateCuda(ctx, sc)
    cam = rzk.Camera(sc.camera)
    recv_t = agg.primary(cam)
    n_vpl = 32768
    vt, vpls, emitted = _spawn(agg, n_vpl, 24000)
    ev = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 1.0)
    tau = _tau(ev, recv_t, cam.n_pixels, vt, n_vpl)
    params = rzk.lightslice_params(num_clusters=1000, max_slice_size=1024, num_neighbor_slices=32,
                                   max_slice_clusters=2000, seed=SEED)
    ls = rzk.LightSliceCuda.create(agg, recv_t, 512, 512, vt, n_vpl, params)
    torch.cuda.synchronize()
    ctx.check()
    ref = RefHarness(sc)
    rls = ref.lightslice(1024, 32, SEED)
    a, b = ls.slices(), rls.slices()
    assert len(a["start"]) == 256
    for key in ("point_pixel", "start", "end", "rep", "neighbors"):
        assert np.array_equal(a[key], b[key]), key
    # reduced matrix: visibility exact; radiance up to the glossy VPLs' transcendentals
    R_ref, V_ref, _ = rls.reduced_matrix(vpls)
    R, V, idx = ls.matrix()
    R, V = R.cpu().numpy(), V.cpu().numpy()
    assert np.array_equal(idx, np.nonzero(vpls["bounce"] <= 1)[0])
    assert np.array_equal(V, V_ref)
    assert np.allclose(R, R_ref, rtol=1e-5, atol=1e-12)
    print(f"PARITY config2: reduced matrix entries bit-equal {float(np.mean(R == R_ref)):.6f}, "
          f"max rel {float(np.max(np.abs(R - R_ref) / np.maximum(np.abs(R_ref), 1e-30))):.2e}")
    # global clustering of the device's matrix: the reference's clustering of the same matrix
    g_rep, g_w, assign = ls.global_clusters()
    _, r_rep, r_w, r_assign = ref.cluster_by_sampling(R, 1000, SEED)
    assert np.array_equal(g_rep, r_rep) and np.array_equal(g_w, r_w) and np.array_equal(assign, r_assign)
    # per-slice refinement and maps from the same global clusters
    rls.refine(R, V, g_rep, g_w, assign, column_magnitudes(R), 2000, SEED)
    ca, cb = ls.clusters(), rls.clusters()
    for key in ("count", "size", "members", "rep", "weight", "upper", "wi", "pdf"):
        assert np.array_equal(ca[key], cb[key]), key
    assert np.allclose(ca["incident"], cb["incident"], rtol=1e-5, atol=1e-12)
    ma, mb = ls.maps(), rls.maps()
    for key in ("valid", "sum", "maps"):
        assert np.array_equal(ma[key], mb[key]), key
    # the clustered gather on seeded pixels
    recv = rzk.records_from_device(recv_t, sg.RECEIVER_DTYPE)
    pick = np.sort(np.random.default_rng(5).choice(cam.n_pixels, 2048, replace=False))
    out = ls.gather(recv_t, cam.n_pixels, rzk.CLAMP_RADIANCE, tau, scale=1.0).cpu().numpy()
    exp = rls.gather(recv[pick].copy(), rzk.CLAMP_RADIANCE, tau)
    rel = _rel(out[pick], exp)
    print(f"PARITY config2: LightSlice gather rel-L2 {rel:.3e} on {len(pick)} pixels, "
          f"bit-equal pixels {float(np.mean(np.all(out[pick] == exp, axis=1))):.4f}")
    assert rel < 1e-5
    assert np.all(np.abs(out[pick] - exp) <= 1e-4 * np.abs(exp) + 1e-9)
    ctx.check()


def test_config3_guided_matches_reference(ctx, oracle_built):
    from oracle import RefHarness, column_magnitudes
    from renzoku_b200 import rzk
    if not RefHarness.available():
        pytest.skip("reference harness not built")
    import torch
    side, spp, mb = 1024, 16, 8
    sc = sg.room_spheres(20000, side, side)
    agg = rzk.AggregateCuda(ctx, sc)
    cam = rzk.Camera(sc.camera)
    recv_t = agg.primary(cam)
    n_vpl = 100_000
    vt, vpls, _ = _spawn(agg, n_vpl, 80_000)
    params = rzk.lightslice_params(num_clusters=4096, max_slice_size=4096, num_neighbor_slices=32,
                                   max_slice_clusters=4096, seed=SEED)
    ls = rzk.LightSliceCuda.create(agg, recv_t, side, side, vt, n_vpl, params)
    torch.cuda.synchronize()
    ctx.check()
    ref = RefHarness(sc)
    rls = ref.lightslice(4096, 32, SEED)
    a, b = ls.slices(), rls.slices()
    for key in ("point_pixel", "start", "end", "rep", "neighbors"):
        assert np.array_equal(a[key], b[key]), key
    # the reference refinement from the device's reduced matrix and global clusters (both
    # stages are pinned against the reference on the scaled scene)
    R, V, _ = ls.matrix()
    R, V = R.cpu().numpy(), V.cpu().numpy()
    assert rls.set_vpls(vpls) == R.shape[0]
    g_rep, g_w, assign = ls.global_clusters()
    rls.refine(R, V, g_rep, g_w, assign, column_magnitudes(R), 4096, SEED)
    ca, cb = ls.clusters(), rls.clusters()
    for key in ("count", "size", "members", "rep", "weight", "upper", "wi", "pdf"):
        assert np.array_equal(ca[key], cb[key]), key
    ma, mb_ = ls.maps(), rls.maps()
    for key in ("valid", "sum", "maps"):
        assert np.array_equal(ma[key], mb_[key]), key
    # paths of seeded pixels, 16 spp, depth 8, roulette beyond depth 3
    img, paths = ls.guided_render(cam, spp, mb, rr_depth=3, rr_prob=0.5, seed=SEED, paths=True)
    ctx.check()
    pix = np.sort(np.random.default_rng(11).choice(cam.n_pixels, 384, replace=False)).astype(np.int32)
    ours = paths[torch.as_tensor(pix, device="cuda").long()].cpu().numpy()
    img = img.cpu().numpy()[pix]
    want = rls.guided(pix, spp, mb, rr_depth=3, rr_prob=0.5, seed=SEED)
    assert np.allclose(img, ours.mean(axis=1), rtol=1e-6, atol=1e-7)
    scale = np.maximum(np.abs(want).max(axis=2), 1e-3)
    close = np.abs(ours - want).max(axis=2) <= 1e-4 * scale + 1e-6
    rel = _rel(ours.mean(axis=1), want.mean(axis=1))
    print(f"PARITY config3: paths agreeing to 1e-4 {float(close.mean()):.5f} of {close.size}; "
          f"image rel-L2 {rel:.3e}")
    assert rel <= 1e-3
