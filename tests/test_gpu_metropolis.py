"""LightSlice's METROPOLIS direction sampler on the device.

The density the chains target and the paths' pdf use (eval_incoming_radiance, FIXED_RADIUS)
is a function of the LightSlice state alone, which both sides build identically: it is
checked against the reference's own function at random points of every valid slice, to float
rounding of its sum.  The chains are random: each slice's states are checked to follow the
density (histogram over the unit square against the density's integral per bin, total
variation distance), and the rendered image's mean against the reference's guided tracer
run with its own METROPOLIS sampler (sequential chains, shuffled 1,024-state caches) on the
same pixels, within the two estimates' standard errors.
"""
import numpy as np
import pytest

from renzoku_b200 import scenegen as sg

pytestmark = pytest.mark.gpu
SEED = 2013


@pytest.fixture(scope="module")
def lightslice(ctx, oracle_built):
    from oracle import RefHarness
    from test_gpu_guided import _setup
    if not RefHarness.available():
        pytest.skip("reference harness not built")
    sc = sg.room_boxes(32, 32)
    return _setup(ctx, sc)


def test_density_matches_reference(ctx, oracle_built, lightslice):
    agg, cam, ls, rls = lightslice
    valid = np.nonzero(rls.maps()["valid"])[0]
    assert len(valid) > 4
    rng = np.random.default_rng(5)
    n = 4000
    slices = rng.choice(valid, n).astype(np.int32)
    xy = rng.random((n, 2), dtype=np.float32)
    ours = ls.density(slices, xy).cpu().numpy()
    ref = rls.density(slices, xy)
    assert (ref > 0).all()
    assert np.allclose(ours, ref, rtol=2e-6, atol=0), np.abs(ours / ref - 1).max()
    # points near cluster directions sum several clusters: the eps floor alone is the minimum
    floor = np.array([ref[slices == s].min() for s in valid])
    assert (ours > floor[np.searchsorted(valid, slices)] * 1.5).mean() > 0.05


def test_chains_follow_the_density(ctx, oracle_built, lightslice):
    agg, cam, ls, rls = lightslice
    valid = np.nonzero(rls.maps()["valid"])[0]
    n = 65536
    ch = ls.chains(SEED, n).cpu().numpy()
    ctx.check()
    invalid = np.setdiff1d(np.arange(ch.shape[0]), valid)
    assert (ch[invalid] == 0).all()
    bins, fine = 8, 128
    g = (np.arange(fine, dtype=np.float32) + 0.5) / fine
    gx, gy = np.meshgrid(g, g, indexing="xy")
    grid = np.stack([gx.ravel(), gy.ravel()], 1)
    tvs = []
    for s in valid:
        st = ch[s]
        assert np.isfinite(st).all() and (st[:, 2] > 0).all()
        # each state's density is the density at its point
        d = ls.density(np.full(256, s, np.int32), st[:256, :2]).cpu().numpy()
        assert np.allclose(st[:256, 2], d, rtol=1e-5)
        hist = np.histogram2d(st[:, 0], st[:, 1], bins=bins, range=[[0, 1], [0, 1]])[0] / n
        f = ls.density(np.full(len(grid), s, np.int32), grid).cpu().numpy()
        want = np.histogram2d(grid[:, 0], grid[:, 1], bins=bins, range=[[0, 1], [0, 1]], weights=f)[0]
        want /= want.sum()
        tvs.append(0.5 * np.abs(hist - want).sum())
    tvs = np.array(tvs)
    assert np.median(tvs) < 0.08 and tvs.max() < 0.15, tvs


def test_metropolis_render_matches_reference_in_mean(ctx, oracle_built, lightslice):
    agg, cam, ls, rls = lightslice
    spp, mb = 16, 6
    img, paths = ls.guided_render(cam, spp, mb, seed=SEED, paths=True, sampler="metropolis")
    ctx.check()
    img2 = ls.guided_render(cam, spp, mb, seed=SEED, sampler="metropolis")
    img, paths, img2 = img.cpu().numpy(), paths.cpu().numpy(), img2.cpu().numpy()
    assert np.isfinite(img).all() and img.sum() > 0
    assert img.tobytes() == img2.tobytes()          # the chains and draws are deterministic
    pix = np.arange(0, cam.n_pixels, 2)
    ref = rls.guided(pix, spp, mb, seed=SEED, sampler="metropolis")
    ours = paths[pix]
    assert np.isfinite(ref).all()
    lum_o = ours.reshape(-1, 3).sum(axis=1)
    lum_r = ref.reshape(-1, 3).sum(axis=1)
    se = np.sqrt(lum_o.var() / lum_o.size + lum_r.var() / lum_r.size)
    assert abs(lum_o.mean() - lum_r.mean()) < 4 * se, (lum_o.mean(), lum_r.mean(), se)
    # a different chain seed changes the image but not its mean beyond noise
    other = ls.guided_render(cam, spp, mb, seed=SEED + 1, sampler="metropolis").cpu().numpy()
    assert other.tobytes() != img.tobytes()


def test_metropolis_rejects_bad_parameters(ctx, lightslice):
    import ctypes
    from renzoku_b200 import rzk
    agg, cam, ls, rls = lightslice
    lib = rzk.load()
    out = np.zeros(1, np.float32)
    for sampler, chain in [(2, 0), (-1, 0), (1, -5)]:
        prm = rzk.GuidedParamsC(1, 4, 0, 1.0, 1, SEED, sampler, chain)
        assert lib.rzk_guided_render(agg.ctx.h, agg.h, ls.h, cam.rec.ctypes.data, ctypes.byref(prm),
                                     ctypes.c_void_p(1), None, None) == rzk.ERR_INVALID
    assert lib.rzk_lightslice_chains(ls.h, SEED, 0, ctypes.c_void_p(1), None) == rzk.ERR_INVALID
