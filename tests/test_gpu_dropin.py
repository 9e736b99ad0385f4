"""The drop-in C++ classes (renzoku_b200/dropin: AggregateCuda, VplGeneratorCuda,
VirtualPointLightCuda, load_scene_cuda) driven through the reference's own interfaces.

A scene file that selects "cuda_lbvh" and "vpl_cuda" is loaded by the factory; its
Aggregate* answers Aggregate::hit(p, q) (one device query per virtual call, and batched)
and closest-hit queries exactly as the reference's AggregateBvh over the same surfaces; its
IVplGenerator* spawns the device's VPLs; its Integrator* renders a frame equal to
rzk_gather_cfg on the same inputs.
"""
import numpy as np
import pytest

from renzoku_b200 import scenegen as sg

SEED = 2013


def _harness():
    from oracle import DropinHarness
    if not DropinHarness.available():
        pytest.skip("drop-in driver not built (needs the reference's headers)")
    return DropinHarness


@pytest.fixture(scope="module")
def scene_file(tmp_path_factory):
    sc = sg.room_objects(300, 64, 48, seed_geo=51, seed_mat=52)
    path = tmp_path_factory.mktemp("dropin") / "room.json"
    sg.write_json(sc, str(path), integrator="vpl_cuda", max_bounce=3, samples=900, traversal="cuda_lbvh")
    return str(path)


def test_factory_keeps_reference_selection(tmp_path, oracle_built):
    """traversal "bvh" and integrator "vpl" stay the reference's own choices (no device)."""
    DH = _harness()
    sc = sg.room_boxes(16, 16)
    path = tmp_path / "ref.json"
    sg.write_json(sc, str(path), integrator="vpl", traversal="bvh")
    assert DH(str(path)).kinds() == {"aggregate_cuda": False, "integrator_cuda": False}


@pytest.mark.gpu
def test_aggregate_cuda_hit_matches_aggregate_bvh(ctx, oracle_built, scene_file):
    DH = _harness()
    dh = DH(scene_file)
    assert dh.kinds() == {"aggregate_cuda": True, "integrator_cuda": True}
    rng = np.random.default_rng(17)
    n = 100_000
    p = rng.uniform(0.02, 0.98, (n, 3)).astype(np.float32)
    q = rng.uniform(0.02, 0.98, (n, 3)).astype(np.float32)
    virt, batch, ref = dh.segments(p, q)
    assert 0.05 < ref.mean() < 0.95
    assert np.array_equal(virt, ref)
    assert np.array_equal(batch, ref)
    # closest hits from the camera region toward the room: the record the reference fills
    m = 4000
    o = np.tile(np.float32([0.5, 0.5, 2.0]), (m, 1)) + rng.uniform(-0.05, 0.05, (m, 3)).astype(np.float32)
    d = np.stack([rng.uniform(-0.3, 0.3, m), rng.uniform(-0.3, 0.3, m), -np.ones(m)], 1).astype(np.float32)
    ours, theirs = dh.closest(o, d)
    assert theirs[:, 0].mean() > 0.9
    assert ours.tobytes() == theirs.tobytes()


@pytest.mark.gpu
def test_vpl_generator_cuda_spawn(ctx, oracle_built, scene_file):
    from renzoku_b200 import rzk
    DH = _harness()
    dh = DH(scene_file)
    got = dh.vpls(SEED, 700, 4)
    sc, _, _ = rzk.import_json(scene_file)
    agg = rzk.AggregateCuda(ctx, sc)
    vt, n = rzk.VplGeneratorCuda(agg).spawn(SEED, 700, 4)
    want = rzk.records_from_device(vt, sg.VPL_DTYPE)
    assert len(got["p"]) == n > 0
    assert np.array_equal(got["p"], want["p"]) and np.array_equal(got["contrib"], want["contrib"])
    assert np.array_equal(got["bounce"], want["bounce"])
    # each VPL's previous reference is its parent on the same path (trace_vpl's push order)
    same = np.r_[False, (want["path"][1:] == want["path"][:-1]) & (want["bounce"][1:] == want["bounce"][:-1] + 1)]
    assert np.array_equal(got["prev"], np.where(same, np.arange(n) - 1, -1))


@pytest.mark.gpu
def test_vpl_cuda_integrator_frame_equals_gather(ctx, oracle_built, scene_file):
    from renzoku_b200 import rzk
    DH = _harness()
    dh = DH(scene_file)
    img, info = dh.render(start_particles=900, max_vpls=1200, seed=SEED, width=64, height=48)
    assert (info["width"], info["height"]) == (64, 48) and info["vpls"] == 1200
    # the same inputs through the Python mirror of the C ABI
    sc, cam, _ = rzk.import_json(scene_file)
    agg = rzk.AggregateCuda(ctx, sc)
    recv = agg.primary(cam)
    vt, n = rzk.VplGeneratorCuda(agg).spawn(SEED, 900, 3)
    vt = vt[: 1200 * 96].contiguous()
    vpls = rzk.records_from_device(vt, sg.VPL_DTYPE)
    assert info["emitted"] == int(vpls["path"][-1]) + 1
    ev = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 1.0)
    mean = ev.mean_contribution(recv, cam.n_pixels, vt, 1200, seed=SEED, n_pairs=65536)
    assert abs(info["tau"] - 0.1 * mean) <= 1e-6 * 0.1 * mean
    ev.clamp_threshold = info["tau"]
    want = ev.gather(recv, cam.n_pixels, vt, 1200, scale=1.0 / info["emitted"], image_width=64).cpu().numpy()
    assert want.sum() > 0
    assert np.array_equal(img, want)
