"""The request loop (rzk_server_*): admitted requests produce the same images as the direct
calls (gathers, and guided renders with either sampler), in batched and in one-at-a-time mode; admission refuses what does not fit the HBM
budget; queued requests can be withdrawn."""
import numpy as np
import pytest

from renzoku_b200 import scenegen as sg

pytestmark = pytest.mark.gpu
SEED = 2013


@pytest.fixture(scope="module")
def world(ctx):
    import dataclasses
    import torch
    from renzoku_b200 import rzk
    scenes = []
    for k, (n_obj, side) in enumerate([(20, 48), (60, 40)]):
        sc = sg.room_objects(n_obj, side, side, seed_geo=10 + k, seed_mat=20 + k)
        agg = rzk.AggregateCuda(ctx, sc)
        cam = rzk.Camera(sc.camera)
        recv = agg.primary(cam)
        vt, n = rzk.VplGeneratorCuda(agg).spawn(SEED + k, 600, 3)
        params = rzk.lightslice_params(max_slice_size=64, num_neighbor_slices=8, num_clusters=40,
                                       max_slice_clusters=80, seed=SEED)
        ls = rzk.LightSliceCuda.create(agg, recv, cam.width, cam.height, vt, n, params)
        scenes.append({"sc": sc, "agg": agg, "vpls": vt, "n": n, "ls": ls})
    torch.cuda.synchronize()
    ctx.check()
    reqs = []
    rng = np.random.default_rng(3)
    for i in range(10):
        w = scenes[i % 2]
        side = int(rng.choice([16, 24, 32, 40]))
        cam = rzk.Camera(dataclasses.replace(w["sc"].camera, width=side, height=side))
        out = torch.full((side * side, 3), float("nan"), dtype=torch.float32, device="cuda")
        r = rzk.RequestC()
        r.kind = rzk.REQ_GATHER if i % 3 else rzk.REQ_GUIDED
        r.scene = w["agg"].h.value
        r.lightslice = w["ls"].h.value
        r.camera = rzk.camera_c(cam)
        nv = int(min(w["n"], rng.integers(100, 500)))
        r.d_vpls = w["vpls"].data_ptr()
        r.n_vpl = nv
        r.clamp_mode = rzk.CLAMP_RADIANCE
        r.tau = 1e-3
        r.scale = 1.0 / 600
        r.spp, r.max_bounce, r.rr_depth, r.rr_prob, r.seed = 2, 4, 2, 0.5, SEED + i
        r.sampler = rzk.GUIDE_METROPOLIS if (i // 3) % 2 else rzk.GUIDE_JENSEN
        r.d_rgb = out.data_ptr()
        reqs.append({"req": r, "out": out, "cam": cam, "w": w})
    return scenes, reqs


def _direct(r):
    import torch
    from renzoku_b200 import rzk
    q, w = r["req"], r["w"]
    if q.kind == rzk.REQ_GATHER:
        recv = w["agg"].primary(r["cam"])
        ev = rzk.VirtualPointLightCuda(w["agg"], q.clamp_mode, q.tau)
        return ev.gather(recv, r["cam"].n_pixels, w["vpls"], q.n_vpl, scale=q.scale,
                         image_width=r["cam"].width).cpu().numpy()
    sampler = "metropolis" if q.sampler == rzk.GUIDE_METROPOLIS else "jensen"
    return w["ls"].guided_render(r["cam"], q.spp, q.max_bounce, rr_depth=q.rr_depth, rr_prob=q.rr_prob,
                                 seed=q.seed, sampler=sampler).cpu().numpy()


@pytest.mark.parametrize("batching", [True, False])
def test_server_results_equal_direct_calls(ctx, world, batching):
    from renzoku_b200 import rzk
    _, reqs = world
    srv = rzk.Server(0, batching=batching)
    for r in reqs:
        r["out"].fill_(float("nan"))
    tickets = [srv.submit(r["req"]) for r in reqs]
    assert all(t is not None for t in tickets)
    for t in tickets:
        st, lat = srv.wait(t, timeout_ms=60000)
        assert st == rzk.OK and lat >= 0.0
    stats = srv.stats()
    assert stats["completed"] == len(reqs) and stats["held_bytes"] == 0
    kind, queue_ms, run_ms = srv.timings()
    assert len(kind) == len(reqs) and sorted(kind) == sorted(int(r["req"].kind) for r in reqs)
    assert np.all(queue_ms >= 0) and np.all(run_ms >= 0)
    srv.close()
    for r in reqs:
        got = r["out"].cpu().numpy()
        assert np.array_equal(got, _direct(r)), r["req"].kind


def test_server_admission_and_cancel(ctx, world):
    from renzoku_b200 import rzk
    _, reqs = world
    tiny = rzk.Server(0, batching=True, hbm_budget_bytes=1024)
    assert tiny.submit(reqs[1]["req"]) is None          # does not fit: refused, not queued
    assert tiny.stats()["rejected"] == 1
    tiny.close()
    srv = rzk.Server(0, batching=True)
    tickets = [srv.submit(r["req"]) for r in reqs * 3]
    c = srv.cancel(tickets[-1])
    assert c in (rzk.OK, rzk.ERR_BUSY)
    for t in tickets:
        st, _ = srv.wait(t, timeout_ms=60000)
        assert st == rzk.OK
    srv.close()
