"""The allocation-free gather entry point (rzk_gather_noalloc), through the C ABI.

It serves callers that cannot let the library call cudaMalloc (device memory owned by
another framework's allocator or held to a fixed budget, or frame loops where an
allocation is not acceptable): its scratch is a fixed static device array.  This file is
collected last so that a run stopping at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest

from renzoku_b200 import scenegen as sg

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 16 << 20


def _noalloc(lib, agg, recv, n_recv, width, vpls, n_vpl, mode, tau, scale, out):
    from renzoku_b200 import rzk
    return lib.rzk_gather_noalloc(agg.h, ctypes.c_void_p(recv.data_ptr()), n_recv, width,
                                  ctypes.c_void_p(vpls.data_ptr()), n_vpl, mode, tau, scale,
                                  ctypes.c_void_p(out.data_ptr()), rzk._stream_ptr())


@pytest.fixture(scope="module")
def scene(ctx, oracle_built):
    from renzoku_b200 import rzk
    sc = sg.room_objects(300, 96, 96, seed_geo=41, seed_mat=42)
    agg = rzk.AggregateCuda(ctx, sc)
    cam = rzk.Camera(sc.camera)
    recv = agg.primary(cam)
    vt, n = rzk.VplGeneratorCuda(agg).spawn(43, 1200, 4)
    return sc, agg, cam, recv, vt, n


def test_noalloc_matches_gather_twice(ctx, scene):
    import torch
    from renzoku_b200 import rzk
    sc, agg, cam, recv, vt, n = scene
    ev = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 0.05)
    ref = ev.gather(recv, cam.n_pixels, vt, n, scale=1.0 / 1200, image_width=96).cpu().numpy()
    assert float(np.abs(ref).sum()) > 0
    lib = rzk.load()
    for call in range(2):
        out = torch.full((cam.n_pixels, 3), float("nan"), dtype=torch.float32, device="cuda")
        st = _noalloc(lib, agg, recv, cam.n_pixels, 96, vt, n, rzk.CLAMP_RADIANCE, 0.05, 1.0 / 1200, out)
        assert st == rzk.OK, (call, lib.rzk_status_string(st))
        got = out.cpu().numpy()
        # rzk_gather's chunk count and VPL order fit in the array: the same sums, bit for bit
        assert np.array_equal(got, ref), (call, np.abs(got - ref).max())
    ctx.check()


def test_noalloc_matches_oracle(ctx, scene):
    """Against the C oracle (the reference's gather restated, summing in push order): the
    device sums Hilbert-ordered chunks, so only the float summation order differs."""
    import torch
    from oracle import Oracle
    from renzoku_b200 import rzk
    sc, agg, cam, recv, vt, n = scene
    lib = rzk.load()
    out = torch.empty((cam.n_pixels, 3), dtype=torch.float32, device="cuda")
    assert _noalloc(lib, agg, recv, cam.n_pixels, 96, vt, n, rzk.CLAMP_RADIANCE, 0.05, 1.0 / 1200, out) == rzk.OK
    got = out.cpu().numpy()
    recv_np = rzk.records_from_device(recv, sg.RECEIVER_DTYPE)
    vpls = rzk.records_from_device(vt, sg.VPL_DTYPE)
    want, want64, _ = Oracle(sc).gather(recv_np, vpls, rzk.CLAMP_RADIANCE, 0.05, 1.0 / 1200, f64=True)
    assert np.linalg.norm(got - want) <= 1e-5 * np.linalg.norm(want)
    assert np.linalg.norm(got - want64) <= 1e-5 * np.linalg.norm(want64)
    assert np.all(np.abs(got - want) <= 1e-4 * np.abs(want) + 1e-7)
    # one chunk (at most 128 VPLs) on an all-Lambertian scene (no transcendental on the
    # path): the oracle's order and values exactly
    lam = sg.room_boxes(32, 32)
    agg1 = rzk.AggregateCuda(ctx, lam)
    recv1 = agg1.primary(rzk.Camera(lam.camera))
    vt1, n1 = rzk.VplGeneratorCuda(agg1).spawn(43, 80, 3)
    n1 = min(n1, 100)
    out1 = torch.empty((32 * 32, 3), dtype=torch.float32, device="cuda")
    assert _noalloc(lib, agg1, recv1, 32 * 32, 32, vt1, n1, rzk.CLAMP_RADIANCE, 0.05, 1.0, out1) == rzk.OK
    want1, _ = Oracle(lam).gather(rzk.records_from_device(recv1, sg.RECEIVER_DTYPE),
                                  rzk.records_from_device(vt1, sg.VPL_DTYPE)[:n1].copy(), rzk.CLAMP_RADIANCE,
                                  0.05, 1.0)
    assert want1.sum() > 0 and np.array_equal(out1.cpu().numpy(), want1)


def test_noalloc_smaller_call_after_larger(ctx, scene):
    """Leftovers of a larger call never reach a later, smaller one: fewer receivers and
    VPLs give the smaller gather's own image, and no VPLs give black."""
    import torch
    from renzoku_b200 import rzk
    sc, agg, cam, recv, vt, n = scene
    lib = rzk.load()
    ev = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 0.05)
    big = torch.empty((cam.n_pixels, 3), dtype=torch.float32, device="cuda")
    assert _noalloc(lib, agg, recv, cam.n_pixels, 96, vt, n, rzk.CLAMP_RADIANCE, 0.05, 1.0, big) == rzk.OK
    m, k = 96 * 40, 700
    small = torch.full((m, 3), float("nan"), dtype=torch.float32, device="cuda")
    assert _noalloc(lib, agg, recv, m, 96, vt, k, rzk.CLAMP_RADIANCE, 0.05, 1.0, small) == rzk.OK
    want = ev.gather(recv, m, vt, k, image_width=96).cpu().numpy()
    assert np.array_equal(small.cpu().numpy(), want)
    zero = torch.full((m, 3), float("nan"), dtype=torch.float32, device="cuda")
    assert _noalloc(lib, agg, recv, m, 96, vt, 0, rzk.CLAMP_RADIANCE, 0.05, 1.0, zero) == rzk.OK
    assert float(zero.abs().sum()) == 0.0
    ctx.check()


def test_noalloc_allocates_nothing(ctx, scene):
    """After the first call on the device, further calls leave the device's free memory
    unchanged (no allocation by the library, the driver or torch)."""
    import torch
    from renzoku_b200 import rzk
    sc, agg, cam, recv, vt, n = scene
    lib = rzk.load()
    out = torch.empty((cam.n_pixels, 3), dtype=torch.float32, device="cuda")
    assert _noalloc(lib, agg, recv, cam.n_pixels, 96, vt, n, rzk.CLAMP_RADIANCE, 0.05, 1.0, out) == rzk.OK
    torch.cuda.synchronize()
    before = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        assert _noalloc(lib, agg, recv, cam.n_pixels, 96, vt, n, rzk.CLAMP_RADIANCE, 0.05, 1.0, out) == rzk.OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == before


def test_noalloc_ring_wraps_matches_gather(ctx):
    """An image whose tiles outnumber the slots of the chunk ring that fit in the array
    (163,840 receivers: 5,120 tiles, about 1,000 slots at 32 chunks) reuses every slot
    several times: the image is still rzk_gather's, bit for bit, with and without an image
    width."""
    import torch
    from renzoku_b200 import rzk
    w, h = 1024, 160
    sc = sg.room_objects(300, w, h, seed_geo=51, seed_mat=52)
    agg = rzk.AggregateCuda(ctx, sc)
    cam = rzk.Camera(sc.camera)
    recv = agg.primary(cam)
    vt, n = rzk.VplGeneratorCuda(agg).spawn(53, 3000, 4)
    assert n >= 32 * 128   # rzk_gather's full 32 chunks
    assert 5120 * 32 * 384 > SCRATCH_BYTES
    ev = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 0.05)
    lib = rzk.load()
    for width in (w, 0):
        ref = ev.gather(recv, cam.n_pixels, vt, n, scale=1.0 / 3000, image_width=width).cpu().numpy()
        assert float(np.abs(ref).sum()) > 0
        out = torch.full((cam.n_pixels, 3), float("nan"), dtype=torch.float32, device="cuda")
        st = _noalloc(lib, agg, recv, cam.n_pixels, width, vt, n, rzk.CLAMP_RADIANCE, 0.05, 1.0 / 3000, out)
        assert st == rzk.OK, lib.rzk_status_string(st)
        got = out.cpu().numpy()
        assert np.array_equal(got, ref), (width, np.abs(got - ref).max())
    ctx.check()


def test_noalloc_large_request(ctx):
    """The array holds the chunk sums of a window of tiles, not of the image: a request of
    2,000,000 receivers (2000 x 1000, more than the array could hold as one chunk plane)
    runs, and matches rzk_gather bit for bit."""
    import torch
    from renzoku_b200 import rzk
    sc = sg.room_objects(100, 2000, 1000, seed_geo=71, seed_mat=72)
    agg = rzk.AggregateCuda(ctx, sc)
    cam = rzk.Camera(sc.camera)
    recv = agg.primary(cam)
    m = cam.n_pixels
    assert 12 * m > SCRATCH_BYTES
    vt, n = rzk.VplGeneratorCuda(agg).spawn(73, 200, 2)
    n = min(n, 300)
    ev = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 0.05)
    lib = rzk.load()
    ref = ev.gather(recv, m, vt, n, scale=1.0 / 200, image_width=2000).cpu().numpy()
    assert float(np.abs(ref).sum()) > 0
    out = torch.full((m, 3), float("nan"), dtype=torch.float32, device="cuda")
    assert _noalloc(lib, agg, recv, m, 2000, vt, n, rzk.CLAMP_RADIANCE, 0.05, 1.0 / 200, out) == rzk.OK
    assert np.array_equal(out.cpu().numpy(), ref)
    ctx.check()
