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


def test_noalloc_matches_gather_twice(ctx):
    import torch
    from renzoku_b200 import rzk
    sc = sg.room_objects(300, 96, 96, seed_geo=41, seed_mat=42)
    agg = rzk.AggregateCuda(ctx, sc)
    cam = rzk.Camera(sc.camera)
    recv = agg.primary(cam)
    vt, n = rzk.VplGeneratorCuda(agg).spawn(43, 1200, 4)
    ev = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 0.05)
    ref = ev.gather(recv, cam.n_pixels, vt, n, scale=1.0 / 1200, image_width=96).cpu().numpy()
    assert float(np.abs(ref).sum()) > 0
    lib = rzk.load()
    for call in range(2):
        out = torch.full((cam.n_pixels, 3), float("nan"), dtype=torch.float32, device="cuda")
        st = _noalloc(lib, agg, recv, cam.n_pixels, 96, vt, n, rzk.CLAMP_RADIANCE, 0.05, 1.0 / 1200, out)
        assert st == rzk.OK, (call, lib.rzk_status_string(st))
        got = out.cpu().numpy()
        # same terms; only the float summation order over VPL chunks may differ
        rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert rel < 1e-5, (call, rel)
        assert np.all(np.abs(got - ref) <= 1e-5 * np.abs(ref) + 1e-7), call
    ctx.check()


def test_noalloc_rejects_oversized_request(ctx):
    import torch
    from renzoku_b200 import rzk
    sc = sg.room_boxes(8, 8)
    agg = rzk.AggregateCuda(ctx, sc)
    lib = rzk.load()
    too_many = (SCRATCH_BYTES - 256) // 12 + 1
    dummy = torch.zeros(256, dtype=torch.uint8, device="cuda")
    st = lib.rzk_gather_noalloc(agg.h, ctypes.c_void_p(dummy.data_ptr()), too_many, 0,
                                ctypes.c_void_p(dummy.data_ptr()), 1, rzk.CLAMP_RADIANCE, 0.05, 1.0,
                                ctypes.c_void_p(dummy.data_ptr()), rzk._stream_ptr())
    assert st == rzk.ERR_CAPACITY
