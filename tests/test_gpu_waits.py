"""Failure path of the bounded waits, without a GPU fault: the chunk ring's slot wait (the
allocation-free gather's persistent kernel) run on a slot that nothing frees must give up
within its limit, report a timeout in the context's error word and leave the context
usable.  Through the C ABI (rzk_debug_ring_wait)."""
import ctypes
import time

import numpy as np
import pytest

from renzoku_b200 import scenegen as sg

pytestmark = pytest.mark.gpu


def test_ring_wait_gives_up_and_context_stays_usable(ctx):
    import torch
    from renzoku_b200 import rzk
    lib = rzk.load()
    ctx.check()   # start from a clear error word
    acquired = ctypes.c_int(-1)
    t0 = time.perf_counter()
    st = lib.rzk_debug_ring_wait(ctx.h, 100, ctypes.byref(acquired), rzk._stream_ptr())
    dt = time.perf_counter() - t0
    assert st == rzk.OK, lib.rzk_status_string(st)
    assert acquired.value == 0
    assert dt < 3.0, dt   # a 100 ms limit, not the gather's 4 s
    assert lib.rzk_context_check(ctx.h, rzk._stream_ptr()) == rzk.ERR_TIMEOUT
    assert lib.rzk_context_check(ctx.h, rzk._stream_ptr()) == rzk.OK   # read and cleared
    # invalid limits are refused before any launch
    assert lib.rzk_debug_ring_wait(ctx.h, 0, ctypes.byref(acquired), rzk._stream_ptr()) == rzk.ERR_INVALID
    assert lib.rzk_debug_ring_wait(ctx.h, 5000, ctypes.byref(acquired), rzk._stream_ptr()) == rzk.ERR_INVALID
    # the context still gathers, and the allocation-free gather (whose ring the wait
    # belongs to) still matches rzk_gather bit for bit
    sc = sg.room_boxes(48, 48)
    agg = rzk.AggregateCuda(ctx, sc)
    recv = agg.primary(rzk.Camera(sc.camera))
    vt, n = rzk.VplGeneratorCuda(agg).spawn(91, 600, 3)
    ev = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 0.05)
    ref = ev.gather(recv, 48 * 48, vt, n, scale=1.0 / 600, image_width=48).cpu().numpy()
    assert float(np.abs(ref).sum()) > 0
    out = torch.full((48 * 48, 3), float("nan"), dtype=torch.float32, device="cuda")
    assert lib.rzk_gather_noalloc(agg.h, ctypes.c_void_p(recv.data_ptr()), 48 * 48, 48,
                                  ctypes.c_void_p(vt.data_ptr()), n, rzk.CLAMP_RADIANCE, 0.05, 1.0 / 600,
                                  ctypes.c_void_p(out.data_ptr()), rzk._stream_ptr()) == rzk.OK
    assert np.array_equal(out.cpu().numpy(), ref)
    ctx.check()
