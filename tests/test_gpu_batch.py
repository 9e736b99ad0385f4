"""Batched gather (rzk_batch_*): many independent gathers in one persistent launch.

Each job's image must equal the single-instance gather (rzk_gather_cfg) with the same VPL
chunking bit for bit - the batch only changes which warp takes which work item, never
which VPLs a partial sum holds or the order it adds them - and a CUDA-graph replay of
rzk_batch_run must reproduce the eager run.
"""
import ctypes

import numpy as np
import pytest

from renzoku_b200 import instances as inst_mod

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_batch(ctx):
    from renzoku_b200 import rzk
    specs = inst_mod.batch_specs(6, seed=77, tris=(2_000, 40_000), side=(40, 160), vpls=(300, 5_000))
    modes = [rzk.CLAMP_RADIANCE, rzk.CLAMP_NONE, rzk.CLAMP_FORM_FACTOR, rzk.CLAMP_REFLECTIVITY,
             rzk.CLAMP_RADIANCE, rzk.CLAMP_NONE]
    insts = [inst_mod.make_instance(ctx, s, clamp_mode=m) for s, m in zip(specs, modes)]
    # the clamp thresholds of the non-radiance modes are the reference's defaults
    for i in insts:
        if i.clamp_mode == rzk.CLAMP_FORM_FACTOR:
            i.tau = 1e-3
        elif i.clamp_mode == rzk.CLAMP_REFLECTIVITY:
            i.tau = 0.1
    ctx.check()
    return insts


def _n_chunks_for(n_vpl, chunk_len):
    """The chunk count whose rzk_gather_cfg chunk length equals chunk_len, or None."""
    for k in range(1, n_vpl + 1):
        c = (n_vpl + k - 1) // k
        c = (c + 127) // 128 * 128
        if c == chunk_len:
            return k
        if c < chunk_len:
            return None
    return None


@pytest.mark.parametrize("chunk_len", [0, 512])
def test_batch_equals_single_gathers(ctx, small_batch, chunk_len):
    import torch
    from renzoku_b200 import rzk
    refs = []
    for i in small_batch:
        k = 0 if chunk_len == 0 else _n_chunks_for(i.n_vpl, chunk_len)
        refs.append(None if k is None else i.gather(out=torch.empty_like(i.out), n_chunks=k).cpu().numpy())
    assert sum(r is not None for r in refs) >= 3
    for v in range(rzk.load().rzk_batch_variants()):
        for i in small_batch:
            i.out.fill_(float("nan"))
        jobs = rzk.make_jobs(i.job() for i in small_batch)
        b = rzk.GatherBatch(ctx, jobs, variant=v, chunk_len=chunk_len)
        b.run()
        torch.cuda.synchronize()
        ctx.check()
        for i, ref in zip(small_batch, refs):
            got = i.out.cpu().numpy()
            assert np.isfinite(got).all()
            if ref is not None:
                bad = np.nonzero(np.any(got != ref, axis=1))[0]
                assert len(bad) == 0, (v, chunk_len, i.spec, bad[:8])
        b.close()


def test_batch_graph_replay(ctx, small_batch):
    import torch
    from renzoku_b200 import rzk
    jobs = rzk.make_jobs(i.job() for i in small_batch)
    b = rzk.GatherBatch(ctx, jobs)
    b.run()
    torch.cuda.synchronize()
    eager = [i.out.clone() for i in small_batch]
    for i in small_batch:
        i.out.zero_()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            b.run(stream=s)
    for _ in range(3):
        for i in small_batch:
            i.out.zero_()
        g.replay()
        torch.cuda.synchronize()
        for i, e in zip(small_batch, eager):
            assert torch.equal(i.out, e)
    ctx.check()
    del g
    b.close()


def test_batch_mixed_shapes_and_empty_vpls(ctx, small_batch):
    """A job with no VPLs gives a zero image; a job without image layout (image_width 0)
    gives the same image as the 8 x 4 tiled layout."""
    import torch
    from renzoku_b200 import rzk
    a = small_batch[0]
    out0 = torch.full_like(a.out, float("nan"))
    out1 = torch.full_like(a.out, float("nan"))
    out2 = torch.full_like(a.out, float("nan"))
    items = [
        (a.agg, a.recv, a.n_recv, a.spec.width, a.vpls, a.n_vpl, a.clamp_mode, a.tau, a.scale, out0),
        (a.agg, a.recv, a.n_recv, 0, a.vpls, a.n_vpl, a.clamp_mode, a.tau, a.scale, out1),
        (a.agg, a.recv, a.n_recv, a.spec.width, a.vpls, 0, a.clamp_mode, a.tau, a.scale, out2),
    ]
    b = rzk.GatherBatch(ctx, rzk.make_jobs(items))
    b.run()
    torch.cuda.synchronize()
    ctx.check()
    assert torch.equal(out0, out1)
    assert float(out2.abs().sum()) == 0.0
    ref = a.gather(out=torch.empty_like(a.out))
    assert torch.equal(out0, ref)
    b.close()


def test_batch_rejects_bad_arguments(ctx, small_batch):
    from renzoku_b200 import rzk
    lib = rzk.load()
    jobs = rzk.make_jobs(i.job() for i in small_batch[:2])
    h = ctypes.c_void_p()
    assert lib.rzk_batch_create(ctx.h, jobs, 2, 0, 100, ctypes.byref(h)) == rzk.ERR_INVALID
    assert lib.rzk_batch_create(ctx.h, jobs, 2, 99, 0, ctypes.byref(h)) == rzk.ERR_INVALID
    assert lib.rzk_batch_create(ctx.h, jobs, 0, 0, 0, ctypes.byref(h)) == rzk.ERR_INVALID
    jobs[1].d_recv = jobs[1].d_recv + 4
    assert lib.rzk_batch_create(ctx.h, jobs, 2, 0, 0, ctypes.byref(h)) == rzk.ERR_INVALID


def test_autotune_picks_a_compiled_configuration(ctx, small_batch):
    from renzoku_b200 import rzk
    jobs = rzk.make_jobs(i.job() for i in small_batch)
    v, c, ms = rzk.autotune_batch(ctx, jobs, max_probe_jobs=3)
    assert 0 <= v < rzk.load().rzk_batch_variants()
    assert c in (0, 512, 1024, 2048)
    assert ms > 0.0


def test_batch_over_one_launch_table(ctx, small_batch):
    """More jobs than one launch's parameter table holds: the batch is split into several
    launches and every job still equals its single gather."""
    import torch
    from renzoku_b200 import rzk
    a, b2 = small_batch[0], small_batch[1]
    ra = a.gather(out=torch.empty_like(a.out))
    rb = b2.gather(out=torch.empty_like(b2.out))
    outs, items = [], []
    for k in range(300):
        x = a if k % 2 == 0 else b2
        o = torch.full_like(x.out, float("nan"))
        outs.append((o, ra if x is a else rb))
        items.append((x.agg, x.recv, x.n_recv, x.spec.width, x.vpls, x.n_vpl, x.clamp_mode, x.tau, x.scale, o))
    bt = rzk.GatherBatch(ctx, rzk.make_jobs(items), variant=0)
    bt.run()
    torch.cuda.synchronize()
    ctx.check()
    for o, r in outs:
        assert torch.equal(o, r)
    bt.close()
