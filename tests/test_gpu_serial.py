"""Warm restart (rzk_scene_serialize / rzk_scene_deserialize) and transport-matrix files
(rzk_matrix_save / rzk_matrix_load).

A restored scene must answer every query exactly like the scene it was saved from: the
same BVH bytes, occlusion, primary hits, VPLs and gather image, and it serialises back to
the same blob.  Matrix files must be byte for byte what the reference's
LightTransportMatrix::save writes for the same matrix, and load back unchanged.
"""
import numpy as np
import pytest

from renzoku_b200 import scenegen as sg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def saved(ctx):
    from renzoku_b200 import rzk
    sc = sg.room_objects(300, 64, 48, seed_geo=51, seed_mat=52)
    agg = rzk.AggregateCuda(ctx, sc)
    blob = agg.serialize()
    return sc, agg, blob


def test_restored_scene_answers_identically(ctx, saved):
    import torch
    from renzoku_b200 import rzk
    sc, agg, blob = saved
    back = rzk.AggregateCuda.restore(ctx, blob, sc)
    assert (back.n_tris, back.n_nodes, back.n_levels) == (agg.n_tris, agg.n_nodes, agg.n_levels)
    for x, y in zip(agg.bvh_dump(), back.bvh_dump()):
        assert x.tobytes() == y.tobytes()
    assert np.array_equal(agg.morton_codes(), back.morton_codes())
    assert np.array_equal(agg.bounding_box(), back.bounding_box())
    cam = rzk.Camera(sc.camera)
    r0, r1 = agg.primary(cam), back.primary(cam)
    assert torch.equal(r0, r1)
    rng = np.random.default_rng(8)
    p = torch.from_numpy(rng.uniform(0, 1, (20000, 3)).astype(np.float32)).cuda()
    q = torch.from_numpy(rng.uniform(0, 1, (20000, 3)).astype(np.float32)).cuda()
    assert torch.equal(agg.hit_segments(p, q), back.hit_segments(p, q))
    v0, n0 = rzk.VplGeneratorCuda(agg).spawn(3, 800, 4)
    v1, n1 = rzk.VplGeneratorCuda(back).spawn(3, 800, 4)
    assert n0 == n1 and torch.equal(v0, v1)
    g0 = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 0.05).gather(r0, cam.n_pixels, v0, n0,
                                                                       image_width=64)
    g1 = rzk.VirtualPointLightCuda(back, rzk.CLAMP_RADIANCE, 0.05).gather(r1, cam.n_pixels, v1, n1,
                                                                        image_width=64)
    assert torch.equal(g0, g1)
    assert back.serialize() == blob
    ctx.check()


def test_rebuilt_scene_still_serialises_the_same(ctx, saved):
    from renzoku_b200 import rzk
    sc, agg, blob = saved
    fresh = rzk.AggregateCuda(ctx, sc)
    fresh.rebuild()
    assert fresh.serialize() == blob


def test_bad_blobs_are_rejected(ctx, saved):
    import ctypes
    from renzoku_b200 import rzk
    sc, agg, blob = saved
    lib = rzk.load()
    h = ctypes.c_void_p()
    bad_magic = b"X" + blob[1:]
    cut = blob[: len(blob) - 7]
    longer = blob + b"\0" * 4
    for b in (bad_magic, cut, longer, blob[:10]):
        assert lib.rzk_scene_deserialize(ctx.h, b, len(b), None, ctypes.byref(h)) == rzk.ERR_INVALID
    ctx.check()


def test_matrix_file_matches_reference_save(ctx, oracle_built, tmp_path):
    import torch
    from oracle import RefHarness
    from renzoku_b200 import rzk
    sc = sg.room_boxes(32, 32)
    agg = rzk.AggregateCuda(ctx, sc)
    recv = agg.primary(rzk.Camera(sc.camera))
    vt, n = rzk.VplGeneratorCuda(agg).spawn(4, 200, 3)
    mat, _ = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_NONE, 0.0).fill(recv, 1024, vt, n)
    ours, ref = tmp_path / "ours.bin", tmp_path / "ref.bin"
    rzk.matrix_save(str(ours), mat)
    RefHarness.matrix_save(mat.cpu().numpy(), str(ref))
    assert ours.read_bytes() == ref.read_bytes()
    back = rzk.matrix_load(str(ref))
    assert back.shape == mat.shape and torch.equal(back, mat)
