"""An OBJ scene imported by rzk_obj_import goes through the device path like a generated
one: scene build, primary hits from its own camera line (bit-identical to the oracle) and
the gather (within the mixed-material tolerance of the oracle)."""
import numpy as np
import pytest

from renzoku_b200 import scenegen as sg

pytestmark = pytest.mark.gpu


def test_imported_obj_scene_renders_like_the_oracle(ctx, oracle_built, tmp_path):
    from oracle import Oracle
    from renzoku_b200 import rzk
    from test_obj_import import _write
    scene, cam, info = rzk.import_obj(str(_write(tmp_path)))
    cam = rzk.Camera.from_focal(cam.spec.eye, cam.spec.lookat, cam.spec.up, float(info["focal"]), 64, 64,
                                info["film_w"], info["film_h"])
    agg = rzk.AggregateCuda(ctx, scene)
    o = Oracle(scene)
    recv_t = agg.primary(cam)
    recv = rzk.records_from_device(recv_t, sg.RECEIVER_DTYPE)
    assert recv.tobytes() == o.primary(cam.rec).tobytes()
    assert (recv["mat"] >= 0).sum() > 100
    vt, n = rzk.VplGeneratorCuda(agg).spawn(11, 400, 3)
    vpls = rzk.records_from_device(vt, sg.VPL_DTYPE)
    img = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 0.05).gather(recv_t, cam.n_pixels, vt, n, n_chunks=1)
    ref, _ = o.gather(recv, vpls, rzk.CLAMP_RADIANCE, 0.05)
    img = img.cpu().numpy()
    rel = np.linalg.norm(img - ref) / np.linalg.norm(ref)
    assert rel < 1e-5, rel
    ctx.check()
