"""A scene read by rzk_obj_import or rzk_json_import goes through the device path like a
generated one: a room written with scenegen.write_obj or write_json and read back renders its
primary hits (through the imported camera, for JSON) and its gather bit for bit like the
oracle (all-Lambertian, one VPL chunk)."""
import numpy as np
import pytest

from renzoku_b200 import scenegen as sg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fmt", ["obj", "json"])
def test_imported_scene_renders_like_the_oracle(ctx, oracle_built, tmp_path, fmt):
    from oracle import Oracle
    from renzoku_b200 import rzk
    src = sg.room_boxes(64, 64)
    if fmt == "obj":
        sg.write_obj(src, str(tmp_path / "room.obj"))
        scene, _, info = rzk.import_obj(str(tmp_path / "room.obj"))
        cam = rzk.Camera(src.camera)
    else:
        sg.write_json(src, str(tmp_path / "room.json"))
        scene, cam, info = rzk.import_json(str(tmp_path / "room.json"))
        assert cam is not None and info["integrator"] == 2
    assert scene.n_prims == src.n_prims
    agg = rzk.AggregateCuda(ctx, scene)
    o = Oracle(scene)
    recv_t = agg.primary(cam)
    recv = rzk.records_from_device(recv_t, sg.RECEIVER_DTYPE)
    assert recv.tobytes() == o.primary(Oracle.camera(src.camera)).tobytes()
    assert (recv["mat"] >= 0).sum() > 1000
    vt, n = rzk.VplGeneratorCuda(agg).spawn(11, 400, 3)
    vpls = rzk.records_from_device(vt, sg.VPL_DTYPE)
    img = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 0.05).gather(recv_t, cam.n_pixels, vt, n, n_chunks=1)
    ref, _ = o.gather(recv, vpls, rzk.CLAMP_RADIANCE, 0.05)
    img = img.cpu().numpy()
    assert float(np.abs(ref).sum()) > 0
    assert np.array_equal(img, ref), np.abs(img - ref).max()
    ctx.check()
