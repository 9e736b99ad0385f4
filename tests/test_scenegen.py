import numpy as np

from renzoku_b200 import scenegen as sg


def test_room_boxes_counts():
    s = sg.room_boxes()
    assert s.n_triangles == 36
    assert (s.prim_mat < 0).sum() == 1
    assert s.camera.width == 256


def test_room_objects_size_and_mix():
    s = sg.room_objects(200, 64, 64)
    assert s.n_triangles == 12 + 100 * 12 + 100 * 288   # room + light + objects
    t = s.mats["type"]
    assert set(np.unique(t)) <= {0, 1, 2}


def test_full_size_config_counts():
    s = sg.room_objects()
    assert 290_000 < s.n_triangles < 310_000
    s3 = sg.room_spheres(2000, 64, 64)
    assert s3.n_triangles == 12 + 2000 * 48


def test_outward_winding_of_spheres():
    t = sg._uv_sphere(16, 10)
    n = np.cross(t[:, 0] - t[:, 1], t[:, 0] - t[:, 2])
    assert ((n * t.mean(axis=1)).sum(-1) > 0).all()
