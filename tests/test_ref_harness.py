"""Oracle against the reference harness on fresh seeded inputs (runs where the reference
tree was available to build oracle/_ref)."""
import numpy as np
import pytest

from renzoku_b200 import scenegen as sg


@pytest.fixture(scope="module")
def pair(oracle_built):
    from oracle import Oracle, RefHarness
    if not RefHarness.available():
        pytest.skip("reference harness not built (reference tree absent)")
    sc = sg.room_objects(120, 40, 40, seed_geo=21, seed_mat=22)
    return sc, Oracle(sc), RefHarness(sc)


def test_bvh_and_primary(pair):
    sc, o, r = pair
    a, b = o.bvh(), r.bvh()
    for x, y in zip(a, b):
        assert x.tobytes() == y.tobytes()
    from oracle import Oracle
    assert Oracle.camera(sc.camera).tobytes() == r.camera().tobytes()
    assert o.primary(Oracle.camera(sc.camera)).tobytes() == r.primary().tobytes()


def test_segments_and_rays(pair):
    sc, o, r = pair
    rng = np.random.default_rng(99)
    p = rng.uniform(0.0, 1.0, (20000, 3)).astype(np.float32)
    q = rng.uniform(0.0, 1.0, (20000, 3)).astype(np.float32)
    assert np.array_equal(o.occluded(p, q)[0], r.occluded(p, q))
    d = rng.normal(size=(5000, 3)).astype(np.float32)
    t1, r1 = o.closest(p[:5000], d)
    t2, r2 = r.closest(p[:5000], d)
    assert t1.tobytes() == t2.tobytes() and r1.tobytes() == r2.tobytes()


def test_vpls_and_gather(pair):
    sc, o, r = pair
    v1 = o.vpl_generate(5, 400, 7)
    v2 = r.vpl_generate(5, 400, 7)
    assert v1.tobytes() == v2.tobytes()
    from oracle import Oracle
    recv = o.primary(Oracle.camera(sc.camera))
    hit = recv[recv["mat"] >= 0][::5]
    for mode, tau in ((0, 0.0), (1, 1e-3), (2, 0.02), (3, 0.02)):
        assert np.array_equal(o.gather(hit, v1[:200], mode, tau)[0], r.gather(hit, v1[:200], mode, tau))
    assert np.array_equal(o.incident(hit[:50], v1[:50], 3, 0.02), r.incident(hit[:50], v1[:50], 3, 0.02))
