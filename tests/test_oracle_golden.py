"""The CPU oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from the reference code): everything bit-exact."""
import hashlib
import os

import numpy as np
import pytest

from renzoku_b200 import scenegen as sg

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
SCENES = {"room_boxes_32": lambda: sg.room_boxes(32, 32),
          "room_objects_60": lambda: sg.room_objects(60, 24, 24)}
TAU = {0: 0.0, 1: 1e-3, 2: 0.05, 3: 0.05}


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module", params=sorted(SCENES))
def case(request, oracle_built):
    from oracle import Oracle
    sc = SCENES[request.param]()
    g = np.load(os.path.join(GOLDEN, request.param + ".npz"))
    return sc, Oracle(sc), g


def test_bvh_bit_exact(case):
    sc, o, g = case
    assert o.n_tris == int(g["n_tris"]) and o.n_nodes == int(g["n_nodes"])
    codes, perm, nodes = o.bvh()
    assert np.array_equal(codes, g["codes"])
    assert np.array_equal(perm, g["perm"])
    assert digest(nodes) == str(g["nodes_sha"])
    # the morton codes are a permutation of the unsorted codes, sorted stably
    raw = o.morton_codes()
    assert np.array_equal(raw[perm], codes)
    assert np.all(np.diff(codes.astype(np.int64)) >= 0)


def test_camera_and_primary_bit_exact(case):
    sc, o, g = case
    from oracle import Oracle
    cam = Oracle.camera(sc.camera)
    assert cam.view(np.uint8).tobytes() == g["camera"].tobytes()
    recv = o.primary(cam, threads=4)
    assert recv.view(np.uint8).tobytes() == g["recv"].tobytes()


def test_occlusion_bit_exact(case):
    sc, o, g = case
    occ, cnt = o.occluded(g["seg_p"], g["seg_q"])
    assert np.array_equal(occ, g["occluded"])
    assert cnt["overflows"] == 0


def test_vpl_generation_bit_exact(case):
    sc, o, g = case
    v = o.vpl_generate(int(g["vpl_seed"]), int(g["vpl_particles"]), int(g["vpl_max_bounce"]))
    assert v.view(np.uint8).tobytes() == g["vpl"].tobytes()


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_gather_bit_exact(case, mode):
    sc, o, g = case
    recv = g["recv"].view(sg.RECEIVER_DTYPE)
    hit = recv[recv["mat"] >= 0]
    vpls = g["vpl"].view(sg.VPL_DTYPE)[:128]
    for cull in (True, False):
        img, _ = o.gather(hit, vpls, mode, TAU[mode], cull=cull, threads=2)
        assert np.array_equal(img, g[f"gather_{mode}"])


def test_gather_f64_close(case):
    sc, o, g = case
    recv = g["recv"].view(sg.RECEIVER_DTYPE)
    hit = recv[recv["mat"] >= 0]
    vpls = g["vpl"].view(sg.VPL_DTYPE)[:128]
    img32, img64, _ = o.gather(hit, vpls, 3, 0.05, f64=True)
    rel = np.linalg.norm(img32 - img64) / np.linalg.norm(img64)
    assert rel < 1e-5
