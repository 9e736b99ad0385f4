"""Seeded light-transport matrices for the clustering tests (shared by the golden-fixture
generator and the tests)."""
import numpy as np

from renzoku_b200 import scenegen as sg


def small_matrix():
    """A 64-row x 600-column matrix: every 9th shading point of a 24x24 view of the mixed
    scene against 600 VPLs, gathered by the oracle (LightTransportMatrix::fill layout)."""
    from oracle import Oracle
    sc = sg.room_objects(120, 24, 24, seed_geo=31, seed_mat=32)
    o = Oracle(sc)
    recv = o.primary(Oracle.camera(sc.camera))
    rows = recv[::9][:64].copy()
    v = o.vpl_generate(33, 700, 4)[:600].copy()
    mat, _ = o.gather_pairs(rows, v, 3, 0.05)
    return mat   # [cols, rows, 3]
