"""LightSlice host stages against the reference's own LightSlice code (no GPU).

The 6-D points, the reduced matrix and the global clusters come from the reference harness
(ls_harness.cc: LightSlice::generate_slices, the reduced-matrix loop of
LightSlice::initialize, ClusterBuilder::cluster_by_sampling); the library's host stages
(rzk_lightslice_host_slice / _host_refine / _host_find) are given the same inputs and must
reproduce the reference bit for bit: the kd-tree's data order, the slices and their
representatives, the nearest-slice lists, every slice's refined clusters (members,
representatives, weights, totals, directions, distribution) and the Jensen maps with their
CDFs.
"""
import numpy as np
import pytest

from renzoku_b200 import scenegen as sg

SEED = 2013


def _cases():
    return [
        ("room_boxes_48", lambda: sg.room_boxes(48, 48), 64, 8, 40, 80),
        ("room_objects_40", lambda: sg.room_objects(60, 40, 40), 48, 6, 30, 60),
    ]


@pytest.fixture(scope="module", params=_cases(), ids=lambda c: c[0])
def staged(request, oracle_built):
    from oracle import RefHarness, column_magnitudes
    from renzoku_b200 import rzk
    if not RefHarness.available():
        pytest.skip("reference harness not built here")
    name, make, slice_size, k, n_clusters, max_sc = request.param
    sc = make()
    ref = RefHarness(sc)
    rls = ref.lightslice(slice_size, k, SEED)
    pts, pix = rls.points()
    params = rzk.lightslice_params(max_slice_size=slice_size, num_neighbor_slices=k, num_clusters=n_clusters,
                                   max_slice_clusters=max_sc, seed=SEED, n_threads=4)
    ours = rzk.LightSliceCuda.from_host(params, pts, pix)
    vpls = ref.vpl_generate(SEED, 300, 3)
    R, V, rep_recv = rls.reduced_matrix(vpls)
    _, g_rep, g_w, assign = ref.cluster_by_sampling(R, n_clusters, SEED)
    mags = column_magnitudes(R)
    vpls1 = np.ascontiguousarray(vpls[vpls["bounce"] <= 1])
    rls.refine(R, V, g_rep, g_w, assign, mags, max_sc, SEED, res=params.map_resolution,
               eps=params.map_epsilon, density_radius=params.density_radius)
    ours.host_refine(R, V, vpls1, rep_recv, g_rep, g_w, assign, mags)
    return {"ref": ref, "rls": rls, "ours": ours, "pts": pts, "pix": pix, "R": R, "V": V}


def test_points_and_slices_match_reference(staged):
    rls, ours = staged["rls"], staged["ours"]
    a, b = ours.slices(), rls.slices()
    assert len(a["start"]) == len(b["start"]) >= 4
    for key in ("point_pixel", "start", "end", "rep", "neighbors"):
        assert np.array_equal(a[key], b[key]), key


def test_find_slice_matches_reference(staged):
    rls, ours, pts = staged["rls"], staged["ours"], staged["pts"]
    rng = np.random.default_rng(5)
    jitter = pts + rng.normal(0.0, 0.02, pts.shape).astype(np.float32)
    for q in (pts, jitter):
        assert np.array_equal(ours.host_find(q), rls.find(q))


def test_refined_clusters_match_reference(staged):
    rls, ours = staged["rls"], staged["ours"]
    a, b = ours.clusters(), rls.clusters()
    assert int(a["count"].sum()) > int(a["count"].shape[0])        # slices were refined
    for key in ("count", "size", "members", "rep", "weight", "upper", "wi", "incident", "pdf"):
        assert np.array_equal(a[key], b[key]), key


def test_maps_match_reference(staged):
    rls, ours = staged["rls"], staged["ours"]
    a, b = ours.maps(), rls.maps()
    assert a["valid"].any()
    for key in ("valid", "sum", "maps"):
        assert np.array_equal(a[key], b[key]), key
    # DiscretePdf2D (pdf.cc:195-229): cell probability = cell / total, and the CDFs are the
    # in-order running sums of rows and of cells within a row
    res = a["maps"].shape[1]
    for s in range(a["maps"].shape[0]):
        m = a["maps"][s]
        rows = np.cumsum(m, axis=1, dtype=np.float32)[:, -1]
        total = np.cumsum(rows, dtype=np.float32)[-1]
        if total > 0:
            assert np.array_equal((m / total).astype(np.float32), b["prob"][s])
        with np.errstate(invalid="ignore", divide="ignore"):
            col = (np.cumsum(m, axis=1, dtype=np.float32) / rows[:, None]).astype(np.float32)
        assert np.array_equal(np.nan_to_num(col, nan=-1.0), np.nan_to_num(a["col_cdf"][s], nan=-1.0))
        assert a["row_cdf"][s].shape == (res,)


def test_reference_builds_maps_only_once_records_are_valid(staged):
    """The reference's own initialize() would build every map before the records' validity
    is set; the pinned maps here are the ones built after it (nonzero for valid slices)."""
    m = staged["ours"].maps()
    v = m["valid"].astype(bool)
    assert (m["maps"][v].reshape(v.sum(), -1).sum(axis=1) > 0).all()
