"""The C-ABI library loads and exports every function include/*.h declares (no GPU calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if not f.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", f)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names.update(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(rzk_[a-z0-9_]+)\s*\(",
                                src, flags=re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "rzk_gather" in names and "rzk_scene_create" in names and len(names) >= 20


def test_library_builds_and_exports_all_symbols():
    from renzoku_b200 import build, rzk
    path = build.build()
    lib = ctypes.CDLL(path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    bound = {n for n, _, _ in rzk.SIGNATURES}
    assert set(declared_functions()) <= bound | set(), set(declared_functions()) - bound


def test_status_strings_without_gpu():
    from renzoku_b200 import rzk
    lib = rzk.load()
    assert lib.rzk_status_string(0) == b"ok"
    assert b"invalid" in lib.rzk_status_string(1)


def test_invalid_arguments_rejected_without_gpu():
    from renzoku_b200 import rzk
    lib = rzk.load()
    assert lib.rzk_scene_create(None, None, None, None) == rzk.ERR_INVALID
    assert lib.rzk_gather(None, None, None, 0, None, 0, 0, 0.0, 1.0, None, None) == rzk.ERR_INVALID
    assert lib.rzk_camera_setup(None, None, None, 45.0, 1, 1, 1.0, 1.0, None) == rzk.ERR_INVALID


def test_new_entry_points_reject_bad_arguments_without_gpu():
    import ctypes
    from renzoku_b200 import rzk
    lib = rzk.load()
    out = ctypes.c_void_p()
    bad = rzk.ServerParamsC(-1, 1, 0)
    assert lib.rzk_server_create(0, ctypes.byref(bad), ctypes.byref(out)) == rzk.ERR_INVALID
    assert lib.rzk_server_submit(None, None, None) == rzk.ERR_INVALID
    assert lib.rzk_guided_render(None, None, None, None, None, None, None, None) == rzk.ERR_INVALID
    assert lib.rzk_lightslice_create(None, None, None, 4, 4, None, 0, None, None, None) == rzk.ERR_INVALID
    assert lib.rzk_batch_create(None, None, 0, 0, 0, None) == rzk.ERR_INVALID
    p = rzk.lightslice_params()
    assert p.num_clusters == 600 and p.max_slice_size == 256 and p.num_neighbor_slices == 16


def test_mrcs_entry_points_reject_bad_arguments_without_gpu():
    import ctypes
    from renzoku_b200 import rzk
    lib = rzk.load()
    p = rzk.mrcs_params()
    # MatrixRowColumnSampling's defaults (mrcs.cc:16-20, 79)
    assert (p.block_size, p.max_clusters, p.max_columns) == (32, 1000, 10000)
    assert abs(p.cluster_ratio - 0.01) < 1e-9
    assert lib.rzk_mrcs_params_default(None) == rzk.ERR_INVALID
    out = ctypes.c_void_p()
    assert lib.rzk_mrcs_create(None, None, None, None, 0, 0, 0.0, ctypes.byref(p), None,
                               ctypes.byref(out)) == rzk.ERR_INVALID
    assert lib.rzk_mrcs_gather(None, None, 0, 0, 1.0, None, None) == rzk.ERR_INVALID
    assert lib.rzk_mrcs_info(None, None, None, None, None, None) == rzk.ERR_INVALID
    assert lib.rzk_mrcs_destroy(None) == rzk.ERR_INVALID


def test_matrix_header_reader_without_gpu(oracle_built, tmp_path):
    """rzk_matrix_file_info reads the header of a file the reference's own
    LightTransportMatrix::save wrote (host code only), and rejects a damaged one."""
    import ctypes
    import numpy as np
    from oracle import RefHarness
    from renzoku_b200 import rzk
    lib = rzk.load()
    m = np.random.default_rng(1).random((9, 4, 3)).astype(np.float32)   # 9 columns x 4 rows
    path = tmp_path / "m.bin"
    RefHarness.matrix_save(m, str(path))
    rows, cols = ctypes.c_int32(), ctypes.c_int32()
    assert lib.rzk_matrix_file_info(str(path).encode(), ctypes.byref(rows), ctypes.byref(cols)) == rzk.OK
    assert (rows.value, cols.value) == (4, 9)
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"4 x\n" + m.tobytes())
    assert lib.rzk_matrix_file_info(str(bad).encode(), ctypes.byref(rows), ctypes.byref(cols)) == rzk.ERR_INVALID
    assert lib.rzk_matrix_file_info(str(tmp_path / "none").encode(), ctypes.byref(rows),
                                    ctypes.byref(cols)) == rzk.ERR_INVALID
    assert lib.rzk_scene_deserialize(None, b"RZKSCN01", 8, None, ctypes.byref(ctypes.c_void_p())) == rzk.ERR_INVALID
