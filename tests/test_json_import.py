"""JSON scene import (rzk_json_import) against the reference's own JsonImporter::load and
get_scene over JsonParser, run through the reference harness on the CPU: the same surfaces in
the same order, vertices, light flags and radiances, BSDF types and parameters, two-sided
flags, area lights in the same order, the first view's camera and integrator, tmin; and what
the path leaves out (glass, mirror, spheres, point / spot / directional lights), counted.
Files the reference stops on (syntax errors, missing keys or files, wrong value types) are
checked against the library alone: the reference exits or dereferences null there."""
import ctypes
import json

import numpy as np
import pytest

pytestmark = pytest.mark.usefixtures("oracle_built")


def _compare(path):
    """Imports `path` with both importers and checks them field by field; returns
    (scene, camera, info, reference facts)."""
    from oracle import RefHarness
    from renzoku_b200 import rzk
    scene, cam, info = rzk.import_json(str(path))
    ref, ref_cam, facts, ref_lights = RefHarness.json_import(str(path))
    keep = (ref["light"] == 1) | (ref["type"] >= 0)
    assert (~keep).sum() == info["surfaces_unsupported_material"]
    r = {k: x[keep] for k, x in ref.items()}
    assert scene.n_prims == len(r["kind"])
    assert np.array_equal(scene.prim_kind, r["kind"])
    assert scene.prim_v.tobytes() == r["v"].tobytes()
    light = scene.prim_mat < 0
    assert np.array_equal(light.astype(np.int32), r["light"])
    assert scene.prim_emit[light].tobytes() == r["emit"][light].tobytes()
    mats = scene.mats[scene.prim_mat[~light]]
    assert np.array_equal(mats["type"], r["type"][~light])
    assert mats["kd"].tobytes() == r["kd"][~light].tobytes()
    is_l = mats["type"] == 0
    assert mats["ks"][~is_l].tobytes() == r["ks"][~light][~is_l].tobytes()
    glossy = np.stack([mats["p0"], mats["p1"]], 1)
    assert glossy[~is_l].tobytes() == r["glossy"][~light][~is_l].tobytes()
    assert np.array_equal((scene.prim_flags & 2) != 0, r["two_sided"] == 1)
    # the area lights in light-list order are the emitting primitives in order (no scene here
    # binds an area light to a sphere)
    assert facts["area_lights"] == int(light.sum())
    assert ref_lights.tobytes() == scene.prim_emit[light].tobytes()
    assert info["point_lights"] == facts["point_lights"]
    assert info["spot_lights"] == facts["spot_lights"]
    assert info["directional_lights"] == facts["directional_lights"]
    assert np.float32(info["tmin"]) == np.float32(facts["tmin"]) and scene.tmin == np.float32(facts["tmin"])
    assert info["two_sided"] == facts["two_sided"]
    assert (cam is None) == (ref_cam is None)
    if cam is not None:
        assert cam.rec.tobytes() == ref_cam.tobytes()
        assert np.float32(info["near_plane"]) == np.float32(facts["near_plane"])
        assert np.float32(info["far_plane"]) == np.float32(facts["far_plane"])
        assert info["integrator"] == facts["integrator"]
        assert info["max_bounce"] == facts["max_bounce"] and info["samples"] == facts["samples"]
    return scene, cam, info, facts


@pytest.mark.parametrize("make,integrator,two_sided", [("room_boxes", "vpl", None),
                                                       ("room_objects", "path", True)])
def test_written_scene_matches_reference_importer(tmp_path, make, integrator, two_sided):
    from renzoku_b200 import scenegen as sg
    sc = sg.room_boxes(64, 64) if make == "room_boxes" else sg.room_objects(60, 64, 64, seed_geo=9, seed_mat=10)
    path = tmp_path / "scene.json"
    sg.write_json(sc, str(path), integrator=integrator, max_bounce=4, samples=16, tmin=2e-3,
                  two_sided=two_sided)
    scene, cam, info, facts = _compare(path)
    assert scene.n_prims == sc.n_prims and info["obj_files"] == 1 and info["skipped"] == 0
    assert info["integrator"] == {"vpl": 2, "path": 1}[integrator] and info["max_bounce"] == 4
    assert info["samples"] == 16 and np.float32(info["tmin"]) == np.float32(2e-3)
    assert info["two_sided"] == (1 if two_sided else 0)
    # same primitives, grouped by material then emitters
    order = np.concatenate([np.nonzero(sc.prim_mat == i)[0] for i in range(len(sc.mats))] +
                           [np.nonzero(sc.prim_mat < 0)[0]])
    assert scene.prim_v.tobytes() == sc.prim_v[order].tobytes()
    assert np.array_equal(scene.mats[scene.prim_mat[scene.prim_mat >= 0]]["kd"],
                          sc.mats[sc.prim_mat[order][sc.prim_mat[order] >= 0]]["kd"])


MESH_ROOM = """# geometry only: objects, no materials
v 0 0 0
v 1 0 0
v 1 0 1
v 0 0 1
v 0 1 0
v 1 1 0
v 1 1 1
v 0 1 1
v 0.4 0.99 0.4
v 0.6 0.99 0.4
v 0.6 0.99 0.6
v 0.4 0.99 0.6
f 1 2 3
f 1 3 4
o floor
f 1 2 3 4
o ceiling
f 5 8 7 6
o wall_a
f 1 5 6
f 1 6 2
o wall_b
f 4 3 7
o lamp
f 9 10 11 12
o lamp_extra
f 9 11 10
o walls
f 2 6 7
vn 0 0 1
o bumpy
f 2//1 3//1 7//1
s 2
f 2 7 6
"""

MESH_PROPS_MTL = """newmtl prop_red
Kd 0.7 0.2 0.2
newmtl prop_glossy
Kd 0.3 0.3 0.3
Ks 0.3 0.3 0.3
Ns 20
newmtl prop_glass
Kd 1 1 1
Ni 1.5
newmtl rz_light_prop
Kd 5 5 4
"""

MESH_PROPS = """# a whole OBJ scene: materials, an emitter, a light quad and a point light
mtllib props.mtl
v 0.2 0.1 0.2
v 0.3 0.1 0.2
v 0.3 0.3 0.2
v 0.2 0.3 0.2
v 0.7 0.1 0.7
v 0.8 0.1 0.7
v 0.8 0.2 0.8
v 0.5 0.98 0.5
lp 8
usemtl rz_light_prop
lq 1 2 3 4
usemtl prop_red
o box
f 1 2 3
f 1 3 4
usemtl prop_glossy
o cone
f 5 6 7
f 5 7 8
usemtl prop_glass
f 6 7 8
usemtl rz_light_prop
o glow
f 2 6 7
"""

MESH_COLOURED = """# geometry whose faces carry materials of their own
mtllib props.mtl
v 0.1 0.5 0.1
v 0.2 0.5 0.1
v 0.2 0.6 0.1
usemtl prop_red
f 1 2 3
"""


def _scene_doc():
    return {
        "geometry": {
            "room": "room.obj",
            "ball": {"type": "sphere", "center": [0.5, 0.3, 0.5], "radius": 0.1},
            "bad_entry": [1, 2, 3],
            "coloured": "coloured.obj",
        },
        "materials": {
            "white": {"type": "lambertian", "kd": [0.75, 0.75, 0.7]},
            "redé\"q": {"type": "lambertian", "kd": [0.6, 0.05, 0.05]},
            "shiny": {"type": "phong", "kd": [0.4, 0.4, 0.4], "ks": [0.3, 0.3, 0.3], "n": 35},
            "brushed": {"type": "ward", "kd": [0.2, 0.25, 0.3], "ks": [0.2, 0.2, 0.2], "ax": 0.15, "ay": 0.35},
            "bright": {"type": "phong", "kd": [0.9, 0.9, 0.9], "ks": [0.5, 0.5, 0.5], "n": 1.0e1},
            "glass": {"type": "glass", "n": 1.5},
            "mirror": {"type": "mirror", "kd": [1, 1, 1]},
            "strange": {"type": "velvet"},
        },
        "light_specs": {
            "ceiling_light": {"type": "area", "radiance": [20, 19, 17.5]},
            "bulb": {"type": "point", "radiance": [1, 1, 1], "position": [0.5, 0.9, 0.5]},
            "spot": {"type": "spot", "radiance": [3, 3, 3], "position": [0.5, 0.9, 0.5],
                     "direction": [0, -1, 0], "phi": 30, "theta": 20, "falloff": 1},
            "sun": {"type": "directional", "radiance": [2, 2, 2], "direction": [0.2, -1, 0.1]},
            "laser": {"type": "laser"},
        },
        "cameras": {
            "main": {"type": "pinhole", "pos": [0.5, 0.5, 2.2], "lookat": [0.5, 0.5, 0], "up": [0, 1, 0],
                     "near": 0.1, "far": 50, "image": [320, 240], "film": [0.036, 0.024], "fov": 40.5},
            "tele": {"type": "pinhole", "pos": [0.5, 0.6, 3.0], "lookat": [0.5, 0.4, 0], "up": [0, 1, 0.1],
                     "near": 0.01, "far": 10.5, "image": [128, 128], "film": [0.025, 0.025], "focal": 0.07},
            "fisheye": {"type": "fisheye"},
        },
        "scene": {
            "world": {
                "surfaces": {
                    "props": "props.obj",
                    "floor": {"mesh": "room.floor", "bsdf": "redé\"q"},
                    "unnamed": {"mesh": "room", "bsdf": "white"},
                    "walls": {"mesh": "room.wall", "bsdf": "shiny"},
                    "walls_all": {"mesh": "room.walls", "bsdf": "brushed"},
                    "hidden": {"mesh": "room.ceiling", "bsdf": "white", "visible": False},
                    "ceiling": {"mesh": "room.ceiling", "bsdf": "bright", "visible": True},
                    "wall_b": {"mesh": "room.wall_b", "bsdf": "glass"},
                    "ball": {"mesh": "ball", "bsdf": "mirror"},
                    "no_mesh": {"mesh": "", "bsdf": "white"},
                    "no_such_bsdf": {"mesh": "room.floor", "bsdf": "nothing"},
                    "obj_material": {"mesh": "room.lamp_extra", "bsdf": "prop_glossy"},
                    "stale": {"mesh": "coloured", "bsdf": "white"},
                    "bumpy": {"mesh": "room.bumpy", "bsdf": "white"},
                },
                "lights": {
                    "top": {"light": "ceiling_light", "mesh": "room.lamp"},
                    "b": "bulb",
                    "s": "spot",
                    "d": "sun",
                    "area_by_name": "ceiling_light",
                    "missing": "nothing",
                    "point_on_mesh": {"light": "bulb", "mesh": "room.floor"},
                },
            },
            # load_camera_views names a view by view->keys[i] with i its position among the
            # views (json_importer.cc:518): a usable view past position 1 would read beyond
            # its own two keys, so the usable ones come first
            "views": {
                "first": {"camera": "tele", "integrator": {"type": "vpl", "max_bounce": 5, "samples": 64}},
                "second": {"camera": "main", "integrator": {"type": "path", "max_bounce": 2, "samples": 4}},
                "broken": {"camera": "nowhere", "integrator": {"type": "vpl", "max_bounce": 2, "samples": 1}},
                "photon": {"camera": "main", "integrator": {"type": "photon", "max_bounce": 2}},
            },
            "options": {"geometry": {"traversal": "none", "tmin": 0.0005, "two_sided_surfaces": True},
                        "opengl": {"shadow_map": {"polygon_offset_factor": 1.5, "polygon_offset_unit": 2},
                                   "sensor": {"multi_sample": "msaa", "num_antialiased_samples": 4}},
                        "experimental": {"note": "kept", "k": 3, "x": 0.5}},
        },
        "ignored_at_root": {"anything": 1},
    }


def _write_tree(tmp_path, doc, text=None):
    (tmp_path / "mesh").mkdir(exist_ok=True)
    (tmp_path / "mesh" / "room.obj").write_text(MESH_ROOM)
    (tmp_path / "mesh" / "props.mtl").write_text(MESH_PROPS_MTL)
    (tmp_path / "mesh" / "props.obj").write_text(MESH_PROPS)
    (tmp_path / "mesh" / "coloured.obj").write_text(MESH_COLOURED)
    p = tmp_path / "test.json"
    p.write_text(text if text is not None else json.dumps(doc, indent=2, ensure_ascii=True))
    return p


def test_every_section_matches_reference_importer(tmp_path):
    """Meshes by object name and prefix, an OBJ scene loaded whole, OBJ material names bound
    from JSON, invisible surfaces, unknown types, unresolved names, a stale OBJ surface index,
    the first usable view, fov and focal cameras, tmin and two-sided options."""
    path = _write_tree(tmp_path, _scene_doc())
    scene, cam, info, facts = _compare(path)
    # what was counted: glass (JSON wall_b and the OBJ's glass face), the mirror sphere, one
    # point light from the OBJ and one from the JSON, spot and directional
    assert info["surfaces_unsupported_material"] == 2
    assert info["spheres"] == 1
    assert info["point_lights"] == 2 and info["spot_lights"] == 1 and info["directional_lights"] == 1
    assert info["obj_files"] == 3
    # first usable view: "tele" with the vpl integrator
    assert info["integrator"] == 2 and info["max_bounce"] == 5 and info["samples"] == 64
    assert cam is not None and info["width"] == 128 and np.float32(info["focal"]) == np.float32(0.07)
    assert info["two_sided"] == 1 and (scene.prim_flags & 2).all()
    # skipped with an error by the reference: the array geometry, velvet, laser, fisheye,
    # the empty mesh name, the unknown bsdf, the stale OBJ index, the area light by name,
    # the unknown light, a point light bound to a mesh, the unknown camera, the photon view
    assert info["skipped"] == 12
    assert info["n_lights"] == 3   # the OBJ's light quad and emitting face, the lamp
    # bound faces the reference shades with interpolated normals: counted
    assert info["faces_with_vertex_normals"] == 1 and info["smoothed_faces"] == 1


def test_fov_camera_matches_reference(tmp_path):
    doc = _scene_doc()
    views = doc["scene"]["views"]
    del views["first"]
    path = _write_tree(tmp_path, doc)
    scene, cam, info, facts = _compare(path)
    assert info["integrator"] == 1 and info["width"] == 320 and info["height"] == 240
    assert np.float32(info["film_w"]) == np.float32(0.036)


def test_sections_apply_in_file_order(tmp_path):
    """The scene section before the materials it names: its surfaces find no material."""
    doc = _scene_doc()
    text = json.dumps(doc)
    order = ["geometry", "light_specs", "cameras", "scene", "materials", "ignored_at_root"]
    text = "{" + ", ".join(json.dumps(k) + ": " + json.dumps(doc[k]) for k in order) + "}"
    path = _write_tree(tmp_path, doc, text)
    scene, cam, info, facts = _compare(path)
    assert (scene.prim_mat < 0).sum() == 3 and info["n_mats"] == 2   # the OBJ scene's own materials


def test_no_options_and_defaults(tmp_path):
    """Without geometry options: tmin RAY_TMIN, one-sided surfaces (the library also reads a
    file without the options object, which the reference's get_scene dereferences)."""
    from renzoku_b200 import rzk
    doc = _scene_doc()
    doc["scene"]["options"] = {"opengl": {}}
    path = _write_tree(tmp_path, doc)
    scene, cam, info, facts = _compare(path)
    assert np.float32(info["tmin"]) == np.float32(1e-3) and (scene.prim_flags == 0).all()
    del doc["scene"]["options"]
    path = _write_tree(tmp_path, doc)
    scene2, _, info2 = rzk.import_json(str(path))
    assert scene2.prim_v.tobytes() == scene.prim_v.tobytes() and info2["two_sided"] == 0


BAD = [
    ("syntax", '{"geometry": {"room": "room.obj",}}'),
    ("truncated", '{"geometry": {"room": "room.obj"}'),
    ("comment", '{"geometry": {"room": "room.obj"}} // trailing'),
    ("scalar_root", '42'),
    ("missing_obj", '{"geometry": {"x": "nowhere.obj"}}'),
    ("material_not_object", '{"materials": {"m": 3}}'),
    ("material_without_type", '{"materials": {"m": {"kd": [1, 1, 1]}}}'),
    ("kd_not_array", '{"materials": {"m": {"type": "lambertian", "kd": 0.5}}}'),
    ("kd_short", '{"materials": {"m": {"type": "lambertian", "kd": [0.5, 0.5]}}}'),
    ("camera_without_near", '{"cameras": {"c": {"type": "pinhole", "pos": [0,0,1], "lookat": [0,0,0], '
                            '"up": [0,1,0], "far": 1, "image": [8,8], "film": [1,1], "fov": 40}}}'),
    ("camera_without_focal", '{"cameras": {"c": {"type": "pinhole", "pos": [0,0,1], "lookat": [0,0,0], '
                             '"up": [0,1,0], "near": 0.1, "far": 1, "image": [8,8], "film": [1,1]}}}'),
    ("real_max_bounce", '{"cameras": {"c": {"type": "pinhole", "pos": [0,0,1], "lookat": [0,0,0], '
                        '"up": [0,1,0], "near": 0.1, "far": 1, "image": [8,8], "film": [1,1], "fov": 40}}, '
                        '"scene": {"world": {"surfaces": {}, "lights": {}}, "views": {"v": {"camera": "c", '
                        '"integrator": {"type": "vpl", "max_bounce": 3.0, "samples": 1}}}}}'),
    ("scene_without_world", '{"scene": {"views": {}}}'),
    ("visible_not_bool", '{"materials": {"m": {"type": "lambertian", "kd": [1,1,1]}}, "scene": {"world": '
                         '{"surfaces": {"s": {"mesh": "room", "bsdf": "m", "visible": 1}}, "lights": {}}, '
                         '"views": {}}}'),
    ("null_pairs_past_values", '{"materials": {"a": null, "b": {"type": "lambertian", "kd": [1,1,1]}}}'),
]
_OPT_SCENE = ('{"cameras": {"c": {"type": "pinhole", "pos": [0,0,1], "lookat": [0,0,0], "up": [0,1,0], '
              '"near": 0.1, "far": 1, "image": [8,8], "film": [1,1], "fov": 40}}, "scene": {"world": '
              '{"surfaces": {}, "lights": {}}, "views": {"v": {"camera": "c", "integrator": {"type": "vpl", '
              '"max_bounce": 3, "samples": 1}}}, "options": %s}}')
BAD += [
    ("shadow_map_without_factor", _OPT_SCENE % '{"opengl": {"shadow_map": {"polygon_offset_unit": 2}}}'),
    ("sensor_samples_real", _OPT_SCENE % '{"opengl": {"sensor": {"multi_sample": "msaa", '
                                         '"num_antialiased_samples": 4.0}}}'),
    ("traversal_not_string", _OPT_SCENE % '{"geometry": {"traversal": 3}}'),
    ("experimental_not_object", _OPT_SCENE % '{"experimental": [1, 2]}'),
]


@pytest.mark.parametrize("name,text", BAD, ids=[b[0] for b in BAD])
def test_files_the_reference_stops_on_are_rejected(tmp_path, name, text):
    from renzoku_b200 import rzk
    path = _write_tree(tmp_path, None, text)
    lib = rzk.load()
    h = ctypes.c_void_p()
    assert lib.rzk_json_import(str(path).encode(), ctypes.byref(h)) == rzk.ERR_INVALID
    assert lib.rzk_json_import(str(tmp_path / "absent.json").encode(), ctypes.byref(h)) == rzk.ERR_INVALID


def test_null_leaves_keys_without_values(tmp_path):
    """A null value adds its key but no value (json_parser.cc:39-41), so the keys after it pair
    with the values after theirs: "kd" after a null reads the next value, as in the reference.
    A null after every key that is read, and one at the root, change nothing."""
    doc = _scene_doc()
    doc["materials"]["white"] = {"type": "lambertian", "x": None, "kd": [0.75, 0.75, 0.7],
                                 "pad": [0.125, 0.25, 0.375]}
    doc["cameras"]["tele"]["comment"] = None
    doc["ignored_at_root"] = None
    path = _write_tree(tmp_path, doc)
    scene, cam, info, facts = _compare(path)
    white = scene.mats["kd"] == np.array([0.125, 0.25, 0.375], np.float32)
    assert white.all(axis=1).sum() == 1 and cam is not None


def test_escapes_and_number_forms_match_reference(tmp_path):
    """Names written with \\u escapes (a surrogate pair included) bind to the same names
    written as raw UTF-8; integers, exponents and -0 read as the reference reads them
    (atoi for integers, atof then float for the rest)."""
    from renzoku_b200 import rzk
    doc = _scene_doc()
    text = json.dumps(doc, ensure_ascii=False)
    text = text.replace('"white": {"type": "lambertian", "kd": [0.75, 0.75, 0.7]}',
                        '"wh\\u00eete\\ud83d\\ude00": {"type": "lambertian", "kd": [7.5E-1, 75e-2, -0]}')
    text = text.replace('"unnamed": {"mesh": "room", "bsdf": "white"}',
                        '"unnamed": {"mesh": "room", "bsdf": "whîte\U0001F600"}')
    text = text.replace('"stale": {"mesh": "coloured", "bsdf": "white"}',
                        '"stale": {"mesh": "coloured", "bsdf": "wh\\u00eete\\ud83d\\ude00"}')
    text = text.replace('"bsdf": "white"', '"bsdf": "whîte😀"')
    assert "white" not in text
    path = _write_tree(tmp_path, None, text)
    scene, cam, info, facts = _compare(path)
    kd = np.array([0.75, 0.75, 0.0], np.float32)
    assert (scene.mats["kd"] == kd).all(axis=1).sum() == 1
    (tmp_path / "plain").mkdir()
    _, _, base = rzk.import_json(str(_write_tree(tmp_path / "plain", _scene_doc())))
    assert info["n_prims"] == base["n_prims"] and info["skipped"] == base["skipped"]
