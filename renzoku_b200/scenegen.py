"""Seeded procedural scenes for the VPL gather workloads.

Each scene is a list of primitives in the reference's own scene model: one Surface per
primitive (surface.h:24-111) whose Shape is a Triangle or a Quad (triangle.h:13,
quad.h:9), with a Lambertian / ModifiedPhong / Ward material (material.h:67-135) or an
area-light emission (surface.cc:19-24).  The arrays map one to one onto
``rzk_scene_desc`` (include/rzk_scene.h).  Geometry is built in numpy float32 so the same
bytes reach the CUDA library, the CPU oracle and the reference harness.

Workloads (sizes and distributions of the gather benchmarks):
  room_boxes    Cornell-style room [0,1]^3 (5 quads, front open), two axis-aligned boxes
                with heights U[0.3,0.6], a 0.25x0.25 ceiling light of radiance 15,
                per-object Lambertian albedo U[0.2,0.8]^3: 36 triangles.
  room_objects  the same room filled with seeded boxes (12 triangles) and UV spheres
                (16 slices x 10 rings, 288 triangles), size log-uniform [0.01,0.1],
                centres U[0.1,0.9]^3, 60/25/15 % Lambertian/Phong/Ward materials.
  room_spheres  the room filled with seeded UV spheres (8 slices x 4 rings, 48 triangles),
                radius log-uniform [0.005,0.03], Lambertian materials.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math

import numpy as np

BSDF_LAMBERTIAN, BSDF_WARD, BSDF_PHONG = 0, 1, 2
PRIM_TRIANGLE, PRIM_QUAD = 3, 4
SURF_FLIPPED, SURF_TWO_SIDED = 1, 2

MATERIAL_DTYPE = np.dtype([("type", "<i4"), ("kd", "<f4", 3), ("ks", "<f4", 3),
                           ("p0", "<f4"), ("p1", "<f4"), ("pad", "<f4", 3)])
RECEIVER_DTYPE = np.dtype([("p", "<f4", 3), ("ng", "<f4", 3), ("ns", "<f4", 3),
                           ("wo", "<f4", 3), ("u", "<f4", 3), ("v", "<f4", 3),
                           ("n", "<f4", 3), ("mat", "<i4"), ("light", "<i4"),
                           ("flags", "<i4")])
VPL_DTYPE = np.dtype([("p", "<f4", 3), ("n", "<f4", 3), ("u", "<f4", 3), ("v", "<f4", 3),
                      ("nn", "<f4", 3), ("wi", "<f4", 3), ("contrib", "<f4", 3),
                      ("mat", "<i4"), ("bounce", "<i4"), ("path", "<i4")])
CAMERA_DTYPE = np.dtype([("eye", "<f4", 3), ("u", "<f4", 3), ("v", "<f4", 3),
                         ("n", "<f4", 3), ("focal", "<f4"), ("cop", "<f4", 2),
                         ("scale", "<f4", 2), ("width", "<i4"), ("height", "<i4"),
                         ("pad", "<i4")])
BVH_NODE_DTYPE = np.dtype([("bmin", "<f4", 3), ("bmax", "<f4", 3), ("start", "<i4"),
                           ("end", "<i4"), ("left", "<i4"), ("right", "<i4"),
                           ("level", "<i4"), ("pad", "<i4")])
assert RECEIVER_DTYPE.itemsize == 96 and VPL_DTYPE.itemsize == 96
assert MATERIAL_DTYPE.itemsize == 48 and CAMERA_DTYPE.itemsize == 80
assert BVH_NODE_DTYPE.itemsize == 48


class SceneDescC(ctypes.Structure):
    """ctypes mirror of rzk_scene_desc."""
    _fields_ = [("n_prims", ctypes.c_int32), ("prim_kind", ctypes.c_void_p),
                ("prim_v", ctypes.c_void_p), ("prim_mat", ctypes.c_void_p),
                ("prim_emit", ctypes.c_void_p), ("prim_flags", ctypes.c_void_p),
                ("n_mats", ctypes.c_int32), ("mats", ctypes.c_void_p),
                ("tmin", ctypes.c_float)]


@dataclasses.dataclass
class CameraSpec:
    """Pinhole camera as the reference's scene JSON gives it (json_importer.cc:398-441)."""
    eye: tuple = (0.5, 0.5, 2.3)
    lookat: tuple = (0.5, 0.5, 0.0)
    up: tuple = (0.0, 1.0, 0.0)
    fov: float = 45.0
    width: int = 256
    height: int = 256
    film_w: float = 0.025
    film_h: float = 0.025


class RefCameraDescC(ctypes.Structure):
    _fields_ = [("eye", ctypes.c_float * 3), ("lookat", ctypes.c_float * 3),
                ("up", ctypes.c_float * 3), ("fov", ctypes.c_float),
                ("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("film_w", ctypes.c_float), ("film_h", ctypes.c_float)]

    @classmethod
    def from_spec(cls, c: CameraSpec) -> "RefCameraDescC":
        return cls((ctypes.c_float * 3)(*c.eye), (ctypes.c_float * 3)(*c.lookat),
                   (ctypes.c_float * 3)(*c.up), c.fov, c.width, c.height, c.film_w,
                   c.film_h)


@dataclasses.dataclass
class Scene:
    """Primitive arrays of one scene (see rzk_scene_desc)."""
    name: str
    prim_kind: np.ndarray     # int32 [P]
    prim_v: np.ndarray        # float32 [P, 12]
    prim_mat: np.ndarray      # int32 [P], -1 = emitter
    prim_emit: np.ndarray     # float32 [P, 3]
    prim_flags: np.ndarray    # int32 [P]
    mats: np.ndarray          # MATERIAL_DTYPE [M]
    camera: CameraSpec
    tmin: float = 1e-3

    @property
    def n_prims(self) -> int:
        return int(self.prim_kind.shape[0])

    @property
    def n_triangles(self) -> int:
        return int(np.where(self.prim_kind == PRIM_QUAD, 2, 1).sum())

    def desc(self) -> SceneDescC:
        """rzk_scene_desc pointing into this object's arrays (keep the Scene alive)."""
        for a in ("prim_kind", "prim_v", "prim_mat", "prim_emit", "prim_flags", "mats"):
            arr = getattr(self, a)
            if not arr.flags["C_CONTIGUOUS"]:
                setattr(self, a, np.ascontiguousarray(arr))
        return SceneDescC(self.n_prims, self.prim_kind.ctypes.data, self.prim_v.ctypes.data,
                          self.prim_mat.ctypes.data, self.prim_emit.ctypes.data,
                          self.prim_flags.ctypes.data, int(self.mats.shape[0]),
                          self.mats.ctypes.data, float(self.tmin))

    def with_camera(self, width: int, height: int) -> "Scene":
        cam = dataclasses.replace(self.camera, width=width, height=height)
        return dataclasses.replace(self, camera=cam)


class _Builder:
    def __init__(self):
        self.kind, self.v, self.mat, self.emit, self.flags = [], [], [], [], []
        self.mats = []

    def material(self, type_, kd, ks=(0.0, 0.0, 0.0), p0=0.0, p1=0.0) -> int:
        self.mats.append((type_, tuple(kd), tuple(ks), p0, p1))
        return len(self.mats) - 1

    @staticmethod
    def _normal(p0, p1, p2):
        a = np.subtract(p0, p1, dtype=np.float64)
        b = np.subtract(p0, p2, dtype=np.float64)
        return np.cross(a, b)

    def quad(self, p0, p1, p2, p3, facing, mat=-1, emit=(0, 0, 0), flags=SURF_TWO_SIDED):
        """Quad whose facet normal unit(cross(p0-p1, p0-p2)) points along ``facing``."""
        if np.dot(self._normal(p0, p1, p2), facing) < 0:
            p1, p3 = p3, p1
        self.kind.append(PRIM_QUAD)
        self.v.append(np.concatenate([p0, p1, p2, p3]).astype(np.float32))
        self.mat.append(mat)
        self.emit.append(emit)
        self.flags.append(flags if mat >= 0 else 0)

    def tri(self, p0, p1, p2, facing, mat, flags=SURF_TWO_SIDED):
        if np.dot(self._normal(p0, p1, p2), facing) < 0:
            p1, p2 = p2, p1
        self.kind.append(PRIM_TRIANGLE)
        self.v.append(np.concatenate([p0, p1, p2, np.zeros(3)]).astype(np.float32))
        self.mat.append(mat)
        self.emit.append((0, 0, 0))
        self.flags.append(flags)

    def tris_bulk(self, verts: np.ndarray, mat_ids: np.ndarray, flags=SURF_TWO_SIDED):
        """Append many triangles at once: verts [T,3,3] already wound outward."""
        n = verts.shape[0]
        v = np.zeros((n, 12), np.float32)
        v[:, :9] = verts.reshape(n, 9)
        self.kind.append(np.full(n, PRIM_TRIANGLE, np.int32))
        self.v.append(v)
        self.mat.append(mat_ids.astype(np.int32))
        self.emit.append(np.zeros((n, 3), np.float32))
        self.flags.append(np.full(n, flags, np.int32))

    def box(self, lo, hi, mat):
        x0, y0, z0 = lo
        x1, y1, z1 = hi
        P = lambda x, y, z: np.array([x, y, z], np.float32)
        self.quad(P(x0, y0, z0), P(x1, y0, z0), P(x1, y0, z1), P(x0, y0, z1), (0, -1, 0), mat)
        self.quad(P(x0, y1, z0), P(x0, y1, z1), P(x1, y1, z1), P(x1, y1, z0), (0, 1, 0), mat)
        self.quad(P(x0, y0, z0), P(x0, y1, z0), P(x1, y1, z0), P(x1, y0, z0), (0, 0, -1), mat)
        self.quad(P(x0, y0, z1), P(x1, y0, z1), P(x1, y1, z1), P(x0, y1, z1), (0, 0, 1), mat)
        self.quad(P(x0, y0, z0), P(x0, y0, z1), P(x0, y1, z1), P(x0, y1, z0), (-1, 0, 0), mat)
        self.quad(P(x1, y0, z0), P(x1, y1, z0), P(x1, y1, z1), P(x1, y0, z1), (1, 0, 0), mat)

    def build(self, name, camera) -> Scene:
        def cat(parts, dtype, shape_tail):
            out = []
            for p in parts:
                a = np.asarray(p, dtype=dtype)
                out.append(a.reshape((-1,) + shape_tail) if shape_tail else a.reshape(-1))
            return np.ascontiguousarray(np.concatenate(out)) if out else np.zeros((0,) + shape_tail, dtype)
        mats = np.zeros(len(self.mats), MATERIAL_DTYPE)
        for i, (t, kd, ks, p0, p1) in enumerate(self.mats):
            mats[i]["type"], mats[i]["kd"], mats[i]["ks"] = t, kd, ks
            mats[i]["p0"], mats[i]["p1"] = p0, p1
        return Scene(name=name, prim_kind=cat(self.kind, np.int32, ()),
                     prim_v=cat(self.v, np.float32, (12,)),
                     prim_mat=cat(self.mat, np.int32, ()),
                     prim_emit=cat(self.emit, np.float32, (3,)),
                     prim_flags=cat(self.flags, np.int32, ()), mats=mats, camera=camera)


def _room(b: _Builder, rng_albedo: np.random.Generator):
    P = lambda x, y, z: np.array([x, y, z], np.float32)
    walls = [
        ((P(0, 0, 0), P(0, 0, 1), P(1, 0, 1), P(1, 0, 0)), (0, 1, 0)),    # floor
        ((P(0, 1, 0), P(1, 1, 0), P(1, 1, 1), P(0, 1, 1)), (0, -1, 0)),   # ceiling
        ((P(0, 0, 0), P(1, 0, 0), P(1, 1, 0), P(0, 1, 0)), (0, 0, 1)),    # back
        ((P(0, 0, 0), P(0, 1, 0), P(0, 1, 1), P(0, 0, 1)), (1, 0, 0)),    # left
        ((P(1, 0, 0), P(1, 0, 1), P(1, 1, 1), P(1, 1, 0)), (-1, 0, 0)),   # right
    ]
    for corners, facing in walls:
        m = b.material(BSDF_LAMBERTIAN, rng_albedo.uniform(0.2, 0.8, 3))
        b.quad(*corners, facing, mat=m)


def _light(b: _Builder, radiance=15.0):
    P = lambda x, y, z: np.array([x, y, z], np.float32)
    h = 0.125
    b.quad(P(0.5 - h, 0.999, 0.5 - h), P(0.5 + h, 0.999, 0.5 - h), P(0.5 + h, 0.999, 0.5 + h),
           P(0.5 - h, 0.999, 0.5 + h), (0, -1, 0), mat=-1, emit=(radiance,) * 3)


def room_boxes(width=256, height=256) -> Scene:
    """Room + two boxes + light: 36 triangles (seeds 1 and 2)."""
    b = _Builder()
    rng_h = np.random.default_rng(1)
    rng_a = np.random.default_rng(2)
    _room(b, rng_a)
    heights = rng_h.uniform(0.3, 0.6, 2)
    for (x0, x1, z0, z1), h in zip([(0.15, 0.4, 0.15, 0.4), (0.55, 0.8, 0.5, 0.75)], heights):
        m = b.material(BSDF_LAMBERTIAN, rng_a.uniform(0.2, 0.8, 3))
        b.box((x0, 0.0, z0), (x1, float(h), z1), m)
    _light(b)
    return b.build("room_boxes", CameraSpec(width=width, height=height))


def _uv_sphere(slices: int, rings: int) -> np.ndarray:
    """Unit UV sphere triangles [T,3,3] (float64), outward winding, caps as triangles."""
    th = np.linspace(0.0, math.pi, rings + 1)
    ph = np.linspace(0.0, 2.0 * math.pi, slices + 1)
    pts = lambda t, p: np.stack([np.sin(t) * np.cos(p), np.cos(t), np.sin(t) * np.sin(p)], -1)
    tris = []
    for r in range(rings):
        for s in range(slices):
            a = pts(th[r], ph[s]); b_ = pts(th[r], ph[s + 1])
            c = pts(th[r + 1], ph[s + 1]); d = pts(th[r + 1], ph[s])
            if r == 0:
                tris.append((a, c, d))
            elif r == rings - 1:
                tris.append((a, b_, c))
            else:
                tris.append((a, b_, c)); tris.append((a, c, d))
    t = np.array(tris, np.float64)
    # wind outward: facet normal cross(p0-p1, p0-p2) must point away from the centre
    n = np.cross(t[:, 0] - t[:, 1], t[:, 0] - t[:, 2])
    flip = (n * t.mean(axis=1)).sum(-1) < 0
    t[flip] = t[flip][:, [0, 2, 1]]
    return t


def _box_tris(lo, hi) -> np.ndarray:
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    c = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], np.float64)
    faces = [(0, 1, 2, 3), (4, 7, 6, 5), (0, 4, 5, 1), (3, 2, 6, 7), (0, 3, 7, 4), (1, 5, 6, 2)]
    out = []
    for f in faces:
        out.append((c[f[0]], c[f[1]], c[f[2]])); out.append((c[f[0]], c[f[2]], c[f[3]]))
    t = np.array(out)
    n = np.cross(t[:, 0] - t[:, 1], t[:, 0] - t[:, 2])
    ctr = (np.asarray(lo) + np.asarray(hi)) * 0.5
    flip = (n * (t.mean(axis=1) - ctr)).sum(-1) < 0
    t[flip] = t[flip][:, [0, 2, 1]]
    return t


def _mixed_material(b: _Builder, rng: np.random.Generator) -> int:
    u = rng.uniform()
    alb = rng.uniform(0.2, 0.8, 3)
    if u < 0.60:
        return b.material(BSDF_LAMBERTIAN, alb)
    if u < 0.85:
        return b.material(BSDF_PHONG, 0.5 * alb, (0.3, 0.3, 0.3), float(rng.uniform(10, 200)))
    a = float(rng.uniform(0.05, 0.3))
    return b.material(BSDF_WARD, 0.5 * alb, (0.3, 0.3, 0.3), a, a)


def room_objects(n_objects=2000, width=512, height=512, seed_geo=3, seed_mat=4) -> Scene:
    """Room + light + n_objects boxes / UV spheres (~300k triangles at 2,000)."""
    b = _Builder()
    _room(b, np.random.default_rng(2))
    _light(b)
    rng = np.random.default_rng(seed_geo)
    rng_m = np.random.default_rng(seed_mat)
    sph = _uv_sphere(16, 10)
    all_v, all_m = [], []
    for i in range(n_objects):
        size = float(np.exp(rng.uniform(math.log(0.01), math.log(0.1))))
        ctr = rng.uniform(0.1, 0.9, 3)
        m = _mixed_material(b, rng_m)
        if i % 2 == 0:
            t = _box_tris(ctr - size, ctr + size)
        else:
            t = sph * size + ctr
        all_v.append(t.astype(np.float32))
        all_m.append(np.full(t.shape[0], m, np.int32))
    b.tris_bulk(np.concatenate(all_v), np.concatenate(all_m))
    return b.build("room_objects", CameraSpec(width=width, height=height))


def room_spheres(n_spheres=20000, width=1024, height=1024, seed=5) -> Scene:
    """Room + light + n_spheres small UV spheres (~960k triangles at 20,000)."""
    b = _Builder()
    rng_a = np.random.default_rng(2)
    _room(b, rng_a)
    _light(b)
    rng = np.random.default_rng(seed)
    sph = _uv_sphere(8, 4)
    radii = np.exp(rng.uniform(math.log(0.005), math.log(0.03), n_spheres))
    ctrs = rng.uniform(0.1, 0.9, (n_spheres, 3))
    mats = np.array([b.material(BSDF_LAMBERTIAN, rng_a.uniform(0.2, 0.8, 3)) for _ in range(64)])
    verts = (sph[None] * radii[:, None, None, None] + ctrs[:, None, None, :]).astype(np.float32)
    mat_ids = np.repeat(mats[np.arange(n_spheres) % 64], sph.shape[0])
    b.tris_bulk(verts.reshape(-1, 3, 3), mat_ids)
    return b.build("room_spheres", CameraSpec(width=width, height=height))


def room_filled(n_tris_target: int, width: int, height: int, seed: int) -> Scene:
    """Room-boxes scene filled with seeded objects to about n_tris_target triangles
    (the batched-gather instances)."""
    n_obj = max(0, int(round((n_tris_target - 36) / 150.0)))
    s = room_objects(n_objects=n_obj, width=width, height=height, seed_geo=seed,
                     seed_mat=seed + 1)
    s.name = f"room_filled_{n_tris_target}"
    return s


def write_obj(scene: Scene, path: str) -> None:
    """Writes `scene` as an OBJ file and its MTL file (same name, .mtl) in the reference's
    OBJ dialect (obj_parser.cpp, obj_importer.cc), which rzk_obj_import reads back: every
    primitive as a face of its own vertices, materials as `mat_<i>` (Lambertian: Kd;
    Phong: Kd, Ks, Ns n; Ward: Kd, Ks, Ns 1/ax 1/ay), each emitter with a material
    `rz_light_<k>` whose Kd is its radiance.  Reals are written with 9 significant digits,
    so float32 values read back unchanged.  The format has no surface flags: surfaces read
    back one-sided, as the reference's importer builds them."""
    import os
    base = os.path.splitext(path)[0]
    mtl_path = base + ".mtl"
    g = lambda x: "%.9g" % float(x)
    with open(mtl_path, "w") as f:
        for i, m in enumerate(scene.mats):
            f.write(f"newmtl mat_{i}\n")
            f.write("Kd " + " ".join(g(x) for x in m["kd"]) + "\n")
            if int(m["type"]) == BSDF_PHONG:
                f.write("Ks " + " ".join(g(x) for x in m["ks"]) + "\n")
                f.write(f"Ns {g(m['p0'])}\n")
            elif int(m["type"]) == BSDF_WARD:
                f.write("Ks " + " ".join(g(x) for x in m["ks"]) + "\n")
                f.write(f"Ns {g(np.float32(1.0) / m['p0'])} {g(np.float32(1.0) / m['p1'])}\n")
        lights = np.nonzero(scene.prim_mat < 0)[0]
        for k, p in enumerate(lights):
            f.write(f"newmtl rz_light_{k}\n")
            f.write("Kd " + " ".join(g(x) for x in scene.prim_emit[p]) + "\n")
    light_of = {int(p): k for k, p in enumerate(lights)}
    with open(path, "w") as f:
        f.write(f"mtllib {os.path.basename(mtl_path)}\n")
        for p in range(scene.n_prims):
            n = int(scene.prim_kind[p])
            for j in range(n):
                f.write("v " + " ".join(g(x) for x in scene.prim_v[p, 3 * j:3 * j + 3]) + "\n")
            name = f"rz_light_{light_of[p]}" if scene.prim_mat[p] < 0 else f"mat_{int(scene.prim_mat[p])}"
            f.write(f"usemtl {name}\n")
            f.write("f " + " ".join(str(-n + j) for j in range(n)) + "\n")


def write_json(scene: Scene, path: str, integrator: str = "vpl", max_bounce: int = 3, samples: int = 1,
               tmin=None, two_sided=None, traversal: str = "bvh") -> None:
    """Writes `scene` as a scene file in the reference's JSON format (json_importer.cc) with
    its geometry in one OBJ file without materials (mesh/<name>.obj beside it, one `o` object
    per material, `m<i>`, and per emitter, `e<k>`), which rzk_json_import reads back:
    materials `mat_<i>` (lambertian kd; phong kd, ks, n; ward kd, ks, ax, ay), area light
    specs `area_<k>` with each emitter's radiance, world surfaces binding `<name>.m<i>` to
    `mat_<i>`, world lights binding `<name>.e<k>` to `area_<k>`, a pinhole camera from the
    scene's camera (fov), one view with the given integrator and the given
    options.geometry.traversal ("bvh", "none" or this library's "cuda_lbvh").  Reals are written with 9
    significant digits, so float32 values read back unchanged; the surfaces come back grouped
    by material, then the emitters."""
    import json
    import os
    root = os.path.dirname(os.path.abspath(path))
    name = os.path.splitext(os.path.basename(path))[0]
    os.makedirs(os.path.join(root, "mesh"), exist_ok=True)
    g = lambda x: "%.9g" % float(x)
    lights = np.nonzero(scene.prim_mat < 0)[0]
    with open(os.path.join(root, "mesh", name + ".obj"), "w") as f:
        def put(p):
            n = int(scene.prim_kind[p])
            for j in range(n):
                f.write("v " + " ".join(g(x) for x in scene.prim_v[p, 3 * j:3 * j + 3]) + "\n")
            f.write("f " + " ".join(str(-n + j) for j in range(n)) + "\n")
        for i in range(len(scene.mats)):
            f.write(f"o m{i}\n")
            for p in np.nonzero(scene.prim_mat == i)[0]:
                put(p)
        for k, p in enumerate(lights):
            f.write(f"o e{k}\n")
            put(p)
    num = lambda x: json.loads(g(x))
    mats = {}
    for i, m in enumerate(scene.mats):
        t = int(m["type"])
        spec = {"kd": [num(x) for x in m["kd"]]}
        if t == BSDF_PHONG:
            spec.update(type="phong", ks=[num(x) for x in m["ks"]], n=num(m["p0"]))
        elif t == BSDF_WARD:
            spec.update(type="ward", ks=[num(x) for x in m["ks"]], ax=num(m["p0"]), ay=num(m["p1"]))
        else:
            spec["type"] = "lambertian"
        mats[f"mat_{i}"] = {"type": spec.pop("type"), **spec}
    cam = scene.camera
    doc = {
        "geometry": {name: name + ".obj"},
        "materials": mats,
        "light_specs": {f"area_{k}": {"type": "area", "radiance": [num(x) for x in scene.prim_emit[p]]}
                        for k, p in enumerate(lights)},
        "cameras": {"cam": {"type": "pinhole", "pos": [num(x) for x in cam.eye],
                            "lookat": [num(x) for x in cam.lookat], "up": [num(x) for x in cam.up],
                            "near": 0.01, "far": 100.0, "image": [int(cam.width), int(cam.height)],
                            "film": [num(cam.film_w), num(cam.film_h)], "fov": num(cam.fov)}},
        "scene": {
            "world": {
                "surfaces": {f"s{i}": {"mesh": f"{name}.m{i}", "bsdf": f"mat_{i}"} for i in range(len(scene.mats))},
                "lights": {f"l{k}": {"light": f"area_{k}", "mesh": f"{name}.e{k}"} for k in range(len(lights))},
            },
            "views": {"main": {"camera": "cam", "integrator": {"type": integrator, "max_bounce": int(max_bounce),
                                                               "samples": int(samples)}}},
            "options": {"geometry": {"traversal": traversal}},
        },
    }
    geo = doc["scene"]["options"]["geometry"]
    if tmin is not None:
        geo["tmin"] = num(tmin)
    if two_sided is not None:
        geo["two_sided_surfaces"] = bool(two_sided)
    with open(path, "w") as f:
        json.dump(doc, f, indent=1)
