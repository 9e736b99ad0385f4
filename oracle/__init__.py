"""TEST INFRASTRUCTURE ONLY: ctypes front-ends for the two CPU checkers.

* ``Oracle``      - liboracle.so, the plain-C restatement in rzk_oracle.c.
* ``RefHarness``  - _ref/librzk_ref.so, the reference's own C++ sources compiled in place
                    (built only where the reference tree exists; the built library
                    travels with the repository copy).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py use this
package, always as the checker.  The product path never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from renzoku_b200 import scenegen as sg

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "librzk_ref.so")
# the reference source tree, read only to compile _ref/librzk_ref.so (absent where the
# prebuilt library travels without it)
REFERENCE_TREE = os.environ.get("RZK_REFERENCE_TREE", "/root/reference")

P = ctypes.c_void_p
I32 = ctypes.c_int32
U32 = ctypes.c_uint32
F32 = ctypes.c_float


class Counters(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in
                ("rays", "root_tests", "inner_pops", "leaf_tests", "overflows", "pairs",
                 "culled")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


def build(ref: bool = True) -> None:
    """Compile liboracle.so and, where the reference tree exists, _ref/librzk_ref.so and the
    drop-in classes' driver _ref/librzk_dropin_test.so."""
    targets = ["oracle"]
    if ref and os.path.isdir(REFERENCE_TREE):
        targets.append("ref")
        if os.path.exists(os.path.join(HERE, "..", "renzoku_b200", "librzk_dropin.so")):
            targets.append("dropin")
    subprocess.run(["make", "-s", "-j8", "-C", HERE, f"REF={REFERENCE_TREE}", *targets], check=True)


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


class Oracle:
    """The C oracle for one scene."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(ORACLE_SO):
                build(ref=False)
            L = ctypes.CDLL(ORACLE_SO)
            L.ro_scene_create.restype = P
            L.ro_scene_create.argtypes = [P]
            L.ro_scene_destroy.argtypes = [P]
            for f in ("ro_num_triangles", "ro_num_nodes", "ro_num_lights"):
                getattr(L, f).restype = I32
                getattr(L, f).argtypes = [P]
            L.ro_morton_codes.argtypes = [P, P]
            L.ro_bvh_dump.argtypes = [P, P, P, P]
            L.ro_camera_setup.argtypes = [P, P, P, F32, I32, I32, F32, F32, P]
            L.ro_primary_rays.argtypes = [P, P, P]
            L.ro_occluded.argtypes = [P, P, P, I32, P, P]
            L.ro_closest.argtypes = [P, P, P, I32, P, P, P]
            L.ro_primary.argtypes = [P, P, P, I32]
            L.ro_gather.argtypes = [P, P, I32, P, I32, I32, F32, F32, I32, P, P, I32, P]
            L.ro_gather_pairs.argtypes = [P, P, I32, P, I32, I32, F32, P, P]
            L.ro_incident.argtypes = [P, P, I32, P, I32, I32, F32, P]
            L.ro_brdf_eval.argtypes = [P, P, P, P, P, I32, P]
            L.ro_mean_contribution.restype = ctypes.c_double
            L.ro_mean_contribution.argtypes = [P, P, P, P, I32, P]
            L.ro_draw_u32.restype = U32
            L.ro_draw_u32.argtypes = [U32, U32, U32, U32]
            L.ro_vpl_generate.restype = I32
            L.ro_vpl_generate.argtypes = [P, U32, I32, I32, P, I32]
            L.ro_ltm_alphas.argtypes = [P, I32, I32, P, P]
            L.ro_cluster_by_sampling.restype = I32
            L.ro_cluster_by_sampling.argtypes = [P, I32, I32, I32, U32, P, P, P, P]
            cls._lib = L
        return cls._lib

    def __init__(self, scene: sg.Scene):
        self.scene = scene
        self._desc = scene.desc()
        self.h = self.lib().ro_scene_create(ctypes.byref(self._desc))
        self.n_tris = self.lib().ro_num_triangles(self.h)
        self.n_nodes = self.lib().ro_num_nodes(self.h)

    def __del__(self):
        if getattr(self, "h", None) and self._lib is not None:
            self._lib.ro_scene_destroy(self.h)
            self.h = None

    def morton_codes(self):
        out = np.zeros(self.n_tris, np.uint32)
        self.lib().ro_morton_codes(self.h, _ptr(out))
        return out

    def bvh(self):
        codes = np.zeros(self.n_tris, np.uint32)
        perm = np.zeros(self.n_tris, np.int32)
        nodes = np.zeros(self.n_nodes, sg.BVH_NODE_DTYPE)
        self.lib().ro_bvh_dump(self.h, _ptr(codes), _ptr(perm), _ptr(nodes))
        return codes, perm, nodes

    @staticmethod
    def camera(spec: sg.CameraSpec) -> np.ndarray:
        cam = np.zeros(1, sg.CAMERA_DTYPE)
        f = lambda t: np.asarray(t, np.float32)
        e, l, u = f(spec.eye), f(spec.lookat), f(spec.up)
        Oracle.lib().ro_camera_setup(_ptr(e), _ptr(l), _ptr(u), spec.fov, spec.width,
                                     spec.height, spec.film_w, spec.film_h, _ptr(cam))
        return cam

    def primary_rays(self, cam: np.ndarray):
        n = int(cam["width"][0]) * int(cam["height"][0])
        o = np.zeros((n, 3), np.float32)
        d = np.zeros((n, 3), np.float32)
        self.lib().ro_primary_rays(_ptr(cam), _ptr(o), _ptr(d))
        return o, d

    def primary(self, cam: np.ndarray, threads: int = 8):
        n = int(cam["width"][0]) * int(cam["height"][0])
        out = np.zeros(n, sg.RECEIVER_DTYPE)
        self.lib().ro_primary(self.h, _ptr(cam), _ptr(out), threads)
        return out

    def occluded(self, p, q):
        p = np.ascontiguousarray(p, np.float32)
        q = np.ascontiguousarray(q, np.float32)
        out = np.zeros(p.shape[0], np.uint8)
        c = Counters()
        self.lib().ro_occluded(self.h, _ptr(p), _ptr(q), p.shape[0], _ptr(out), ctypes.byref(c))
        return out, c.as_dict()

    def closest(self, o, d):
        o = np.ascontiguousarray(o, np.float32)
        d = np.ascontiguousarray(d, np.float32)
        t = np.zeros(o.shape[0], np.float32)
        rec = np.zeros(o.shape[0], sg.RECEIVER_DTYPE)
        self.lib().ro_closest(self.h, _ptr(o), _ptr(d), o.shape[0], _ptr(t), _ptr(rec), None)
        return t, rec

    def gather(self, recv, vpls, clamp_mode, tau, scale=1.0, cull=True, f64=False,
               threads=8):
        n = recv.shape[0]
        out = np.zeros((n, 3), np.float32)
        out64 = np.zeros((n, 3), np.float64) if f64 else None
        c = Counters()
        self.lib().ro_gather(self.h, _ptr(recv), n, _ptr(vpls), vpls.shape[0], clamp_mode,
                             tau, scale, int(cull), _ptr(out),
                             _ptr(out64) if f64 else None, threads, ctypes.byref(c))
        return (out, out64, c.as_dict()) if f64 else (out, c.as_dict())

    def gather_pairs(self, recv, vpls, clamp_mode, tau):
        n, m = recv.shape[0], vpls.shape[0]
        rgb = np.zeros((m, n, 3), np.float32)
        vis = np.zeros((m, n), np.uint8)
        self.lib().ro_gather_pairs(self.h, _ptr(recv), n, _ptr(vpls), m, clamp_mode, tau,
                                   _ptr(rgb), _ptr(vis))
        return rgb, vis

    def incident(self, recv, vpls, clamp_mode, tau):
        n, m = recv.shape[0], vpls.shape[0]
        rgb = np.zeros((m, n, 3), np.float32)
        self.lib().ro_incident(self.h, _ptr(recv), n, _ptr(vpls), m, clamp_mode, tau, _ptr(rgb))
        return rgb

    def brdf_eval(self, mat, uvn9, wo, wi):
        n = mat.shape[0]
        out = np.zeros((n, 3), np.float32)
        self.lib().ro_brdf_eval(self.h, _ptr(mat), _ptr(uvn9), _ptr(wo), _ptr(wi), n, _ptr(out))
        return out

    def mean_contribution(self, recv, recv_idx, vpl_idx, vpls):
        recv_idx = np.ascontiguousarray(recv_idx, np.int32)
        vpl_idx = np.ascontiguousarray(vpl_idx, np.int32)
        return float(self.lib().ro_mean_contribution(self.h, _ptr(recv), _ptr(recv_idx),
                                                     _ptr(vpl_idx), recv_idx.shape[0],
                                                     _ptr(vpls)))

    def vpl_generate(self, seed, n_particles, max_bounce, cap=None):
        cap = cap or n_particles * max(1, max_bounce - 1)
        out = np.zeros(cap, sg.VPL_DTYPE)
        n = self.lib().ro_vpl_generate(self.h, seed, n_particles, max_bounce, _ptr(out), cap)
        return out[:min(n, cap)]

    @staticmethod
    def draw_u32(seed, stream, path, d):
        return int(Oracle.lib().ro_draw_u32(seed, stream, path, d))

    @staticmethod
    def ltm_alphas(mat):
        """mat: float32 [cols, rows, 3] (column-major MatrixC<Rgb>)."""
        mat = np.ascontiguousarray(mat, np.float32)
        cols, rows = mat.shape[0], mat.shape[1]
        a = np.zeros(cols, np.float32)
        n = np.zeros(cols, np.float32)
        Oracle.lib().ro_ltm_alphas(_ptr(mat), rows, cols, _ptr(a), _ptr(n))
        return a, n

    @staticmethod
    def cluster_by_sampling(mat, num_clusters, seed):
        mat = np.ascontiguousarray(mat, np.float32)
        cols, rows = mat.shape[0], mat.shape[1]
        cap = max(num_clusters, cols)
        c = np.zeros(cap, np.int32); r = np.zeros(cap, np.int32); w = np.zeros(cap, np.float32)
        a = np.zeros(cols, np.int32)
        n = Oracle.lib().ro_cluster_by_sampling(_ptr(mat), rows, cols, num_clusters, seed, _ptr(c),
                                                _ptr(r), _ptr(w), _ptr(a))
        return c[:n], r[:n], w[:n], a


class RefHarness:
    """The reference's own classes for one scene (see ref/ref_harness.cc)."""

    _lib = None

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    @classmethod
    def lib(cls):
        if cls._lib is None:
            L = ctypes.CDLL(REF_SO)
            L.rref_create.restype = P
            L.rref_create.argtypes = [P, P, U32]
            L.rref_destroy.argtypes = [P]
            L.rref_num_triangles.restype = I32
            L.rref_num_triangles.argtypes = [P]
            L.rref_num_nodes.restype = I32
            L.rref_num_nodes.argtypes = [P]
            L.rref_bvh_dump.restype = I32
            L.rref_bvh_dump.argtypes = [P, P, P, P, I32]
            L.rref_camera.argtypes = [P, P]
            L.rref_occluded.argtypes = [P, P, P, I32, P]
            L.rref_closest.argtypes = [P, P, P, I32, P, P]
            L.rref_primary.argtypes = [P, P]
            L.rref_primary_rays.argtypes = [P, P, P]
            L.rref_vpl_generate.restype = I32
            L.rref_vpl_generate.argtypes = [P, U32, I32, I32, P, I32]
            L.rref_gather.argtypes = [P, P, I32, P, I32, I32, F32, P, P, P]
            L.rref_incident.argtypes = [P, P, I32, P, I32, I32, F32, P]
            L.rref_brdf_eval.argtypes = [P, P, P, P, P, I32, P]
            L.rref_rng_stream.argtypes = [U32, U32, U32]
            L.rref_gather_mt.argtypes = [P, P, I32, P, I32, I32, F32, F32, P, I32]
            L.rref_ltm_alphas.argtypes = [P, I32, I32, P, P]
            L.rref_cluster_by_sampling.restype = I32
            L.rref_cluster_by_sampling.argtypes = [P, P, I32, I32, I32, U32, P, P, P, P]
            L.rref_ls_create.restype = P
            L.rref_ls_create.argtypes = [P, I32, I32, U32]
            L.rref_ls_num_points.restype = I32
            L.rref_ls_num_points.argtypes = [P]
            L.rref_ls_num_slices.restype = I32
            L.rref_ls_num_slices.argtypes = [P]
            L.rref_ls_points.argtypes = [P, P, P]
            L.rref_ls_slices.argtypes = [P, P, P, P, P]
            L.rref_ls_neighbors.argtypes = [P, P]
            L.rref_ls_find.argtypes = [P, P, I32, P]
            L.rref_ls_reduced_matrix.restype = I32
            L.rref_ls_reduced_matrix.argtypes = [P, P, I32, I32, F32, P, P, P]
            L.rref_ls_set_vpls.restype = I32
            L.rref_ls_set_vpls.argtypes = [P, P, I32]
            L.rref_ls_refine.argtypes = [P, P, P, I32, I32, P, P, P, P, I32, U32, I32, F32, F32]
            L.rref_ls_num_slice_clusters.restype = I32
            L.rref_ls_num_slice_clusters.argtypes = [P]
            L.rref_ls_clusters.argtypes = [P, P, P, P, P, P, P, P, P, P, P]
            L.rref_ls_maps.argtypes = [P, P, P, P, P]
            L.rref_ls_gather.argtypes = [P, P, I32, I32, F32, P]
            L.rref_ls_gather_mt.argtypes = [P, P, I32, I32, F32, P, I32]
            L.rref_ls_guided.argtypes = [P, P, I32, I32, I32, I32, F32, I32, U32, P]
            L.rref_ls_density.argtypes = [P, P, P, I32, P]
            L.rref_ls_set_sampler.argtypes = [P, I32]
            L.rref_matrix_save.argtypes = [P, I32, I32, ctypes.c_char_p]
            L.rref_obj_import.restype = I32
            L.rref_obj_import.argtypes = [ctypes.c_char_p, I32, P, P, P, P, P, P, P, P, P, P, P]
            L.rref_json_import.restype = I32
            L.rref_json_import.argtypes = [ctypes.c_char_p, I32, P, P, P, P, P, P, P, P, P, P, P, P, P, I32]
            L.rref_mrcs.restype = I32
            L.rref_mrcs.argtypes = [P, P, I32, I32, F32, U32, I32, F32, I32, P, I32, P, P, P, P, I32]
            cls._lib = L
        return cls._lib

    def __init__(self, scene: sg.Scene, seed: int = 2013):
        self.scene = scene
        self._desc = scene.desc()
        self._cam = sg.RefCameraDescC.from_spec(scene.camera)
        self.h = self.lib().rref_create(ctypes.byref(self._desc), ctypes.byref(self._cam), seed)
        self.n_tris = self.lib().rref_num_triangles(self.h)
        self.n_nodes = self.lib().rref_num_nodes(self.h)

    def bvh(self):
        codes = np.zeros(self.n_tris, np.uint32)
        perm = np.zeros(self.n_tris, np.int32)
        nodes = np.zeros(self.n_nodes, sg.BVH_NODE_DTYPE)
        n = self.lib().rref_bvh_dump(self.h, _ptr(codes), _ptr(perm), _ptr(nodes), self.n_nodes)
        assert n == self.n_nodes
        return codes, perm, nodes

    def camera(self):
        cam = np.zeros(1, sg.CAMERA_DTYPE)
        self.lib().rref_camera(self.h, _ptr(cam))
        return cam

    def primary(self):
        n = self.scene.camera.width * self.scene.camera.height
        out = np.zeros(n, sg.RECEIVER_DTYPE)
        self.lib().rref_primary(self.h, _ptr(out))
        return out

    def primary_rays(self):
        n = self.scene.camera.width * self.scene.camera.height
        o = np.zeros((n, 3), np.float32)
        d = np.zeros((n, 3), np.float32)
        self.lib().rref_primary_rays(self.h, _ptr(o), _ptr(d))
        return o, d

    def occluded(self, p, q):
        p = np.ascontiguousarray(p, np.float32)
        q = np.ascontiguousarray(q, np.float32)
        out = np.zeros(p.shape[0], np.uint8)
        self.lib().rref_occluded(self.h, _ptr(p), _ptr(q), p.shape[0], _ptr(out))
        return out

    def closest(self, o, d):
        o = np.ascontiguousarray(o, np.float32)
        d = np.ascontiguousarray(d, np.float32)
        t = np.zeros(o.shape[0], np.float32)
        rec = np.zeros(o.shape[0], sg.RECEIVER_DTYPE)
        self.lib().rref_closest(self.h, _ptr(o), _ptr(d), o.shape[0], _ptr(t), _ptr(rec))
        return t, rec

    def vpl_generate(self, seed, n_particles, max_bounce, cap=None):
        cap = cap or n_particles * max(1, max_bounce - 1) + 16
        out = np.zeros(cap, sg.VPL_DTYPE)
        n = self.lib().rref_vpl_generate(self.h, seed, n_particles, max_bounce, _ptr(out), cap)
        return out[:min(n, cap)]

    def gather(self, recv, vpls, clamp_mode, tau, pairs=False):
        n, m = recv.shape[0], vpls.shape[0]
        out = np.zeros((n, 3), np.float32)
        rgb = np.zeros((m, n, 3), np.float32) if pairs else None
        vis = np.zeros((m, n), np.uint8) if pairs else None
        self.lib().rref_gather(self.h, _ptr(recv), n, _ptr(vpls), m, clamp_mode, tau,
                               _ptr(out), _ptr(rgb) if pairs else None,
                               _ptr(vis) if pairs else None)
        return (out, rgb, vis) if pairs else out

    def gather_mt(self, recv, vpls, clamp_mode, tau, scale=1.0, threads=None):
        """The reference gather on `threads` host threads (all cores by default)."""
        threads = threads or os.cpu_count() or 1
        out = np.zeros((recv.shape[0], 3), np.float32)
        self.lib().rref_gather_mt(self.h, _ptr(recv), recv.shape[0], _ptr(vpls), vpls.shape[0],
                                  clamp_mode, tau, scale, _ptr(out), threads)
        return out

    def ltm_alphas(self, mat):
        mat = np.ascontiguousarray(mat, np.float32)
        cols, rows = mat.shape[0], mat.shape[1]
        a = np.zeros(cols, np.float32)
        n = np.zeros(cols, np.float32)
        self.lib().rref_ltm_alphas(_ptr(mat), rows, cols, _ptr(a), _ptr(n))
        return a, n

    def cluster_by_sampling(self, mat, num_clusters, seed):
        mat = np.ascontiguousarray(mat, np.float32)
        cols, rows = mat.shape[0], mat.shape[1]
        cap = max(num_clusters, cols)
        c = np.zeros(cap, np.int32); r = np.zeros(cap, np.int32); w = np.zeros(cap, np.float32)
        a = np.zeros(cols, np.int32)
        n = self.lib().rref_cluster_by_sampling(self.h, _ptr(mat), rows, cols, num_clusters, seed,
                                                _ptr(c), _ptr(r), _ptr(w), _ptr(a))
        return c[:n], r[:n], w[:n], a

    @classmethod
    def obj_import(cls, path, cap=100000):
        """The reference's ObjImporter::load on `path`: per triangle / quad surface in order,
        (kind, vertices [12], is_light, radiance, Bsdf::Type or -1, kd, ks, glossy [2]), the
        camera record (or None) and the total surface count."""
        kind = np.zeros(cap, np.int32); v = np.zeros((cap, 12), np.float32)
        light = np.zeros(cap, np.int32); emit = np.zeros((cap, 3), np.float32)
        mtype = np.zeros(cap, np.int32); kd = np.zeros((cap, 3), np.float32)
        ks = np.zeros((cap, 3), np.float32); gl = np.zeros((cap, 2), np.float32)
        cam = np.zeros(1, sg.CAMERA_DTYPE)
        has_cam, n_surf = ctypes.c_int32(), ctypes.c_int32()
        k = cls.lib().rref_obj_import(str(path).encode(), cap, _ptr(kind), _ptr(v), _ptr(light), _ptr(emit),
                                      _ptr(mtype), _ptr(kd), _ptr(ks), _ptr(gl), _ptr(cam),
                                      ctypes.byref(has_cam), ctypes.byref(n_surf))
        out = {"kind": kind[:k], "v": v[:k], "light": light[:k], "emit": emit[:k], "type": mtype[:k],
               "kd": kd[:k], "ks": ks[:k], "glossy": gl[:k]}
        return out, (cam if has_cam.value else None), n_surf.value

    @classmethod
    def json_import(cls, path, cap=100000, light_cap=100000):
        """The reference's JsonImporter::load and get_scene on `path`: the per-surface fields
        of obj_import plus each surface's two-sided flag, the first view's camera record (or
        None), a dict of scene facts (surface count, integrator 1 path / 2 vpl, max_bounce,
        samples, light counts by kind, two-sided option, tmin, near and far planes) and the
        area lights' radiances in light-list order."""
        kind = np.zeros(cap, np.int32); v = np.zeros((cap, 12), np.float32)
        light = np.zeros(cap, np.int32); emit = np.zeros((cap, 3), np.float32)
        mtype = np.zeros(cap, np.int32); kd = np.zeros((cap, 3), np.float32)
        ks = np.zeros((cap, 3), np.float32); gl = np.zeros((cap, 2), np.float32)
        two = np.zeros(cap, np.int32)
        cam = np.zeros(1, sg.CAMERA_DTYPE)
        meta = np.zeros(16, np.int32); fmeta = np.zeros(4, np.float32)
        lemit = np.zeros((light_cap, 3), np.float32)
        k = cls.lib().rref_json_import(str(path).encode(), cap, _ptr(kind), _ptr(v), _ptr(light), _ptr(emit),
                                       _ptr(mtype), _ptr(kd), _ptr(ks), _ptr(gl), _ptr(two), _ptr(cam),
                                       _ptr(meta), _ptr(fmeta), _ptr(lemit), light_cap)
        out = {"kind": kind[:k], "v": v[:k], "light": light[:k], "emit": emit[:k], "type": mtype[:k],
               "kd": kd[:k], "ks": ks[:k], "glossy": gl[:k], "two_sided": two[:k]}
        facts = {"n_surfaces": int(meta[0]), "integrator": int(meta[2]), "max_bounce": int(meta[3]),
                 "samples": int(meta[4]), "point_lights": int(meta[5]), "spot_lights": int(meta[6]),
                 "directional_lights": int(meta[7]), "area_lights": int(meta[8]), "two_sided": int(meta[9]),
                 "tmin": float(fmeta[0]), "near_plane": float(fmeta[1]), "far_plane": float(fmeta[2])}
        return out, (cam if meta[1] else None), facts, lemit[:min(int(meta[8]), light_cap)]

    @classmethod
    def matrix_save(cls, mat, path):
        """The reference's LightTransportMatrix::save of a column-major matrix [cols, rows, 3]."""
        mat = np.ascontiguousarray(mat, np.float32)
        cls.lib().rref_matrix_save(_ptr(mat), mat.shape[1], mat.shape[0], str(path).encode())

    def mrcs(self, vpls, clamp_mode, tau, seed, recv, block_size=32, cluster_ratio=0.01, max_clusters=1000):
        """The reference's MatrixRowColumnSampling::initialize on `vpls` (its draws from the
        stream (seed, 7, 0)), then gather_clusters for every receiver (unscaled).  Returns
        (image [n, 3], centres, representatives, weights)."""
        vpls = np.ascontiguousarray(vpls)
        recv = np.ascontiguousarray(recv)
        n = recv.shape[0]
        out = np.zeros((n, 3), np.float32)
        cap = max(1, vpls.shape[0])
        c = np.zeros(cap, np.int32); r = np.zeros(cap, np.int32); w = np.zeros(cap, np.float32)
        k = self.lib().rref_mrcs(self.h, _ptr(vpls), vpls.shape[0], clamp_mode, tau, seed, block_size,
                                 cluster_ratio, max_clusters, _ptr(recv), n, _ptr(out), _ptr(c), _ptr(r),
                                 _ptr(w), cap)
        k = min(k, cap)
        return out, c[:k], r[:k], w[:k]

    def incident(self, recv, vpls, clamp_mode, tau):
        n, m = recv.shape[0], vpls.shape[0]
        rgb = np.zeros((m, n, 3), np.float32)
        self.lib().rref_incident(self.h, _ptr(recv), n, _ptr(vpls), m, clamp_mode, tau, _ptr(rgb))
        return rgb

    def brdf_eval(self, mat, uvn9, wo, wi):
        n = mat.shape[0]
        out = np.zeros((n, 3), np.float32)
        self.lib().rref_brdf_eval(self.h, _ptr(mat), _ptr(uvn9), _ptr(wo), _ptr(wi), n, _ptr(out))
        return out

    def lightslice(self, max_slice_size: int, num_neighbors: int, seed: int):
        """LightSlice::generate_slices on this scene (stream (seed, 4, 0))."""
        return RefLightSlice(self, max_slice_size, num_neighbors, seed)


class RefLightSlice:
    """The reference's LightSlice stages on a RefHarness scene (see ref/ls_harness.cc)."""

    def __init__(self, ref: RefHarness, max_slice_size: int, num_neighbors: int, seed: int):
        self.ref = ref
        self.k = num_neighbors
        L = RefHarness.lib()
        self.h = L.rref_ls_create(ref.h, max_slice_size, num_neighbors, seed)
        self.n_points = L.rref_ls_num_points(self.h)
        self.n_slices = L.rref_ls_num_slices(self.h)
        self.n_vpl1 = 0
        self.res = 0

    def points(self):
        pts = np.zeros((self.n_points, 6), np.float32)
        pix = np.zeros(self.n_points, np.int32)
        RefHarness.lib().rref_ls_points(self.h, _ptr(pts), _ptr(pix))
        return pts, pix

    def slices(self):
        ns = self.n_slices
        pp = np.zeros(self.n_points, np.int32)
        st, en, rp = (np.zeros(ns, np.int32) for _ in range(3))
        RefHarness.lib().rref_ls_slices(self.h, _ptr(pp), _ptr(st), _ptr(en), _ptr(rp))
        nb = np.zeros((ns, self.k), np.int32)
        RefHarness.lib().rref_ls_neighbors(self.h, _ptr(nb))
        return {"point_pixel": pp, "start": st, "end": en, "rep": rp, "neighbors": nb}

    def find(self, pts):
        pts = np.ascontiguousarray(pts, np.float32)
        out = np.zeros(len(pts), np.int32)
        RefHarness.lib().rref_ls_find(self.h, _ptr(pts), len(pts), _ptr(out))
        return out

    def reduced_matrix(self, vpls, inc_mode=0, inc_tau=0.0):
        vpls = np.ascontiguousarray(vpls)
        n1 = int((vpls["bounce"] <= 1).sum())
        R = np.zeros((n1, self.n_slices, 3), np.float32)
        V = np.zeros((n1, self.n_slices), np.uint8)
        rep = np.zeros(self.n_slices, sg.RECEIVER_DTYPE)
        got = RefHarness.lib().rref_ls_reduced_matrix(self.h, _ptr(vpls), len(vpls), inc_mode, inc_tau, _ptr(R),
                                                      _ptr(V), _ptr(rep))
        assert got == n1
        self.n_vpl1 = n1
        return R, V, rep

    def set_vpls(self, vpls):
        """Loads the one-bounce VPLs without tracing the reduced matrix (for a matrix computed
        elsewhere and passed to refine)."""
        vpls = np.ascontiguousarray(vpls)
        self.n_vpl1 = RefHarness.lib().rref_ls_set_vpls(self.h, _ptr(vpls), len(vpls))
        return self.n_vpl1

    def refine(self, R, V, g_rep, g_weight, assign, mags, max_slice_clusters, seed, res=32, eps=1e-3,
               density_radius=0.1):
        R = np.ascontiguousarray(R, np.float32)
        V = np.ascontiguousarray(V, np.uint8)
        g_rep = np.ascontiguousarray(g_rep, np.int32)
        g_weight = np.ascontiguousarray(g_weight, np.float32)
        assign = np.ascontiguousarray(assign, np.int32)
        mags = np.ascontiguousarray(mags, np.float32)
        self.res = res
        RefHarness.lib().rref_ls_refine(self.h, _ptr(R), _ptr(V), R.shape[0], len(g_rep), _ptr(g_rep),
                                        _ptr(g_weight), _ptr(assign), _ptr(mags), max_slice_clusters, seed, res,
                                        eps, density_radius)

    def clusters(self):
        L = RefHarness.lib()
        nc = L.rref_ls_num_slice_clusters(self.h)
        cnt = np.zeros(self.n_slices, np.int32)
        rep, size = np.zeros(nc, np.int32), np.zeros(nc, np.int32)
        w, pdf = np.zeros(nc, np.float32), np.zeros(nc, np.float32)
        up = np.zeros(nc, np.uint8)
        wi, inc = np.zeros((nc, 3), np.float32), np.zeros((nc, 3), np.float32)
        mem = np.zeros(self.n_slices * max(self.n_vpl1, 1), np.int32)
        cone = np.zeros((nc, 4), np.float32)
        L.rref_ls_clusters(self.h, _ptr(cnt), _ptr(rep), _ptr(w), _ptr(up), _ptr(wi), _ptr(inc), _ptr(pdf),
                           _ptr(size), _ptr(mem), _ptr(cone))
        return {"count": cnt, "rep": rep, "weight": w, "upper": up, "wi": wi, "incident": inc, "pdf": pdf,
                "size": size, "members": mem[: int(size.sum())], "cone": cone}

    def maps(self):
        ns, res = self.n_slices, self.res
        m = np.zeros((ns, res, res), np.float32)
        v = np.zeros(ns, np.uint8)
        sm = np.zeros(ns, np.float32)
        pr = np.zeros((ns, res, res), np.float32)
        RefHarness.lib().rref_ls_maps(self.h, _ptr(m), _ptr(v), _ptr(sm), _ptr(pr))
        return {"maps": m, "valid": v, "sum": sm, "prob": pr}

    def gather(self, recv, clamp_mode, tau, threads=1):
        recv = np.ascontiguousarray(recv)
        out = np.zeros((len(recv), 3), np.float32)
        if threads > 1:
            RefHarness.lib().rref_ls_gather_mt(self.h, _ptr(recv), len(recv), clamp_mode, tau, _ptr(out), threads)
        else:
            RefHarness.lib().rref_ls_gather(self.h, _ptr(recv), len(recv), clamp_mode, tau, _ptr(out))
        return out


    def density(self, slices, xy):
        """LightSlice::eval_incoming_radiance (the METROPOLIS density) of slices[i] at xy[i]."""
        sl = np.ascontiguousarray(slices, np.int32)
        pts = np.ascontiguousarray(xy, np.float32).reshape(-1, 2)
        out = np.zeros(len(sl), np.float32)
        RefHarness.lib().rref_ls_density(self.h, _ptr(sl), _ptr(pts), len(sl), _ptr(out))
        return out

    def guided(self, pixels, spp, max_bounce, rr_depth=0, rr_prob=1.0, direct=True, seed=2013, sampler="jensen"):
        """Per-path radiance [len(pixels)][spp][3] of the reference's guided path tracer with
        its "jensen" or "metropolis" sampler (the Metropolis chains start afresh each call)."""
        RefHarness.lib().rref_ls_set_sampler(self.h, {"jensen": 0, "metropolis": 1}[sampler])
        pixels = np.ascontiguousarray(pixels, np.int32)
        out = np.zeros((len(pixels), spp, 3), np.float32)
        RefHarness.lib().rref_ls_guided(self.h, _ptr(pixels), len(pixels), spp, max_bounce, rr_depth, rr_prob,
                                        1 if direct else 0, seed, _ptr(out))
        return out

class DropinHarness:
    """A scene file loaded by the drop-in factory (load_scene_cuda) and driven through the
    reference's interfaces, beside the reference's AggregateBvh (see ref/dropin_harness.cc)."""

    _lib = None
    SO = os.path.join(HERE, "_ref", "librzk_dropin_test.so")

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.SO) and RefHarness.available()

    @classmethod
    def lib(cls):
        if cls._lib is None:
            RefHarness.lib()
            L = ctypes.CDLL(cls.SO, mode=ctypes.RTLD_GLOBAL)
            L.rdi_load.restype = P
            L.rdi_load.argtypes = [ctypes.c_char_p, I32]
            L.rdi_kinds.restype = I32
            L.rdi_kinds.argtypes = [P]
            L.rdi_segments.restype = I32
            L.rdi_segments.argtypes = [P, P, P, I32, P, P, P]
            L.rdi_closest.restype = I32
            L.rdi_closest.argtypes = [P, P, P, I32, P]
            L.rdi_vpls.restype = I32
            L.rdi_vpls.argtypes = [P, U32, I32, I32, P, P, P, P, I32]
            L.rdi_render.restype = I32
            L.rdi_render.argtypes = [P, I32, I32, U32, P, I32, P]
            cls._lib = L
        return cls._lib

    def __init__(self, path: str, device: int = 0):
        self.h = self.lib().rdi_load(str(path).encode(), device)
        if not self.h:
            raise RuntimeError(f"load_scene_cuda failed on {path}")

    def kinds(self):
        k = self.lib().rdi_kinds(self.h)
        return {"aggregate_cuda": bool(k & 1), "integrator_cuda": bool(k & 2)}

    def segments(self, p, q):
        p = np.ascontiguousarray(p, np.float32)
        q = np.ascontiguousarray(q, np.float32)
        n = len(p)
        virt, batch, ref = (np.zeros(n, np.uint8) for _ in range(3))
        assert self.lib().rdi_segments(self.h, _ptr(p), _ptr(q), n, _ptr(virt), _ptr(batch), _ptr(ref)) == 0
        return virt, batch, ref

    def closest(self, o, d):
        o = np.ascontiguousarray(o, np.float32)
        d = np.ascontiguousarray(d, np.float32)
        rec = np.zeros((len(o), 2, 14), np.float32)
        assert self.lib().rdi_closest(self.h, _ptr(o), _ptr(d), len(o), _ptr(rec)) == 0
        return rec[:, 0], rec[:, 1]

    def vpls(self, seed, particles, max_bounce, cap=None):
        cap = cap or particles * max(1, max_bounce - 1)
        p, c = np.zeros((cap, 3), np.float32), np.zeros((cap, 3), np.float32)
        b, pv = np.zeros(cap, np.int32), np.zeros(cap, np.int32)
        n = self.lib().rdi_vpls(self.h, seed, particles, max_bounce, _ptr(p), _ptr(c), _ptr(b), _ptr(pv), cap)
        assert n >= 0
        n = min(n, cap)
        return {"p": p[:n], "contrib": c[:n], "bounce": b[:n], "prev": pv[:n]}

    def render(self, start_particles, max_vpls, seed, width, height):
        img = np.zeros((height * width, 3), np.float32)
        info = np.zeros(5, np.float32)
        st = self.lib().rdi_render(self.h, start_particles, max_vpls, seed, _ptr(img), img.size, _ptr(info))
        assert st == 0, st
        return img, {"width": int(info[0]), "height": int(info[1]), "vpls": int(info[2]),
                     "emitted": int(info[3]), "tau": float(info[4])}


def column_magnitudes(mat: np.ndarray) -> np.ndarray:
    """The magnitude of every flattened column [cols][rows][3] summed in order, as
    ClusterBuilder's magnitude() (cluster_builder.cc:14-20) computes it in float."""
    flat = np.ascontiguousarray(mat, np.float32).reshape(mat.shape[0], -1)
    sq = flat * flat
    return np.sqrt(np.cumsum(sq, axis=1, dtype=np.float32)[:, -1]).astype(np.float32)
