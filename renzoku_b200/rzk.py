"""ctypes bindings for librzk_cuda.so (include/rzk.h) and the Python-side mirror of the
reference's plugin interfaces for the VPL gather path.

The classes keep the reference's names and argument meanings so that callers and tests
read like the reference's own code:

  AggregateCuda           Aggregate / AggregateBvh (aggregate.h:15-91, aggregate_bvh.h:22)
                          hit(p, q) -> occluded, hit(ray) -> closest hit, BVH dump
  VplGeneratorCuda        IVplGenerator::spawn (vpl_generator.h:8-21)
  VirtualPointLightCuda   IVirtualPointLightEvaluator::radiance / incident_radiance
                          (vpl_interface.h:126-139) batched: gather, transport matrix fill
  Camera                  Camera::set_perspective / shoot_ray (camera.cc:23-65)

Device buffers are torch CUDA tensors (PyTorch is used for device memory and streams
only); every computation runs in the CUDA library.  There is no CPU fallback: on a
machine without the built library or a GPU these classes raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import scenegen as sg

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librzk_cuda.so")

P = ctypes.c_void_p
I32 = ctypes.c_int32
U32 = ctypes.c_uint32
F32 = ctypes.c_float

# status codes (rzk_types.h)
OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_TIMEOUT, ERR_STACK, ERR_CAPACITY, ERR_UNSUPPORTED, ERR_BUSY = range(9)
CLAMP_NONE, CLAMP_FORM_FACTOR, CLAMP_REFLECTIVITY, CLAMP_RADIANCE = range(4)

# every symbol include/rzk.h declares: (name, restype, argtypes)
SIGNATURES = [
    ("rzk_status_string", ctypes.c_char_p, [I32]),
    ("rzk_context_create", I32, [I32, P]),
    ("rzk_context_destroy", I32, [P]),
    ("rzk_context_check", I32, [P, P]),
    ("rzk_context_rays", I32, [P, P, I32, P]),
    ("rzk_debug_ring_wait", I32, [P, I32, P, P]),
    ("rzk_scene_create", I32, [P, P, P, P]),
    ("rzk_scene_destroy", I32, [P]),
    ("rzk_scene_info", I32, [P, P, P, P, P]),
    ("rzk_scene_bounding_box", I32, [P, P]),
    ("rzk_scene_rebuild", I32, [P, P]),
    ("rzk_scene_serialized_size", I32, [P, P]),
    ("rzk_scene_serialize", I32, [P, P, ctypes.c_size_t, P, P]),
    ("rzk_scene_deserialize", I32, [P, P, ctypes.c_size_t, P, P]),
    ("rzk_matrix_save", I32, [ctypes.c_char_p, P, I32, I32, P]),
    ("rzk_matrix_file_info", I32, [ctypes.c_char_p, P, P]),
    ("rzk_matrix_load", I32, [ctypes.c_char_p, P, I32, I32, P]),
    ("rzk_bvh_dump", I32, [P, P, P, P, I32, P]),
    ("rzk_morton_codes", I32, [P, P, P]),
    ("rzk_occluded_batch", I32, [P, P, P, I32, P, P]),
    ("rzk_closest_batch", I32, [P, P, P, I32, P, P, P]),
    ("rzk_ray_query_batch", I32, [P, P, I32, I32, P, P]),
    ("rzk_primary", I32, [P, P, P, P]),
    ("rzk_camera_setup", I32, [P, P, P, F32, I32, I32, F32, F32, P]),
    ("rzk_camera_setup_focal", I32, [P, P, P, F32, I32, I32, F32, F32, P]),
    ("rzk_obj_import", I32, [ctypes.c_char_p, P]),
    ("rzk_obj_get_info", I32, [P, P]),
    ("rzk_obj_scene_desc", I32, [P, P]),
    ("rzk_obj_destroy", I32, [P]),
    ("rzk_json_import", I32, [ctypes.c_char_p, P]),
    ("rzk_json_get_info", I32, [P, P]),
    ("rzk_json_scene_desc", I32, [P, P]),
    ("rzk_json_destroy", I32, [P]),
    ("rzk_vpl_generate", I32, [P, U32, I32, I32, P, I32, P, P]),
    ("rzk_gather", I32, [P, P, P, I32, P, I32, I32, F32, F32, P, P]),
    ("rzk_gather_variants", I32, []),
    ("rzk_gather_cfg", I32, [P, P, P, I32, I32, P, I32, I32, F32, F32, P, I32, I32, P]),
    ("rzk_gather_host", I32, [P, P, P, I32, I32, P, I32, I32, F32, F32, P, P]),
    ("rzk_gather_matrix", I32, [P, P, I32, P, I32, I32, F32, P, P, P]),
    ("rzk_incident_matrix", I32, [P, P, I32, P, I32, I32, F32, P, P]),
    ("rzk_mean_contribution", I32, [P, P, P, I32, P, I32, U32, I32, P, P]),
    ("rzk_gather_noalloc", I32, [P, P, I32, I32, P, I32, I32, F32, F32, P, P]),
    ("rzk_ltm_alphas", I32, [P, I32, I32, P, P, P]),
    ("rzk_cluster_by_sampling", I32, [P, I32, I32, I32, U32, P, P, P, P, P, P]),
    ("rzk_mrcs_params_default", I32, [P]),
    ("rzk_mrcs_create", I32, [P, P, P, P, I32, I32, F32, P, P, P]),
    ("rzk_mrcs_destroy", I32, [P]),
    ("rzk_mrcs_info", I32, [P, P, P, P, P, P]),
    ("rzk_mrcs_clusters", I32, [P, P, P, P, P]),
    ("rzk_mrcs_gather", I32, [P, P, I32, I32, F32, P, P]),
    ("rzk_batch_variants", I32, []),
    ("rzk_batch_create", I32, [P, P, I32, I32, I32, P]),
    ("rzk_batch_run", I32, [P, P]),
    ("rzk_batch_destroy", I32, [P]),
    ("rzk_batch_autotune", I32, [P, P, I32, I32, P, P, P, P, P]),
    ("rzk_batch_variant_info", I32, [I32, P, P, P, P]),
    ("rzk_lightslice_params_default", I32, [P]),
    ("rzk_lightslice_create", I32, [P, P, P, I32, I32, P, I32, P, P, P]),
    ("rzk_lightslice_destroy", I32, [P]),
    ("rzk_lightslice_info", I32, [P, P, P, P, P, P, P]),
    ("rzk_lightslice_slices", I32, [P, P, P, P, P, P]),
    ("rzk_lightslice_global", I32, [P, P, P, P]),
    ("rzk_lightslice_clusters", I32, [P, P, P, P, P, P, P, P, P, P]),
    ("rzk_lightslice_maps", I32, [P, P, P, P, P, P]),
    ("rzk_lightslice_matrix", I32, [P, P, P, P, P]),
    ("rzk_lightslice_find_slice", I32, [P, P, I32, P, P]),
    ("rzk_lightslice_host_slice", I32, [P, P, P, I32, P]),
    ("rzk_lightslice_host_refine", I32, [P, P, P, I32, P, P, I32, P, P, P, P]),
    ("rzk_lightslice_host_find", I32, [P, P, I32, P]),
    ("rzk_lightslice_gather", I32, [P, P, I32, I32, F32, F32, P, P]),
    ("rzk_guided_render", I32, [P, P, P, P, P, P, P, P]),
    ("rzk_lightslice_density", I32, [P, P, P, I32, P, P]),
    ("rzk_lightslice_chains", I32, [P, U32, I32, P, P]),
    ("rzk_server_create", I32, [I32, P, P]),
    ("rzk_server_destroy", I32, [P]),
    ("rzk_server_submit", I32, [P, P, P]),
    ("rzk_server_poll", I32, [P, ctypes.c_uint64, P, P]),
    ("rzk_server_wait", I32, [P, ctypes.c_uint64, I32, P]),
    ("rzk_server_cancel", I32, [P, ctypes.c_uint64]),
    ("rzk_server_stats", I32, [P, P, P, P, P, P, P]),
    ("rzk_server_timings", I32, [P, P, P, P, I32, P]),
]

_LIB = None


class RzkError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        msg = _LIB.rzk_status_string(status).decode() if _LIB is not None else str(status)
        super().__init__(f"{what}: {msg} (status {status})")


def load(path: str = LIB_PATH):
    """Load librzk_cuda.so; raises when it has not been built (no fallback)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run renzoku_b200/build.py (no CPU fallback)")
        L = ctypes.CDLL(path)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(status: int, what: str) -> None:
    if status != OK:
        raise RzkError(status, what)


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("renzoku_b200 needs a CUDA device (no CPU fallback)")
    return torch


def _stream_ptr(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _dptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def records_to_device(arr: np.ndarray, device="cuda"):
    """numpy structured records -> contiguous uint8 CUDA tensor of the same bytes."""
    torch = _torch()
    raw = np.ascontiguousarray(arr).view(np.uint8).reshape(-1)
    return torch.from_numpy(raw.copy()).to(device)


def records_from_device(t, dtype) -> np.ndarray:
    return t.detach().cpu().numpy().view(dtype).reshape(-1)


class Context:
    """One device + the library's scratch buffers (rzk_context)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        self.device = device
        h = ctypes.c_void_p()
        check(self.lib.rzk_context_create(device, ctypes.byref(h)), "rzk_context_create")
        self.h = h

    def check(self, stream=None) -> None:
        check(self.lib.rzk_context_check(self.h, _stream_ptr(stream)), "device error word")

    def rays(self, reset: bool = False, stream=None) -> int:
        """Shadow rays the gather kernels traced since creation or the last reset
        (rzk_context_rays)."""
        n = ctypes.c_uint64()
        check(self.lib.rzk_context_rays(self.h, ctypes.byref(n), 1 if reset else 0, _stream_ptr(stream)),
              "rzk_context_rays")
        return int(n.value)

    def close(self):
        if getattr(self, "h", None):
            self.lib.rzk_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Camera:
    """Camera::set_perspective + Sensor: the pinhole parameters (rzk_camera)."""

    def __init__(self, spec: sg.CameraSpec):
        lib = load()
        self.spec = spec
        self.rec = np.zeros(1, sg.CAMERA_DTYPE)
        f = lambda t: np.asarray(t, np.float32)
        e, l, u = f(spec.eye), f(spec.lookat), f(spec.up)
        check(lib.rzk_camera_setup(e.ctypes.data, l.ctypes.data, u.ctypes.data, spec.fov,
                                   spec.width, spec.height, spec.film_w, spec.film_h,
                                   self.rec.ctypes.data), "rzk_camera_setup")

    @classmethod
    def from_focal(cls, eye, lookat, up, focal: float, width: int, height: int, film_w: float,
                   film_h: float) -> "Camera":
        """Camera::set_perspective with a focal length (the OBJ camera line)."""
        self = cls.__new__(cls)
        self.spec = sg.CameraSpec(tuple(eye), tuple(lookat), tuple(up), float("nan"), width, height, film_w, film_h)
        self.rec = np.zeros(1, sg.CAMERA_DTYPE)
        f = lambda t: np.asarray(t, np.float32)
        e, l, u = f(eye), f(lookat), f(up)
        check(load().rzk_camera_setup_focal(e.ctypes.data, l.ctypes.data, u.ctypes.data, focal, width, height,
                                            film_w, film_h, self.rec.ctypes.data), "rzk_camera_setup_focal")
        return self

    @property
    def n_pixels(self) -> int:
        return self.spec.width * self.spec.height

    @property
    def width(self) -> int:
        return self.spec.width

    @property
    def height(self) -> int:
        return self.spec.height


class ObjInfoC(ctypes.Structure):
    """ctypes mirror of rzk_obj_info."""
    _fields_ = [("n_prims", I32), ("n_mats", I32), ("n_lights", I32), ("has_camera", I32),
                ("eye", F32 * 3), ("lookat", F32 * 3), ("up", F32 * 3), ("focal", F32),
                ("width", I32), ("height", I32), ("film_w", F32), ("film_h", F32),
                ("point_lights", I32), ("spheres", I32), ("faces_without_material", I32),
                ("faces_unsupported_material", I32), ("short_faces", I32),
                ("faces_with_vertex_normals", I32), ("smoothed_faces", I32), ("mtl_files_missing", I32)]


def _scene_from_desc(name: str, d, info):
    """A scenegen.Scene copied out of a filled rzk_scene_desc, with the info's camera."""
    n, m = d.n_prims, d.n_mats

    def arr(ptr, dtype, count):
        if count == 0:
            return np.zeros(0, dtype)
        return np.frombuffer(ctypes.string_at(ptr, np.dtype(dtype).itemsize * count), dtype).copy()

    spec = sg.CameraSpec(tuple(info.eye), tuple(info.lookat), tuple(info.up), float("nan"), info.width,
                         info.height, info.film_w, info.film_h)
    return sg.Scene(name, arr(d.prim_kind, np.int32, n),
                    arr(d.prim_v, np.float32, 12 * n).reshape(n, 12), arr(d.prim_mat, np.int32, n),
                    arr(d.prim_emit, np.float32, 3 * n).reshape(n, 3), arr(d.prim_flags, np.int32, n),
                    arr(d.mats, sg.MATERIAL_DTYPE, m), spec, d.tmin)


def _import_scene_file(path, kind: str, info_cls):
    lib = load()
    h = ctypes.c_void_p()
    check(getattr(lib, f"rzk_{kind}_import")(str(path).encode(), ctypes.byref(h)), f"rzk_{kind}_import")
    try:
        info = info_cls()
        check(getattr(lib, f"rzk_{kind}_get_info")(h, ctypes.byref(info)), f"rzk_{kind}_get_info")
        d = sg.SceneDescC()
        check(getattr(lib, f"rzk_{kind}_scene_desc")(h, ctypes.byref(d)), f"rzk_{kind}_scene_desc")
        scene = _scene_from_desc(os.path.splitext(os.path.basename(str(path)))[0], d, info)
        cam = (Camera.from_focal(info.eye, info.lookat, info.up, info.focal, info.width, info.height,
                                 info.film_w, info.film_h) if info.has_camera else None)
        out = {k: getattr(info, k) for k, _ in info_cls._fields_ if k not in ("eye", "lookat", "up")}
        return scene, cam, out
    finally:
        getattr(lib, f"rzk_{kind}_destroy")(h)


def import_obj(path: str):
    """A Wavefront OBJ scene in the reference's dialect (rzk_obj_import): returns
    (scenegen.Scene, Camera or None, info dict of what was counted and left out)."""
    return _import_scene_file(path, "obj", ObjInfoC)


class JsonInfoC(ctypes.Structure):
    """ctypes mirror of rzk_json_info."""
    _fields_ = [("n_prims", I32), ("n_mats", I32), ("n_lights", I32), ("has_camera", I32),
                ("eye", F32 * 3), ("lookat", F32 * 3), ("up", F32 * 3), ("focal", F32),
                ("width", I32), ("height", I32), ("film_w", F32), ("film_h", F32),
                ("near_plane", F32), ("far_plane", F32), ("integrator", I32), ("max_bounce", I32),
                ("samples", I32), ("tmin", F32), ("two_sided", I32), ("obj_files", I32),
                ("point_lights", I32), ("spot_lights", I32), ("directional_lights", I32), ("spheres", I32),
                ("surfaces_unsupported_material", I32), ("skipped", I32), ("faces_with_vertex_normals", I32),
                ("smoothed_faces", I32), ("traversal", I32)]


JSON_INTEGRATORS = {0: None, 1: "path", 2: "vpl", 3: "vpl_cuda"}
JSON_TRAVERSALS = {0: "bvh", 1: "none", 2: "cuda_lbvh"}


def import_json(path: str):
    """A scene file in the reference's JSON format (rzk_json_import; JsonImporter::load and
    get_scene, json_importer.cc): returns (scenegen.Scene, Camera or None, info dict with the
    first view's integrator, max_bounce and samples and what was counted and left out)."""
    return _import_scene_file(path, "json", JsonInfoC)


class AggregateCuda:
    """Device-resident scene + LBVH; the Aggregate interface (aggregate.h:15-91)."""

    def __init__(self, ctx: Context, scene: sg.Scene, stream=None):
        self.ctx = ctx
        self.lib = ctx.lib
        self.scene = scene
        self._desc = scene.desc()
        h = ctypes.c_void_p()
        check(self.lib.rzk_scene_create(ctx.h, ctypes.byref(self._desc), _stream_ptr(stream),
                                        ctypes.byref(h)), "rzk_scene_create")
        self.h = h
        self._info()
        self.tmin = scene.tmin

    def _info(self):
        nt, nn, nl = I32(), I32(), I32()
        nb = ctypes.c_size_t()
        check(self.lib.rzk_scene_info(self.h, ctypes.byref(nt), ctypes.byref(nn), ctypes.byref(nl),
                                      ctypes.byref(nb)), "rzk_scene_info")
        self.n_tris, self.n_nodes, self.n_levels, self.device_bytes = nt.value, nn.value, nl.value, nb.value

    def serialize(self, stream=None) -> bytes:
        """The built scene as one blob (rzk_scene_serialize), for a warm restart."""
        n = ctypes.c_size_t()
        check(self.lib.rzk_scene_serialized_size(self.h, ctypes.byref(n)), "rzk_scene_serialized_size")
        buf = ctypes.create_string_buffer(n.value)
        w = ctypes.c_size_t()
        check(self.lib.rzk_scene_serialize(self.h, buf, n.value, ctypes.byref(w), _stream_ptr(stream)),
              "rzk_scene_serialize")
        return buf.raw[: w.value]

    @classmethod
    def restore(cls, ctx: Context, blob: bytes, scene: sg.Scene, stream=None) -> "AggregateCuda":
        """A scene rebuilt from serialize()'s blob without building its trees again; `scene`
        is the description it was made from (kept for the Python-side fields)."""
        self = cls.__new__(cls)
        self.ctx, self.lib, self.scene = ctx, ctx.lib, scene
        h = ctypes.c_void_p()
        check(self.lib.rzk_scene_deserialize(ctx.h, blob, len(blob), _stream_ptr(stream), ctypes.byref(h)),
              "rzk_scene_deserialize")
        self.h = h
        self._info()
        self.tmin = scene.tmin
        return self

    def close(self):
        if getattr(self, "h", None):
            self.lib.rzk_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rebuild(self, stream=None):
        check(self.lib.rzk_scene_rebuild(self.h, _stream_ptr(stream)), "rzk_scene_rebuild")

    def bvh_dump(self):
        codes = np.zeros(self.n_tris, np.uint32)
        perm = np.zeros(self.n_tris, np.int32)
        nodes = np.zeros(self.n_nodes, sg.BVH_NODE_DTYPE)
        check(self.lib.rzk_bvh_dump(self.h, codes.ctypes.data, perm.ctypes.data, nodes.ctypes.data,
                                    self.n_nodes, _stream_ptr()), "rzk_bvh_dump")
        return codes, perm, nodes

    def bounding_box(self) -> np.ndarray:
        """Aggregate::get_bounding_box: float32 [6] = min xyz, max xyz."""
        box = np.zeros(6, np.float32)
        check(self.lib.rzk_scene_bounding_box(self.h, box.ctypes.data), "rzk_scene_bounding_box")
        return box

    def morton_codes(self):
        codes = np.zeros(self.n_tris, np.uint32)
        check(self.lib.rzk_morton_codes(self.h, codes.ctypes.data, _stream_ptr()), "rzk_morton_codes")
        return codes

    def hit_segments(self, p, q, stream=None):
        """Aggregate::hit(p, q, tmin, time) for device tensors p, q [n,3] float32: uint8 [n]."""
        torch = _torch()
        n = p.shape[0]
        out = torch.empty(n, dtype=torch.uint8, device=p.device)
        check(self.lib.rzk_occluded_batch(self.h, _dptr(p), _dptr(q), n, _dptr(out),
                                          _stream_ptr(stream)), "rzk_occluded_batch")
        return out

    def hit_rays(self, o, d, stream=None):
        """Closest hits of rays (o, d): (t [n] float32, receivers [n*96] uint8)."""
        torch = _torch()
        n = o.shape[0]
        t = torch.empty(n, dtype=torch.float32, device=o.device)
        recv = torch.empty(n * 96, dtype=torch.uint8, device=o.device)
        check(self.lib.rzk_closest_batch(self.h, _dptr(o), _dptr(d), n, _dptr(t), _dptr(recv),
                                         _stream_ptr(stream)), "rzk_closest_batch")
        return t, recv

    def primary(self, camera: Camera, out=None, stream=None):
        """One pixel-centre primary hit per pixel as receiver records (uint8 tensor)."""
        torch = _torch()
        if out is None:
            out = torch.empty(camera.n_pixels * 96, dtype=torch.uint8, device="cuda")
        check(self.lib.rzk_primary(self.h, camera.rec.ctypes.data, _dptr(out), _stream_ptr(stream)),
              "rzk_primary")
        return out


class VplGeneratorCuda:
    """IVplGenerator::spawn (vpl_generator.h:12-14) on the device."""

    def __init__(self, aggregate: AggregateCuda):
        self.agg = aggregate

    def spawn(self, seed: int, num_start_particles: int, max_bounce: int, cap: int | None = None,
              stream=None):
        torch = _torch()
        cap = cap or num_start_particles * max(1, max_bounce - 1)
        out = torch.zeros(cap * 96, dtype=torch.uint8, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        check(self.agg.lib.rzk_vpl_generate(self.agg.h, seed, num_start_particles, max_bounce,
                                            _dptr(out), cap, _dptr(cnt), _stream_ptr(stream)),
              "rzk_vpl_generate")
        n = int(cnt.item())
        return out[: min(n, cap) * 96], n


class VirtualPointLightCuda:
    """The VPL evaluator (IVirtualPointLightEvaluator, vpl_interface.h:126-139) batched over
    receivers x VPLs, with the reference's clamp modes (vpl_interface.h:155-162)."""

    def __init__(self, aggregate: AggregateCuda, clamp_mode: int = CLAMP_FORM_FACTOR,
                 clamp_threshold: float = 1e-3):
        # VirtualPointLight::VirtualPointLight defaults (vpl.cc:180-202)
        self.agg = aggregate
        self.ctx = aggregate.ctx
        self.clamp_mode = clamp_mode
        self.clamp_threshold = clamp_threshold

    def gather(self, recv, n_recv, vpls, n_vpl, scale=1.0, out=None, image_width=0, variant=0,
               n_chunks=0, stream=None):
        """Per-receiver sum of gather_point over all VPLs, times `scale`.  image_width > 0
        declares the receivers a row-major image (8 x 4 pixel warp tiles)."""
        torch = _torch()
        if out is None:
            out = torch.empty((n_recv, 3), dtype=torch.float32, device="cuda")
        check(self.agg.lib.rzk_gather_cfg(self.ctx.h, self.agg.h, _dptr(recv), n_recv, image_width,
                                          _dptr(vpls), n_vpl, self.clamp_mode, self.clamp_threshold,
                                          scale, _dptr(out), variant, n_chunks, _stream_ptr(stream)),
              "rzk_gather")
        return out

    def gather_host(self, recv_np: np.ndarray, vpls_np: np.ndarray, scale=1.0,
                    image_width=0) -> np.ndarray:
        """End-to-end call on host buffers (pinned or pageable numpy arrays)."""
        out = np.zeros((recv_np.shape[0], 3), np.float32)
        check(self.agg.lib.rzk_gather_host(self.ctx.h, self.agg.h, recv_np.ctypes.data,
                                           recv_np.shape[0], image_width, vpls_np.ctypes.data,
                                           vpls_np.shape[0], self.clamp_mode, self.clamp_threshold,
                                           scale, out.ctypes.data, _stream_ptr()), "rzk_gather_host")
        return out

    def fill(self, recv, n_recv, vpls, n_vpl, with_visibility=True, stream=None):
        """TransportMatrix::fill: column-major [n_vpl, n_recv, 3] matrix (+ visibility)."""
        torch = _torch()
        mat = torch.empty((n_vpl, n_recv, 3), dtype=torch.float32, device="cuda")
        vis = torch.empty((n_vpl, n_recv), dtype=torch.uint8, device="cuda") if with_visibility else None
        check(self.agg.lib.rzk_gather_matrix(self.agg.h, _dptr(recv), n_recv, _dptr(vpls), n_vpl,
                                             self.clamp_mode, self.clamp_threshold, _dptr(mat),
                                             _dptr(vis) if vis is not None else None,
                                             _stream_ptr(stream)), "rzk_gather_matrix")
        return mat, vis

    def incident_radiance(self, recv, n_recv, vpls, n_vpl, threshold=None, stream=None):
        torch = _torch()
        mat = torch.empty((n_vpl, n_recv, 3), dtype=torch.float32, device="cuda")
        tau = self.clamp_threshold if threshold is None else threshold
        check(self.agg.lib.rzk_incident_matrix(self.agg.h, _dptr(recv), n_recv, _dptr(vpls), n_vpl,
                                               self.clamp_mode, tau, _dptr(mat), _stream_ptr(stream)),
              "rzk_incident_matrix")
        return mat

    def mean_contribution(self, recv, n_recv, vpls, n_vpl, seed=0, n_pairs=65536, stream=None):
        m = ctypes.c_double()
        check(self.agg.lib.rzk_mean_contribution(self.ctx.h, self.agg.h, _dptr(recv), n_recv,
                                                 _dptr(vpls), n_vpl, seed, n_pairs, ctypes.byref(m),
                                                 _stream_ptr(stream)), "rzk_mean_contribution")
        return m.value


def pair_indices(seed: int, n_pairs: int, n_recv: int, n_vpl: int, draw_u32):
    """The seeded (receiver, VPL) pairs of rzk_mean_contribution, from a draw function."""
    ri = np.array([draw_u32(seed, 3, k, 0) % n_recv for k in range(n_pairs)], np.int32)
    vi = np.array([draw_u32(seed, 3, k, 1) % n_vpl for k in range(n_pairs)], np.int32)
    return ri, vi


def matrix_save(path: str, mat, stream=None) -> None:
    """Writes a device matrix [cols, rows, 3] in MatrixC<Rgb>::save's format."""
    check(load().rzk_matrix_save(str(path).encode(), _dptr(mat), mat.shape[1], mat.shape[0],
                                 _stream_ptr(stream)), "rzk_matrix_save")


def matrix_load(path: str, stream=None):
    """Reads a MatrixC<Rgb>::save file into a new device matrix [cols, rows, 3]."""
    torch = _torch()
    rows, cols = I32(), I32()
    check(load().rzk_matrix_file_info(str(path).encode(), ctypes.byref(rows), ctypes.byref(cols)),
          "rzk_matrix_file_info")
    mat = torch.empty((cols.value, rows.value, 3), dtype=torch.float32, device="cuda")
    check(load().rzk_matrix_load(str(path).encode(), _dptr(mat), rows.value, cols.value, _stream_ptr(stream)),
          "rzk_matrix_load")
    return mat


class ClusterBuilderCuda:
    """ClusterBuilder::cluster_by_sampling (cluster_builder.h:10-27) and the matrix
    statistics it uses, on a device matrix [cols, rows, 3] (column-major MatrixC<Rgb>)."""

    def __init__(self):
        self.lib = load()

    def alphas(self, mat, stream=None):
        torch = _torch()
        cols, rows = mat.shape[0], mat.shape[1]
        a = torch.empty(cols, dtype=torch.float32, device=mat.device)
        n = torch.empty(cols, dtype=torch.float32, device=mat.device)
        check(self.lib.rzk_ltm_alphas(_dptr(mat), rows, cols, _dptr(a), _dptr(n), _stream_ptr(stream)),
              "rzk_ltm_alphas")
        return a, n

    def cluster_by_sampling(self, mat, num_clusters, seed, stream=None):
        """Returns (centers, representatives, weights, assignment) as numpy arrays."""
        cols, rows = mat.shape[0], mat.shape[1]
        cap = max(num_clusters, cols)
        c = np.zeros(cap, np.int32)
        r = np.zeros(cap, np.int32)
        w = np.zeros(cap, np.float32)
        a = np.zeros(max(cols, 1), np.int32)
        n = I32()
        check(self.lib.rzk_cluster_by_sampling(_dptr(mat), rows, cols, num_clusters, seed, ctypes.byref(n),
                                               c.ctypes.data, r.ctypes.data, w.ctypes.data, a.ctypes.data,
                                               _stream_ptr(stream)), "rzk_cluster_by_sampling")
        k = n.value
        return c[:k], r[:k], w[:k], a[:cols]


class MrcsParamsC(ctypes.Structure):
    """ctypes mirror of rzk_mrcs_params."""
    _fields_ = [("block_size", I32), ("cluster_ratio", F32), ("max_clusters", I32), ("max_columns", I32),
                ("seed", U32)]


def mrcs_params(**kw) -> MrcsParamsC:
    """MatrixRowColumnSampling's defaults (mrcs.cc:16-20) with keyword overrides."""
    p = MrcsParamsC()
    check(load().rzk_mrcs_params_default(ctypes.byref(p)), "rzk_mrcs_params_default")
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class MrcsCuda:
    """MatrixRowColumnSampling (mrcs.h:17-45): initialize() at construction on device VPLs,
    gather_clusters() for every receiver with gather()."""

    def __init__(self, agg: "AggregateCuda", camera: "Camera", vpls, n_vpl: int, clamp_mode: int, tau: float,
                 params: MrcsParamsC | None = None, stream=None):
        self.lib = load()
        self.agg = agg
        self.params = params or mrcs_params()
        h = ctypes.c_void_p()
        check(self.lib.rzk_mrcs_create(agg.ctx.h, agg.h, camera.rec.ctypes.data, _dptr(vpls) if n_vpl else None,
                                       n_vpl, clamp_mode, tau, ctypes.byref(self.params),
                                       _stream_ptr(stream), ctypes.byref(h)), "rzk_mrcs_create")
        self.h = h

    def info(self) -> dict:
        rows, cols, target, n = I32(), I32(), I32(), I32()
        ms = np.zeros(4, np.float32)
        check(self.lib.rzk_mrcs_info(self.h, ctypes.byref(rows), ctypes.byref(cols), ctypes.byref(target),
                                     ctypes.byref(n), ms.ctypes.data), "rzk_mrcs_info")
        return {"rows": rows.value, "columns": cols.value, "num_clusters": target.value, "clusters": n.value,
                "stage_ms": ms.tolist()}

    def clusters(self):
        """(pixels [rows, 2] (x, y), centres, representatives, weights)."""
        i = self.info()
        px = np.zeros((i["rows"], 2), np.int32)
        c = np.zeros(max(i["clusters"], 1), np.int32)
        r = np.zeros_like(c)
        w = np.zeros(c.shape[0], np.float32)
        check(self.lib.rzk_mrcs_clusters(self.h, px.ctypes.data, c.ctypes.data, r.ctypes.data, w.ctypes.data),
              "rzk_mrcs_clusters")
        k = i["clusters"]
        return px, c[:k], r[:k], w[:k]

    def gather(self, recv, n_recv, scale=1.0, out=None, image_width=0, stream=None):
        torch = _torch()
        if out is None:
            out = torch.empty((n_recv, 3), dtype=torch.float32, device="cuda")
        check(self.lib.rzk_mrcs_gather(self.h, _dptr(recv), n_recv, image_width, scale, _dptr(out),
                                       _stream_ptr(stream)), "rzk_mrcs_gather")
        return out

    def close(self):
        if getattr(self, "h", None):
            self.lib.rzk_mrcs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GatherJobC(ctypes.Structure):
    """ctypes mirror of rzk_gather_job."""
    _fields_ = [("scene", P), ("d_recv", P), ("n_recv", I32), ("image_width", I32), ("d_vpls", P),
                ("n_vpl", I32), ("clamp_mode", I32), ("tau", F32), ("scale", F32), ("d_rgb", P)]


def make_jobs(items):
    """items: iterable of (AggregateCuda, recv tensor, n_recv, image_width, vpl tensor, n_vpl,
    clamp_mode, tau, scale, out tensor) -> ctypes array of rzk_gather_job."""
    items = list(items)
    arr = (GatherJobC * len(items))()
    for k, (agg, recv, n_recv, w, vpls, n_vpl, mode, tau, scale, out) in enumerate(items):
        arr[k] = GatherJobC(agg.h.value, recv.data_ptr(), n_recv, w, vpls.data_ptr(), n_vpl, mode, tau,
                            scale, out.data_ptr())
    return arr


class GatherBatch:
    """Many gathers in one persistent launch (rzk_batch_*); run() is graph-capturable."""

    def __init__(self, ctx: Context, jobs, variant=0, chunk_len=0):
        self.lib = load()
        self.jobs = jobs
        h = ctypes.c_void_p()
        check(self.lib.rzk_batch_create(ctx.h, jobs, len(jobs), variant, chunk_len, ctypes.byref(h)),
              "rzk_batch_create")
        self.h = h

    def run(self, stream=None):
        check(self.lib.rzk_batch_run(self.h, _stream_ptr(stream)), "rzk_batch_run")

    def close(self):
        if getattr(self, "h", None):
            self.lib.rzk_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_variant_info(variant: int) -> dict:
    """A batch variant's tile shape (rzk_batch_variant_info)."""
    lib = load()
    w, t, m, tw = I32(), I32(), I32(), I32()
    check(lib.rzk_batch_variant_info(variant, ctypes.byref(w), ctypes.byref(t), ctypes.byref(m), ctypes.byref(tw)),
          "rzk_batch_variant_info")
    return {"warps": w.value, "vpl_tile": t.value, "ctas_per_sm": m.value,
            "warp_tile": f"{tw.value}x{32 // tw.value}"}


def autotune_batch(ctx: Context, jobs, max_probe_jobs=8, stream=None, table: bool = False):
    """Returns (variant, chunk_len, probe_ms) of the fastest batch configuration, and with
    table=True also every probe's time [variants][4 chunk lengths: default, 512, 1024, 2048]."""
    lib = load()
    v, c, ms = I32(), I32(), ctypes.c_float()
    probes = np.zeros((lib.rzk_batch_variants(), 4), np.float32)
    check(lib.rzk_batch_autotune(ctx.h, jobs, len(jobs), max_probe_jobs, ctypes.byref(v), ctypes.byref(c),
                                 ctypes.byref(ms), probes.ctypes.data, _stream_ptr(stream)), "rzk_batch_autotune")
    if table:
        return v.value, c.value, ms.value, probes
    return v.value, c.value, ms.value


class LightSliceParamsC(ctypes.Structure):
    """ctypes mirror of rzk_lightslice_params."""
    _fields_ = [("num_clusters", I32), ("max_slice_size", I32), ("num_neighbor_slices", I32),
                ("max_slice_clusters", I32), ("map_resolution", I32), ("map_epsilon", F32),
                ("density_radius", F32), ("incident_clamp_mode", I32), ("incident_tau", F32),
                ("seed", U32), ("n_threads", I32)]


def lightslice_params(**kw) -> LightSliceParamsC:
    """The reference's defaults (lightslice.cc:23-85) with keyword overrides."""
    p = LightSliceParamsC()
    check(load().rzk_lightslice_params_default(ctypes.byref(p)), "rzk_lightslice_params_default")
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class GuidedParamsC(ctypes.Structure):
    """ctypes mirror of rzk_guided_params."""
    _fields_ = [("spp", I32), ("max_bounce", I32), ("rr_depth", I32), ("rr_prob", F32),
                ("direct_lighting", I32), ("seed", U32), ("sampler", I32), ("chain_samples", I32)]


GUIDE_JENSEN = 0
GUIDE_METROPOLIS = 1


class LightSliceCuda:
    """LightSlice (lightslice.cc): slicing, reduced matrix, clustering, per-slice refinement and
    maps built from an image's receivers and a VPL set; gather() is gather_clusters for every
    pixel.  Built from host inputs (from_host) it holds the host stages only."""

    def __init__(self, handle, params, lib=None, agg=None):
        self.lib = lib or load()
        self.h = handle
        self.params = params
        self.agg = agg

    @classmethod
    def create(cls, agg: "AggregateCuda", recv, width: int, height: int, vpls, n_vpl: int, params=None,
               stream=None):
        params = params or lightslice_params()
        h = ctypes.c_void_p()
        check(agg.lib.rzk_lightslice_create(agg.ctx.h, agg.h, _dptr(recv), width, height, _dptr(vpls), n_vpl,
                                            ctypes.byref(params), ctypes.byref(h), _stream_ptr(stream)),
              "rzk_lightslice_create")
        return cls(h, params, agg.lib, agg)

    @classmethod
    def from_host(cls, params, points: np.ndarray, pixels: np.ndarray):
        lib = load()
        pts = np.ascontiguousarray(points, np.float32)
        pix = np.ascontiguousarray(pixels, np.int32)
        h = ctypes.c_void_p()
        check(lib.rzk_lightslice_host_slice(ctypes.byref(params), pts.ctypes.data, pix.ctypes.data, len(pix),
                                            ctypes.byref(h)), "rzk_lightslice_host_slice")
        return cls(h, params, lib)

    def host_refine(self, R: np.ndarray, V: np.ndarray, vpls_used: np.ndarray, rep_recv: np.ndarray,
                    g_rep, g_weight, assign, mags):
        R = np.ascontiguousarray(R, np.float32)
        V = np.ascontiguousarray(V, np.uint8)
        vpls_used = np.ascontiguousarray(vpls_used)
        rep_recv = np.ascontiguousarray(rep_recv)
        g_rep = np.ascontiguousarray(g_rep, np.int32)
        g_weight = np.ascontiguousarray(g_weight, np.float32)
        assign = np.ascontiguousarray(assign, np.int32)
        mags = np.ascontiguousarray(mags, np.float32)
        check(self.lib.rzk_lightslice_host_refine(self.h, R.ctypes.data, V.ctypes.data, len(vpls_used),
                                                  vpls_used.ctypes.data, rep_recv.ctypes.data, len(g_rep),
                                                  g_rep.ctypes.data, g_weight.ctypes.data, assign.ctypes.data,
                                                  mags.ctypes.data), "rzk_lightslice_host_refine")

    def info(self):
        v = [I32() for _ in range(5)]
        ms = (ctypes.c_double * 8)()
        check(self.lib.rzk_lightslice_info(self.h, *[ctypes.byref(x) for x in v], ms), "rzk_lightslice_info")
        n_points, n_slices, n_vpl, n_global, n_sc = [x.value for x in v]
        return {"points": n_points, "slices": n_slices, "vpls_used": n_vpl, "global_clusters": n_global,
                "slice_clusters": n_sc, "ms": list(ms)}

    def slices(self):
        inf = self.info()
        ns, k = inf["slices"], self.params.num_neighbor_slices
        pp = np.zeros(inf["points"], np.int32)
        st, en, rp = (np.zeros(ns, np.int32) for _ in range(3))
        nb = np.zeros((ns, k), np.int32)
        check(self.lib.rzk_lightslice_slices(self.h, pp.ctypes.data, st.ctypes.data, en.ctypes.data, rp.ctypes.data,
                                             nb.ctypes.data), "rzk_lightslice_slices")
        return {"point_pixel": pp, "start": st, "end": en, "rep": rp, "neighbors": nb}

    def global_clusters(self):
        """The global clustering (rzk_lightslice_global): representatives, weights and each
        one-bounce column's cluster."""
        inf = self.info()
        rep = np.zeros(inf["global_clusters"], np.int32)
        w = np.zeros(inf["global_clusters"], np.float32)
        assign = np.zeros(inf["vpls_used"], np.int32)
        check(self.lib.rzk_lightslice_global(self.h, rep.ctypes.data, w.ctypes.data, assign.ctypes.data),
              "rzk_lightslice_global")
        return rep, w, assign

    def clusters(self):
        inf = self.info()
        ns, nc = inf["slices"], inf["slice_clusters"]
        cnt = np.zeros(ns, np.int32)
        rep, size = np.zeros(nc, np.int32), np.zeros(nc, np.int32)
        w, pdf = np.zeros(nc, np.float32), np.zeros(nc, np.float32)
        up = np.zeros(nc, np.uint8)
        wi, inc = np.zeros((nc, 3), np.float32), np.zeros((nc, 3), np.float32)
        check(self.lib.rzk_lightslice_clusters(self.h, cnt.ctypes.data, rep.ctypes.data, w.ctypes.data,
                                               up.ctypes.data, wi.ctypes.data, inc.ctypes.data, pdf.ctypes.data,
                                               size.ctypes.data, None), "rzk_lightslice_clusters")
        mem = np.zeros(int(size.sum()), np.int32)
        check(self.lib.rzk_lightslice_clusters(self.h, None, None, None, None, None, None, None, None,
                                               mem.ctypes.data), "rzk_lightslice_clusters")
        return {"count": cnt, "rep": rep, "weight": w, "upper": up, "wi": wi, "incident": inc, "pdf": pdf,
                "size": size, "members": mem}

    def maps(self):
        ns, res = self.info()["slices"], self.params.map_resolution
        m = np.zeros((ns, res, res), np.float32)
        v = np.zeros(ns, np.uint8)
        sm = np.zeros(ns, np.float32)
        rc = np.zeros((ns, res), np.float32)
        cc = np.zeros((ns, res, res), np.float32)
        check(self.lib.rzk_lightslice_maps(self.h, m.ctypes.data, v.ctypes.data, sm.ctypes.data, rc.ctypes.data,
                                           cc.ctypes.data), "rzk_lightslice_maps")
        return {"maps": m, "valid": v, "sum": sm, "row_cdf": rc, "col_cdf": cc}

    def matrix(self):
        torch = _torch()
        inf = self.info()
        ns, n1 = inf["slices"], inf["vpls_used"]
        R = torch.empty((n1, ns, 3), dtype=torch.float32, device="cuda")
        V = torch.empty((n1, ns), dtype=torch.uint8, device="cuda")
        idx = np.zeros(n1, np.int32)
        check(self.lib.rzk_lightslice_matrix(self.h, _dptr(R), _dptr(V), idx.ctypes.data, _stream_ptr()),
              "rzk_lightslice_matrix")
        return R, V, idx

    def host_find(self, points: np.ndarray) -> np.ndarray:
        pts = np.ascontiguousarray(points, np.float32)
        out = np.zeros(len(pts), np.int32)
        check(self.lib.rzk_lightslice_host_find(self.h, pts.ctypes.data, len(pts), out.ctypes.data),
              "rzk_lightslice_host_find")
        return out

    def find_slice(self, recv, n_recv, stream=None):
        torch = _torch()
        out = torch.empty(n_recv, dtype=torch.int32, device="cuda")
        check(self.lib.rzk_lightslice_find_slice(self.h, _dptr(recv), n_recv, _dptr(out), _stream_ptr(stream)),
              "rzk_lightslice_find_slice")
        return out

    def gather(self, recv, n_recv, clamp_mode, tau, scale=1.0, out=None, stream=None):
        torch = _torch()
        if out is None:
            out = torch.empty((n_recv, 3), dtype=torch.float32, device="cuda")
        check(self.lib.rzk_lightslice_gather(self.h, _dptr(recv), n_recv, clamp_mode, tau, scale, _dptr(out),
                                             _stream_ptr(stream)), "rzk_lightslice_gather")
        return out

    def guided_render(self, cam: "Camera", spp: int, max_bounce: int, rr_depth: int = 0, rr_prob: float = 1.0,
                      direct: bool = True, seed: int = 2013, paths: bool = False, out=None, stream=None,
                      sampler: str = "jensen", chain_samples: int = 0):
        """LightSlice-guided path tracing (rzk_guided_render) with the "jensen" or "metropolis"
        direction sampler: the per-pixel mean image, and the per-path radiance [W*H, spp, 3]
        when paths=True."""
        torch = _torch()
        n = cam.n_pixels
        if out is None:
            out = torch.empty((n, 3), dtype=torch.float32, device="cuda")
        pt = torch.empty((n, spp, 3), dtype=torch.float32, device="cuda") if paths else None
        mode = {"jensen": GUIDE_JENSEN, "metropolis": GUIDE_METROPOLIS}[sampler]
        prm = GuidedParamsC(spp, max_bounce, rr_depth, rr_prob, 1 if direct else 0, seed, mode, chain_samples)
        check(self.lib.rzk_guided_render(self.agg.ctx.h, self.agg.h, self.h, cam.rec.ctypes.data, ctypes.byref(prm),
                                         _dptr(out), _dptr(pt) if pt is not None else None, _stream_ptr(stream)),
              "rzk_guided_render")
        return (out, pt) if paths else out

    def density(self, slices, xy, stream=None):
        """The METROPOLIS sampler's density (rzk_lightslice_density): eval_incoming_radiance of
        slices[i] at the unit-square point xy[i]; a float32 tensor [n] on the device."""
        torch = _torch()
        sl = torch.as_tensor(np.ascontiguousarray(slices, np.int32), device="cuda")
        pts = torch.as_tensor(np.ascontiguousarray(xy, np.float32).reshape(-1, 2), device="cuda")
        out = torch.empty(sl.shape[0], dtype=torch.float32, device="cuda")
        check(self.lib.rzk_lightslice_density(self.h, _dptr(sl), _dptr(pts), int(sl.shape[0]), _dptr(out),
                                              _stream_ptr(stream)), "rzk_lightslice_density")
        return out

    def chains(self, seed: int, n_samples: int, stream=None):
        """The METROPOLIS chains (rzk_lightslice_chains): [n_slices, n_samples, 4] states after
        the warm-up as (unit-square x, y, density, 0), on the device."""
        torch = _torch()
        out = torch.empty((self.info()["slices"], n_samples, 4), dtype=torch.float32, device="cuda")
        check(self.lib.rzk_lightslice_chains(self.h, seed, n_samples, _dptr(out), _stream_ptr(stream)),
              "rzk_lightslice_chains")
        return out

    def close(self):
        if getattr(self, "h", None):
            self.lib.rzk_lightslice_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


REQ_GATHER, REQ_GUIDED = 0, 1


class CameraC(ctypes.Structure):
    """ctypes mirror of rzk_camera (80 bytes)."""
    _fields_ = [("eye", F32 * 3), ("u", F32 * 3), ("v", F32 * 3), ("n", F32 * 3), ("focal", F32),
                ("cop", F32 * 2), ("scale", F32 * 2), ("width", I32), ("height", I32), ("pad", I32)]


class RequestC(ctypes.Structure):
    """ctypes mirror of rzk_request."""
    _fields_ = [("kind", I32), ("scene", P), ("lightslice", P), ("camera", CameraC), ("d_vpls", P),
                ("n_vpl", I32), ("clamp_mode", I32), ("tau", F32), ("scale", F32), ("spp", I32),
                ("max_bounce", I32), ("rr_depth", I32), ("rr_prob", F32), ("seed", U32), ("d_rgb", P),
                ("sampler", I32)]


class ServerParamsC(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_int64), ("batching", I32), ("max_batch", I32)]


def camera_c(cam: "Camera") -> CameraC:
    c = CameraC()
    ctypes.memmove(ctypes.byref(c), cam.rec.ctypes.data, ctypes.sizeof(CameraC))
    return c


class Server:
    """The request loop (rzk_server_*): submit() returns a ticket or None when not admitted."""

    def __init__(self, device=0, batching=True, hbm_budget_bytes=0, max_batch=0):
        self.lib = load()
        prm = ServerParamsC(hbm_budget_bytes, 1 if batching else 0, max_batch)
        h = ctypes.c_void_p()
        check(self.lib.rzk_server_create(device, ctypes.byref(prm), ctypes.byref(h)), "rzk_server_create")
        self.h = h

    def submit(self, req: RequestC):
        t = ctypes.c_uint64()
        st = self.lib.rzk_server_submit(self.h, ctypes.byref(req), ctypes.byref(t))
        if st == ERR_BUSY:
            return None
        check(st, "rzk_server_submit")
        return t.value

    def poll(self, ticket):
        state, lat = I32(), ctypes.c_double()
        st = self.lib.rzk_server_poll(self.h, ticket, ctypes.byref(state), ctypes.byref(lat))
        return state.value, (lat.value if state.value >= 2 else None), st

    def wait(self, ticket, timeout_ms=-1):
        lat = ctypes.c_double()
        st = self.lib.rzk_server_wait(self.h, ticket, timeout_ms, ctypes.byref(lat))
        return st, lat.value

    def cancel(self, ticket):
        return self.lib.rzk_server_cancel(self.h, ticket)

    def stats(self):
        v = [ctypes.c_int64() for _ in range(6)]
        check(self.lib.rzk_server_stats(self.h, *[ctypes.byref(x) for x in v]), "rzk_server_stats")
        return dict(zip(["submitted", "rejected", "completed", "launches", "held_bytes", "budget_bytes"],
                        [x.value for x in v]))

    def timings(self):
        """Per completed request (completion order): kind, queue wait and run time in ms
        (rzk_server_timings)."""
        n = I32()
        check(self.lib.rzk_server_timings(self.h, None, None, None, 0, ctypes.byref(n)), "rzk_server_timings")
        k = n.value
        kind = np.zeros(k, np.int32)
        qm, rm = np.zeros(k, np.float64), np.zeros(k, np.float64)
        check(self.lib.rzk_server_timings(self.h, kind.ctypes.data, qm.ctypes.data, rm.ctypes.data, k,
                                          ctypes.byref(n)), "rzk_server_timings")
        return kind, qm, rm

    def close(self):
        if getattr(self, "h", None):
            self.lib.rzk_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
