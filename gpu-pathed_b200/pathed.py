"""ctypes binding of libpathed.so (the C ABI declared in include/pathed.h).

This is the call path tests and benchmarks use: every call goes through the C ABI into the
sm_100a kernels; there is no Python or CPU fallback. Importing this module loads the
in-tree libpathed.so and raises if it is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpathed.so")

PT_OK = 0
PT_ERR_ARG = -1
PT_ERR_STATE = -2
PT_ERR_CUDA = -3
PT_ERR_SCENE = -4
PT_ERR_DEVICE = -5

LAMBERTIAN, MIRROR, GLASS, MICROFACET = 0, 1, 2, 3
METAL = 5  # Beckmann microfacet with a Schlick Fresnel of RGB F0 = albedo (no reference counterpart)

# every symbol declared in include/pathed.h
EXPORTED = [
    "pt_create", "pt_destroy", "pt_last_error", "pt_set_device", "pt_load_config", "pt_load_config_level",
    "pt_load_arrays", "pt_scene_counts_get", "pt_export_scene", "pt_set_bvh", "pt_check_bvh", "pt_set_camera",
    "pt_set_material", "pt_set_max_depth", "pt_set_nee", "pt_set_seed", "pt_set_guiding", "pt_reset",
    "pt_set_launch", "pt_get_launch", "pt_render_async", "pt_poll", "pt_wait", "pt_get_spp", "pt_get_stats",
    "pt_readback", "pt_readback_pass", "pt_readback_rgba8", "pt_hit_test", "pt_trace_rays",
    "pt_trace_rays_device", "pt_occluded", "pt_version", "pt_set_profiling", "pt_get_profile",
    "pt_trace_rays_static", "pt_autotune", "pt_guide_reset", "pt_set_consistent_mis", "pt_guide_get_info",
    "pt_guide_get_params", "pt_guide_set_params", "pt_guide_forward", "pt_guide_gradients", "pt_set_guide_options",
    "pt_batch_generate", "pt_load_batch", "pt_batch_get_info", "pt_batch_readback", "pt_set_guide_inference",
    "pt_set_bvh_builder",
    "pt_set_renderer",
    "pt_load_request",
    "pt_load_reference_scene",
    "pt_read_exr",
    "pt_save_exr",
    "pt_write_exr",
    "pt_set_guide_fraction",
    "pt_set_bvh_nodes",
    "pt_readback_async",
    "pt_readback_wait",
    "pt_measure_l2_read",
    "pt_set_test_limits",
    "pt_set_watertight",
    "pt_set_guide_training",
]

MESH_OBJ, MESH_PLY = 0, 1  # PT_MESH_OBJ, PT_MESH_PLY
RENDERER_CUDA, RENDERER_OPTIX, RENDERER_NORMALS = 0, 1, 2  # PT_RENDERER_*

GUIDE_PARAMS = 16104

STATIC_MAX_RAYS = 65536  # PT_STATIC_MAX_RAYS

STAGES = ("camera", "extend", "sort", "shade", "shadow", "accumulate", "guide")


class PathedError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"pathed error {code}: {msg}")
        self.code = code


class SceneDesc(C.Structure):
    _fields_ = [
        ("num_triangles", C.c_int), ("tri_vertices", C.c_void_p), ("tri_normals", C.c_void_p),
        ("tri_materials", C.c_void_p), ("num_spheres", C.c_int), ("spheres", C.c_void_p),
        ("sphere_materials", C.c_void_p), ("num_materials", C.c_int), ("material_types", C.c_void_p),
        ("material_albedo", C.c_void_p), ("material_emit", C.c_void_p), ("material_ior", C.c_void_p),
        ("material_alpha", C.c_void_p), ("env_width", C.c_int), ("env_height", C.c_int),
        ("env_rgba", C.c_void_p),
    ]


class MeshFile(C.Structure):
    _fields_ = [("path", C.c_char_p), ("format", C.c_int), ("default_material", C.c_int)]


class SceneRequest(C.Structure):
    _fields_ = [
        ("num_files", C.c_int), ("files", C.c_void_p), ("num_materials", C.c_int), ("material_types", C.c_void_p),
        ("material_albedo", C.c_void_p), ("material_emit", C.c_void_p), ("material_ior", C.c_void_p),
        ("material_alpha", C.c_void_p), ("num_spheres", C.c_int), ("spheres", C.c_void_p),
        ("sphere_materials", C.c_void_p), ("env_exr", C.c_char_p), ("camera", C.c_void_p),
    ]


class SceneCounts(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "num_triangles", "num_spheres", "num_materials", "num_lights", "env_width", "env_height",
        "bvh_width", "bvh_nodes", "bvh_depth", "bvh_max_leaf", "res_x", "res_y", "default_spp",
        "default_depth", "default_nee")] + [("bvh_build_ms", C.c_double)]


class SceneExport(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "tri_vertices", "tri_normals", "tri_materials", "spheres", "sphere_materials", "material_types",
        "material_albedo", "material_emit", "material_ior", "material_alpha", "light_types",
        "light_indices", "env_rgba", "camera")]


class LaunchConfig(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "wave_paths", "block_extend", "block_shade", "block_shadow", "blocks_per_sm", "sort_materials",
        "use_graph", "sort_rays", "refill_idle", "speculate", "split_shade", "overlap_shadow", "shadow_order",
        "fuse_camera")]


class Stats(C.Structure):
    _fields_ = [("rays_camera", C.c_ulonglong), ("rays_extend", C.c_ulonglong), ("rays_shadow", C.c_ulonglong),
                ("last_frame_ms", C.c_float), ("last_frame_spp", C.c_int), ("total_spp", C.c_int),
                ("frames", C.c_int)]


class GuideInfo(C.Structure):
    _fields_ = [("enabled", C.c_int), ("mode", C.c_int), ("steps", C.c_int), ("params", C.c_int),
                ("samples", C.c_ulonglong), ("loss", C.c_float)]


class TuneResult(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("bvh_width", "sort_materials", "blocks_per_sm", "block", "wave_paths")] + \
               [("best_ms", C.c_float), ("default_ms", C.c_float), ("trials", C.c_int), ("from_cache", C.c_int),
                ("sort_rays", C.c_int), ("speculate", C.c_int), ("split_shade", C.c_int), ("max_leaf", C.c_int),
                ("bvh_builder", C.c_int), ("shadow_order", C.c_int), ("fuse_camera", C.c_int)]


class BatchScene(C.Structure):
    _fields_ = [("config", C.c_int), ("level", C.c_int), ("seed", C.c_ulonglong), ("width", C.c_int),
                ("height", C.c_int), ("spp", C.c_int), ("max_depth", C.c_int), ("guided", C.c_int),
                ("pad", C.c_int)]


class BatchInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("num_triangles", "num_spheres", "num_lights", "width", "height", "spp",
                                       "max_depth", "guided", "spp_accumulated")] + \
               [("first_pixel", C.c_longlong), ("first_path", C.c_longlong)]


BATCH_FIELDS = ("config", "level", "seed", "width", "height", "spp", "max_depth", "guided")


def read_exr(path) -> np.ndarray:
    """OpenEXR image as (height, width, 4) float32 RGBA, rows top first (LoadEXR's layout)."""
    w, h = C.c_int(), C.c_int()
    p = os.fsencode(path)
    rc = lib.pt_read_exr(p, C.byref(w), C.byref(h), None, 0)
    if rc != 0:
        raise PathedError(rc, lib.pt_last_error(None).decode())
    out = np.empty((h.value, w.value, 4), np.float32)
    rc = lib.pt_read_exr(p, C.byref(w), C.byref(h), out.ctypes.data, out.size)
    if rc != 0:
        raise PathedError(rc, lib.pt_last_error(None).decode())
    return out


def write_exr(path, rgb: np.ndarray):
    """(height, width, 3) radiances, row 0 = image bottom, written as the reference's
    Image::save writes them (HALF B, G, R, top row first)."""
    a = np.ascontiguousarray(rgb, np.float32)
    rc = lib.pt_write_exr(os.fsencode(path), a.shape[1], a.shape[0], a.ctypes.data)
    if rc != 0:
        raise PathedError(rc, lib.pt_last_error(None).decode())


def batch_generate(seed: int, n: int) -> list[dict]:
    """Configuration 4's seeded draw of n scenes (dicts of BATCH_FIELDS)."""
    arr = (BatchScene * n)()
    rc = lib.pt_batch_generate(C.c_ulonglong(seed), n, arr)
    if rc != 0:
        raise PathedError(rc, "pt_batch_generate failed")
    return [{k: getattr(a, k) for k in BATCH_FIELDS} for a in arr]


class Profile(C.Structure):
    _fields_ = [("stage_ms", C.c_float * 7), ("stage_launches", C.c_int * 7), ("extend_nodes", C.c_ulonglong),
                ("extend_prims", C.c_ulonglong), ("shadow_nodes", C.c_ulonglong), ("shadow_prims", C.c_ulonglong),
                ("bvh_width", C.c_int), ("node_bytes", C.c_int), ("prim_bytes", C.c_int), ("wave_paths", C.c_int),
                ("graph_captures", C.c_int)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libpathed.so not built ({LIB_PATH}); run gpu-pathed_b200/build.py")
    lib = C.CDLL(LIB_PATH)
    lib.pt_last_error.restype = C.c_char_p
    lib.pt_last_error.argtypes = [C.c_void_p]
    lib.pt_version.restype = C.c_char_p
    lib.pt_create.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_void_p)]
    lib.pt_destroy.argtypes = [C.c_void_p]
    lib.pt_load_config.argtypes = [C.c_void_p, C.c_int, C.c_uint64]
    lib.pt_load_config_level.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_int]
    lib.pt_set_seed.argtypes = [C.c_void_p, C.c_uint64]
    lib.pt_set_camera.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_int]
    lib.pt_set_material.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_float, C.c_float]
    lib.pt_poll.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_float)]
    lib.pt_wait.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
    lib.pt_readback.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    lib.pt_readback_async.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    lib.pt_readback_wait.argtypes = [C.c_void_p]
    lib.pt_readback_pass.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    lib.pt_readback_rgba8.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    lib.pt_batch_generate.argtypes = [C.c_ulonglong, C.c_int, C.c_void_p]
    lib.pt_load_batch.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    lib.pt_batch_get_info.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    lib.pt_batch_readback.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, C.c_int]
    lib.pt_trace_rays.argtypes = [C.c_void_p] + [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 5
    lib.pt_trace_rays_device.argtypes = [C.c_void_p] + [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 5
    lib.pt_trace_rays_static.argtypes = [C.c_void_p] + [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 5
    lib.pt_occluded.argtypes = [C.c_void_p] + [C.c_void_p] * 4 + [C.c_int, C.c_void_p]
    lib.pt_hit_test.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int)]
    lib.pt_load_request.argtypes = [C.c_void_p, C.c_void_p]
    lib.pt_load_reference_scene.argtypes = [C.c_void_p, C.c_int, C.c_char_p]
    lib.pt_save_exr.argtypes = [C.c_void_p, C.c_char_p]
    lib.pt_set_guide_fraction.argtypes = [C.c_void_p, C.c_float]
    lib.pt_write_exr.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p]
    lib.pt_read_exr.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p, C.c_size_t]
    for name in ("pt_set_device", "pt_set_max_depth", "pt_set_nee", "pt_set_guiding", "pt_render_async",
                 "pt_set_bvh_builder", "pt_set_renderer", "pt_set_bvh_nodes", "pt_set_watertight",
                 "pt_set_guide_training"):
        getattr(lib, name).argtypes = [C.c_void_p, C.c_int]
    lib.pt_set_bvh.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.pt_set_test_limits.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.pt_measure_l2_read.argtypes = [C.c_int, C.c_size_t, C.c_int, C.c_int, C.POINTER(C.c_double),
                                       C.POINTER(C.c_double)]
    lib.pt_set_profiling.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.pt_autotune.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_void_p]
    lib.pt_guide_reset.argtypes = [C.c_void_p]
    lib.pt_set_guide_options.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int]
    lib.pt_set_consistent_mis.argtypes = [C.c_void_p, C.c_int]
    lib.pt_guide_get_info.argtypes = [C.c_void_p, C.c_void_p]
    lib.pt_guide_get_params.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    lib.pt_guide_set_params.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    lib.pt_guide_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    lib.pt_guide_gradients.argtypes = [C.c_void_p] * 4 + [C.c_int, C.c_void_p]
    lib.pt_get_profile.argtypes = [C.c_void_p, C.c_void_p]
    for name in ("pt_reset", "pt_check_bvh"):
        getattr(lib, name).argtypes = [C.c_void_p]
    for name in ("pt_scene_counts_get", "pt_export_scene", "pt_set_launch", "pt_get_launch", "pt_get_stats",
                 "pt_load_arrays", "pt_get_spp"):
        getattr(lib, name).argtypes = [C.c_void_p, C.c_void_p]
    return lib


lib = _load()


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def _f32(a, n=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} floats, got {a.size}")
    return a


class Session:
    """One render session (RenderSession + its PathTracer) on the current CUDA device."""

    def __init__(self, width: int, height: int):
        h = C.c_void_p()
        rc = lib.pt_create(width, height, C.byref(h))
        if rc != PT_OK:
            raise PathedError(rc, lib.pt_last_error(None).decode())
        self._h = h
        self.width, self.height = width, height

    def close(self):
        if getattr(self, "_h", None):
            lib.pt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != PT_OK:
            raise PathedError(rc, lib.pt_last_error(self._h).decode())
        return rc

    def set_device(self, device: int):
        """Select the CUDA device (the library's runtime keeps its own current device)."""
        self._check(lib.pt_set_device(self._h, device))

    # ---- scene
    def load_config(self, config: int, seed: int = 0x5EED, level: int | None = None):
        if level is None:
            self._check(lib.pt_load_config(self._h, config, seed))
        else:
            self._check(lib.pt_load_config_level(self._h, config, seed, level))

    def load_arrays(self, tri_vertices=None, tri_normals=None, tri_materials=None, spheres=None,
                    sphere_materials=None, material_types=None, material_albedo=None, material_emit=None,
                    material_ior=None, material_alpha=None, env_rgba=None):
        keep = []

        def f(a, dt=np.float32):
            if a is None:
                return None, None
            arr = np.ascontiguousarray(np.asarray(a, dtype=dt))
            keep.append(arr)
            return arr, arr.ctypes.data

        tv, tvp = f(tri_vertices)
        _, tnp = f(tri_normals)
        _, tmp = f(tri_materials, np.int32)
        sp, spp = f(spheres)
        _, smp = f(sphere_materials, np.int32)
        mt, mtp = f(material_types, np.int32)
        d = SceneDesc()
        d.num_triangles = 0 if tv is None else tv.size // 9
        d.tri_vertices, d.tri_normals, d.tri_materials = tvp, tnp, tmp
        d.num_spheres = 0 if sp is None else sp.size // 4
        d.spheres, d.sphere_materials = spp, smp
        d.num_materials = 0 if mt is None else mt.size
        d.material_types = mtp
        d.material_albedo = f(material_albedo)[1]
        d.material_emit = f(material_emit)[1]
        d.material_ior = f(material_ior)[1]
        d.material_alpha = f(material_alpha)[1]
        if env_rgba is not None:
            e, ep = f(env_rgba)
            d.env_height, d.env_width = e.shape[0], e.shape[1]
            d.env_rgba = ep
        self._check(lib.pt_load_arrays(self._h, C.byref(d)))

    def load_request(self, files, material_types, camera, material_albedo=None, material_emit=None,
                     material_ior=None, material_alpha=None, spheres=None, sphere_materials=None, env_exr=None):
        """Scene files (SceneAdapter::ParseRequest): `files` is a list of (path, MESH_OBJ |
        MESH_PLY, default material id); camera = origin, target, up, vfov (radians), flip."""
        keep = []

        def f(a, dt=np.float32):
            if a is None:
                return None
            arr = np.ascontiguousarray(np.asarray(a, dtype=dt))
            keep.append(arr)
            return arr

        mf = (MeshFile * max(1, len(files)))()
        for m, (path, fmt, mat) in zip(mf, files):
            m.path, m.format, m.default_material = os.fsencode(path), int(fmt), int(mat)
        r = SceneRequest()
        r.num_files, r.files = len(files), C.cast(mf, C.c_void_p)
        mt = f(material_types, np.int32)
        r.num_materials, r.material_types = mt.size, mt.ctypes.data
        for name, a in (("material_albedo", material_albedo), ("material_emit", material_emit),
                        ("material_ior", material_ior), ("material_alpha", material_alpha)):
            arr = f(a)
            setattr(r, name, None if arr is None else arr.ctypes.data)
        if spheres is not None:
            sp, sm = f(spheres), f(sphere_materials, np.int32)
            r.num_spheres, r.spheres, r.sphere_materials = sp.size // 4, sp.ctypes.data, sm.ctypes.data
        r.env_exr = None if env_exr is None else os.fsencode(env_exr)
        cam = f(camera)
        if cam is None or cam.size != 11:
            raise ValueError("camera needs 11 floats")
        r.camera = cam.ctypes.data
        self._check(lib.pt_load_request(self._h, C.byref(r)))

    def save_exr(self, path):
        """The accumulated radiance as the reference's Image::save writes it (HALF B, G, R)."""
        self._check(lib.pt_save_exr(self._h, os.fsencode(path)))

    def load_reference_scene(self, index: int, scenes_dir: str):
        """The reference's built-in scene 0-3, read from its scenes/ directory."""
        self._check(lib.pt_load_reference_scene(self._h, int(index), os.fsencode(scenes_dir)))

    def counts(self) -> SceneCounts:
        c = SceneCounts()
        self._check(lib.pt_scene_counts_get(self._h, C.byref(c)))
        return c

    def export_scene(self) -> dict:
        c = self.counts()
        out = {
            "tri_vertices": np.zeros((c.num_triangles, 9), np.float32),
            "tri_normals": np.zeros((c.num_triangles, 9), np.float32),
            "tri_materials": np.zeros(c.num_triangles, np.int32),
            "spheres": np.zeros((c.num_spheres, 4), np.float32),
            "sphere_materials": np.zeros(c.num_spheres, np.int32),
            "material_types": np.zeros(c.num_materials, np.int32),
            "material_albedo": np.zeros((c.num_materials, 3), np.float32),
            "material_emit": np.zeros((c.num_materials, 3), np.float32),
            "material_ior": np.zeros(c.num_materials, np.float32),
            "material_alpha": np.zeros(c.num_materials, np.float32),
            "light_types": np.zeros(c.num_lights, np.int32),
            "light_indices": np.zeros(c.num_lights, np.int32),
            "env_rgba": np.zeros((c.env_height, c.env_width, 4), np.float32) if c.env_width else None,
            "camera": np.zeros(11, np.float32),
        }
        e = SceneExport()
        for k, v in out.items():
            setattr(e, k, _ptr(v) if v is not None and v.size else None)
        self._check(lib.pt_export_scene(self._h, C.byref(e)))
        out["counts"] = c
        return out

    def set_bvh(self, width: int, max_leaf: int = 4):
        self._check(lib.pt_set_bvh(self._h, width, max_leaf))

    def check_bvh(self) -> int:
        return lib.pt_check_bvh(self._h)

    # ---- model edits
    def set_camera(self, origin, target, up, vfov_radians: float, flip: bool = False):
        o, t, u = _f32(origin, 3), _f32(target, 3), _f32(up, 3)
        self._check(lib.pt_set_camera(self._h, o.ctypes.data, t.ctypes.data, u.ctypes.data, vfov_radians, int(flip)))

    def set_material(self, material_id, mtype, albedo=(0, 0, 0), emit=(0, 0, 0), ior=1.0, alpha=0.1):
        a, e = _f32(albedo, 3), _f32(emit, 3)
        self._check(lib.pt_set_material(self._h, material_id, mtype, a.ctypes.data, e.ctypes.data, ior, alpha))

    def set_max_depth(self, d: int):
        self._check(lib.pt_set_max_depth(self._h, d))

    def set_nee(self, on: bool):
        self._check(lib.pt_set_nee(self._h, int(bool(on))))

    def set_seed(self, seed: int):
        self._check(lib.pt_set_seed(self._h, seed))

    def set_guiding(self, on: bool):
        self._check(lib.pt_set_guiding(self._h, int(bool(on))))

    def reset(self):
        self._check(lib.pt_reset(self._h))

    def set_launch(self, **kw):
        c = LaunchConfig()
        for k, v in kw.items():
            setattr(c, k, int(v))
        self._check(lib.pt_set_launch(self._h, C.byref(c)))

    def get_launch(self) -> dict:
        c = LaunchConfig()
        self._check(lib.pt_get_launch(self._h, C.byref(c)))
        return {k: getattr(c, k) for k, _ in LaunchConfig._fields_}

    # ---- rendering
    def render_async(self, spp: int):
        self._check(lib.pt_render_async(self._h, spp))

    def poll(self):
        done, ms = C.c_int(), C.c_float()
        self._check(lib.pt_poll(self._h, C.byref(done), C.byref(ms)))
        return bool(done.value), ms.value

    def wait(self) -> float:
        ms = C.c_float()
        self._check(lib.pt_wait(self._h, C.byref(ms)))
        return ms.value

    def render(self, spp: int) -> float:
        self.render_async(spp)
        return self.wait()

    def spp(self) -> int:
        v = C.c_int()
        self._check(lib.pt_get_spp(self._h, C.byref(v)))
        return v.value

    def stats(self) -> dict:
        s = Stats()
        self._check(lib.pt_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    # ---- learned path guiding
    def guide_reset(self):
        self._check(lib.pt_guide_reset(self._h))

    def set_guide_options(self, steps_per_frame=-1, batch=0, lr=0.0, warmup_steps=-1):
        """steps_per_frame 0 selects the automatic schedule; -1 (and batch 0, lr 0, warmup
        -1) keep the current setting."""
        self._check(lib.pt_set_guide_options(self._h, steps_per_frame, batch, lr, warmup_steps))

    def set_consistent_mis(self, on: bool):
        self._check(lib.pt_set_consistent_mis(self._h, int(bool(on))))

    def guide_info(self) -> dict:
        g = GuideInfo()
        self._check(lib.pt_guide_get_info(self._h, C.byref(g)))
        return {k: getattr(g, k) for k, _ in GuideInfo._fields_}

    def set_guide_training(self, tc: bool):
        """Guide training on tcgen05 / tensor memory (True) or mma.sync (False)."""
        self._check(lib.pt_set_guide_training(self._h, int(bool(tc))))

    def set_guide_inference(self, tc: bool):
        """Guide inference on tcgen05 / tensor memory (True) or mma.sync (False)."""
        self._check(lib.pt_set_guide_inference(self._h, int(bool(tc))))

    def set_guide_fraction(self, fraction: float):
        """Probability of sampling the guide at a non-delta vertex (default 0.7)."""
        self._check(lib.pt_set_guide_fraction(self._h, float(fraction)))

    def guide_params(self) -> np.ndarray:
        out = np.empty(GUIDE_PARAMS, np.float32)
        self._check(lib.pt_guide_get_params(self._h, out.ctypes.data, out.size))
        return out

    def set_guide_params(self, p):
        p = _f32(p, GUIDE_PARAMS)
        self._check(lib.pt_guide_set_params(self._h, p.ctypes.data, p.size))

    def guide_forward(self, x) -> np.ndarray:
        x = _f32(x).reshape(-1, 80)
        raw = np.empty((x.shape[0], 40), np.float32)
        self._check(lib.pt_guide_forward(self._h, x.ctypes.data, x.shape[0], raw.ctypes.data))
        return raw

    def guide_gradients(self, x, wi, w) -> np.ndarray:
        x, wi, w = _f32(x).reshape(-1, 80), _f32(wi).reshape(-1, 3), _f32(w).reshape(-1)
        g = np.empty(GUIDE_PARAMS, np.float32)
        self._check(lib.pt_guide_gradients(self._h, x.ctypes.data, wi.ctypes.data, w.ctypes.data, x.shape[0],
                                           g.ctypes.data))
        return g

    def autotune(self, spp: int, cache_path: str | None = None) -> dict:
        r = TuneResult()
        self._check(lib.pt_autotune(self._h, spp, cache_path.encode() if cache_path else None, C.byref(r)))
        return {k: getattr(r, k) for k, _ in TuneResult._fields_}

    def set_profiling(self, stage_timing: bool = True, work_counters: bool = False):
        self._check(lib.pt_set_profiling(self._h, int(bool(stage_timing)), int(bool(work_counters))))

    def profile(self) -> dict:
        p = Profile()
        self._check(lib.pt_get_profile(self._h, C.byref(p)))
        d = {k: getattr(p, k) for k, _ in Profile._fields_ if k not in ("stage_ms", "stage_launches")}
        d["stage_ms"] = dict(zip(STAGES, list(p.stage_ms)))
        d["stage_launches"] = dict(zip(STAGES, list(p.stage_launches)))
        return d

    def readback(self, out: np.ndarray | None = None, pass_only: bool = False) -> np.ndarray:
        if out is None:
            out = np.empty((self.height, self.width, 3), np.float32)
        fn = lib.pt_readback_pass if pass_only else lib.pt_readback
        self._check(fn(self._h, out.ctypes.data, out.size))
        return out

    def readback_async(self, out: np.ndarray):
        """Start copying the running mean as of the last enqueued frame into `out` (float32
        H x W x 3, ideally page-locked); it overlaps the next frame. readback_wait() finishes it."""
        if out.dtype != np.float32 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a contiguous float32 array")
        self._check(lib.pt_readback_async(self._h, out.ctypes.data, out.size))
        self._pending_out = out  # keep the buffer alive until the copy is waited for

    def readback_wait(self) -> np.ndarray | None:
        self._check(lib.pt_readback_wait(self._h))
        out, self._pending_out = getattr(self, "_pending_out", None), None
        return out

    def set_bvh_builder(self, gpu):
        """Build the BVH on the host (SAH; False or 0) or on the GPU, collapsed to the wide
        format: True or 1 a linear BVH (Karras radix tree), 2 PLOC clustering."""
        self._check(lib.pt_set_bvh_builder(self._h, int(gpu)))

    def set_bvh_quantized(self, on: bool):
        """Traverse quantized wide nodes (widths 4 and 8) instead of float nodes."""
        self._check(lib.pt_set_bvh_nodes(self._h, int(bool(on))))

    def set_watertight(self, on: bool):
        """Watertight ray/triangle test (Woop, Benthin and Wald 2013) instead of the
        reference's Triangle::hit arithmetic (the default)."""
        self._check(lib.pt_set_watertight(self._h, int(bool(on))))

    def set_test_limits(self, stack_entries: int = 0, mma_polls: int = 0):
        """Test hook for the device-error paths: cap the traversal stack and the tensor-core
        inference waits (0: off); calls that hit a limit raise PathedError(PT_ERR_DEVICE)."""
        self._check(lib.pt_set_test_limits(self._h, int(stack_entries), int(mma_polls)))

    def set_renderer(self, kind: int):
        """RENDERER_CUDA (the path tracer) or RENDERER_NORMALS (the normals G-buffer: one
        pixel-centre ray per pixel and frame)."""
        self._check(lib.pt_set_renderer(self._h, int(kind)))

    # ---- batched frames (configuration 4)
    def load_batch(self, scenes: list[dict]):
        arr = (BatchScene * len(scenes))()
        for a, d in zip(arr, scenes):
            for k in BATCH_FIELDS:
                setattr(a, k, int(d.get(k, -1 if k == "level" else 0)))
        self._check(lib.pt_load_batch(self._h, arr, len(scenes)))

    def batch_info(self, scene: int) -> dict:
        b = BatchInfo()
        self._check(lib.pt_batch_get_info(self._h, scene, C.byref(b)))
        return {k: getattr(b, k) for k, _ in BatchInfo._fields_}

    def batch_readback(self, scene: int, pass_only: bool = False) -> np.ndarray:
        i = self.batch_info(scene)
        out = np.empty((i["height"], i["width"], 3), np.float32)
        self._check(lib.pt_batch_readback(self._h, scene, out.ctypes.data, out.size, int(pass_only)))
        return out

    def readback_rgba8(self) -> np.ndarray:
        out = np.empty((self.height, self.width, 4), np.uint8)
        self._check(lib.pt_readback_rgba8(self._h, out.ctypes.data, out.size))
        return out

    # ---- queries
    def hit_test(self, x: int, y: int) -> int:
        m = C.c_int()
        self._check(lib.pt_hit_test(self._h, x, y, C.byref(m)))
        return m.value

    def trace_rays(self, o, d, tmin, tmax, with_bary=False):
        o = _f32(o).reshape(-1, 3)
        d = _f32(d).reshape(-1, 3)
        n = o.shape[0]
        tmin = _f32(np.broadcast_to(np.asarray(tmin, np.float32), (n,)))
        tmax = _f32(np.broadcast_to(np.asarray(tmax, np.float32), (n,)))
        pt_ = np.empty(n, np.int32)
        pid = np.empty(n, np.int32)
        mid = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        bary = np.empty((n, 2), np.float32) if with_bary else None
        self._check(lib.pt_trace_rays(self._h, o.ctypes.data, d.ctypes.data, tmin.ctypes.data, tmax.ctypes.data,
                                      n, pt_.ctypes.data, pid.ctypes.data, mid.ctypes.data, t.ctypes.data,
                                      _ptr(bary)))
        res = {"prim_type": pt_, "prim_id": pid, "mat_id": mid, "t": t}
        if with_bary:
            res["bary"] = bary
        return res

    def occluded(self, o, d, tmin, tmax):
        o = _f32(o).reshape(-1, 3)
        d = _f32(d).reshape(-1, 3)
        n = o.shape[0]
        tmin = _f32(np.broadcast_to(np.asarray(tmin, np.float32), (n,)))
        tmax = _f32(np.broadcast_to(np.asarray(tmax, np.float32), (n,)))
        occ = np.empty(n, np.int32)
        self._check(lib.pt_occluded(self._h, o.ctypes.data, d.ctypes.data, tmin.ctypes.data, tmax.ctypes.data, n,
                                    occ.ctypes.data))
        return occ


def version() -> str:
    return lib.pt_version().decode()


def measure_l2_read(device: int = 0, nbytes: int = 32 << 20, reps: int = 64, trials: int = 5):
    """Read bandwidth (GB/s) of an L2-resident buffer of `nbytes` on `device`, and the best
    launch's ms (pt_measure_l2_read): the roofline denominator of traversal on scenes whose
    nodes and leaf entries fit in L2."""
    gbs, ms = C.c_double(), C.c_double()
    rc = lib.pt_measure_l2_read(int(device), int(nbytes), int(reps), int(trials), C.byref(gbs), C.byref(ms))
    if rc != 0:
        raise PathedError(rc, "pt_measure_l2_read failed")
    return gbs.value, ms.value
