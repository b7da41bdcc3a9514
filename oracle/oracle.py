"""ORACLE - test infrastructure, not product code.

ctypes wrappers of liboracle.so (the CPU restatement of the reference integrator, built from
oracle/oracle.cpp) and of _ref/libref_cpu.so (the reference's own sources compiled for the
host CPU by `make -C oracle ref`). Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_cpu.so")
# Where the reference tree lies: $PATHED_REFERENCE, else the path the last build() was
# given (recorded in _ref/REFERENCE_TREE), else None (tests that read it then skip).
_TREE_NOTE = os.path.join(HERE, "_ref", "REFERENCE_TREE")


def _reference_tree():
    t = os.environ.get("PATHED_REFERENCE")
    if not t and os.path.exists(_TREE_NOTE):
        with open(_TREE_NOTE) as f:
            t = f.read().strip()
    return t or None


REF_TREE = _reference_tree()


def build(ref_tree=None) -> None:
    """Compile liboracle.so and, when `ref_tree` names an existing reference tree, the
    reference's CPU and GPU builds from its sources (on a machine without it, the prebuilt
    _ref/ libraries are used as they are). The tree's path is recorded for the tests."""
    global REF_TREE
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if ref_tree and os.path.isdir(ref_tree):
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", "refbench", "refassets", f"REF={ref_tree}"],
                       check=True)
        os.makedirs(os.path.dirname(_TREE_NOTE), exist_ok=True)
        with open(_TREE_NOTE, "w") as f:
            f.write(os.path.abspath(ref_tree) + "\n")
        REF_TREE = os.path.abspath(ref_tree)


def _f(a):
    return np.ascontiguousarray(np.asarray(a, np.float32))


def _i(a):
    return np.ascontiguousarray(np.asarray(a, np.int32))


class _SceneLib:
    """Common scene handling of the two libraries (same create signature)."""

    prefix = ""

    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        p = self.prefix
        getattr(self.lib, p + "scene_create").restype = C.c_void_p
        getattr(self.lib, p + "scene_create").argtypes = (
            [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
            + [C.c_void_p] * 5 + [C.c_int, C.c_int, C.c_void_p])
        getattr(self.lib, p + "scene_destroy").argtypes = [C.c_void_p]

    def scene(self, sc: dict, accel: bool = False, watertight: bool = False):
        """Create a scene from an export dict (pathed.Session.export_scene layout). With
        `accel` (oracle only), queries run through the parity accelerator, which gives the
        linear scan's results on meshes the scan is too slow for. With `watertight` (oracle
        only), triangles take the watertight test of the CUDA path's opt-in mode."""
        keep = [
            _f(sc["tri_vertices"]), _f(sc["tri_normals"]), _i(sc["tri_materials"]), _f(sc["spheres"]),
            _i(sc["sphere_materials"]), _i(sc["material_types"]), _f(sc["material_albedo"]),
            _f(sc["material_emit"]), _f(sc["material_ior"]), _f(sc["material_alpha"]),
        ]
        env = sc.get("env_rgba")
        env = None if env is None or env.size == 0 else _f(env)
        ew, eh = (0, 0) if env is None else (env.shape[1], env.shape[0])
        h = getattr(self.lib, self.prefix + "scene_create")(
            keep[0].shape[0] if keep[0].ndim > 1 else keep[0].size // 9, keep[0].ctypes.data,
            keep[1].ctypes.data, keep[2].ctypes.data,
            keep[3].size // 4, keep[3].ctypes.data if keep[3].size else None,
            keep[4].ctypes.data if keep[4].size else None,
            keep[5].size, keep[5].ctypes.data, keep[6].ctypes.data, keep[7].ctypes.data, keep[8].ctypes.data,
            keep[9].ctypes.data, ew, eh, None if env is None else env.ctypes.data)
        if watertight:
            getattr(self.lib, self.prefix + "scene_watertight")(h, 1)
        if accel:
            getattr(self.lib, self.prefix + "scene_accel")(h)
        return _SceneHandle(self, h, keep + [env])


class _SceneHandle:
    def __init__(self, owner, h, keep):
        self.owner, self.h, self._keep = owner, h, keep

    def __del__(self):
        try:
            getattr(self.owner.lib, self.owner.prefix + "scene_destroy")(self.h)
        except Exception:
            pass


class Oracle(_SceneLib):
    prefix = "oracle_"

    def __init__(self, path=ORACLE_LIB):
        super().__init__(path)
        L = self.lib
        L.oracle_scene_accel.argtypes = [C.c_void_p]
        L.oracle_scene_watertight.argtypes = [C.c_void_p, C.c_int]
        L.oracle_trace.argtypes = [C.c_void_p] + [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 4 + [C.c_int]
        L.oracle_render.argtypes = ([C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                     C.c_int, C.c_uint64, C.c_uint64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_int, C.c_int])
        L.oracle_bsdf_sample.argtypes = [C.c_int, C.c_void_p, C.c_float, C.c_float, C.c_void_p, C.c_float,
                                         C.c_float, C.c_void_p]
        L.oracle_bsdf_eval.argtypes = [C.c_int, C.c_void_p, C.c_float, C.c_float, C.c_void_p, C.c_void_p,
                                       C.c_void_p]
        L.oracle_light_sample.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_void_p]
        L.oracle_camera_ray.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                        C.c_void_p]
        L.oracle_normals.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int]
        L.oracle_dist1d.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p]
        L.oracle_dist2d.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p]
        L.oracle_phitheta_pdf.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                          C.c_void_p, C.c_int, C.c_void_p]
        L.oracle_env_sample.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_void_p]
        L.oracle_rng.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_int, C.c_void_p]
        L.oracle_num_lights.argtypes = [C.c_void_p]
        L.oracle_guide_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.oracle_guide_grad.argtypes = [C.c_void_p] * 4 + [C.c_int, C.c_int, C.c_void_p]
        L.oracle_guide_grad.restype = C.c_double
        L.oracle_guide_loss_exact.argtypes = [C.c_void_p] * 4 + [C.c_int]
        L.oracle_guide_loss_exact.restype = C.c_double

    def guide_forward(self, params, x, quant=True):
        params, x = _f(params), _f(x).reshape(-1, 80)
        out = np.zeros((x.shape[0], 40), np.float64)
        self.lib.oracle_guide_forward(params.ctypes.data, x.ctypes.data, x.shape[0], int(quant), out.ctypes.data)
        return out

    def guide_grad(self, params, x, wi, w, quant=False):
        params, x, wi, w = _f(params), _f(x).reshape(-1, 80), _f(wi).reshape(-1, 3), _f(w)
        g = np.zeros(params.size, np.float64)
        loss = self.lib.oracle_guide_grad(params.ctypes.data, x.ctypes.data, wi.ctypes.data, w.ctypes.data,
                                          x.shape[0], int(quant), g.ctypes.data)
        return loss, g

    def guide_loss_exact(self, params64, x, wi, w):
        p = np.ascontiguousarray(np.asarray(params64, np.float64))
        x, wi, w = _f(x).reshape(-1, 80), _f(wi).reshape(-1, 3), _f(w)
        return self.lib.oracle_guide_loss_exact(p.ctypes.data, x.ctypes.data, wi.ctypes.data, w.ctypes.data,
                                                x.shape[0])

    def trace(self, scene, o, d, tmin, tmax, threads=0):
        o, d = _f(o).reshape(-1, 3), _f(d).reshape(-1, 3)
        n = o.shape[0]
        tmin = _f(np.broadcast_to(np.asarray(tmin, np.float32), (n,)))
        tmax = _f(np.broadcast_to(np.asarray(tmax, np.float32), (n,)))
        out = {"prim_type": np.empty(n, np.int32), "prim_id": np.empty(n, np.int32),
               "mat_id": np.empty(n, np.int32), "t": np.empty(n, np.float32)}
        self.lib.oracle_trace(scene.h, o.ctypes.data, d.ctypes.data, tmin.ctypes.data, tmax.ctypes.data, n,
                              out["prim_type"].ctypes.data, out["prim_id"].ctypes.data, out["mat_id"].ctypes.data,
                              out["t"].ctypes.data, threads)
        return out

    def render(self, scene, camera, width, height, pixels, spp, max_depth, nee=True, seed=0x5EED, sample_base=0,
               trace_once=True, threads=0, consistent_mis=False):
        pixels = _i(pixels)
        n = pixels.size
        mean = np.zeros((n, 3), np.float64)
        var = np.zeros((n, 3), np.float64)
        counts = np.zeros(3, np.uint64)
        cam = _f(camera)
        self.lib.oracle_render(scene.h, cam.ctypes.data, width, height, pixels.ctypes.data, n, spp, max_depth,
                               int(bool(nee)), seed, sample_base, int(bool(trace_once)), mean.ctypes.data,
                               var.ctypes.data, counts.ctypes.data, threads, int(bool(consistent_mis)))
        return mean, var, counts

    def normals(self, scene, camera, width, height, threads=0):
        """normals G-buffer image, (height, width, 3), row 0 = camera row 0"""
        out = np.empty((height, width, 3), np.float32)
        cam = _f(camera)
        self.lib.oracle_normals(scene.h, cam.ctypes.data, width, height, out.ctypes.data, threads)
        return out

    def rng(self, seed, sample, pixel, n):
        out = np.empty(n, np.float32)
        self.lib.oracle_rng(seed, sample, pixel, n, out.ctypes.data)
        return out


class RefCPU(_SceneLib):
    """The reference's own routines compiled for the host CPU."""

    prefix = "ref_"

    def __init__(self, path=REF_LIB):
        super().__init__(path)
        L = self.lib
        L.ref_trace.argtypes = [C.c_void_p] + [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 4
        L.ref_bsdf_sample.argtypes = [C.c_int, C.c_void_p, C.c_float, C.c_float, C.c_void_p, C.c_float, C.c_float,
                                      C.c_void_p]
        L.ref_bsdf_eval.argtypes = [C.c_int, C.c_void_p, C.c_float, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_light_sample.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_void_p]
        L.ref_camera_ray.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                     C.c_void_p]
        L.ref_dist1d.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p]
        L.ref_dist2d.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p]
        L.ref_phitheta_pdf.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                       C.c_int, C.c_void_p]
        L.ref_env_sample.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_void_p]
        L.ref_normals.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]

    def normals(self, scene, camera, width, height):
        out = np.empty((height, width, 3), np.float32)
        cam = _f(camera)
        self.lib.ref_normals(scene.h, cam.ctypes.data, width, height, out.ctypes.data)
        return out

    def trace(self, scene, o, d, tmin, tmax):
        o, d = _f(o).reshape(-1, 3), _f(d).reshape(-1, 3)
        n = o.shape[0]
        tmin = _f(np.broadcast_to(np.asarray(tmin, np.float32), (n,)))
        tmax = _f(np.broadcast_to(np.asarray(tmax, np.float32), (n,)))
        out = {"prim_type": np.empty(n, np.int32), "prim_id": np.empty(n, np.int32),
               "mat_id": np.empty(n, np.int32), "t": np.empty(n, np.float32)}
        self.lib.ref_trace(scene.h, o.ctypes.data, d.ctypes.data, tmin.ctypes.data, tmax.ctypes.data, n,
                           out["prim_type"].ctypes.data, out["prim_id"].ctypes.data, out["mat_id"].ctypes.data,
                           out["t"].ctypes.data)
        return out


REF_ASSETS_LIB = os.path.join(HERE, "_ref", "libref_assets.so")


class RefAssets:
    """The reference's OBJ/MTL/PLY parsers and its vendored LoadEXR, compiled for the host."""

    def __init__(self, path=REF_ASSETS_LIB):
        self.lib = L = C.CDLL(path)
        L.ref_mesh_parse.restype = C.c_void_p
        L.ref_mesh_parse.argtypes = [C.c_char_p, C.c_int]
        for name in ("ref_mesh_faces", "ref_mesh_mtls"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.ref_mesh_copy.argtypes = [C.c_void_p] * 5
        L.ref_mesh_free.argtypes = [C.c_void_p]
        L.ref_exr_load.restype = C.c_void_p
        L.ref_exr_load.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.ref_exr_free.argtypes = [C.c_void_p]
        L.ref_image_save.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_char_p]
        L.ref_exr_save_piz.argtypes = [C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_int, C.c_void_p, C.c_char_p]

    def exr_save_piz(self, path, planes, names=b"BGRA"[:3], half=False):
        """tinyexr's SaveEXRImageToFile with PIZ compression of (channels, height, width)
        FP32 planes, stored as HALF or FLOAT"""
        a = np.ascontiguousarray(planes, np.float32)
        code = self.lib.ref_exr_save_piz(a.shape[2], a.shape[1], a.shape[0], names, 1 if half else 2, a.ctypes.data,
                                         os.fsencode(path))
        if code != 0:
            raise RuntimeError(f"SaveEXRImageToFile failed with {code}")

    def image_save(self, path, rgb):
        """Image::save of (height, width, 3) radiances, row 0 = image bottom"""
        a = np.ascontiguousarray(rgb, np.float32)
        self.lib.ref_image_save(a.shape[1], a.shape[0], a.ctypes.data, os.fsencode(path))

    def mesh(self, path, ply=False) -> dict:
        """faces as p (n, 9), n (n, 9), per-face MTL index, MTL table (m, 6: Kd, Ke)"""
        h = self.lib.ref_mesh_parse(os.fsencode(path), int(ply))
        try:
            nf, nm = self.lib.ref_mesh_faces(h), self.lib.ref_mesh_mtls(h)
            out = {"p": np.empty((nf, 9), np.float32), "n": np.empty((nf, 9), np.float32),
                   "mtl": np.empty(nf, np.int32), "mtls": np.empty((nm, 6), np.float32)}
            self.lib.ref_mesh_copy(h, out["p"].ctypes.data, out["n"].ctypes.data, out["mtl"].ctypes.data,
                                   out["mtls"].ctypes.data)
            return out
        finally:
            self.lib.ref_mesh_free(h)

    def exr(self, path) -> np.ndarray:
        w, h, code = C.c_int(), C.c_int(), C.c_int()
        p = self.lib.ref_exr_load(os.fsencode(path), C.byref(w), C.byref(h), C.byref(code))
        if not p:
            raise RuntimeError(f"LoadEXR failed with {code.value}")
        try:
            return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_float)), (h.value, w.value, 4)).copy()
        finally:
            self.lib.ref_exr_free(p)


REFBENCH_LIB = os.path.join(HERE, "_ref", "librefbench.so")
REFBENCH_NOFMA_LIB = os.path.join(HERE, "_ref", "librefbench_nofma.so")


class RefBench:
    """The reference's own CUDA integrator (renderKernel + updateFramebuffer, World::hit),
    built from the reference sources by `make -C oracle refbench`. GPU only."""

    def __init__(self, nofma: bool = False):
        path = REFBENCH_NOFMA_LIB if nofma else REFBENCH_LIB
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = self.lib = C.CDLL(path)
        L.refbench_create.restype = C.c_void_p
        L.refbench_create.argtypes = ([C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                       C.c_int] + [C.c_void_p] * 5 + [C.c_int, C.c_int, C.c_void_p])
        L.refbench_init.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.refbench_render.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float)]
        L.refbench_readback.argtypes = [C.c_void_p, C.c_void_p]
        L.refbench_trace.argtypes = [C.c_void_p] + [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 4
        L.refbench_destroy.argtypes = [C.c_void_p]
        self.h = None

    def load(self, sc: dict, width: int, height: int):
        # the reference has no metallic Beckmann (type 5): it renders those materials as its own
        # Microfacet (type 3, dielectric Fresnel of eta 1.5), the closest material it has
        types = np.where(_i(sc["material_types"]) == 5, 3, _i(sc["material_types"])).astype(np.int32)
        keep = [_f(sc["tri_vertices"]), _f(sc["tri_normals"]), _i(sc["tri_materials"]), _f(sc["spheres"]),
                _i(sc["sphere_materials"]), types, _f(sc["material_albedo"]),
                _f(sc["material_emit"]), _f(sc["material_ior"]), _f(sc["material_alpha"])]
        env = sc.get("env_rgba")
        env = None if env is None or env.size == 0 else _f(env)
        ew, eh = (0, 0) if env is None else (env.shape[1], env.shape[0])
        self.h = self.lib.refbench_create(
            keep[0].size // 9, keep[0].ctypes.data, keep[1].ctypes.data, keep[2].ctypes.data, keep[3].size // 4,
            keep[3].ctypes.data if keep[3].size else None, keep[4].ctypes.data if keep[4].size else None,
            keep[5].size, keep[5].ctypes.data, keep[6].ctypes.data, keep[7].ctypes.data, keep[8].ctypes.data,
            keep[9].ctypes.data, ew, eh, None if env is None else env.ctypes.data)
        if not self.h:
            raise RuntimeError("refbench_create failed")
        cam = _f(sc["camera"])
        self.w, self.hgt = width, height
        if self.lib.refbench_init(self.h, cam.ctypes.data, width, height) != 0:
            raise RuntimeError("refbench_init failed")

    def render(self, spp, max_depth, nee=True) -> float:
        ms = C.c_float()
        if self.lib.refbench_render(self.h, spp, max_depth, int(bool(nee)), C.byref(ms)) != 0:
            raise RuntimeError("refbench_render failed")
        return ms.value

    def readback(self):
        out = np.empty((self.hgt, self.w, 3), np.float32)
        if self.lib.refbench_readback(self.h, out.ctypes.data) != 0:
            raise RuntimeError("refbench_readback failed")
        return out

    def trace(self, o, d, tmin, tmax):
        o, d = _f(o).reshape(-1, 3), _f(d).reshape(-1, 3)
        n = o.shape[0]
        tmin = _f(np.broadcast_to(np.asarray(tmin, np.float32), (n,)))
        tmax = _f(np.broadcast_to(np.asarray(tmax, np.float32), (n,)))
        out = {"prim_type": np.empty(n, np.int32), "prim_id": np.empty(n, np.int32),
               "mat_id": np.empty(n, np.int32), "t": np.empty(n, np.float32)}
        if self.lib.refbench_trace(self.h, o.ctypes.data, d.ctypes.data, tmin.ctypes.data, tmax.ctypes.data, n,
                                   out["prim_type"].ctypes.data, out["prim_id"].ctypes.data,
                                   out["mat_id"].ctypes.data, out["t"].ctypes.data) != 0:
            raise RuntimeError("refbench_trace failed")
        return out

    def close(self):
        if self.h:
            self.lib.refbench_destroy(self.h)
            self.h = None


def call_pair(fn_o, fn_r, *args, nout):
    """Run the same unit routine in both libraries; returns (oracle_out, reference_out)."""
    a = np.zeros(nout, np.float32)
    b = np.zeros(nout, np.float32)
    fn_o(*args, a.ctypes.data)
    fn_r(*args, b.ctypes.data)
    return a, b


def dist1d(lib, values, xis):
    """1-D distribution pmf/total/sample of either library ('oracle_' or 'ref_' prefix)."""
    v, x = _f(values), _f(xis)
    pmf = np.zeros(v.size, np.float32)
    total = np.zeros(1, np.float32)
    idx = np.zeros(x.size, np.int32)
    spmf = np.zeros(x.size, np.float32)
    fn = getattr(lib.lib, lib.prefix + "dist1d")
    fn(v.ctypes.data, v.size, x.ctypes.data, x.size, pmf.ctypes.data, total.ctypes.data, idx.ctypes.data,
       spmf.ctypes.data)
    return pmf, float(total[0]), idx, spmf


def dist2d(lib, values, w, h, xis):
    v, x = _f(values), _f(xis).reshape(-1, 2)
    pmf = np.zeros(w * h, np.float32)
    sx = np.zeros(x.shape[0], np.int32)
    sy = np.zeros(x.shape[0], np.int32)
    spmf = np.zeros(x.shape[0], np.float32)
    fn = getattr(lib.lib, lib.prefix + "dist2d")
    fn(v.ctypes.data, w, h, x.ctypes.data, x.shape[0], pmf.ctypes.data, sx.ctypes.data, sy.ctypes.data,
       spmf.ctypes.data)
    return pmf.reshape(h, w), sx, sy, spmf


def phitheta_pdf(lib, values, w, h, canon, dirs):
    v = _f(values)
    c = _f(canon).reshape(-1, 2)
    d = _f(dirs).reshape(-1, 3)
    pc = np.zeros(c.shape[0], np.float32)
    pd = np.zeros(d.shape[0], np.float32)
    fn = getattr(lib.lib, lib.prefix + "phitheta_pdf")
    fn(v.ctypes.data, w, h, c.ctypes.data, c.shape[0], pc.ctypes.data, d.ctypes.data, d.shape[0], pd.ctypes.data)
    return pc, pd
