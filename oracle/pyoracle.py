"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline leg as the checker.  The product package never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "ref_render")

f3 = C.c_float * 3


class Material(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("kd", f3), ("alpha", C.c_float), ("reserved", f3)]


class Light(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("position", f3), ("intensity", f3), ("left", f3), ("up", f3),
                ("normal", f3), ("area", C.c_float)]


class MediumS(C.Structure):
    _fields_ = [("enabled", C.c_uint32), ("sigma_a", f3), ("sigma_s", f3), ("g", C.c_float)]


class SceneS(C.Structure):
    _fields_ = [("vertices", C.POINTER(C.c_float)), ("num_vertices", C.c_uint32),
                ("triangles", C.POINTER(C.c_uint32)), ("num_triangles", C.c_uint32),
                ("triangle_material", C.POINTER(C.c_uint32)),
                ("materials", C.POINTER(Material)), ("num_materials", C.c_uint32),
                ("lights", C.POINTER(Light)), ("num_lights", C.c_uint32),
                ("medium", MediumS)]


class CameraS(C.Structure):
    _fields_ = [("position", f3), ("nv", f3), ("uv", f3), ("vv", f3), ("focal_distance", C.c_float)]


class FilmS(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("time_bins", C.c_uint32),
                ("exposure", C.c_float), ("offset", C.c_float), ("camera_unwarp", C.c_uint32),
                ("bounce_films", C.c_uint32), ("components", C.c_uint32)]


class IntegratorS(C.Structure):
    _fields_ = [("max_bounces", C.c_uint32), ("sqrt_spp", C.c_uint32), ("incoming_samples", C.c_uint32),
                ("flags", C.c_uint32), ("seed", C.c_uint64)]


class Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("prim_id", C.c_uint32), ("u", C.c_float), ("v", C.c_float)]


HIT_DTYPE = np.dtype([("t", np.float32), ("prim_id", np.uint32), ("u", np.float32), ("v", np.float32)])


def build(force=False):
    """Compile liboracle.so with the committed Makefile (gcc, -ffp-contract=off)."""
    if force or not os.path.exists(LIB_PATH) or \
            os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "tr_oracle.c")):
        subprocess.check_call(["make", "-s", "-C", HERE, "all"])
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        L.orc_create.restype = C.c_int
        L.orc_create.argtypes = [C.POINTER(SceneS), C.POINTER(CameraS), C.POINTER(FilmS),
                                 C.POINTER(IntegratorS), C.POINTER(C.c_void_p)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_bvh_info.argtypes = [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                   C.POINTER(C.c_uint32)]
        L.orc_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p,
                                C.c_void_p]
        L.orc_trace_moller.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
        L.orc_moller_terms.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32] + [C.c_void_p] * 4
        L.orc_render_ex.restype = C.c_int
        L.orc_render_ex.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                    C.c_uint32, C.c_int] + [C.c_void_p] * 10
        L.orc_render.restype = C.c_int
        L.orc_render.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                 C.c_uint32, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_path_records.restype = C.c_int
        L.orc_path_records.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32,
                                       C.c_void_p, C.c_void_p, C.c_int]
        L.orc_log.restype = C.c_float
        L.orc_log.argtypes = [C.c_float]
        L.orc_exp.restype = C.c_float
        L.orc_exp.argtypes = [C.c_float]
        L.orc_sincos2pi.argtypes = [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.orc_ggx_sample.restype = C.c_int
        L.orc_ggx_sample.argtypes = [C.c_void_p, C.c_float, C.c_void_p, C.c_void_p, C.c_float, C.c_float,
                                     C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_ggx_eval_cos.argtypes = [C.c_void_p, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_hg_eval.argtypes = [C.c_float, C.c_float]
        L.orc_hg_eval.restype = C.c_float
        L.orc_hg_sample_cos.argtypes = [C.c_float, C.c_float]
        L.orc_hg_sample_cos.restype = C.c_float
        L.orc_pcg32_first.restype = C.c_uint32
        L.orc_pcg32_first.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32]
        _lib = L
    return _lib


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class Oracle:
    """CPU restatement of the transient path tracer for one scene."""

    def __init__(self, scene):
        self.scene = scene
        v, t, m = scene.flatten()
        self._keep = [v, t, m]
        mats = (Material * len(scene.materials))()
        for i, mm in enumerate(scene.materials):
            mats[i].kind = mm.kind
            mats[i].kd = f3(*mm.kd)
            mats[i].alpha = mm.alpha
        lights = (Light * len(scene.lights))()
        for i, L in enumerate(scene.lights):
            lights[i].kind = L.kind
            lights[i].position = f3(*L.position)
            lights[i].intensity = f3(*L.intensity)
            lights[i].left = f3(*L.left)
            lights[i].up = f3(*L.up)
            lights[i].normal = f3(*L.normal)
            lights[i].area = L.area
        med = MediumS()
        if scene.medium is not None:
            med.enabled = 1
            med.sigma_a = f3(*scene.medium.sigma_a)
            med.sigma_s = f3(*scene.medium.sigma_s)
            med.g = scene.medium.g
        self._keep += [mats, lights]
        s = SceneS(_ptr(v, C.c_float), len(v), _ptr(t, C.c_uint32), len(t), _ptr(m, C.c_uint32),
                   mats, len(scene.materials), lights, len(scene.lights), med)
        pos, nv, uv, vv, fd = scene.camera.basis()
        cam = CameraS(f3(*pos), f3(*nv), f3(*uv), f3(*vv), float(fd))
        film = FilmS(scene.width, scene.height, scene.time_bins, scene.exposure, scene.offset,
                     int(getattr(scene, "camera_unwarp", 0)), int(getattr(scene, "bounce_films", 0)),
                     int(getattr(scene, "components", 0)))
        integ = IntegratorS(scene.max_bounces, scene.sqrt_spp, scene.incoming_samples, scene.flags, scene.seed)
        h = C.c_void_p()
        rc = lib().orc_create(C.byref(s), C.byref(cam), C.byref(film), C.byref(integ), C.byref(h))
        if rc != 0:
            raise ValueError("orc_create failed")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bvh_info(self):
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        lib().orc_bvh_info(self.h, C.byref(a), C.byref(b), C.byref(c))
        return {"interior_nodes": a.value, "leaves": b.value, "depth": c.value}

    def trace(self, rays, any_hit=False, counts=False):
        rays = np.ascontiguousarray(rays, np.float32)
        n = len(rays)
        out = np.zeros(n, HIT_DTYPE)
        nv = np.zeros(n, np.uint32) if counts else None
        nt = np.zeros(n, np.uint32) if counts else None
        lib().orc_trace(self.h, rays.ctypes.data, n, int(any_hit), out.ctypes.data,
                        nv.ctypes.data if counts else None, nt.ctypes.data if counts else None)
        return (out, nv, nt) if counts else out

    def trace_moller(self, rays):
        rays = np.ascontiguousarray(rays, np.float32)
        out = np.zeros(len(rays), HIT_DTYPE)
        lib().orc_trace_moller(self.h, rays.ctypes.data, len(rays), out.ctypes.data)
        return out

    def moller_terms(self, rays, ids):
        """Embree's Moeller-Trumbore terms of ray i against triangle ids[i]: dict of float32
        arrays T, absden, u, v (unnormalised; the distance is T / absden)."""
        rays = np.ascontiguousarray(rays, np.float32)
        ids = np.ascontiguousarray(ids, np.uint32)
        out = {k: np.zeros(len(rays), np.float32) for k in ("T", "absden", "u", "v")}
        lib().orc_moller_terms(self.h, rays.ctypes.data, ids.ctypes.data, len(rays),
                               *(out[k].ctypes.data for k in ("T", "absden", "u", "v")))
        return out

    def render(self, sample_begin=0, sample_count=None, window=None, nthreads=1,
               streak=True, steady=True, weight=True, bounces=False, components=False):
        """Adds the camera samples into fresh full-frame films.  With bounces=True (the scene's
        film has bounce_films = N > 0) also returns the per-bounce films "bstreak"
        [N][H][W][T][3], "bsteady" [N][H][W][3], "bweight" [N][H][W]; with components=True the
        per-pixel sums "depth" [H][W], "positions" and "normals" [H][W][3]."""
        sc = self.scene
        if sample_count is None:
            sample_count = sc.spp
        x0, y0, x1, y1 = window if window is not None else (0, 0, sc.width, sc.height)
        H, W, T = sc.height, sc.width, sc.time_bins
        NB = int(getattr(sc, "bounce_films", 0)) if bounces else 0
        st = np.zeros((H, W, T, 3), np.float64) if streak else None
        sd = np.zeros((H, W, 3), np.float64) if steady else None
        wt = np.zeros((H, W), np.float64) if weight else None
        bst = np.zeros((NB, H, W, T, 3), np.float64) if NB else None
        bsd = np.zeros((NB, H, W, 3), np.float64) if NB else None
        bwt = np.zeros((NB, H, W), np.float64) if NB else None
        cd = np.zeros((H, W), np.float64) if components else None
        cp = np.zeros((H, W, 3), np.float64) if components else None
        cn = np.zeros((H, W, 3), np.float64) if components else None
        stats = np.zeros(8, np.uint64)
        ptr = lambda a: a.ctypes.data if a is not None else None
        rc = lib().orc_render_ex(self.h, x0, y0, x1, y1, sample_begin, sample_count, nthreads,
                                 ptr(st), ptr(sd), ptr(wt), ptr(bst), ptr(bsd), ptr(bwt), ptr(cd), ptr(cp), ptr(cn),
                                 stats.ctypes.data)
        if rc != 0:
            raise ValueError("orc_render failed")
        out = {"streak": st, "steady": sd, "weight": wt,
               "stats": dict(zip(["paths", "closest_rays", "shadow_rays", "splats", "closest_nodes",
                                  "closest_tris", "shadow_nodes", "shadow_tris"], map(int, stats)))}
        if NB:
            out.update(bstreak=bst, bsteady=bsd, bweight=bwt)
        if components:
            out.update(depth=cd, positions=cp, normals=cn)
        return out

    def path_records(self, x, y, s, j=0, cap=256):
        bins = np.zeros(cap, np.uint32)
        rgb = np.zeros((cap, 3), np.float32)
        n = lib().orc_path_records(self.h, x, y, s, j, bins.ctypes.data, rgb.ctypes.data, cap)
        return bins[:n], rgb[:n]
