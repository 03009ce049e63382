"""ctypes binding of the C ABI declared in include/transient_b200.h.

The product path: every call goes to libtransient_b200.so (CUDA, sm_100a).  There is no CPU
fallback; importing this module fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libtransient_b200.so")

f3 = C.c_float * 3


class Material(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("kd", f3), ("alpha", C.c_float), ("reserved", f3)]


class Light(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("position", f3), ("intensity", f3), ("left", f3), ("up", f3),
                ("normal", f3), ("area", C.c_float)]


class Medium(C.Structure):
    _fields_ = [("enabled", C.c_uint32), ("sigma_a", f3), ("sigma_s", f3), ("g", C.c_float)]


class Scene(C.Structure):
    _fields_ = [("vertices", C.POINTER(C.c_float)), ("num_vertices", C.c_uint32),
                ("triangles", C.POINTER(C.c_uint32)), ("num_triangles", C.c_uint32),
                ("triangle_material", C.POINTER(C.c_uint32)),
                ("materials", C.POINTER(Material)), ("num_materials", C.c_uint32),
                ("lights", C.POINTER(Light)), ("num_lights", C.c_uint32),
                ("medium", Medium)]


class Camera(C.Structure):
    _fields_ = [("position", f3), ("nv", f3), ("uv", f3), ("vv", f3), ("focal_distance", C.c_float)]


class Film(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("time_bins", C.c_uint32),
                ("exposure", C.c_float), ("offset", C.c_float), ("camera_unwarp", C.c_uint32),
                ("bounce_films", C.c_uint32), ("components", C.c_uint32)]


class Integrator(C.Structure):
    _fields_ = [("max_bounces", C.c_uint32), ("sqrt_spp", C.c_uint32), ("incoming_samples", C.c_uint32),
                ("flags", C.c_uint32), ("seed", C.c_uint64)]


class Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("prim_id", C.c_uint32), ("u", C.c_float), ("v", C.c_float)]


class Stats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("camera_samples", C.c_uint64), ("closest_rays", C.c_uint64),
                ("shadow_rays", C.c_uint64), ("splats", C.c_uint64), ("render_ms", C.c_double),
                ("bvh_build_ms", C.c_double), ("bvh_nodes", C.c_uint32), ("bvh_depth", C.c_uint32),
                ("device_bytes", C.c_uint64), ("kernel_launches", C.c_uint64),
                ("raygen_ms", C.c_double), ("extend_ms", C.c_double), ("shade_ms", C.c_double),
                ("shadow_ms", C.c_double), ("splat_ms", C.c_double),
                ("extend_launches", C.c_uint64), ("shadow_launches", C.c_uint64),
                ("guide_ms", C.c_double), ("train_steps", C.c_uint64), ("train_loss", C.c_float),
                ("trace_ms", C.c_double)]


FILM_F64, FILM_F32, FILM_RGBE = 0, 1, 2     # tr_render_film delivery types


class BatchConfig(C.Structure):
    _fields_ = [("capacity", C.c_uint32), ("shade_block", C.c_uint32), ("splat_div", C.c_uint32),
                ("use_graph", C.c_uint32)]


TR_OK = 0
STATUS = {0: "TR_OK", 1: "TR_ERR_INVALID_ARGUMENT", 2: "TR_ERR_CUDA", 3: "TR_ERR_OUT_OF_MEMORY",
          4: "TR_ERR_NOT_SUPPORTED", 5: "TR_ERR_TIMEOUT", 6: "TR_ERR_NO_DEVICE", 7: "TR_ERR_IO"}

# every exported symbol of include/transient_b200.h with its prototype
PROTOTYPES = {
    "tr_create": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.POINTER(Film), C.POINTER(Integrator),
                            C.c_int, C.POINTER(C.c_void_p)]),
    "tr_render": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32]),
    "tr_render_region": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                   C.c_uint32]),
    "tr_clear_film": (C.c_int, [C.c_void_p]),
    "tr_get_film": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tr_release_cached_memory": (C.c_int, [C.c_int]),
    "tr_render_film": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tr_get_film_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tr_get_film_bounce": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tr_get_film_components": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tr_write_film": (C.c_int, [C.c_void_p, C.c_char_p]),
    "tr_trace_rays": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p]),
    "tr_trace_rays_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p]),
    "tr_render_region_noalloc": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                           C.c_uint64, C.c_uint32, C.c_void_p]),
    "tr_guide_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
    "tr_guide_set_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tr_guide_get_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tr_guide_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "tr_guide_train_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_float,
                                      C.POINTER(C.c_float), C.c_void_p]),
    "tr_guide_get_grads": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tr_guide_destroy": (C.c_int, [C.c_void_p]),
    "tr_guide_set_wait_limit": (C.c_int, [C.c_void_p, C.c_uint32]),
    "tr_set_guide": (C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_uint32]),
    "tr_set_guide_scope": (C.c_int, [C.c_void_p, C.c_uint32, C.c_float]),
    "tr_stats_get": (C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    "tr_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_uint32, C.POINTER(C.c_void_p)]),
    "tr_batch_set_config": (C.c_int, [C.c_void_p, C.POINTER(BatchConfig)]),
    "tr_batch_get_config": (C.c_int, [C.c_void_p, C.POINTER(BatchConfig)]),
    "tr_batch_render": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
    "tr_batch_autotune": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                    C.POINTER(BatchConfig), C.POINTER(C.c_uint32)]),
    "tr_batch_set_guide": (C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_uint32]),
    "tr_batch_stats": (C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    "tr_batch_destroy": (C.c_int, [C.c_void_p]),
    "tr_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tr_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "tr_destroy": (C.c_int, [C.c_void_p]),
    "tr_status_string": (C.c_char_p, [C.c_int]),
    "tr_last_error": (C.c_char_p, []),
    "tr_abi_version": (C.c_int, []),
}


class TransientError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


_lib = None


def lib():
    """Load libtransient_b200.so (raises if it was not built; there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with "
                              "`make -C jarabotransientrendering_b200/csrc` (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != TR_OK:
        msg = lib().tr_last_error()
        raise TransientError(status, msg.decode() if msg else "")
