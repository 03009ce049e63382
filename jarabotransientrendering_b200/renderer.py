"""Host-side API of the B200 transient path tracer.

Two layers over the C ABI (include/transient_b200.h):

* :class:`Context` - one device-resident scene + streak film (``tr_create`` ... ``tr_destroy``);
* the reference-shaped classes (``World``, ``Lambertian``, ``PointLightSource``,
  ``RectangularAreaLightSource``, ``HomogeneousMedium``, ``HenyeyGreenstein``,
  ``PinholeCamera``, ``StreakCameraFilm``, ``StratifiedSampler``,
  ``BidirectionalPathTracing``, ``TransientRenderer``) with the names, argument meaning and
  error behaviour of the reference renderer's classes, so that a scene set up the way
  ``src/bunnykiller.cpp:main`` sets it up renders on the GPU with
  ``TransientRenderer().render(name, world, integrator, camera, film, sampler)``
  (``src/Renderer/TransientRenderer.h:76-201``).
"""
from __future__ import annotations

import ctypes as C
import math
import os
from typing import List, Optional

import numpy as np

from . import _abi
from . import scenes as S

HIT_DTYPE = np.dtype([("t", np.float32), ("prim_id", np.uint32), ("u", np.float32), ("v", np.float32)])
INVALID_ID = 0xFFFFFFFF


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class Context:
    """A scene uploaded to one GPU with its BVH and FP64 streak film (``tr_create``)."""

    def __init__(self, scene: S.Scene, device: int = 0, arrays=None):
        """``arrays``: optional pre-flattened (vertices f32 [nv,3], triangles u32 [nt,3],
        triangle materials u32 [nt]) host arrays, e.g. in pinned memory."""
        L = _abi.lib()
        self.scene = scene
        v, t, m = arrays if arrays is not None else scene.flatten()
        self._keep = [v, t, m]
        mats = (_abi.Material * len(scene.materials))()
        for i, mm in enumerate(scene.materials):
            mats[i].kind = mm.kind
            mats[i].kd = _abi.f3(*mm.kd)
            mats[i].alpha = mm.alpha
        lights = (_abi.Light * max(1, len(scene.lights)))()
        for i, Lt in enumerate(scene.lights):
            lights[i].kind = Lt.kind
            lights[i].position = _abi.f3(*Lt.position)
            lights[i].intensity = _abi.f3(*Lt.intensity)
            lights[i].left = _abi.f3(*Lt.left)
            lights[i].up = _abi.f3(*Lt.up)
            lights[i].normal = _abi.f3(*Lt.normal)
            lights[i].area = Lt.area
        med = _abi.Medium()
        if scene.medium is not None:
            med.enabled = 1
            med.sigma_a = _abi.f3(*scene.medium.sigma_a)
            med.sigma_s = _abi.f3(*scene.medium.sigma_s)
            med.g = scene.medium.g
        self._keep += [mats, lights]
        sc = _abi.Scene(_ptr(v, C.c_float), len(v), _ptr(t, C.c_uint32), len(t), _ptr(m, C.c_uint32),
                        mats, len(scene.materials), lights, len(scene.lights), med)
        pos, nv, uv, vv, fd = scene.camera.basis()
        cam = _abi.Camera(_abi.f3(*pos), _abi.f3(*nv), _abi.f3(*uv), _abi.f3(*vv), float(fd))
        film = _abi.Film(scene.width, scene.height, scene.time_bins, scene.exposure, scene.offset,
                         int(scene.camera_unwarp), int(scene.bounce_films), int(scene.components))
        integ = _abi.Integrator(scene.max_bounces, scene.sqrt_spp, scene.incoming_samples, scene.flags, scene.seed)
        h = C.c_void_p()
        _abi.check(L.tr_create(C.byref(sc), C.byref(cam), C.byref(film), C.byref(integ), device, C.byref(h)))
        self.h = h
        self.device = device

    # -- rendering ------------------------------------------------------------------------
    def render(self, sample_begin: int = 0, sample_count: Optional[int] = None, window=None):
        """Adds camera samples [sample_begin, sample_begin+sample_count) of every pixel (or of
        the pixel window (x0, y0, x1, y1)) to the film."""
        if sample_count is None:
            sample_count = self.scene.spp
        if window is None:
            _abi.check(_abi.lib().tr_render(self.h, sample_begin, sample_count))
        else:
            x0, y0, x1, y1 = window
            _abi.check(_abi.lib().tr_render_region(self.h, x0, y0, x1, y1, sample_begin, sample_count))
        return self

    def clear(self):
        _abi.check(_abi.lib().tr_clear_film(self.h))

    def film(self, streak=True, steady=True, weight=True):
        sc = self.scene
        H, W, T = sc.height, sc.width, sc.time_bins
        st = np.empty((H, W, T, 3), np.float64) if streak else None
        sd = np.empty((H, W, 3), np.float64) if steady else None
        wt = np.empty((H, W), np.float64) if weight else None
        _abi.check(_abi.lib().tr_get_film(self.h, st.ctypes.data if st is not None else None,
                                          sd.ctypes.data if sd is not None else None,
                                          wt.ctypes.data if wt is not None else None))
        return {"streak": st, "steady": sd, "weight": wt}

    def bounce_film(self, bounce, streak=True, steady=True, weight=True):
        """Per-bounce film ``bounce`` (scenes with bounce_films > 0), as ``film``."""
        sc = self.scene
        H, W, T = sc.height, sc.width, sc.time_bins
        st = np.empty((H, W, T, 3), np.float64) if streak else None
        sd = np.empty((H, W, 3), np.float64) if steady else None
        wt = np.empty((H, W), np.float64) if weight else None
        _abi.check(_abi.lib().tr_get_film_bounce(self.h, bounce, st.ctypes.data if st is not None else None,
                                                 sd.ctypes.data if sd is not None else None,
                                                 wt.ctypes.data if wt is not None else None))
        return {"streak": st, "steady": sd, "weight": wt}

    def components(self):
        """Per-pixel sums of the enabled film components: {"depth": [H][W], "positions",
        "normals": [H][W][3]} (None for a component the film does not have)."""
        sc = self.scene
        H, W = sc.height, sc.width
        c = sc.components
        d = np.empty((H, W), np.float64) if c & S.COMP_DEPTH else None
        p = np.empty((H, W, 3), np.float64) if c & S.COMP_POSITIONS else None
        n = np.empty((H, W, 3), np.float64) if c & S.COMP_NORMALS else None
        ptr = lambda a: a.ctypes.data if a is not None else None
        _abi.check(_abi.lib().tr_get_film_components(self.h, ptr(d), ptr(p), ptr(n)))
        return {"depth": d, "positions": p, "normals": n}

    def film_into(self, streak=None, steady=None, weight=None):
        """tr_get_film into caller-provided (e.g. pinned) float64 host arrays."""
        _abi.check(_abi.lib().tr_get_film(self.h, streak.ctypes.data if streak is not None else None,
                                          steady.ctypes.data if steady is not None else None,
                                          weight.ctypes.data if weight is not None else None))

    def render_film(self, sample_begin, sample_count, streak=None, steady=None, weight=None):
        """tr_render_film: render and stream the film into caller-provided host arrays (pinned
        arrays let the copies overlap the rendering).  float64 or float32 arrays receive the
        sums (streak [H][W][T][3], steady [H][W][3], weight [H][W]); uint8 arrays receive the
        averaged cells RGBE-encoded as the .hdr files hold them (streak [H][W][T][4], steady
        [H][W][4], no weight).  Returns nothing; the arrays hold the film when it returns."""
        arrs = [a for a in (streak, steady, weight) if a is not None]
        dt = arrs[0].dtype if arrs else np.dtype(np.float64)
        if any(a.dtype != dt for a in arrs) or dt not in (np.float64, np.float32, np.uint8):
            raise ValueError("film arrays must all be float64, all float32 or all uint8")
        sc = self.scene
        H, W, T = sc.height, sc.width, sc.time_bins
        ch = 4 if dt == np.uint8 else 3
        if dt == np.uint8 and weight is not None:
            raise ValueError("RGBE delivery has no weight array")
        for a, shape in ((streak, (H, W, T, ch)), (steady, (H, W, ch)), (weight, (H, W))):
            if a is not None and (a.shape != shape or not a.flags["C_CONTIGUOUS"]):
                raise ValueError(f"film array must be C-contiguous with shape {shape}")
        kind = {np.dtype(np.float32): _abi.FILM_F32, np.dtype(np.uint8): _abi.FILM_RGBE}.get(np.dtype(dt),
                                                                                           _abi.FILM_F64)
        _abi.check(_abi.lib().tr_render_film(self.h, int(sample_begin), int(sample_count), kind,
                                             streak.ctypes.data if streak is not None else None,
                                             steady.ctypes.data if steady is not None else None,
                                             weight.ctypes.data if weight is not None else None))

    def write(self, name: str):
        _abi.check(_abi.lib().tr_write_film(self.h, name.encode()))

    # -- ray queries ----------------------------------------------------------------------
    def trace(self, rays, any_hit=False):
        rays = np.ascontiguousarray(rays, np.float32)
        assert rays.ndim == 2 and rays.shape[1] == 8
        out = np.zeros(len(rays), HIT_DTYPE)
        _abi.check(_abi.lib().tr_trace_rays(self.h, rays.ctypes.data, len(rays), int(any_hit), out.ctypes.data))
        return out

    def trace_device(self, d_rays_ptr, n, d_out_ptr, any_hit=False, stream_ptr=None):
        _abi.check(_abi.lib().tr_trace_rays_device(self.h, C.c_void_p(d_rays_ptr), n, int(any_hit),
                                                   C.c_void_p(d_out_ptr), C.c_void_p(stream_ptr)))

    def set_guide(self, guide, mix_prob=0.5, learning_rate=1e-3, train_pool=262144):
        """Render with the learned proposal (tr_set_guide); guide=None detaches."""
        _abi.check(_abi.lib().tr_set_guide(self.h, guide.h if guide is not None else None, mix_prob,
                                           learning_rate, train_pool))
        self._guide = guide

    def set_guide_scope(self, depths=0xFFFFFFFF, min_roughness=0.5):
        """Surface vertices at path depth < depths on Lambertian or GGX (roughness >= min_roughness)
        materials sample with the proposal (tr_set_guide_scope); the others sample their BSDF."""
        _abi.check(_abi.lib().tr_set_guide_scope(self.h, depths, min_roughness))

    def stats(self):
        s = _abi.Stats()
        _abi.check(_abi.lib().tr_stats_get(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in _abi.Stats._fields_}

    def close(self):
        if getattr(self, "h", None):
            _abi.lib().tr_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Several contexts rendered together in shared wavefront batches, one captured CUDA graph
    replayed per batch (``tr_batch_*``).  Each context's film receives exactly the samples a
    ``Context.render`` of the same sample range would give it."""

    def __init__(self, contexts):
        self.contexts = list(contexts)
        arr = (C.c_void_p * len(self.contexts))(*[c.h.value for c in self.contexts])
        h = C.c_void_p()
        _abi.check(_abi.lib().tr_batch_create(arr, len(self.contexts), C.byref(h)))
        self.h = h

    def _arrays(self, begin, count):
        n = len(self.contexts)
        begin = [begin] * n if np.isscalar(begin) else list(begin)
        count = [count] * n if np.isscalar(count) else list(count)
        assert len(begin) == n and len(count) == n
        return (C.c_uint64 * n)(*begin), (C.c_uint32 * n)(*count)

    def render(self, sample_begin, sample_count):
        """Adds samples [sample_begin[i], sample_begin[i] + sample_count[i]) of every pixel of
        scene i (scalars apply to every scene)."""
        b, c = self._arrays(sample_begin, sample_count)
        _abi.check(_abi.lib().tr_batch_render(self.h, b, c))
        return self

    def config(self):
        cfg = _abi.BatchConfig()
        _abi.check(_abi.lib().tr_batch_get_config(self.h, C.byref(cfg)))
        return {k: getattr(cfg, k) for k, _ in _abi.BatchConfig._fields_}

    def set_config(self, **kw):
        cur = self.config()
        cur.update(kw)
        cfg = _abi.BatchConfig(*[cur[k] for k, _ in _abi.BatchConfig._fields_])
        _abi.check(_abi.lib().tr_batch_set_config(self.h, C.byref(cfg)))

    def autotune(self, sample_begin, trial_samples):
        """Runs the autotuner (trial renders add to the films); returns (best config, trials)."""
        b, c = self._arrays(sample_begin, trial_samples)
        best = _abi.BatchConfig()
        trials = C.c_uint32()
        _abi.check(_abi.lib().tr_batch_autotune(self.h, b, c, C.byref(best), C.byref(trials)))
        return {k: getattr(best, k) for k, _ in _abi.BatchConfig._fields_}, trials.value

    def set_guide(self, guide, mix_prob=0.5, learning_rate=1e-3, train_pool=262144):
        _abi.check(_abi.lib().tr_batch_set_guide(self.h, guide.h if guide is not None else None, mix_prob,
                                                 learning_rate, train_pool))
        self._guide = guide

    def stats(self):
        s = _abi.Stats()
        _abi.check(_abi.lib().tr_batch_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in _abi.Stats._fields_}

    def close(self):
        if getattr(self, "h", None):
            _abi.lib().tr_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Guide:
    """Learned directional proposal: MLP -> mixture of 8 von Mises-Fisher lobes (tr_guide_*)."""

    PARAMS = 16640

    def __init__(self, device: int = 0, seed: int = 1):
        h = C.c_void_p()
        _abi.check(_abi.lib().tr_guide_create(device, seed, C.byref(h)))
        self.h = h

    def params(self):
        p = np.zeros(self.PARAMS, np.float32)
        _abi.check(_abi.lib().tr_guide_get_params(self.h, p.ctypes.data))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.PARAMS
        _abi.check(_abi.lib().tr_guide_set_params(self.h, p.ctypes.data))

    def close(self):
        if getattr(self, "h", None):
            _abi.lib().tr_guide_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# =========================================================================================
# Reference-shaped interface
# =========================================================================================

class Lambertian:
    """``-lambertian r g b``: UberMaterial holding one Lambertian(Kd) (bunnykiller.cpp:328-337)."""

    def __init__(self, Kd=(0.67, 0.67, 0.67)):
        self.Kd = tuple(float(k) for k in (Kd if np.ndim(Kd) else (Kd,) * 3))

    def _material(self):
        return S.Material(S.MAT_LAMBERTIAN, self.Kd)


class GGX:
    """Microfacet reflector (no reference counterpart): Schlick F0 = ``R``, roughness ``alpha``."""

    def __init__(self, R=(0.9, 0.9, 0.9), alpha=0.2):
        self.R = tuple(float(k) for k in (R if np.ndim(R) else (R,) * 3))
        self.alpha = float(alpha)

    def _material(self):
        return S.Material(S.MAT_GGX, self.R, self.alpha)


class PointLightSource:
    """``-point-light-source x y z r g b`` (PointLightSource.h:141-171)."""

    def __init__(self, world, position, intensities):
        self.position = tuple(map(float, position))
        self.intensities = tuple(map(float, intensities))

    def _light(self):
        return S.Light(S.LIGHT_POINT, self.position, self.intensities)


class RectangularAreaLightSource:
    """``-rectangular-area-light-source px py pz tx ty tz sx sy I``: corner ``position``, normal
    towards ``target`` (bunnykiller.cpp:1242-1262), frame of ``setup()``
    (RectangularAreaLightSource.h:66-80)."""

    def __init__(self, world, position, target, size, intensity):
        self._l = S.rect_light(position, target, size, intensity)

    def _light(self):
        return self._l


class HenyeyGreenstein:
    def __init__(self, g, mean_time=0.0):
        if mean_time != 0.0:
            raise NotImplementedError("phase-function time delay (-pf-time) is not supported")
        self.g = float(g)


class HomogeneousMedium:
    """``-homogeneous-medium sa sa sa ss ss ss -pf-hg g`` (bunnykiller.cpp:184-227)."""

    def __init__(self, sigma_a, sigma_s, phase: HenyeyGreenstein):
        self.sigma_a = tuple(map(float, sigma_a))
        self.sigma_s = tuple(map(float, sigma_s))
        self.g = phase.g


def _obj_parse(path):
    """OBJ reader with the rules of World::add_triangle_mesh (World.h:209-420): ``v`` (optional
    w), ``vt``, ``vn``, ``vp``; faces ``f a b c`` / ``a/t`` / ``a//n`` / ``a/t/n``, 1-based or
    negative indices; anything but triangles is an error."""
    if not os.path.exists(path):
        raise RuntimeError(f'Error: failed to open model file: "{path}"')
    verts, faces = [], []
    nvt = nvn = 0

    def index(tok, n, line_num):
        i = int(tok)
        j = i - 1 if i > 0 else n + i
        if j > n - 1 or j < 0:
            raise IndexError(f'Error: reading open model file "{path}": out of range index {i} at line {line_num}')
        return j

    with open(path) as fh:
        for line_num, line in enumerate(fh, 1):
            tok = line.split()
            if not tok or tok[0].startswith("#"):
                continue
            if tok[0] == "v":
                if len(tok) not in (4, 5):
                    raise RuntimeError(f'Error: reading open model file "{path}" at line {line_num}')
                verts.append([float(tok[1]), float(tok[2]), float(tok[3])])
            elif tok[0] == "vt":
                nvt += 1
            elif tok[0] == "vn":
                nvn += 1
            elif tok[0] in ("vp",):
                continue
            elif tok[0].startswith("v"):
                raise RuntimeError(f'Error: reading open model file "{path}" at line {line_num}')
            elif tok[0] == "f":
                if len(tok) != 4:
                    raise RuntimeError(f'Error: reading open model file "{path}": invalid face at line {line_num}')
                tri = []
                for t in tok[1:]:
                    parts = t.split("/")
                    tri.append(index(parts[0], len(verts), line_num))
                    if len(parts) > 1 and parts[1]:
                        index(parts[1], nvt, line_num)
                    if len(parts) > 2 and parts[2]:
                        index(parts[2], nvn, line_num)
                faces.append(tri)
    return np.asarray(verts, np.float32).reshape(-1, 3), np.asarray(faces, np.uint32).reshape(-1, 3)


class World:
    """Scene container: meshes with materials, lights and the world medium (World.h:98-787)."""

    def __init__(self):
        self._meshes: List[S.Mesh] = []
        self._materials: List[S.Material] = []
        self._lights: List[S.Light] = []
        self._medium: Optional[S.Medium] = None

    def add_triangle_mesh(self, name_file, mat):
        v, t = _obj_parse(name_file)
        self.add_triangles(v, t, mat, name=os.path.basename(name_file))

    def add_triangles(self, vertices, triangles, mat, name="mesh"):
        self._materials.append(mat._material())
        self._meshes.append(S.Mesh(name, np.asarray(vertices, np.float32), np.asarray(triangles, np.uint32),
                                   len(self._materials) - 1))

    def add_light(self, ls):
        self._lights.append(ls._light())

    def set_medium(self, m: HomogeneousMedium):
        self._medium = S.Medium(m.sigma_a, m.sigma_s, m.g)

    def nb_lights(self):
        return len(self._lights)

    def freeze(self):
        """The BVH is built on the GPU side of the boundary (tr_create)."""


class PinholeCamera:
    def __init__(self, position, focus, up, focal_distance):
        self.position, self.focus, self.up = tuple(position), tuple(focus), tuple(up)
        self.focal_distance = float(focal_distance)

    @staticmethod
    def focal_from_fov(fov_deg):
        """``-camera-fov`` (bunnykiller.cpp:1156-1161): fd = 1 / tan(fov/2)."""
        return 1.0 / math.tan(math.pi / 180.0 * fov_deg / 2.0)


class StreakCameraFilm:
    """Streak film of ``time_resolution`` bins of ``exposure`` (StreakCameraFilm.h:91-121).
    After a render it holds the accumulated sums (``streak``, ``steady``, ``weight``)."""

    bounce_films = 0

    def __init__(self, w, h, t, exposure, camera_unwarp=False, filter=None, comp=1):
        """comp: FilmComponents bits (1 radiance | 2 depth | 8 positions | 16 normals); the
        variance bit (4) is ignored, as the reference's Film keeps no variance image."""
        self.width, self.height, self.time_resolution = int(w), int(h), int(t)
        self.exposure = float(exposure)
        self.camera_unwarp = bool(camera_unwarp)
        self.components = int(comp) & (S.COMP_DEPTH | S.COMP_POSITIONS | S.COMP_NORMALS)
        self.offset = 0.0
        self.streak = self.steady = self.weight = None
        self._ctx = None

    def set_offset(self, offset):
        self.offset = float(offset)

    def get_time_length(self):
        return self.time_resolution * self.exposure + self.offset

    def get_exposure_time(self):
        return self.exposure

    def average(self):
        """Streak and steady images divided by the per-pixel weight (NaN -> 0)."""
        with np.errstate(invalid="ignore", divide="ignore"):
            st = self.streak / self.weight[:, :, None, None]
            sd = self.steady / self.weight[:, :, None]
        return np.nan_to_num(st, nan=0.0), np.nan_to_num(sd, nan=0.0)

    def write(self, name):
        if self._ctx is None:
            raise RuntimeError("film has not been rendered")
        self._ctx.write(name)


class MultibounceStreakFilm(StreakCameraFilm):
    """``nb_bounces`` per-bounce streak films (MultibounceStreakCameraFilm.h:63-83,151-171):
    a radiance sample of bounce b goes to film min(b, nb_bounces - 1).  After a render
    ``bounce_streak``/``bounce_steady``/``bounce_weight`` hold the per-bounce sums and
    ``steady`` the base film's image of all samples."""

    def __init__(self, w, h, t, exposure, nb_bounces, filter=None, camera_unwarp=False, comp=1):
        super().__init__(w, h, t, exposure, camera_unwarp, filter, comp)
        if not 1 <= int(nb_bounces) <= 32:
            raise ValueError("nb_bounces must be in [1, 32]")
        self.bounce_films = int(nb_bounces)
        self.bounce_streak = self.bounce_steady = self.bounce_weight = None

    def bounce_streak_image(self, b=0, y=0):
        """Averaged streak image (time x width) of scanline y of bounce film b."""
        with np.errstate(invalid="ignore", divide="ignore"):
            img = self.bounce_streak[b, y] / self.bounce_weight[b, y][:, None, None]
        return np.nan_to_num(img, nan=0.0).transpose(1, 0, 2)


class StratifiedSampler:
    def __init__(self, size_x, size_y, sqrt_spp, jittered=True):
        if not jittered:
            raise NotImplementedError("only jittered stratified sampling is supported")
        self.size_x, self.size_y, self.sqrt_spp = int(size_x), int(size_y), int(sqrt_spp)

    def get_nb_samples(self):
        return self.size_x * self.size_y * self.sqrt_spp * self.sqrt_spp


class BidirectionalPathTracing:
    """Path tracing with next-event estimation, the mode the reference CLI runs
    (BidirectionalPathTracing.h:122-137; ProgramParams.h:162-164), or, after
    ``set_path_tracing_only(False)``, with light subpaths and eye-light vertex connections
    (TR_FLAG_BIDIRECTIONAL: with a time-sampling renderer, scenes without a medium)."""

    def __init__(self, world, incoming_samples=1, f_log=None, film=None):
        self.world = world
        self.incoming_samples = int(incoming_samples)
        self.max_path_size = 30
        self.seed = 0
        self.path_tracing_only = True

    def set_max_path_size(self, n):
        self.max_path_size = int(n)

    def set_path_tracing_only(self, on):
        # BidirectionalPathTracing::set_path_tracing_only (BidirectionalPathTracing.h:214-217)
        self.path_tracing_only = bool(on)

    def set_seed(self, seed):
        self.seed = int(seed)


class TransientRenderer:
    """GPU replacement of ``TransientRenderer::render`` (TransientRenderer.h:76-201)."""

    def __init__(self, f_log=None, time_sampling=False, device=0):
        # time_sampling: TransientRenderer(f_log, true) -> set_mode(SamplingMode::Transient)
        # (TransientRenderer.h:61-74, BidirectionalPathTracing.h:189-206)
        self.time_sampling = bool(time_sampling)
        self.device = device

    def render(self, name, world: World, integrator: BidirectionalPathTracing, camera: PinholeCamera,
               film: StreakCameraFilm, sampler: StratifiedSampler):
        if integrator is None:
            raise RuntimeError("Error: Need to define an integrator for rendering\n")
        fov = 2.0 * math.degrees(math.atan(1.0 / camera.focal_distance))
        scene = S.Scene("render", list(world._meshes), list(world._materials), list(world._lights),
                        S.Camera(camera.position, camera.focus, camera.up, fov, camera.focal_distance),
                        film.width, film.height, film.time_resolution, film.exposure, film.offset,
                        integrator.max_path_size, sampler.sqrt_spp, integrator.incoming_samples,
                        world._medium, integrator.seed)
        scene.camera_unwarp = int(film.camera_unwarp)
        scene.bounce_films = int(film.bounce_films)
        scene.components = int(film.components)
        if self.time_sampling:
            scene.flags |= S.FLAG_TIME_SAMPLING
        if not integrator.path_tracing_only:
            scene.flags |= S.FLAG_BIDIRECTIONAL
        ctx = Context(scene, self.device)
        ctx.render(0, scene.spp)
        f = ctx.film()
        film.streak, film.steady, film.weight = f["streak"], f["steady"], f["weight"]
        if film.bounce_films:
            b = [ctx.bounce_film(k) for k in range(film.bounce_films)]
            film.bounce_streak = np.stack([x["streak"] for x in b])
            film.bounce_steady = np.stack([x["steady"] for x in b])
            film.bounce_weight = np.stack([x["weight"] for x in b])
        if film.components:
            film.component_sums = ctx.components()
        film._ctx = ctx
        if name:
            ctx.write(name)
        return film
