"""Drive the reference renderer harness (oracle/_ref/ref_render) on a generated scene.

TEST INFRASTRUCTURE ONLY.  Writes the harness's text scene format and reads back its raw
double-precision film.  Used by tests/ to pin the CPU oracle statistically against the
reference's own integrator and by bench.py's CPU baseline.
"""
from __future__ import annotations

import json
import os
import subprocess
import tempfile

import numpy as np

from .pyoracle import HERE, REF_BIN


def ref_available():
    return os.path.exists(REF_BIN)


# where the reference sources lie: $TR_REFERENCE_SRC, else the build container's location
REF_SRC = os.environ.get("TR_REFERENCE_SRC", "/root/reference/src")


def sources_available(ref_src=REF_SRC):
    return os.path.isdir(ref_src)


def build_ref(ref_src=REF_SRC):
    """Compile the reference programs (oracle/_ref: the renderer with Embree and with the
    reference's own BVH, the hit harness) from the reference sources, only where those sources
    exist; the first build compiles the vendored Embree (about three minutes on eight cores)."""
    if os.path.isdir(ref_src):
        subprocess.check_call(["make", "-s", "-j", str(os.cpu_count() or 4), "-C", HERE, "ref",
                               f"REF_SRC={ref_src}"])
        lib = os.path.join(os.path.dirname(HERE), "jarabotransientrendering_b200", "libtransient_b200.so")
        if os.path.exists(lib):             # the adaptor program links the CUDA library
            subprocess.check_call(["make", "-s", "-C", HERE, "adaptor", f"REF_SRC={ref_src}"])
    return ref_available()


def write_scene(scene, path, seed=None):
    lines = []
    lines.append(f"film {scene.width} {scene.height} {scene.time_bins} {scene.exposure!r} {scene.offset!r}")
    uw, nb = int(getattr(scene, "camera_unwarp", 0)), int(getattr(scene, "bounce_films", 0))
    cm = int(getattr(scene, "components", 0))
    if uw or nb or cm:
        lines.append(f"filmopts {uw} {nb} {cm}")
    if int(getattr(scene, "flags", 0)) & 2:                  # time-sampling mode
        lines.append("mode transient")
    if int(getattr(scene, "flags", 0)) & 4:                  # light subpaths + vertex connections
        lines.append("bidir 1")
    c = scene.camera
    lines.append("camera " + " ".join(repr(float(v)) for v in (*c.position, *c.focus, *c.up)) + f" {c.fov_deg!r}")
    lines.append(f"integrator {scene.max_bounces} {scene.sqrt_spp} {scene.incoming_samples} "
                 f"{scene.seed if seed is None else seed}")
    if scene.medium is not None:
        m = scene.medium
        lines.append("medium 1 " + " ".join(repr(float(v)) for v in (*m.sigma_a, *m.sigma_s, m.g)))
    for m in scene.materials:
        lines.append(f"material {m.kind} {m.kd[0]!r} {m.kd[1]!r} {m.kd[2]!r} {m.alpha!r}")
    for L in scene.lights:
        if L.kind == 0:
            lines.append("light point " + " ".join(repr(float(v)) for v in (*L.position, *L.intensity)))
        else:
            lines.append("light rect " + " ".join(repr(float(v)) for v in (*L.position, *L.target, *L.size))
                         + f" {float(L.intensity[0])!r}")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
        for mesh in scene.meshes:
            v = np.asarray(mesh.vertices, np.float32)
            t = np.asarray(mesh.triangles, np.int64)
            fh.write(f"mesh {len(v)} {len(t)} {mesh.material}\n")
            np.savetxt(fh, v, fmt="%.9g")
            np.savetxt(fh, t, fmt="%d")
        fh.write("end\n")


def render(scene, seed=None, rows=None, keep_streak=True, workdir=None, binary=None):
    """Run the reference renderer (`binary`, default oracle/_ref/ref_render: the Embree build);
    returns dict(streak, steady, weight, seconds, paths).  rows=(y0, y1) renders scanlines
    [y0, y1) only and returns films of y1 - y0 rows."""
    wd = workdir or tempfile.mkdtemp(prefix="bk_ref_")
    sp = os.path.join(wd, "scene.txt")
    op = os.path.join(wd, "film.bin")
    write_scene(scene, sp, seed)
    cmd = [binary or REF_BIN, sp, op]
    if rows is not None:
        cmd += [str(rows[0]), str(rows[1])]
    if not keep_streak:
        cmd += ["--no-streak"]
    res = subprocess.run(cmd, check=True, capture_output=True, text=True)
    info = json.loads(res.stderr.strip().splitlines()[-1])
    H, W, T = scene.height, scene.width, scene.time_bins
    if rows is not None:                     # a band holds only its own scanlines
        H = rows[1] - rows[0]
    raw = np.fromfile(op, np.float64)
    off = 0
    streak = None
    if keep_streak:
        streak = raw[:H * W * T * 3].reshape(H, W, T, 3)
        off = H * W * T * 3
    steady = raw[off:off + H * W * 3].reshape(H, W, 3)
    off += H * W * 3
    weight = raw[off:off + H * W].reshape(H, W)
    off += H * W
    extra = {}
    NB = int(getattr(scene, "bounce_films", 0))
    if NB:
        n = NB * H * W * T * 3
        extra["bstreak"] = raw[off:off + n].reshape(NB, H, W, T, 3)
        off += n
        extra["bsteady"] = raw[off:off + NB * H * W * 3].reshape(NB, H, W, 3)
        off += NB * H * W * 3
        extra["bweight"] = raw[off:off + NB * H * W].reshape(NB, H, W)
    if int(getattr(scene, "components", 0)):
        extra["depth"] = raw[off:off + H * W].reshape(H, W)
        off += H * W
        extra["positions"] = raw[off:off + H * W * 3].reshape(H, W, 3)
        off += H * W * 3
        extra["normals"] = raw[off:off + H * W * 3].reshape(H, W, 3)
    if workdir is None:
        for p in (sp, op):
            os.remove(p)
        os.rmdir(wd)
    return {"streak": streak, "steady": steady, "weight": weight, **extra, **info}
