"""C ABI and host logic checks that need no GPU: the library loads and exports every entry point
declared in include/transient_b200.h; argument validation (the reference's exceptions become
status codes); the reference-shaped OBJ reader; the seeded scene generators."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, cuda_available
from jarabotransientrendering_b200 import _abi, scenes as S
import jarabotransientrendering_b200 as T

HEADER = os.path.join(ROOT, "include", "transient_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\**(tr_\w+)\s*\(", src, re.M)))


def test_header_declares_expected_api():
    syms = declared_symbols()
    for s in ["tr_create", "tr_render", "tr_render_region", "tr_get_film", "tr_trace_rays", "tr_stats_get",
              "tr_destroy", "tr_status_string", "tr_last_error", "tr_write_film"]:
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = _abi.lib()
    for s in declared_symbols():
        assert hasattr(lib, s), s
        assert s in _abi.PROTOTYPES, f"{s} has no ctypes prototype"
    assert lib.tr_abi_version() == 2


def test_status_strings():
    lib = _abi.lib()
    for code in range(8):
        assert lib.tr_status_string(code)
    assert lib.tr_status_string(99) == b"unknown status"


def _scene_structs(sc):
    """Builds C structs for a scene without creating a context."""
    v, t, m = sc.flatten()
    mats = (_abi.Material * len(sc.materials))()
    for i, mm in enumerate(sc.materials):
        mats[i].kind = mm.kind
        mats[i].kd = _abi.f3(*mm.kd)
        mats[i].alpha = mm.alpha
    lights = (_abi.Light * max(1, len(sc.lights)))()
    for i, L in enumerate(sc.lights):
        lights[i].kind = L.kind
        lights[i].position = _abi.f3(*L.position)
        lights[i].intensity = _abi.f3(*L.intensity)
        lights[i].area = L.area
    keep = [v, t, m, mats, lights]
    s = _abi.Scene(v.ctypes.data_as(C.POINTER(C.c_float)), len(v), t.ctypes.data_as(C.POINTER(C.c_uint32)), len(t),
                   m.ctypes.data_as(C.POINTER(C.c_uint32)), mats, len(sc.materials), lights, len(sc.lights),
                   _abi.Medium())
    cam = _abi.Camera(_abi.f3(0.5, 0.5, -1.37), _abi.f3(0, 0, 1), _abi.f3(-1, 0, 0), _abi.f3(0, 1, 0), 2.7)
    film = _abi.Film(sc.width, sc.height, sc.time_bins, sc.exposure, 0.0)
    integ = _abi.Integrator(sc.max_bounces, sc.sqrt_spp, sc.incoming_samples, 0, 1)
    return s, cam, film, integ, keep


def _create(s, cam, film, integ):
    h = C.c_void_p()
    rc = _abi.lib().tr_create(C.byref(s), C.byref(cam), C.byref(film), C.byref(integ), 0, C.byref(h))
    return rc, h, _abi.lib().tr_last_error().decode()


def test_validation_rejects_bad_scenes_before_touching_a_device():
    sc = S.cornell()
    s, cam, film, integ, keep = _scene_structs(sc)
    # material index out of range (reference: dangling material / bad mesh)
    bad = np.array(keep[2], copy=True)
    bad[3] = 99
    s.triangle_material = bad.ctypes.data_as(C.POINTER(C.c_uint32))
    rc, _, msg = _create(s, cam, film, integ)
    assert rc == 1 and "material index" in msg
    s.triangle_material = keep[2].ctypes.data_as(C.POINTER(C.c_uint32))
    # no light source
    s.num_lights = 0
    rc, _, msg = _create(s, cam, film, integ)
    assert rc == 1 and "light" in msg
    s.num_lights = 1
    # zero-sized film and bad exposure
    film.time_bins = 0
    assert _create(s, cam, film, integ)[0] == 1
    film.time_bins = 64
    film.exposure = 0.0
    assert _create(s, cam, film, integ)[0] == 1
    film.exposure = 0.005
    # depth beyond the supported path length
    integ.max_bounces = 200
    assert _create(s, cam, film, integ)[0] == 1
    integ.max_bounces = 6
    # NaN albedo
    keep[3][0].kd = _abi.f3(float("nan"), 0.5, 0.5)
    rc, _, msg = _create(s, cam, film, integ)
    assert rc == 1 and "not finite" in msg


def test_vertex_index_and_nan_geometry_rejected():
    if cuda_available():
        pytest.skip("on a GPU machine the valid path proceeds to device set-up")
    sc = S.cornell()
    s, cam, film, integ, keep = _scene_structs(sc)
    rc, _, msg = _create(s, cam, film, integ)
    assert rc == 6, msg         # valid scene, but no CUDA device on this machine


def test_obj_reader_follows_reference_rules(tmp_path):
    p = tmp_path / "m.obj"
    p.write_text("# comment\nv 0 0 0\nv 1 0 0 1.0\nv 0 1 0\nvt 0 0\nvn 0 0 1\n"
                 "f 1 2 3\nf -3 -2 -1\nf 1/1 2/1 3/1\nf 1//1 2//1 3//1\nf 1/1/1 2/1/1 3/1/1\n")
    v, t = T.renderer._obj_parse(str(p))
    assert v.shape == (3, 3) and t.shape == (5, 3)
    assert (t == np.array([0, 1, 2], np.uint32)).all()
    q = tmp_path / "bad.obj"
    q.write_text("v 0 0 0\nv 1 0 0\nf 1 2 5\n")
    with pytest.raises(IndexError):
        T.renderer._obj_parse(str(q))
    r = tmp_path / "quad.obj"
    r.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\n")
    with pytest.raises(RuntimeError):
        T.renderer._obj_parse(str(r))
    with pytest.raises(RuntimeError):
        T.renderer._obj_parse(str(tmp_path / "missing.obj"))


def test_scene_generators_deterministic_and_oriented(tmp_path):
    a, b = S.icosphere(subdiv=3), S.icosphere(subdiv=3)
    va, ta, ma = a.flatten()
    vb, tb, mb = b.flatten()
    assert (va == vb).all() and (ta == tb).all()
    assert S.icosphere(subdiv=7).num_triangles == 10 + 24 + 20 * 4 ** 7
    c = S.cornell()
    assert c.num_triangles == 34
    # room normals point inward: camera-facing back wall normal has -z
    back = [m for m in c.meshes if m.name == "back"][0]
    v, t = back.vertices.astype(np.float64), back.triangles
    n = np.cross(v[t[:, 2]] - v[t[:, 0]], v[t[:, 1]] - v[t[:, 0]])
    assert (n[:, 2] < 0).all()
    # OBJ files round-trip through the reference-rules reader
    paths = c.write_obj(str(tmp_path))
    w = T.World()
    for path in paths:
        w.add_triangle_mesh(path, T.Lambertian(0.5))
    assert sum(len(m.triangles) for m in w._meshes) == 34


def test_rect_light_frame_matches_reference_setup():
    L = S.rect_light((0.525, 0.99, 0.525), (0.525, 0.0, 0.525), (0.05, 0.05), 40.0)
    assert np.allclose(L.normal, (0, -1, 0))
    # normal parallel to +-y: up = z, left = n x up, up = n x left (scaled by size)
    assert np.allclose(L.left, (-0.05, 0, 0)) and np.allclose(L.up, (0, 0, -0.05))
    assert abs(L.area - 0.0025) < 1e-9


def test_c_header_is_plain_c(tmp_path):
    """include/transient_b200.h compiles as C99 (no C++ types cross the boundary)."""
    import subprocess
    src = tmp_path / "t.c"
    src.write_text('#include "transient_b200.h"\nint main(void){ tr_stats s; (void)s; return tr_abi_version() * 0; }\n')
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", f"-I{ROOT}/include", str(src)])


def test_python_structs_match_the_c_layout(tmp_path):
    """The ctypes mirrors in _abi.py have the C structs' sizes and field offsets."""
    import ctypes as C
    import subprocess
    from jarabotransientrendering_b200 import _abi
    checks = {"tr_stats": (_abi.Stats, ["render_ms", "guide_ms", "train_loss", "trace_ms"]),
              "tr_batch_config": (_abi.BatchConfig, ["splat_div", "use_graph"])}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "transient_b200.h"', 'int main(void){']
    for cname, (_, fields) in checks.items():
        lines.append(f'printf("%zu\\n", sizeof({cname}));')
        lines += [f'printf("%zu\\n", offsetof({cname}, {f}));' for f in fields]
    lines.append('return 0; }')
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.check_call(["gcc", "-std=c99", f"-I{ROOT}/include", str(src), "-o", str(exe)])
    got = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    want = []
    for cname, (py, fields) in checks.items():
        want.append(C.sizeof(py))
        want += [getattr(py, f).offset for f in fields]
    assert got == want


def test_reference_adaptor_compiles():
    """include/bunnykiller_gpu.hpp derives from the reference's TransientRenderer and overrides
    its render() signature (needs the reference sources; skipped where they are absent)."""
    import subprocess
    from oracle import refscene
    ref = refscene.REF_SRC
    if not refscene.sources_available():
        pytest.skip("reference sources not present on this machine")
    subprocess.check_call(["g++", "-fsyntax-only", "-std=c++14", "-w", "-include",
                           os.path.join(ROOT, "oracle", "ref_globals.h"), f"-I{ref}", f"-I{ROOT}/include",
                           os.path.join(ROOT, "tests", "adaptor_check.cpp")])


@pytest.mark.parametrize("workload", ["cornell", "icosphere"])
def test_product_bvh_builder_invariants(tmp_path, workload):
    """The host BVH builder of the CUDA path (csrc/bvh_build.cpp, multithreaded binned SAH collapsed
    to four-child nodes): every triangle exactly once in leaf order with its vertices, boxes
    enclose their leaves, all nodes reachable, the reported stack bounds the traversal, and the
    four-child tree has about half the binary tree's depth."""
    import json
    import subprocess
    exe = tmp_path / "bvh_check"
    csrc = os.path.join(ROOT, "jarabotransientrendering_b200", "csrc")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-pthread", "-ffp-contract=off", f"-I{csrc}",
                           os.path.join(ROOT, "tests", "bvh_check.cpp"), os.path.join(csrc, "bvh_build.cpp"),
                           "-o", str(exe)])
    v, t, _ = S.WORKLOADS[workload]().flatten()
    raw = tmp_path / "mesh.bin"
    with open(raw, "wb") as fh:
        fh.write(np.array([len(v), len(t)], np.uint32).tobytes())
        fh.write(v.tobytes())
        fh.write(t.tobytes())
    out = subprocess.run([str(exe), str(raw)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout
    info = json.loads(out.stdout)
    assert info["stack"] <= 96 and info["depth"] * 2 <= info["binary_depth"] + 2
