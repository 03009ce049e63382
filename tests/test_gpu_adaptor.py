"""The reference-side C++ adaptor (include/bunnykiller_gpu.hpp) run for real.

oracle/_ref/adaptor_render (tests/adaptor_render.cpp, built where the reference sources are)
sets up the reference's own World (with its Embree scene), PinholeCamera, StreakCameraFilm,
StratifiedSampler and BidirectionalPathTracing as the reference's main() does, captures the same
OBJ files with tr::SceneCapture and calls tr::GpuTransientRenderer::render through a
RenderEngine pointer (bunnykiller.cpp:1824).  Its per-scanline <name>_%04d.hdr files and
<name>.hdr must equal what the library writes for the same scene rendered from Python
(tr_write_film), and a sampler that disagrees with the captured configuration must be refused.
"""
import math
import os
import subprocess

import numpy as np
import pytest

from jarabotransientrendering_b200 import scenes as S

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "adaptor_render")


def adaptor_scene(W, H, T, exposure, sqrt_spp):
    """The scene tests/adaptor_render.cpp writes: a room of floor, ceiling and back wall, a box on
    the floor, a point light at (0.5, 0.9, 0.5), depth 6, seed 7."""
    room_v = np.array([[0, 0, 0], [1, 0, 0], [1, 0, 1], [0, 0, 1], [0, 1, 0], [1, 1, 0], [1, 1, 1], [0, 1, 1]],
                      np.float32)
    room_t = np.array([[1, 3, 2], [1, 4, 3], [5, 6, 7], [5, 7, 8], [4, 7, 3], [4, 8, 7]], np.uint32) - 1
    box_v = np.array([[0.3, 0, 0.3], [0.6, 0, 0.3], [0.6, 0, 0.6], [0.3, 0, 0.6],
                      [0.3, 0.4, 0.3], [0.6, 0.4, 0.3], [0.6, 0.4, 0.6], [0.3, 0.4, 0.6]], np.float32)
    box_t = np.array([[5, 6, 7], [5, 7, 8], [1, 2, 6], [1, 6, 5], [2, 3, 7], [2, 7, 6], [3, 4, 8], [3, 8, 7],
                      [4, 1, 5], [4, 5, 8]], np.uint32) - 1
    mats = [S.Material(S.MAT_LAMBERTIAN, (0.75, 0.75, 0.75)), S.Material(S.MAT_LAMBERTIAN, (0.25, 0.75, 0.25))]
    meshes = [S.Mesh("room", room_v, room_t, 0), S.Mesh("box", box_v, box_t, 1)]
    light = S.Light(S.LIGHT_POINT, (0.5, 0.9, 0.5), (1.0, 1.0, 1.0))
    fd = float(np.float32(1.0 / math.tan(math.pi / 180.0 * 40.0 / 2.0)))
    cam = S.Camera((0.5, 0.5, -1.37), (0.5, 0.5, 0.5), (0.0, 1.0, 0.0), 40.0, focal_distance=fd)
    return S.Scene("adaptor", meshes, mats, [light], cam, W, H, T, exposure, 0.0, 6, sqrt_spp, 1, None, 7)


def read_hdr(path):
    from test_gpu_parity import read_hdr as rd
    return rd(path)


def test_adaptor_renders_the_reference_setup_through_the_library(gpu, tmp_path):
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/adaptor_render is built where the reference sources are")
    W, H, T, exposure, sqrt_spp = 24, 16, 64, 0.05, 4
    out = subprocess.run([EXE, str(tmp_path), "adp", str(W), str(H), str(T), str(exposure), str(sqrt_spp)],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    sc = adaptor_scene(W, H, T, exposure, sqrt_spp)
    with gpu.Context(sc) as ctx:
        ctx.render(0, sc.spp)
        ctx.write(str(tmp_path / "py"))
        f = ctx.film()
    assert f["streak"].sum() > 0
    for y in range(H):
        a = read_hdr(str(tmp_path / f"adp_{y:04d}.hdr"))
        b = read_hdr(str(tmp_path / f"py_{y:04d}.hdr"))
        assert a.shape == (W, T, 3) and a.shape == b.shape
        assert np.allclose(a, b, rtol=1 / 64, atol=1e-30), y
    a, b = read_hdr(str(tmp_path / "adp.hdr")), read_hdr(str(tmp_path / "py.hdr"))
    assert a.shape == (H, W, 3) and np.allclose(a, b, rtol=1 / 64, atol=1e-30)
    assert a.sum() > 0


def test_adaptor_refuses_a_sampler_that_disagrees_with_the_capture(gpu, tmp_path):
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/adaptor_render is built where the reference sources are")
    out = subprocess.run([EXE, str(tmp_path), "bad", "24", "16", "64", "0.05", "4", "3"],
                         capture_output=True, text=True)
    assert out.returncode == 3 and "sampler" in out.stdout, out.stdout + out.stderr
    assert not os.path.exists(tmp_path / "bad.hdr")
