"""The library's .hdr film writer (csrc/tr_film_io.cpp, the reference's StreakCameraFilm output:
StreakCameraFilm.h:356-437, ImageIO.h:146-193), built on the CPU and driven with raw sums:
its bytes equal the RGBE restatement (average in double rounded to float, NaN -> 0, shared
exponent from frexp of the largest channel, channels truncated to [0, 255]) that the GPU tests
compare the device encoding with, for both streak layouts (T >= 8 rows x, T < 8 transposed)."""
import os
import subprocess

import numpy as np
import pytest

from test_gpu_render_film import _hdr_pixels, _rgbe_np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "jarabotransientrendering_b200", "csrc")


@pytest.fixture(scope="module")
def film_check(tmp_path_factory):
    exe = tmp_path_factory.mktemp("film") / "film_check"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-ffp-contract=off", f"-I{CSRC}",
                           os.path.join(ROOT, "tests", "film_check.cpp"), os.path.join(CSRC, "tr_film_io.cpp"),
                           "-o", str(exe)])
    return str(exe)


def _film(rng, H, W, T):
    # sums spanning many exponents, exact zeros, channels far apart (clamped at 255), and
    # pixels of weight 0 (their sums are 0: average NaN -> 0)
    scale = 10.0 ** rng.integers(-40, 12, size=(H, W, T, 1))
    streak = rng.exponential(1.0, (H, W, T, 3)) * scale
    streak[rng.random((H, W, T)) < 0.3] = 0.0
    streak[..., 1] *= np.where(rng.random((H, W, T)) < 0.1, 1e-9, 1.0)
    steady = rng.exponential(1.0, (H, W, 3)) * 10.0 ** rng.integers(-5, 5, size=(H, W, 1))
    weight = rng.integers(0, 300, size=(H, W)).astype(np.float64)
    streak[weight == 0] = 0.0
    steady[weight == 0] = 0.0
    return streak, steady, weight


@pytest.mark.parametrize("T", [64, 5])
def test_written_film_bytes_equal_the_rgbe_restatement(film_check, tmp_path, T):
    rng = np.random.default_rng(7 + T)
    H, W = 6, 11
    streak, steady, weight = _film(rng, H, W, T)
    src = tmp_path / "film.bin"
    with open(src, "wb") as fh:
        fh.write(np.ascontiguousarray(streak).tobytes())
        fh.write(np.ascontiguousarray(steady).tobytes())
        fh.write(np.ascontiguousarray(weight).tobytes())
    name = str(tmp_path / "out")
    subprocess.check_call([film_check, str(src), name, str(W), str(H), str(T)])
    want = _rgbe_np(streak, weight[..., None])
    for y in range(H):
        h, w, pix = _hdr_pixels(f"{name}_{y:04d}.hdr")
        if T >= 8:
            assert (h, w) == (W, T) and (pix == want[y]).all()
        else:
            assert (h, w) == (T, W) and (pix == want[y].transpose(1, 0, 2)).all()
    h, w, pix = _hdr_pixels(name + ".hdr")
    assert (h, w) == (H, W) and (pix == _rgbe_np(steady, weight)).all()
    assert (want[..., 3] > 0).mean() > 0.2 and (want[..., 3] == 0).mean() > 0.2
