"""GPU tests of the film options against the CPU oracle (which is pinned to the reference's own
integrator for them in tests/test_oracle.py): camera unwarp (StreakCameraFilm.h:167) and
per-bounce films (MultibounceStreakCameraFilm.h:151-171).  GPU and oracle replay the same
random walks, so the films agree per bin up to the FP32 rounding of warp-group sums."""
import os

import numpy as np
import pytest

from jarabotransientrendering_b200 import scenes as S

pytestmark = pytest.mark.gpu

RTOL = 2e-5


def _scenes():
    c = S.cornell(width=24, height=20, time_bins=96, exposure=0.05, sqrt_spp=2, max_bounces=6)
    m = S.medium(width=20, height=20, time_bins=128, exposure=0.04, sqrt_spp=2, incoming_samples=2, max_bounces=8)
    a = S.guided(width=20, height=20, time_bins=64, exposure=0.08, sqrt_spp=2, max_bounces=6)
    return {"cornell": c, "medium": m, "arealight": a}


def _same(a, b):
    assert ((a != 0) == (b != 0)).all()
    assert np.allclose(a, b, rtol=RTOL, atol=1e-12)


@pytest.mark.parametrize("name", ["cornell", "medium", "arealight"])
def test_camera_unwarp_matches_oracle(gpu, oracle_lib, name):
    sc = _scenes()[name]
    sc.camera_unwarp = 1
    with gpu.Context(sc) as c:
        c.render(0, 12)
        f = c.film()
    o = oracle_lib.Oracle(sc).render(sample_count=12, nthreads=8)
    _same(f["streak"], o["streak"])
    _same(f["steady"], o["steady"])
    assert (f["weight"] == o["weight"]).all()
    # unwarping moves samples earlier: the film must differ from the warped one
    sc.camera_unwarp = 0
    with gpu.Context(sc) as c:
        c.render(0, 12)
        g = c.film()
    assert not np.allclose(f["streak"], g["streak"])


@pytest.mark.parametrize("name,nb,unwarp", [("cornell", 3, 0), ("medium", 4, 0), ("arealight", 2, 1),
                                            ("medium", 1, 1)])
def test_bounce_films_match_oracle(gpu, oracle_lib, name, nb, unwarp):
    sc = _scenes()[name]
    sc.bounce_films = nb
    sc.camera_unwarp = unwarp
    with gpu.Context(sc) as c:
        c.render(0, 12)
        f = c.film()
        b = [c.bounce_film(k) for k in range(nb)]
        with pytest.raises(gpu.TransientError):
            c.bounce_film(nb)
    o = oracle_lib.Oracle(sc).render(sample_count=12, nthreads=8, bounces=True)
    _same(f["streak"], o["streak"])
    _same(f["steady"], o["steady"])
    assert (f["weight"] == o["weight"]).all()
    for k in range(nb):
        _same(b[k]["streak"], o["bstreak"][k])
        _same(b[k]["steady"], o["bsteady"][k])
        assert (b[k]["weight"] == o["bweight"][k]).all()
    # the bounce films partition the in-window samples of the film (each film sums its records in
    # its own FP32 warp groups, hence the FP32 tolerance)
    assert np.allclose(sum(x["streak"] for x in b), f["streak"], rtol=RTOL, atol=1e-12)


def test_bounce_films_written_like_the_reference(gpu, tmp_path):
    sc = _scenes()["cornell"]
    sc.bounce_films = 2
    with gpu.Context(sc) as c:
        c.render(0, 4)
        c.write(str(tmp_path / "frame"))
    names = sorted(os.listdir(tmp_path))
    assert "frame.hdr" in names                           # base steady image
    for b in (1, 2):
        rows = [n for n in names if n.startswith(f"frame_b{b:02d}_")]
        assert len(rows) == sc.height                     # one streak image per scanline
    assert not any(n.startswith("frame_0") for n in names)  # no main streak film in this mode


def test_noalloc_film_modes_match_render(gpu):
    import ctypes as C
    from jarabotransientrendering_b200 import _abi
    sc = _scenes()["medium"]
    sc.bounce_films = 2
    sc.camera_unwarp = 1
    with gpu.Context(sc) as c:
        c.render(0, 6)
        f = c.film()
        b = [c.bounce_film(k) for k in range(2)]
    with gpu.Context(sc) as c:
        for y0 in range(0, sc.height, 10):
            _abi.check(_abi.lib().tr_render_region_noalloc(c.h, 0, y0, sc.width, min(sc.height, y0 + 10), 0, 6, None))
        g = c.film()
        h = [c.bounce_film(k) for k in range(2)]
    _same(g["streak"], f["streak"])
    _same(g["steady"], f["steady"])
    for k in range(2):
        _same(h[k]["streak"], b[k]["streak"])
        assert (h[k]["weight"] == b[k]["weight"]).all()


def test_batch_camera_unwarp_and_bounce_films(gpu):
    scs = list(_scenes().values())
    for sc in scs:
        sc.camera_unwarp = 1
    singles = []
    for sc in scs:
        with gpu.Context(sc) as c:
            c.render(0, 5)
            singles.append(c.film())
    ctxs = [gpu.Context(sc) for sc in scs]
    try:
        with gpu.Batch(ctxs) as B:
            B.set_config(capacity=65536)
            B.render(0, 5)
        for c, s in zip(ctxs, singles):
            f = c.film()
            _same(f["streak"], s["streak"])
            _same(f["steady"], s["steady"])
    finally:
        for c in ctxs:
            c.close()
    sc = scs[0]
    sc.bounce_films = 2
    with gpu.Context(sc) as c:
        with pytest.raises(gpu.TransientError):
            gpu.Batch([c])


@pytest.mark.parametrize("name", ["cornell", "medium"])
def test_film_components_match_oracle(gpu, oracle_lib, name):
    """Depth / positions / normals (Film::add_components): one camera-ray record per camera
    sample, the closest surface at any distance (in the medium scene too); FLT_MAX depth and
    zero position / normal where the camera ray leaves the open room."""
    sc = _scenes()[name]
    sc.components = S.COMP_DEPTH | S.COMP_POSITIONS | S.COMP_NORMALS
    sc.camera_unwarp = 1 if name == "medium" else 0
    sc.bounce_films = 2 if name == "medium" else 0
    with gpu.Context(sc) as c:
        c.render(0, 12)
        f = c.film()
        comp = c.components()
    o = oracle_lib.Oracle(sc).render(sample_count=12, nthreads=8, components=True)
    _same(f["streak"], o["streak"])
    for key in ("depth", "positions", "normals"):
        # FP64 sums of identical FP32 records, in another order (atomics)
        assert np.allclose(comp[key], o[key], rtol=1e-12, atol=1e-9), key
    assert (comp["depth"] > 0).all()


def test_film_components_written_and_batched(gpu, tmp_path):
    scs = list(_scenes().values())
    for sc in scs:
        sc.components = S.COMP_DEPTH | S.COMP_NORMALS
    with gpu.Context(scs[0]) as c:
        c.render(0, 3)
        c.write(str(tmp_path / "frame"))
        single = c.components()
        w = c.film(streak=False, steady=False)["weight"]
    names = set(os.listdir(tmp_path))
    assert {"frame.hdr", "frame_depth.hdr", "frame_normals.raw"} <= names and "frame_positions.raw" not in names
    raw = np.fromfile(tmp_path / "frame_normals.raw", np.float32).reshape(scs[0].height, scs[0].width, 3)
    assert np.allclose(raw, (single["normals"] / w[:, :, None]).astype(np.float32), rtol=1e-6, atol=1e-7)
    ctxs = [gpu.Context(sc) for sc in scs]
    try:
        with gpu.Batch(ctxs) as B:
            B.set_config(capacity=65536)
            B.render(0, 3)
        batched = ctxs[0].components()
    finally:
        for c in ctxs:
            c.close()
    for key in ("depth", "normals"):
        assert np.allclose(batched[key], single[key], rtol=1e-12, atol=1e-9)
