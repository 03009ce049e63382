"""GPU tests of time sampling (TR_FLAG_TIME_SAMPLING; the reference's -time-sampling, i.e.
BidirectionalPathTracing::set_mode(SamplingMode::Transient)) against the CPU oracle, which is
pinned to the reference's own renderer in tests/test_oracle.py.  GPU and oracle replay the same
random walks: per-path light point, time-based free flights, no Russian roulette, time-angular
directions in the medium (including the reference's rare tiny densities), so the films agree per
bin up to the FP32 rounding of warp-group sums."""
import numpy as np
import pytest

from jarabotransientrendering_b200 import scenes as S

pytestmark = pytest.mark.gpu

RTOL = 2e-5


def _scenes():
    m = S.medium(width=20, height=20, time_bins=128, exposure=0.04, sqrt_spp=2, incoming_samples=2, max_bounces=10)
    c = S.cornell(width=24, height=20, time_bins=96, exposure=0.05, sqrt_spp=2, max_bounces=6)
    a = S.guided(width=20, height=20, time_bins=64, exposure=0.08, sqrt_spp=2, max_bounces=6)
    # a medium lit by an area light: the path's light point is drawn on the rectangle
    r = S.medium(width=16, height=16, time_bins=96, exposure=0.05, sqrt_spp=2, incoming_samples=1, max_bounces=8)
    r.lights = [S.rect_light((0.6, 0.8, 0.6), (0.6, 0.0, 0.6), (0.3, 0.2), 4.0)]
    out = {"medium": m, "cornell": c, "arealight": a, "medium_rect": r}
    for sc in out.values():
        sc.flags |= S.FLAG_TIME_SAMPLING
    return out


def _same(a, b):
    assert ((a != 0) == (b != 0)).all()
    assert np.allclose(a, b, rtol=RTOL, atol=1e-12)


@pytest.mark.parametrize("name", ["medium", "cornell", "arealight", "medium_rect"])
def test_time_sampling_matches_oracle(gpu, oracle_lib, name):
    sc = _scenes()[name]
    with gpu.Context(sc) as c:
        c.render(0, 16)
        f = c.film()
        st = c.stats()
    o = oracle_lib.Oracle(sc).render(sample_count=16, nthreads=8)
    _same(f["streak"], o["streak"])
    _same(f["steady"], o["steady"])
    assert (f["weight"] == o["weight"]).all()
    assert st["paths"] == sc.width * sc.height * 16 * sc.incoming_samples
    # the mode changes the walks: the film differs from the standard-sampling one
    sc.flags &= ~S.FLAG_TIME_SAMPLING
    with gpu.Context(sc) as c:
        c.render(0, 16)
        g = c.film()
    assert not np.allclose(f["streak"], g["streak"])


def test_time_sampling_with_film_options(gpu, oracle_lib):
    """Camera unwarp and per-bounce films on top of time sampling."""
    sc = _scenes()["medium"]
    sc.camera_unwarp = 1
    sc.bounce_films = 3
    with gpu.Context(sc) as c:
        c.render(0, 12)
        f = c.film()
        b = [c.bounce_film(k) for k in range(3)]
    o = oracle_lib.Oracle(sc).render(sample_count=12, nthreads=8, bounces=True)
    _same(f["streak"], o["streak"])
    for k in range(3):
        _same(b[k]["streak"], o["bstreak"][k])
        assert (b[k]["weight"] == o["bweight"][k]).all()


def test_time_sampling_noalloc_matches_render(gpu):
    import ctypes as C  # noqa: F401
    from jarabotransientrendering_b200 import _abi
    sc = _scenes()["medium"]
    with gpu.Context(sc) as c:
        c.render(0, 6)
        f = c.film()
    with gpu.Context(sc) as c:
        for y0 in range(0, sc.height, 5):
            _abi.check(_abi.lib().tr_render_region_noalloc(c.h, 0, y0, sc.width, min(sc.height, y0 + 5), 0, 6, None))
        g = c.film()
    _same(g["streak"], f["streak"])
    assert (g["weight"] == f["weight"]).all()


def test_time_sampling_in_batch_with_standard_contexts(gpu):
    """A batch mixing time-sampling and standard contexts renders each as its own context."""
    scs = list(_scenes().values())[:3]
    plain = S.medium(width=16, height=16, time_bins=64, exposure=0.05, sqrt_spp=2, incoming_samples=1, max_bounces=6)
    scs.append(plain)
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
            assert (f["weight"] == s["weight"]).all()
    finally:
        for c in ctxs:
            c.close()


def test_time_sampling_reference_renderer_api(gpu, tmp_path):
    """TransientRenderer(f_log, time_sampling=True) selects the mode, as the reference's
    constructor argument does (TransientRenderer.h:61-62, bunnykiller.cpp:1337-1345)."""
    from test_gpu_parity import small
    sc = small("cornell")
    paths = sc.write_obj(str(tmp_path))
    w = gpu.World()
    kd = {"left": S.RED, "right": S.GREEN}
    for p, m in zip(paths, sc.meshes):
        w.add_triangle_mesh(p, gpu.Lambertian(kd.get(m.name, S.WHITE)))
    w.add_light(gpu.PointLightSource(w, (0.5, 0.99, 0.5), (1, 1, 1)))
    cam = gpu.PinholeCamera((0.5, 0.5, -1.37), (0.5, 0.5, 0.5), (0, 1, 0), gpu.PinholeCamera.focal_from_fov(40))
    film = gpu.StreakCameraFilm(sc.width, sc.height, sc.time_bins, sc.exposure)
    sampler = gpu.StratifiedSampler(sc.width, sc.height, sc.sqrt_spp)
    bpt = gpu.BidirectionalPathTracing(w, 1)
    bpt.set_max_path_size(sc.max_bounces)
    bpt.set_seed(sc.seed)
    gpu.TransientRenderer(None, time_sampling=True).render(None, w, bpt, cam, film, sampler)
    sc.flags |= S.FLAG_TIME_SAMPLING
    with gpu.Context(sc) as ctx:
        ctx.render(0, sc.spp)
        f = ctx.film()
    assert np.allclose(film.streak, f["streak"], rtol=1e-4, atol=1e-9)
    sc.flags &= ~S.FLAG_TIME_SAMPLING
    with gpu.Context(sc) as ctx:
        ctx.render(0, sc.spp)
        g = ctx.film()
    assert not np.allclose(film.streak, g["streak"])


def _chunk_energies(ctx, chunks, spp):
    e, prev = [], 0.0
    for k in range(chunks):
        ctx.render(k * spp, spp)
        tot = float(ctx.film(steady=False, weight=False)["streak"].sum())
        e.append(tot - prev)
        prev = tot
    return np.array(e)


def test_time_sampling_with_learned_proposal_is_unbiased(gpu):
    """The learned proposal on surfaces under time sampling (no Russian roulette: the guided
    vertex carries probability 1): per-chunk energies agree with plain time sampling."""
    sc = _scenes()["arealight"]
    sc.flags |= S.FLAG_ORTHONORMAL_FRAME
    with gpu.Context(sc) as c:
        plain = _chunk_energies(c, 24, 16)
    g = gpu.Guide(seed=3)
    with gpu.Context(sc) as c:
        c.set_guide(g, mix_prob=0.5, learning_rate=1e-3, train_pool=65536)
        guided = _chunk_energies(c, 24, 16)
    g.close()
    assert np.isfinite(guided).all() and (guided > 0).all()
    se = np.sqrt(plain.var(ddof=1) / len(plain) + guided.var(ddof=1) / len(guided))
    z = (guided.mean() - plain.mean()) / se
    assert abs(z) < 4.5, (guided.mean(), plain.mean(), z)
