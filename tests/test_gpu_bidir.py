"""GPU tests of bidirectional connections (TR_FLAG_BIDIRECTIONAL: light subpaths and eye-light
vertex connections, BidirectionalPathTracing with set_path_tracing_only(false), in time-sampling
mode) against the CPU oracle, which is pinned to the reference's own renderer in
tests/test_oracle.py.  GPU and oracle replay the same eye walks, light subpaths (their own
random stream) and connections, so the films agree per bin up to the FP32 rounding of
warp-group sums."""
import numpy as np
import pytest

from jarabotransientrendering_b200 import scenes as S

pytestmark = pytest.mark.gpu

RTOL = 2e-5
BD = S.FLAG_TIME_SAMPLING | S.FLAG_BIDIRECTIONAL


def _scenes():
    c = S.cornell(width=24, height=20, time_bins=96, exposure=0.05, sqrt_spp=2, max_bounces=6)
    a = S.guided(width=20, height=20, time_bins=64, exposure=0.08, sqrt_spp=2, max_bounces=5, lambertian_floor=True)
    a.lights = [S.rect_light((0.6, 0.8, 0.6), (0.6, 0.0, 0.6), (0.3, 0.2), 4.0)]
    o = S.cornell(width=16, height=16, time_bins=64, exposure=0.05, sqrt_spp=2, max_bounces=8, incoming_samples=2)
    o.flags = S.FLAG_ORTHONORMAL_FRAME
    i = S.icosphere(subdiv=3, width=16, height=16, time_bins=128, exposure=0.02, sqrt_spp=2, max_bounces=4)
    out = {"cornell": c, "arealight": a, "ortho_ninc2": o, "icosphere": i}
    for sc in out.values():
        sc.flags |= BD
    return out


def _same(a, b):
    assert ((a != 0) == (b != 0)).all()
    assert np.allclose(a, b, rtol=RTOL, atol=1e-12)


@pytest.mark.parametrize("name", ["cornell", "arealight", "ortho_ninc2", "icosphere"])
def test_bidirectional_matches_oracle(gpu, oracle_lib, name):
    sc = _scenes()[name]
    with gpu.Context(sc) as c:
        c.render(0, 12)
        f = c.film()
        st = c.stats()
    o = oracle_lib.Oracle(sc).render(sample_count=12, nthreads=8)
    _same(f["streak"], o["streak"])
    _same(f["steady"], o["steady"])
    assert (f["weight"] == o["weight"]).all()
    # same rays: closest hits of both subpaths, next-event and connection shadow rays
    assert st["closest_rays"] == o["stats"]["closest_rays"] and st["shadow_rays"] == o["stats"]["shadow_rays"]
    # the eye walks are the time-sampling path tracer's (the light subpaths draw from their own
    # stream): the connections only add, bin by bin, and carry energy
    sc.flags &= ~S.FLAG_BIDIRECTIONAL
    with gpu.Context(sc) as c:
        c.render(0, 12)
        g = c.film()
    assert (f["streak"] - g["streak"] >= -RTOL * np.abs(g["streak"]) - 1e-12).all()
    assert f["streak"].sum() > 1.01 * g["streak"].sum()


def test_bidirectional_with_film_options(gpu, oracle_lib):
    """Camera unwarp and per-bounce films (connections carry bounce ie + il + 1)."""
    sc = _scenes()["cornell"]
    sc.camera_unwarp = 1
    sc.bounce_films = 4
    with gpu.Context(sc) as c:
        c.render(0, 8)
        f = c.film()
        b = [c.bounce_film(k) for k in range(4)]
    o = oracle_lib.Oracle(sc).render(sample_count=8, nthreads=8, bounces=True)
    _same(f["streak"], o["streak"])
    _same(f["steady"], o["steady"])
    for k in range(4):
        _same(b[k]["streak"], o["bstreak"][k])
        _same(b[k]["steady"], o["bsteady"][k])
        assert (b[k]["weight"] == o["bweight"][k]).all()


def test_bidirectional_progressive_and_batched_calls(gpu):
    """Additive renders over several wavefront batches equal one render."""
    sc = _scenes()["cornell"]
    with gpu.Context(sc) as c:
        c.render(0, 16)
        f = c.film()
    with gpu.Context(sc) as c:
        for s0 in range(0, 16, 4):
            c.render(s0, 4)
        g = c.film()
    _same(g["streak"], f["streak"])


def test_bidirectional_unsupported_combinations(gpu):
    """Refused with TR_ERR_NOT_SUPPORTED: no time sampling (the reference's light sample is then
    uninitialised), a medium (the reference dereferences a null medium), GGX, more than 16
    bounces; and the modes that have no subpath storage (batches, learned proposal, the
    allocation-free path)."""
    base = _scenes()["cornell"]
    cases = []
    s1 = _scenes()["cornell"]; s1.flags = S.FLAG_BIDIRECTIONAL; cases.append(s1)
    s2 = S.medium(width=8, height=8, time_bins=32, exposure=0.1, sqrt_spp=1, max_bounces=4); s2.flags = BD; cases.append(s2)
    s3 = S.guided(width=8, height=8, time_bins=32, exposure=0.1, sqrt_spp=1, max_bounces=4); s3.flags |= BD; cases.append(s3)
    s4 = _scenes()["cornell"]; s4.max_bounces = 17; cases.append(s4)
    for sc in cases:
        with pytest.raises(gpu.TransientError) as ei:
            gpu.Context(sc)
        assert ei.value.status == 4, sc.name
    from jarabotransientrendering_b200 import _abi
    with gpu.Context(base) as c:
        with pytest.raises(gpu.TransientError):
            gpu.Batch([c])
        with pytest.raises(gpu.TransientError):
            _abi.check(_abi.lib().tr_render_region_noalloc(c.h, 0, 0, 4, 4, 0, 1, None))
    o = _scenes()["ortho_ninc2"]
    g = gpu.Guide(seed=1)
    with gpu.Context(o) as c:
        with pytest.raises(gpu.TransientError):
            c.set_guide(g)
    g.close()


def test_bidirectional_reference_renderer_api(gpu, tmp_path):
    """BidirectionalPathTracing.set_path_tracing_only(False) with a time-sampling
    TransientRenderer selects light subpaths, as in the reference's API."""
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
    bpt.set_path_tracing_only(False)
    gpu.TransientRenderer(None, time_sampling=True).render(None, w, bpt, cam, film, sampler)
    sc.flags |= BD
    with gpu.Context(sc) as ctx:
        ctx.render(0, sc.spp)
        f = ctx.film()
    assert np.allclose(film.streak, f["streak"], rtol=1e-4, atol=1e-9)
