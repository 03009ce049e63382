"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle and the reference's
golden films.

* ray batches: triangle ids, distances and barycentrics bit-identical to the oracle (same
  watertight test, same fixed operation order), occlusion booleans identical;
* renders: per-path random walks are bit-identical (same PCG32 streams, same IEEE operation
  sequence), so every (pixel, bin) sum agrees with the oracle up to the FP32 rounding of the
  warp-group sums added to the FP64 film (relative 2e-5);
* statistics against the reference renderer's own films (tests/golden): per-bin z-scores and
  total energy;
* size-independent properties at the full benchmark sizes: weight = samples per pixel,
  steady = time-integrated streak, additivity of progressive renders.
"""
import os

import numpy as np
import pytest

from jarabotransientrendering_b200 import scenes as S

pytestmark = pytest.mark.gpu

RTOL_TILE = 2e-5     # FP32 warp-group sums vs FP64 oracle sums of the same records


def small(name):
    if name == "cornell":
        return S.cornell(width=32, height=24, time_bins=256, exposure=0.02, sqrt_spp=4, max_bounces=6)
    if name == "medium":
        return S.medium(width=24, height=24, time_bins=256, exposure=0.04, sqrt_spp=4, incoming_samples=2,
                        max_bounces=12)
    if name == "icosphere":
        return S.icosphere(subdiv=5, width=32, height=32, time_bins=512, exposure=0.01, sqrt_spp=4, max_bounces=8)
    if name == "ggx":
        return S.guided(width=24, height=24, time_bins=256, exposure=0.02, sqrt_spp=4, max_bounces=6)
    if name == "arealight":
        s = S.guided(width=24, height=24, time_bins=256, exposure=0.02, sqrt_spp=4, max_bounces=6,
                     lambertian_floor=True)
        s.lights = [S.rect_light((0.6, 0.8, 0.6), (0.6, 0.0, 0.6), (0.2, 0.2), 4.0)]
        return s
    raise KeyError(name)


@pytest.mark.parametrize("name,nrays", [("cornell", 200000), ("icosphere7", 200000)])
def test_trace_rays_bit_identical_to_oracle(gpu, oracle_lib, name, nrays):
    sc = S.icosphere() if name == "icosphere7" else S.cornell()
    rays = S.random_rays(nrays, seed=11)
    with gpu.Context(sc) as ctx:
        hg = ctx.trace(rays)
        ag = ctx.trace(rays, any_hit=True)
    o = oracle_lib.Oracle(sc)
    ho = o.trace(rays)
    ao = o.trace(rays, any_hit=True)
    assert (hg["prim_id"] == ho["prim_id"]).all()
    assert (hg["t"].view(np.uint32) == ho["t"].view(np.uint32)).all()
    hit = ho["prim_id"] != 0xFFFFFFFF
    assert (hg["u"][hit].view(np.uint32) == ho["u"][hit].view(np.uint32)).all()
    assert (hg["v"][hit].view(np.uint32) == ho["v"][hit].view(np.uint32)).all()
    assert ((ag["prim_id"] != 0xFFFFFFFF) == (ao["prim_id"] != 0xFFFFFFFF)).all()
    assert hit.mean() > 0.5


@pytest.mark.parametrize("name", ["icosphere7", "cornell"])
def test_trace_matches_reference_embree_all_rays(gpu, oracle_lib, name):
    """The full seeded correctness batch (1,048,576 rays over the subdivision-7 icosphere scene;
    262,144 over the Cornell box) on the GPU against the reference's own Embree records
    (tests/golden/embree_hits_*.npz): every triangle id equal except classified ties, every
    distance within 2 ulp except the reference's reciprocal rounding (tests/test_embree_hits.py)."""
    from oracle import refhits
    from test_embree_hits import check_report, load
    sc, rays, fx = load(name)
    with gpu.Context(sc) as ctx:
        hg = ctx.trace(rays)
    o = oracle_lib.Oracle(sc)
    ho = o.trace(rays)
    assert (hg["prim_id"] == ho["prim_id"]).all()
    assert (hg["t"].view(np.uint32) == ho["t"].view(np.uint32)).all()
    gid, t = refhits.decode(fx, ho)
    rep = refhits.classify(o, sc.flatten()[1], rays, hg, gid, t)
    check_report(rep)


def test_trace_rays_edge_cases(gpu, oracle_lib):
    sc = S.cornell()
    rays = np.array([
        [0.9, 0.5, 0.1, 1e-5, 0.0, -1.0, 0.0, np.inf],     # straight down onto the floor
        [0.9, 0.5, 0.1, 1e-5, 0.0, -1.0, 0.0, 0.25],       # tfar before the floor
        [0.9, 0.5, 0.1, 0.75, 0.0, -1.0, 0.0, np.inf],     # tnear beyond the floor
        [0.9, 0.5, 0.1, 1e-5, 0.0, 0.0, -1.0, np.inf],     # out of the open front
        [1.0, 0.5, 1.0, 1e-5, 0.0, -1.0, 0.0, np.inf],     # along the back-right edge to a corner
        [0.5, 0.5, 0.5, 1e-5, 0.0, 0.0, 0.0, np.inf],      # zero direction (invalid; must not fault)
        [0.0, 0.0, 0.0, 1e-5, 1.0, 1.0, 1.0, np.inf],      # from a room corner, diagonal
    ], np.float32)
    with gpu.Context(sc) as ctx:
        assert len(ctx.trace(np.zeros((0, 8), np.float32))) == 0
        h = ctx.trace(rays)
        a = ctx.trace(rays, any_hit=True)
    o = oracle_lib.Oracle(sc)
    ho = o.trace(rays)
    assert (h["prim_id"] == ho["prim_id"]).all()
    assert (h["t"].view(np.uint32) == ho["t"].view(np.uint32)).all()
    assert h["prim_id"][0] in (0, 1) and abs(h["t"][0] - 0.5) < 1e-6
    assert h["prim_id"][1] == 0xFFFFFFFF and h["t"][1] == np.float32(0.25)
    assert h["prim_id"][2] == 0xFFFFFFFF and h["prim_id"][3] == 0xFFFFFFFF
    assert h["prim_id"][4] != 0xFFFFFFFF        # watertight: the shared corner is not a crack
    assert ((a["prim_id"] != 0xFFFFFFFF) == (h["prim_id"] != 0xFFFFFFFF)).all()


@pytest.mark.parametrize("name", ["cornell", "medium", "icosphere", "arealight", "ggx"])
def test_render_matches_oracle_per_path(gpu, oracle_lib, name):
    sc = small(name)
    with gpu.Context(sc) as ctx:
        ctx.render(0, sc.spp)
        fg = ctx.film()
        st = ctx.stats()
    fo = oracle_lib.Oracle(sc).render(sample_count=sc.spp, nthreads=8)
    assert (fg["weight"] == fo["weight"]).all()
    # identical random walks: the same (pixel, bin) cells are touched
    assert ((fg["streak"] != 0) == (fo["streak"] != 0)).all()
    assert np.allclose(fg["streak"], fo["streak"], rtol=RTOL_TILE, atol=1e-12)
    assert np.allclose(fg["steady"], fo["steady"], rtol=RTOL_TILE, atol=1e-12)
    assert st["splats"] == fo["stats"]["splats"]
    assert st["shadow_rays"] == fo["stats"]["shadow_rays"]
    assert st["closest_rays"] == fo["stats"]["closest_rays"]


@pytest.mark.parametrize("sqrt_spp", [1, 4])
def test_long_film_matches_oracle(gpu, oracle_lib, sqrt_spp):
    # 65,536 time bins (a pixel's streak row is 1.5 MiB of FP64); one sample per pixel puts 32
    # pixels in each warp's records, 16 samples two pixels
    sc = S.cornell(width=16, height=12, time_bins=65536, exposure=0.0002, sqrt_spp=sqrt_spp, max_bounces=6)
    with gpu.Context(sc) as ctx:
        ctx.render(0, sc.spp)
        fg = ctx.film()
        st = ctx.stats()
    fo = oracle_lib.Oracle(sc).render(sample_count=sc.spp, nthreads=8)
    assert (fg["weight"] == fo["weight"]).all()
    assert ((fg["streak"] != 0) == (fo["streak"] != 0)).all()
    assert np.allclose(fg["streak"], fo["streak"], rtol=RTOL_TILE, atol=1e-12)
    assert np.allclose(fg["steady"], fo["steady"], rtol=RTOL_TILE, atol=1e-12)
    assert st["splats"] == fo["stats"]["splats"] > 0


@pytest.mark.parametrize("flags", [0, S.FLAG_TIME_SAMPLING])
def test_batches_on_wave_lanes_match_oracle(gpu, oracle_lib, flags):
    # 96 x 96 pixels x 1024 samples = 9.4 M paths: five pixel batches of the 2^21-slot wave,
    # dealt in turn to the wave lanes (buffers and streams), so one lane takes two batches
    sc = S.cornell(width=96, height=96, time_bins=128, exposure=0.04, sqrt_spp=32, max_bounces=4)
    sc.flags |= flags
    with gpu.Context(sc) as ctx:
        ctx.render(0, sc.spp)
        fg = ctx.film()
        st = ctx.stats()
    fo = oracle_lib.Oracle(sc).render(sample_count=sc.spp, nthreads=8)
    assert (fg["weight"] == fo["weight"]).all()
    assert ((fg["streak"] != 0) == (fo["streak"] != 0)).all()
    assert np.allclose(fg["streak"], fo["streak"], rtol=RTOL_TILE, atol=1e-12)
    assert np.allclose(fg["steady"], fo["steady"], rtol=RTOL_TILE, atol=1e-12)
    assert st["splats"] == fo["stats"]["splats"]
    assert st["shadow_rays"] == fo["stats"]["shadow_rays"]
    assert st["closest_rays"] == fo["stats"]["closest_rays"]


def test_time_bins_beyond_the_bin_field_are_refused(gpu):
    sc = S.cornell(width=1, height=1, time_bins=(1 << 24) - 1, exposure=1e-6, sqrt_spp=1)
    with pytest.raises(gpu.TransientError, match="time_bins") as ei:
        gpu.Context(sc)
    assert ei.value.status == 1


def test_render_region_and_progressive_additivity(gpu, oracle_lib):
    sc = small("cornell")
    with gpu.Context(sc) as ctx:
        ctx.render(0, 5)
        ctx.render(5, 11)
        a = ctx.film()
        ctx.clear()
        ctx.render(0, 16)
        b = ctx.film()
        ctx.clear()
        ctx.render(0, 16, window=(3, 2, 17, 9))
        w = ctx.film()
    assert np.allclose(a["streak"], b["streak"], rtol=RTOL_TILE, atol=1e-12)
    assert (a["weight"] == b["weight"]).all()
    fo = oracle_lib.Oracle(sc).render(sample_count=16, window=(3, 2, 17, 9))
    assert (w["weight"] == fo["weight"]).all()
    assert np.allclose(w["streak"], fo["streak"], rtol=RTOL_TILE, atol=1e-12)
    assert w["streak"][:2].sum() == 0 and w["streak"][:, :3].sum() == 0


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", ["cornell", "medium", "arealight"])
def test_gpu_matches_reference_statistics(gpu, name):
    from test_oracle import _golden_scene, compare_to_golden
    g = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    sc = _golden_scene(name)
    K = len(g["energy"])
    films = []
    with gpu.Context(sc) as ctx:
        for k in range(K):
            ctx.clear()
            ctx.render(64 * k, 64)
            films.append(ctx.film(steady=False, weight=False)["streak"])
    r = compare_to_golden(np.array(films), g)
    assert r["frac_z3"] < 0.02 and abs(r["mean_z"]) < 0.1 and abs(r["energy_z"]) < 4.0, r
    assert r["one_sided_bins"] == 0, r


@pytest.mark.parametrize("workload", ["cornell", "icosphere", "medium", "guided"])
def test_full_size_properties(gpu, workload):
    """Benchmark-size renders: weights, steady = sum over time, finiteness, determinism."""
    sc = S.WORKLOADS[workload]()
    spp = min(sc.spp, 16)
    with gpu.Context(sc) as ctx:
        ctx.render(0, spp)
        f = ctx.film()
        st = ctx.stats()
        ctx.clear()
        ctx.render(0, spp)
        f2 = ctx.film(streak=False)
    assert (f["weight"] == spp).all()
    assert np.isfinite(f["streak"]).all() and (f["streak"] >= 0).all()
    tsum = f["streak"].sum(axis=2)
    assert np.allclose(tsum, f["steady"], rtol=1e-4, atol=1e-9)
    assert np.allclose(f2["steady"], f["steady"], rtol=1e-5, atol=1e-12)   # same walks; atomics reorder sums
    assert st["paths"] == sc.width * sc.height * spp * sc.incoming_samples
    assert f["steady"].sum() > 0


def test_write_film_reference_layout(gpu, tmp_path):
    sc = S.cornell(width=16, height=8, time_bins=64, exposure=0.08, sqrt_spp=2)
    with gpu.Context(sc) as ctx:
        ctx.render(0, 4)
        f = ctx.film()
        name = str(tmp_path / "streak")
        ctx.write(name)
    files = sorted(os.listdir(tmp_path))
    assert len(files) == 8 + 1 and "streak.hdr" in files and "streak_0007.hdr" in files
    img = read_hdr(name + "_0003.hdr")
    assert img.shape == (16, 64, 3)                 # height W (x), width T (time)
    ref = f["streak"][3] / f["weight"][3][:, None, None]
    m = ref.max(axis=2) > 1e-3 * ref.max()
    assert np.allclose(img[m], ref[m], rtol=0.02, atol=1e-6)
    st = read_hdr(name + ".hdr")
    assert st.shape == (8, 16, 3)


def read_hdr(path):
    """Minimal reader of flat (non run-length) Radiance RGBE files."""
    data = open(path, "rb").read()
    head, _, rest = data.partition(b"\n\n")
    dims, _, pix = rest.partition(b"\n")
    _, h, _, w = dims.split()
    h, w = int(h), int(w)
    a = np.frombuffer(pix, np.uint8).reshape(h, w, 4).astype(np.float64)
    e = a[..., 3:4]
    scale = np.where(e > 0, np.ldexp(1.0, (e - 136).astype(np.int32)), 0.0)
    return (a[..., :3] + 0.5 * (e > 0)) * scale


def test_errors_surface_as_status(gpu):
    sc = small("cornell")
    with gpu.Context(sc) as ctx:
        with pytest.raises(gpu.TransientError) as ei:
            ctx.render(0, 4, window=(0, 0, sc.width + 1, 1))
        assert ei.value.status == 1
        with pytest.raises(gpu.TransientError):
            ctx.render((1 << 32) - 2, 4)
    big = S.cornell(width=65535, height=65535, time_bins=4096)
    with pytest.raises(gpu.TransientError) as ei:
        gpu.Context(big)
    assert ei.value.status == 3                       # film does not fit


def test_host_nan_inputs_keep_film_finite(gpu):
    """Fault injection on the host: a NaN light intensity makes every contribution non-finite;
    like TransientRenderer.h:167-171 those samples are dropped and the film stays finite."""
    sc = small("cornell")
    sc.lights = [S.Light(S.LIGHT_POINT, (0.5, 0.8, 0.5), (float("nan"), 1.0, 1.0))]
    with gpu.Context(sc) as ctx:
        ctx.render(0, 4)
        f = ctx.film()
    assert np.isfinite(f["streak"]).all() and f["streak"].sum() == 0


def test_reference_shaped_api(gpu, tmp_path):
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
    gpu.TransientRenderer().render(None, w, bpt, cam, film, sampler)
    with gpu.Context(sc) as ctx:
        ctx.render(0, sc.spp)
        f = ctx.film()
    assert (film.weight == sc.spp).all()
    assert np.allclose(film.streak, f["streak"], rtol=1e-4, atol=1e-9)
    with pytest.raises(RuntimeError):
        gpu.TransientRenderer().render(None, w, None, cam, film, sampler)


def test_render_on_a_caller_stream_with_wave_lanes(gpu):
    # tr_set_stream: the lanes fork from the caller's stream and join it again before the call
    # returns; the film equals a render on the context's own stream
    import torch
    from jarabotransientrendering_b200 import _abi
    sc = S.cornell(width=96, height=96, time_bins=128, exposure=0.04, sqrt_spp=32, max_bounces=4)
    with gpu.Context(sc) as ctx:
        ctx.render(0, sc.spp)
        ref = ctx.film()
    stream = torch.cuda.Stream()
    busy = torch.empty(1 << 28, dtype=torch.uint8, device="cuda")
    with gpu.Context(sc) as ctx:
        _abi.check(_abi.lib().tr_set_stream(ctx.h, stream.cuda_stream))
        with torch.cuda.stream(stream):
            busy.fill_(1)                      # work queued ahead of the render on that stream
        ctx.render(0, sc.spp)
        assert stream.query()                  # nothing of the render is left in flight
        got = ctx.film()
    assert (got["weight"] == ref["weight"]).all()
    assert ((got["streak"] != 0) == (ref["streak"] != 0)).all()
    assert np.allclose(got["streak"], ref["streak"], rtol=RTOL_TILE, atol=1e-12)


def test_deferred_profiling_sums_the_renders_since_the_last_read(gpu):
    # tr_set_profiling(ctx, 2): the events of every timed launch are read out at tr_stats_get,
    # as sums over the renders since the previous read
    from jarabotransientrendering_b200 import _abi
    sc = S.cornell(width=96, height=96, time_bins=128, exposure=0.04, sqrt_spp=32, max_bounces=4)
    keys = ("raygen_ms", "extend_ms", "shade_ms", "shadow_ms", "splat_ms", "trace_ms")
    with gpu.Context(sc) as ctx:
        ctx.render(0, sc.spp)                                   # allocations, lanes
        _abi.check(_abi.lib().tr_set_profiling(ctx.h, 1))
        one = []
        for _ in range(3):
            ctx.render(0, sc.spp)
            one.append(ctx.stats())
        _abi.check(_abi.lib().tr_set_profiling(ctx.h, 2))
        ctx.render(0, sc.spp)
        ctx.render(0, sc.spp)
        two = ctx.stats()
        again = ctx.stats()                                     # nothing pending: unchanged
    per = {k: np.median([s[k] for s in one]) for k in keys}
    for k in keys:
        assert per[k] > 0 and 1.2 * per[k] < two[k] < 3.0 * per[k], (k, per[k], two[k])
        assert again[k] == two[k]
    assert two["trace_ms"] <= two["extend_ms"] + two["shadow_ms"]
    with gpu.Context(sc) as ctx:
        with pytest.raises(gpu.TransientError, match="profiling"):
            _abi.check(_abi.lib().tr_set_profiling(ctx.h, 3))
