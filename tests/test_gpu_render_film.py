"""tr_render_film: rendering with the film streamed to host memory as pixel rows complete.

Checked against tr_render + tr_get_film on the same scene: FP64 delivery equals the device film,
FP32 delivery equals it rounded to float, the film delivered is the accumulated one (earlier
renders included), and renders that need several pixel batches or several sample chunks (only
the last chunk's rows are final) deliver every row."""
import numpy as np
import pytest

from jarabotransientrendering_b200 import scenes as S

pytestmark = pytest.mark.gpu

RTOL = 2e-5          # FP32 warp-group sums, as in the other film comparisons


def _arrays(sc, dtype, pinned):
    H, W, T = sc.height, sc.width, sc.time_bins
    if pinned:
        import torch
        mk = lambda shape: torch.empty(shape, dtype=getattr(torch, np.dtype(dtype).name), pin_memory=True).numpy()
    else:
        mk = lambda shape: np.empty(shape, dtype)
    a = (mk((H, W, T, 3)), mk((H, W, 3)), mk((H, W)))
    for x in a:
        x.fill(-1)
    return a


def _close(a, b, rtol=RTOL):
    assert ((a != 0) == (b != 0)).all()
    assert np.allclose(a, b, rtol=rtol, atol=1e-12)


@pytest.mark.parametrize("pinned", [True, False])
def test_render_film_f64_and_f32_match_get_film(gpu, pinned):
    # 256 x 256 pixels x 64 samples: two pixel batches of the 2^21-slot wave
    sc = S.cornell(width=256, height=256, time_bins=64, exposure=0.08, sqrt_spp=8, max_bounces=4)
    with gpu.Context(sc) as ref:
        ref.render(0, 64)
        f = ref.film()
    st, sd, wt = _arrays(sc, np.float64, pinned)
    with gpu.Context(sc) as c:
        c.render_film(0, 64, st, sd, wt)
    _close(st, f["streak"])
    _close(sd, f["steady"])
    assert (wt == f["weight"]).all()
    st, sd, wt = _arrays(sc, np.float32, pinned)
    with gpu.Context(sc) as c:
        c.render_film(0, 64, st, sd, wt)
    _close(st, f["streak"].astype(np.float32))
    _close(sd, f["steady"].astype(np.float32))
    assert (wt == f["weight"].astype(np.float32)).all()


def test_render_film_delivers_the_accumulated_film(gpu):
    sc = S.medium(width=32, height=24, time_bins=128, exposure=0.04, sqrt_spp=4, incoming_samples=2, max_bounces=8)
    with gpu.Context(sc) as ref:
        ref.render(0, 8)
        f = ref.film()
    st, sd, wt = _arrays(sc, np.float64, False)
    with gpu.Context(sc) as c:
        c.render(0, 3)
        c.render_film(3, 5, st, sd, wt)
        g = c.film()
    _close(st, f["streak"])
    _close(st, g["streak"], rtol=0)
    assert (wt == f["weight"]).all()


def test_render_film_over_several_sample_chunks(gpu):
    # one pixel x 2.5 M samples: more samples than one wave of 2^21 paths holds, so they are
    # rendered in two chunks and the pixel is delivered after the last one
    sc = S.cornell(width=1, height=1, time_bins=16, exposure=0.3, sqrt_spp=1, max_bounces=2)
    n = 2_500_000
    with gpu.Context(sc) as ref:
        ref.render(0, n)
        f = ref.film()
    st, sd, wt = _arrays(sc, np.float64, False)
    with gpu.Context(sc) as c:
        c.render_film(0, n, st, sd, wt)
    assert (wt == n).all()
    # 2.5 M samples: FP32 warp-group sums added to the FP64 film in launch-dependent order
    _close(st, f["streak"], rtol=1e-3)


def test_render_film_rejects_mixed_or_bad_arrays(gpu):
    sc = S.cornell(width=8, height=8, time_bins=16, exposure=0.3, sqrt_spp=1, max_bounces=2)
    with gpu.Context(sc) as c:
        with pytest.raises(ValueError):
            c.render_film(0, 1, np.empty((8, 8, 16, 3)), np.empty((8, 8, 3), np.float32))
        with pytest.raises(ValueError):
            c.render_film(0, 1, np.empty((8, 8, 15, 3)))
        from jarabotransientrendering_b200 import _abi
        assert _abi.lib().tr_render_film(c.h, 0, 1, 7, None, None, None) == 1


def test_device_memory_is_kept_for_reuse_and_released_on_request(gpu):
    """Destroyed contexts leave their device memory in the library's pool (a second context
    of the same size takes it without the free device memory dropping again);
    tr_release_cached_memory hands it back to the driver."""
    import torch
    from jarabotransientrendering_b200 import _abi
    sc = S.cornell(width=128, height=128, time_bins=2048, exposure=0.005, sqrt_spp=1, max_bounces=2)
    film_bytes = sc.width * sc.height * sc.time_bins * 3 * 8          # 805 MB
    _abi.check(_abi.lib().tr_release_cached_memory(0))
    free0 = torch.cuda.mem_get_info()[0]
    with gpu.Context(sc) as c:
        c.render(0, 1)
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 >= film_bytes                                  # kept by the pool
    with gpu.Context(sc) as c:
        c.render(0, 1)
    free2 = torch.cuda.mem_get_info()[0]
    assert abs(free2 - free1) < film_bytes // 4                         # reused, not mapped again
    _abi.check(_abi.lib().tr_release_cached_memory(0))
    free3 = torch.cuda.mem_get_info()[0]
    assert free3 - free2 >= film_bytes
    assert _abi.lib().tr_release_cached_memory(99) == 1


@pytest.mark.parametrize("workload", ["cornell", "icosphere"])
def test_device_bvh_build_matches_the_host_builder(gpu, tmp_path, workload):
    """tr_create builds the BVH on the device with the host builder's split rules: the same
    four-child tree (node count and depth) as csrc/bvh_build.cpp on the same mesh."""
    import json
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    csrc = os.path.join(root, "jarabotransientrendering_b200", "csrc")
    exe = tmp_path / "bvh_check"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-pthread", "-ffp-contract=off", f"-I{csrc}",
                           os.path.join(root, "tests", "bvh_check.cpp"), os.path.join(csrc, "bvh_build.cpp"),
                           "-o", str(exe)])
    sc = S.WORKLOADS[workload]()
    v, t, _ = sc.flatten()
    raw = tmp_path / "mesh.bin"
    with open(raw, "wb") as fh:
        fh.write(np.array([len(v), len(t)], np.uint32).tobytes())
        fh.write(v.tobytes())
        fh.write(t.tobytes())
    host = json.loads(subprocess.run([str(exe), str(raw)], capture_output=True, text=True, check=True).stdout)
    small = S.WORKLOADS[workload](width=8, height=8, time_bins=16)
    with gpu.Context(small) as c:
        st = c.stats()
    assert st["bvh_nodes"] == host["nodes"] and st["bvh_depth"] == host["depth"], (st, host)


def _rgbe_np(sums, weight):
    """The .hdr writer's encoding restated in numpy: average in double rounded to float (NaN ->
    0), v = max channel = m 2^e, channels * (m 256 / v) truncated to [0, 255], e + 128."""
    with np.errstate(invalid="ignore", divide="ignore"):
        avg = (sums / weight[..., None]).astype(np.float32)
    avg[np.isnan(avg)] = 0.0
    v = avg.max(axis=-1)
    m, e = np.frexp(v)
    ok = v >= np.float32(1e-32)
    with np.errstate(invalid="ignore", divide="ignore", over="ignore"):
        scale = (m * np.float32(256.0)).astype(np.float32) / v
        s = avg * scale[..., None]
    q = np.where(s > 0, np.where(s < 255, s, 255), 0).astype(np.uint8)
    out = np.zeros(avg.shape[:-1] + (4,), np.uint8)
    out[..., :3] = np.where(ok[..., None], q, 0)
    out[..., 3] = np.where(ok, e + 128, 0).astype(np.uint8)
    return out


def _hdr_pixels(path):
    data = open(path, "rb").read()
    head, _, rest = data.partition(b"\n\n")
    dims, _, pix = rest.partition(b"\n")
    _, h, _, w = dims.split()
    return int(h), int(w), np.frombuffer(pix, np.uint8).reshape(int(h), int(w), 4)


@pytest.mark.parametrize("time_bins", [64, 4])
def test_render_film_rgbe_is_the_written_files_pixel_data(gpu, tmp_path, time_bins):
    """RGBE delivery: the averaged film encoded on the device equals, byte for byte, the pixel
    data tr_write_film writes (per-scanline streak files, steady image) and the encoding
    restated in numpy from the FP64 sums."""
    sc = S.cornell(width=40, height=24, time_bins=time_bins, exposure=5.12 / time_bins, sqrt_spp=4, max_bounces=4)
    H, W, T = sc.height, sc.width, sc.time_bins
    st = np.full((H, W, T, 4), 7, np.uint8)
    sd = np.full((H, W, 4), 7, np.uint8)
    name = str(tmp_path / "film")
    with gpu.Context(sc) as c:
        c.render_film(0, 16, st, sd)
        f = c.film()
        c.write(name)
    assert (st == _rgbe_np(f["streak"], f["weight"][..., None])).all()
    assert (sd == _rgbe_np(f["steady"], f["weight"])).all()
    assert (st[..., 3] > 0).mean() > 0.05          # a populated film, not only zero cells
    for y in range(H):
        h, w, pix = _hdr_pixels(f"{name}_{y:04d}.hdr")
        if T >= 8:
            assert (h, w) == (W, T) and (pix == st[y]).all()
        else:
            assert (h, w) == (T, W) and (pix == st[y].transpose(1, 0, 2)).all()
    h, w, pix = _hdr_pixels(name + ".hdr")
    assert (h, w) == (H, W) and (pix == sd).all()
    with gpu.Context(sc) as c:
        with pytest.raises(ValueError):
            c.render_film(0, 1, st, sd, np.empty((H, W), np.uint8))


def test_render_film_with_a_short_last_sample_chunk(gpu):
    """256 paths per camera sample and 9,000 samples per pixel: the 2^21-slot wave holds 8,192
    samples of a pixel, so the samples come in two chunks and the short last one packs ten
    pixels into each batch; every delivered row equals the device film (F32 and RGBE)."""
    sc = S.cornell(width=4, height=4, time_bins=32, exposure=0.1, sqrt_spp=1, max_bounces=2,
                   incoming_samples=256)
    H, W, T = sc.height, sc.width, sc.time_bins
    n = 9000
    st, sd, wt = _arrays(sc, np.float32, False)
    with gpu.Context(sc) as c:
        c.render_film(0, n, st, sd, wt)
        f = c.film()
    assert (wt == n).all()
    assert (st == f["streak"].astype(np.float32)).all() and (sd == f["steady"].astype(np.float32)).all()
    s8 = np.zeros((H, W, T, 4), np.uint8)
    d8 = np.zeros((H, W, 4), np.uint8)
    with gpu.Context(sc) as c:
        c.render_film(0, n, s8, d8)
        f = c.film()
    assert (s8 == _rgbe_np(f["streak"], f["weight"][..., None])).all()
    assert (d8 == _rgbe_np(f["steady"], f["weight"])).all()


def test_render_film_rgbe_after_earlier_samples(gpu):
    """RGBE delivery of a film that already held samples (an earlier tr_render) and of one whose
    earlier samples were cleared: both equal the encoding of the final sums."""
    sc = S.medium(width=32, height=24, time_bins=128, exposure=0.04, sqrt_spp=4, incoming_samples=2, max_bounces=8)
    H, W, T = sc.height, sc.width, sc.time_bins
    for clear in (False, True):
        st = np.full((H, W, T, 4), 7, np.uint8)
        sd = np.full((H, W, 4), 7, np.uint8)
        with gpu.Context(sc) as c:
            c.render(0, 4)
            if clear:
                c.clear()
            c.render_film(4, 8, st, sd)
            f = c.film()
        assert (f["weight"] == (8 if clear else 12)).all()
        assert (st == _rgbe_np(f["streak"], f["weight"][..., None])).all()
        assert (sd == _rgbe_np(f["steady"], f["weight"])).all()
        assert (st[..., 3] > 0).mean() > 0.02


def test_render_film_rgbe_when_the_touched_cells_do_not_fit_shared_memory(gpu):
    """One sample per pixel puts 512 pixels in a splat block; with 1,024 bins their cell bitmap
    (64 KB) exceeds the 32 KB the launcher allows, so the blocks read every cell back instead."""
    sc = S.cornell(width=64, height=32, time_bins=1024, exposure=0.005, sqrt_spp=1, max_bounces=4)
    H, W, T = sc.height, sc.width, sc.time_bins
    st = np.full((H, W, T, 4), 7, np.uint8)
    sd = np.full((H, W, 4), 7, np.uint8)
    with gpu.Context(sc) as c:
        c.render_film(0, 1, st, sd)
        f = c.film()
    assert (st == _rgbe_np(f["streak"], f["weight"][..., None])).all()
    assert (sd == _rgbe_np(f["steady"], f["weight"])).all()
    assert (st[..., 3] > 0).sum() > 100
