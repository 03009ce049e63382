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
