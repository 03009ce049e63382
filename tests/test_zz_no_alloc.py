"""tr_render_region_noalloc: the render entry point that allocates no GPU memory.

It serves callers that cannot allocate GPU memory once set up -- under an engine whose memory
pool owns the device, or in a frame loop that cannot pay cudaMalloc's device-wide
synchronisation mid-frame.  Its per-path state lives in one fixed array inside the library;
this file checks, through the C ABI, that it renders exactly what tr_render renders, on two
calls in a row (the array keeps the previous call's contents), that its calls allocate no device
memory and count their rays like tr_render's, and that requests beyond its stated limits are
refused.  Named test_zz_* so pytest runs it last; it also passes alone in
a fresh process, where its first call performs the per-device set-up.
"""
import ctypes as C

import numpy as np
import pytest

from jarabotransientrendering_b200 import _abi, scenes as S

pytestmark = pytest.mark.gpu

RTOL_TILE = 2e-5     # same tolerance as the other GPU film comparisons (FP32 warp-group sums)


def _noalloc(ctx, window, s0, n, stream=None):
    x0, y0, x1, y1 = window
    return _abi.lib().tr_render_region_noalloc(ctx.h, x0, y0, x1, y1, s0, n, stream)


def test_noalloc_matches_tr_render_two_calls_in_a_row(gpu):
    sc = S.cornell(width=32, height=24, time_bins=256, exposure=0.02, sqrt_spp=4, max_bounces=6)
    window = (0, 0, sc.width, sc.height)            # 768 pixels x 4 samples = 3072 paths per call
    with gpu.Context(sc) as ref, gpu.Context(sc) as na:
        for s0 in (0, 4):                           # two calls in a row on the same scratch array
            ref.render(s0, 4)
            _abi.check(_noalloc(na, window, s0, 4))
            a, b = ref.film(), na.film()            # tr_get_film synchronises the context stream
            assert (a["weight"] == b["weight"]).all()
            assert ((a["streak"] != 0) == (b["streak"] != 0)).all()
            assert np.allclose(a["streak"], b["streak"], rtol=RTOL_TILE, atol=1e-12)
            assert np.allclose(a["steady"], b["steady"], rtol=RTOL_TILE, atol=1e-12)
            assert b["streak"].sum() > 0


def test_noalloc_windows_cover_a_larger_render(gpu):
    """A frame too large for one call, rendered as several windows, equals one tr_render."""
    sc = S.medium(width=64, height=48, time_bins=512, exposure=0.02, sqrt_spp=4, incoming_samples=2, max_bounces=12)
    with gpu.Context(sc) as ref, gpu.Context(sc) as na:
        ref.render(0, 16)
        rows = 16                                   # 64 x 16 pixels x 16 samples x 2 = 32768 paths
        for y in range(0, sc.height, rows):
            _abi.check(_noalloc(na, (0, y, sc.width, y + rows), 0, 16))
        a, b = ref.film(), na.film()
    assert (a["weight"] == b["weight"]).all()
    assert np.allclose(a["streak"], b["streak"], rtol=RTOL_TILE, atol=1e-12)


def test_noalloc_refuses_requests_beyond_its_limits(gpu):
    sc = S.cornell(width=256, height=256, time_bins=64, exposure=0.08, sqrt_spp=2, max_bounces=6)
    with gpu.Context(sc) as ctx:
        rc = _noalloc(ctx, (0, 0, 256, 256), 0, 4)   # 262144 paths > 65536
        assert rc == 1 and b"65536" in _abi.lib().tr_last_error()
        rc = _noalloc(ctx, (0, 0, 300, 1), 0, 1)     # window outside the film
        assert rc == 1
    deep = S.cornell(width=8, height=8, time_bins=64, exposure=0.08, sqrt_spp=2, max_bounces=20)
    with gpu.Context(deep) as ctx:
        rc = _noalloc(ctx, (0, 0, 8, 8), 0, 1)
        assert rc == 1 and b"max_bounces" in _abi.lib().tr_last_error()


def test_noalloc_calls_allocate_nothing_and_count_their_rays(gpu):
    """After set-up (tr_create), further calls change neither the device's free memory nor the
    context's device bytes, and the context's ray and splat counters match tr_render's."""
    import torch
    sc = S.cornell(width=32, height=24, time_bins=256, exposure=0.02, sqrt_spp=4, max_bounces=6)
    window = (0, 0, sc.width, sc.height)
    with gpu.Context(sc) as ref, gpu.Context(sc) as na:
        _abi.check(_noalloc(na, window, 0, 4))       # warm-up call
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        bytes0 = na.stats()["device_bytes"]
        for s0 in (4, 8, 12):
            _abi.check(_noalloc(na, window, s0, 4))
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        st = na.stats()
        assert free1 == free0 and st["device_bytes"] == bytes0
        ref.render(0, 16)
        sr = ref.stats()
        for k in ("paths", "camera_samples", "closest_rays", "shadow_rays", "splats"):
            assert st[k] == sr[k] and st[k] > 0, k
