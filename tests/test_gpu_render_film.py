"""tr_render_film: rendering with the film streamed to host memory as pixel rows complete.

Checked against tr_render + tr_get_film on the same scene: FP64 delivery equals the device film,
FP32 delivery equals it rounded to float, the film delivered is the accumulated one (earlier
renders included), and renders that need several pixel batches or several sample chunks (only
the last chunk's rows are final) deliver every row."""
import numpy as np
import pytest

from jarabotransientrendering_b200 import scenes as S

pytestmark = pytest.mark.gpu

RTOL = 2e-5          # FP32 shared-memory tile sums, as in the other film comparisons


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
    # 2.5 M samples summed in FP32 shared-memory tiles, in launch-dependent order
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
