"""GPU tests of guided rendering: the learned proposal combined with BSDF sampling by one-sample
MIS must leave the estimator unbiased (guided and plain films agree statistically, whether the
network is untrained or trained online during the renders), and the orthonormal-frame plain
sampler it is compared against is bit-for-bit the oracle's."""
import numpy as np
import pytest

from jarabotransientrendering_b200 import scenes as S

pytestmark = pytest.mark.gpu

RTOL_TILE = 2e-5


def guided_scene(width=32, height=32, time_bins=128, exposure=0.04):
    sc = S.guided(width=width, height=height, time_bins=time_bins, exposure=exposure, sqrt_spp=4, max_bounces=6)
    sc.flags = S.FLAG_ORTHONORMAL_FRAME
    return sc


def test_orthonormal_frame_matches_oracle(gpu, oracle_lib):
    for sc in (S.cornell(width=24, height=24, time_bins=256, exposure=0.02, sqrt_spp=4), guided_scene(24, 24, 256, 0.02)):
        sc.flags = S.FLAG_ORTHONORMAL_FRAME
        with gpu.Context(sc) as ctx:
            ctx.render(0, 16)
            fg = ctx.film()
        fo = oracle_lib.Oracle(sc).render(sample_count=16, nthreads=8)
        assert ((fg["streak"] != 0) == (fo["streak"] != 0)).all()
        assert np.allclose(fg["streak"], fo["streak"], rtol=RTOL_TILE, atol=1e-12)


def _films(gpu, sc, K, spp, guide=None, train_pool=0, min_roughness=None):
    out = []
    with gpu.Context(sc) as ctx:
        if guide is not None:
            ctx.set_guide(guide, mix_prob=0.5, learning_rate=1e-3, train_pool=train_pool)
            if min_roughness is not None:
                ctx.set_guide_scope(min_roughness=min_roughness)
        for k in range(K):
            ctx.clear()
            ctx.render(spp * k, spp)
            out.append(ctx.film(steady=False, weight=False)["streak"])
        st = ctx.stats()
    return np.array(out), st


def _z(a, b):
    se = np.sqrt(a.var(0, ddof=1) / len(a) + b.var(0, ddof=1) / len(b))
    m = se > 0
    return (a.mean(0) - b.mean(0))[m] / se[m]


def _compare(a, b, tile=8, window=8):
    """Two-sample z-scores of aggregates that each sum thousands of paths, so are close to
    normal: total energy, 8x8-pixel tiles and 8-bin time windows. Single bins or pixels are
    sparse and heavy-tailed, and their tails differ between the samplers (one-sample MIS with an
    untrained mixture gives rarer, larger contributions than BSDF sampling), which skews their
    z-scores even when both estimators are unbiased."""
    K, H, W, T, _ = a.shape

    def tiles(x):
        return x.sum(axis=(3, 4)).reshape(len(x), H // tile, tile, W // tile, tile).sum(axis=(2, 4)).reshape(len(x), -1)

    def windows(x):
        return x.sum(axis=(1, 2, 4)).reshape(len(x), T // window, window).sum(axis=2)

    ez = _z(a.sum(axis=(1, 2, 3, 4)), b.sum(axis=(1, 2, 3, 4)))[0]
    zt, zw = _z(tiles(a), tiles(b)), _z(windows(a), windows(b))
    return {"energy_z": float(ez), "energy_rel": float(a.sum() / b.sum() * len(b) / len(a) - 1),
            "tile_max_z": float(np.abs(zt).max()), "tile_mean_z": float(zt.mean()),
            "window_max_z": float(np.abs(zw).max()), "window_mean_z": float(zw.mean())}


@pytest.mark.parametrize("train,min_roughness", [(False, None), (True, None), (True, 0.0)])
def test_guided_render_is_unbiased(gpu, train, min_roughness):
    """Untrained and trained proposals; min_roughness 0 guides the GGX floor's vertices too (by
    default only rougher GGX and Lambertian vertices are guided)."""
    sc = guided_scene()
    K = 40
    plain, _ = _films(gpu, sc, K, 64)
    g = gpu.Guide(seed=5)
    try:
        guided, st = _films(gpu, sc, K, 64, guide=g, train_pool=32768 if train else 0, min_roughness=min_roughness)
    finally:
        g.close()
    r = _compare(guided, plain)
    assert abs(r["energy_z"]) < 4.0 and abs(r["energy_rel"]) < 0.05, r
    assert r["tile_max_z"] < 4.5 and r["window_max_z"] < 4.5, r
    if train:
        assert st["train_steps"] >= 1 and np.isfinite(st["train_loss"])


def test_guided_render_on_wave_lanes_is_unbiased_and_trains(gpu):
    # 96 x 96 pixels x 1024 samples per render: five pixel batches dealt to the wave lanes,
    # several of them filling the training pool at once (entries tagged by batch)
    sc = guided_scene(96, 96, 128, 0.04)
    K = 20
    plain, _ = _films(gpu, sc, K, 1024)
    g = gpu.Guide(seed=7)
    try:
        guided, st = _films(gpu, sc, K, 1024, guide=g, train_pool=65536)
    finally:
        g.close()
    r = _compare(guided, plain, tile=16, window=16)
    assert abs(r["energy_z"]) < 4.0 and abs(r["energy_rel"]) < 0.02, r
    assert r["tile_max_z"] < 4.5 and r["window_max_z"] < 4.5, r
    assert st["train_steps"] >= 1 and np.isfinite(st["train_loss"])


def test_guided_training_updates_the_network(gpu):
    """Each render call trains the proposal on the previous call's samples (beside its own
    rendering), so the first call trains nothing and every later one at least one step."""
    sc = guided_scene(64, 64, 128, 0.04)
    g = gpu.Guide(seed=9)
    try:
        p0 = g.params()
        with gpu.Context(sc) as ctx:
            ctx.set_guide(g, mix_prob=0.5, learning_rate=1e-3, train_pool=65536)
            losses = []
            for k in range(6):
                ctx.render(16 * k, 16)
                st = ctx.stats()
                if k == 0:
                    assert st["train_steps"] == 0
                    assert np.array_equal(g.params(), p0)
                    continue
                assert st["train_steps"] >= 1
                losses.append(st["train_loss"])
            f = ctx.film()
        p1 = g.params()
    finally:
        g.close()
    assert np.isfinite(losses).all()
    assert np.abs(p1 - p0).max() > 1e-4
    assert np.isfinite(f["streak"]).all() and f["streak"].sum() > 0


def test_guide_requires_orthonormal_frame(gpu):
    sc = S.guided(width=16, height=16, time_bins=64, exposure=0.08, sqrt_spp=2)
    g = gpu.Guide()
    try:
        with gpu.Context(sc) as ctx:
            with pytest.raises(gpu.TransientError):
                ctx.set_guide(g)
    finally:
        g.close()


def test_trained_proposal_lowers_the_film_error_at_equal_samples(gpu):
    """What the learned proposal gains: on a small version of the guided workload (GGX floor,
    small area light hidden above an occluder slab, so indirect light dominates), after online
    training on the renderer's own samples, a film of N samples per pixel drawn with the trained
    proposal has a clearly lower rel-L2 error against a converged plain render than a film of
    the same N samples drawn with plain BSDF sampling (both on the same pixels, both unbiased)."""
    import torch
    from jarabotransientrendering_b200 import convergence as CV, renderer as R
    sc = S.guided(width=64, height=64, time_bins=256, exposure=0.02, sqrt_spp=4, max_bounces=6)
    sc.flags = S.FLAG_ORTHONORMAL_FRAME
    ref = CV.Reference(sc, 16384)               # 2 x 16,384 spp plain (its own noise is subtracted)
    n_spp = 1024
    with R.Context(sc, 0) as ctx:                 # plain BSDF sampling
        ctx.render(1 << 20, n_spp)
        err_plain = ref.rel_l2(CV.film_device(ctx), n_spp)
    g = R.Guide(device=0, seed=1)
    try:
        with R.Context(sc, 0) as ctx:
            ctx.set_guide(g, mix_prob=0.7, learning_rate=3e-3, train_pool=65536)
            s = 1 << 21
            for _ in range(48):                   # online training on 48 passes of 64 spp
                ctx.render(s, 64)
                s += 64
            ctx.clear()
            for _ in range(n_spp // 64):          # the measured film, still training
                ctx.render(s, 64)
                s += 64
            err_guided = ref.rel_l2(CV.film_device(ctx), n_spp)
    finally:
        g.close()
    del ref
    torch.cuda.empty_cache()
    print(f"rel-L2 at {n_spp} spp: plain {err_plain:.4f}, guided {err_guided:.4f}")
    assert err_guided < 0.8 * err_plain, (err_plain, err_guided)
