"""GPU tests of multi-scene batches (tr_batch_*): several contexts rendered in shared wavefront
batches replayed from a captured CUDA graph.  Each scene's film must equal the film of rendering
that context alone over the same sample range (same per-path random streams; sums differ only by
the grouping of FP32 warp sums and the order of FP64 film additions), whatever the queue
capacity, shade block, pixels per splat block or graph use; the autotuner must return a valid configuration; a learned proposal shared by
the batch must leave every scene's estimate unbiased."""
import numpy as np
import pytest

from jarabotransientrendering_b200 import scenes as S

pytestmark = pytest.mark.gpu

RTOL = 2e-5


def small_scenes():
    a = S.cornell(width=64, height=48, time_bins=128, exposure=0.04, sqrt_spp=2, max_bounces=5)
    b = S.medium(width=48, height=48, time_bins=256, exposure=0.02, sqrt_spp=2, incoming_samples=2, max_bounces=7)
    c = S.icosphere(subdiv=3, width=64, height=64, time_bins=64, exposure=0.08, sqrt_spp=2, max_bounces=6)
    d = S.guided(width=32, height=32, time_bins=96, exposure=0.05, sqrt_spp=2)
    for sc in (a, b, c, d):
        sc.flags = S.FLAG_ORTHONORMAL_FRAME
    return [a, b, c, d]


def _single_films(gpu, scs, begins, counts):
    out = []
    for sc, b0, n in zip(scs, begins, counts):
        with gpu.Context(sc) as c:
            if n:
                c.render(b0, n)
            out.append(c.film())
    return out


def _check_same(films, singles):
    for f, s in zip(films, singles):
        assert ((f["streak"] != 0) == (s["streak"] != 0)).all()
        assert np.allclose(f["streak"], s["streak"], rtol=RTOL, atol=1e-12)
        assert np.allclose(f["steady"], s["steady"], rtol=RTOL, atol=1e-12)
        assert (f["weight"] == s["weight"]).all()


@pytest.mark.parametrize("cfg", [dict(capacity=1 << 21, use_graph=1),
                                 dict(capacity=65536, use_graph=1),
                                 dict(capacity=65536, use_graph=0, shade_block=128, splat_div=2),
                                 dict(capacity=131072, use_graph=1, shade_block=128, splat_div=4)])
def test_batch_matches_single_contexts(gpu, cfg):
    scs = small_scenes()
    begins, counts = [0, 3, 1, 2], [16, 5, 6, 4]
    singles = _single_films(gpu, scs, begins, counts)
    ctxs = [gpu.Context(sc) for sc in scs]
    try:
        with gpu.Batch(ctxs) as B:
            B.set_config(**cfg)
            B.render(begins, counts)
            st = B.stats()
        films = [c.film() for c in ctxs]
    finally:
        for c in ctxs:
            c.close()
    _check_same(films, singles)
    assert st["paths"] == sum(sc.width * sc.height * n * sc.incoming_samples for sc, n in zip(scs, counts))
    assert st["kernel_launches"] > 0


def test_batch_repeated_calls_reuse_the_graph(gpu):
    """Two calls with the same plan shape replay one graph; a third with other counts recaptures."""
    scs = small_scenes()
    ctxs = [gpu.Context(sc) for sc in scs]
    try:
        with gpu.Batch(ctxs) as B:
            B.set_config(capacity=65536, use_graph=1)
            B.render([0, 0, 0, 0], [4, 4, 4, 4])
            B.render([4, 4, 4, 4], [4, 4, 4, 4])
            B.render([8, 8, 8, 8], [1, 0, 2, 3])
        films = [c.film() for c in ctxs]
    finally:
        for c in ctxs:
            c.close()
    singles = _single_films(gpu, scs, [0, 0, 0, 0], [9, 8, 10, 11])
    _check_same(films, singles)


def test_batch_autotune(gpu):
    scs = small_scenes()
    ctxs = [gpu.Context(sc) for sc in scs]
    try:
        with gpu.Batch(ctxs) as B:
            best, trials = B.autotune(0, 1)
            assert trials >= 6
            assert best["capacity"] in (1 << 19, 1 << 20, 1 << 21, 1 << 22)
            assert best["shade_block"] in (128, 256) and best["splat_div"] in (1, 2, 4)
            assert B.config() == best
            B.render(trials, 2)
        films = [c.film() for c in ctxs]
    finally:
        for c in ctxs:
            c.close()
    singles = _single_films(gpu, scs, [0] * 4, [trials + 2] * 4)
    _check_same(films, singles)


def test_batch_guided_is_unbiased(gpu):
    scs = small_scenes()[::3]            # Cornell + the guided scene
    K = 24
    plain = [[], []]
    for k in range(K):
        for i, sc in enumerate(scs):
            with gpu.Context(sc) as c:
                c.render(16 * k, 16)
                plain[i].append(c.film(steady=False, weight=False)["streak"].sum())
    g = gpu.Guide(seed=4)
    guided = [[], []]
    ctxs = [gpu.Context(sc) for sc in scs]
    try:
        with gpu.Batch(ctxs) as B:
            B.set_guide(g, mix_prob=0.7, learning_rate=3e-3, train_pool=32768)
            for k in range(K):
                for c in ctxs:
                    c.clear()
                B.render(1000 + 16 * k, 16)
                for i, c in enumerate(ctxs):
                    guided[i].append(c.film(steady=False, weight=False)["streak"].sum())
            st = B.stats()
    finally:
        for c in ctxs:
            c.close()
        g.close()
    assert st["train_steps"] >= 1
    for i in range(2):
        a, b = np.array(guided[i]), np.array(plain[i])
        z = (a.mean() - b.mean()) / np.sqrt(a.var(ddof=1) / K + b.var(ddof=1) / K)
        assert abs(z) < 4.0, (i, z, a.mean() / b.mean())


def test_batch_errors(gpu):
    sc = S.cornell(width=16, height=16, time_bins=32, exposure=0.16, sqrt_spp=1)
    ctxs = [gpu.Context(sc) for _ in range(17)]
    try:
        with pytest.raises(gpu.TransientError):
            gpu.Batch(ctxs)
        with gpu.Batch(ctxs[:2]) as B:
            with pytest.raises(gpu.TransientError):
                B.set_config(capacity=1000)
            with pytest.raises(gpu.TransientError):
                B.set_config(shade_block=96)
            g = gpu.Guide()
            try:
                with pytest.raises(gpu.TransientError):       # contexts lack orthonormal frames
                    B.set_guide(g)
            finally:
                g.close()
            B.render([0, 0], [1, 0])
    finally:
        for c in ctxs:
            c.close()
