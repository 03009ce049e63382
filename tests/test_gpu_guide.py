"""GPU tests of the learned directional proposal (BF16 tcgen05 MLP forward/backward, vMF-mixture
loss, Adam) through the C ABI, against the numpy oracle (oracle/guide_oracle.py)."""
import ctypes as C

import numpy as np
import pytest

from jarabotransientrendering_b200 import _abi
from oracle import guide_oracle as G

pytestmark = pytest.mark.gpu


def _guide(seed=1):
    h = C.c_void_p()
    _abi.check(_abi.lib().tr_guide_create(0, seed, C.byref(h)))
    return h


def _dev(a, dtype):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dtype=dtype, device="cuda")


def _features(rng, n):
    x = G.bf16(rng.normal(0.0, 1.0, (n, 64)).astype(np.float32))
    x[:, 46:] = 0.0
    return x


def _bits(x):
    import torch
    return torch.from_numpy(G.to_bf16_bits(x).view(np.int16)).cuda()


def _ready():
    """Inputs and outputs are made on torch's stream; the guide's entry points called with a
    NULL stream run on the guide's own stream, which is not ordered after torch's work."""
    import torch
    torch.cuda.synchronize()


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 65536])
def test_forward_matches_oracle(gpu, n):
    import torch
    rng = np.random.default_rng(n)
    params = rng.normal(0, 0.15, G.NP).astype(np.float32)
    x = _features(rng, n)
    g = _guide()
    try:
        _abi.check(_abi.lib().tr_guide_set_params(g, params.ctypes.data))
        xd = _bits(x)
        out = torch.zeros((n, 40), dtype=torch.float32, device="cuda")
        _ready()
        _abi.check(_abi.lib().tr_guide_forward(g, C.c_void_p(xd.data_ptr()), n, C.c_void_p(out.data_ptr()), None))
        got = out.cpu().numpy()
    finally:
        _abi.lib().tr_guide_destroy(g)
    ref, _ = G.forward(params, x)
    scale = np.abs(ref).max() + 1e-6
    # BF16 hidden activations may round differently where FP32 sums differ in the last bits
    assert np.abs(got - ref).max() <= 2e-2 * scale, np.abs(got - ref).max() / scale
    assert np.abs(got - ref).mean() <= 1e-3 * scale


def test_gradients_match_oracle(gpu):
    import torch
    rng = np.random.default_rng(7)
    n = 4096
    params = rng.normal(0, 0.15, G.NP).astype(np.float32)
    x = _features(rng, n)
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    w = (rng.random(n) + 0.05).astype(np.float32)
    g = _guide()
    try:
        _abi.check(_abi.lib().tr_guide_set_params(g, params.ctypes.data))
        xd = _bits(x)
        dd = _dev(dirs.astype(np.float32), torch.float32)
        wd = _dev(w, torch.float32)
        loss = C.c_float()
        _ready()
        _abi.check(_abi.lib().tr_guide_train_step(g, C.c_void_p(xd.data_ptr()), C.c_void_p(dd.data_ptr()),
                                                  C.c_void_p(wd.data_ptr()), n, 0.0, C.byref(loss), None))
        grads = np.zeros(G.NP, np.float32)
        _abi.check(_abi.lib().tr_guide_get_grads(g, grads.ctypes.data))
    finally:
        _abi.lib().tr_guide_destroy(g)
    ref_loss, ref = G.gradients(params, x, dirs, w)
    assert abs(loss.value - ref_loss) <= 1e-3 * abs(ref_loss) + 1e-4
    for l in range(4):
        a, b = grads[l * 4096:(l + 1) * 4096], ref[l * 4096:(l + 1) * 4096]
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-12)
        assert rel < 0.05, (l, rel)
    gb, rb = grads[4 * 4096:], ref[4 * 4096:]
    assert np.linalg.norm(gb - rb) / (np.linalg.norm(rb) + 1e-12) < 0.05


def test_training_fits_a_feature_dependent_distribution(gpu):
    """Online-style training (Adam, lr 1e-3, batches of 65,536): on directions drawn from a
    vMF lobe whose mean depends on the input features, the loss drops well below the loss of
    the initial (broad) mixture; one Adam step matches the oracle's Adam."""
    import torch
    rng = np.random.default_rng(11)
    n = 65536
    g = _guide(seed=3)
    try:
        p0 = np.zeros(G.NP, np.float32)
        _abi.check(_abi.lib().tr_guide_get_params(g, p0.ctypes.data))
        losses = []
        for it in range(150):
            x = np.zeros((n, 64), np.float32)
            ang = rng.random(n) * 2 * np.pi
            x[:, 0], x[:, 1] = np.sin(ang), np.cos(ang)
            x = G.bf16(x)
            mu = np.stack([np.cos(ang), np.sin(ang), np.zeros(n)], 1)
            dirs = G.sample_vmf(mu, np.full(n, 20.0), rng.random(n), rng.random(n))
            w = np.ones(n, np.float32)
            xd, dd, wd = _bits(x), _dev(dirs.astype(np.float32), torch.float32), _dev(w, torch.float32)
            loss = C.c_float()
            _ready()
            _abi.check(_abi.lib().tr_guide_train_step(g, C.c_void_p(xd.data_ptr()), C.c_void_p(dd.data_ptr()),
                                                      C.c_void_p(wd.data_ptr()), n, 1e-3, C.byref(loss), None))
            losses.append(loss.value)
            if it == 0:
                p1 = np.zeros(G.NP, np.float32)
                _abi.check(_abi.lib().tr_guide_get_params(g, p1.ctypes.data))
                gr = np.zeros(G.NP, np.float32)
                _abi.check(_abi.lib().tr_guide_get_grads(g, gr.ctypes.data))
                exp, _, _ = G.adam(p0, gr, np.zeros(G.NP), np.zeros(G.NP), 1, 1e-3)
                assert np.allclose(p1, exp, atol=1e-6, rtol=1e-5)
    finally:
        _abi.lib().tr_guide_destroy(g)
    # uniform density on the sphere has -log q = log(4 pi) = 2.53; a kappa-20 lobe has ~-0.58
    assert losses[0] > 1.5
    assert np.mean(losses[-10:]) < losses[0] - 1.5, (losses[0], losses[-10:])


def test_guide_errors(gpu):
    g = _guide()
    try:
        rc = _abi.lib().tr_guide_train_step(g, None, None, None, 0, 1e-3, None, None)
        assert rc == 1
    finally:
        _abi.lib().tr_guide_destroy(g)


def test_wait_timeout_is_reported_and_the_guide_recovers(gpu):
    """With a wait limit of 0 every tensor-core completion wait gives up at once: the forward
    pass, a training step and a guided render each return TR_ERR_TIMEOUT (the kernels first let
    their in-flight MMAs land and free their tensor memory); with the limit restored, the same
    guide and context compute correct results again."""
    import torch
    import jarabotransientrendering_b200 as T
    from jarabotransientrendering_b200 import renderer as R, scenes as S
    L = _abi.lib()
    rng = np.random.default_rng(5)
    n = 1000
    params = rng.normal(0, 0.15, G.NP).astype(np.float32)
    x = _features(rng, n)
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    w = (rng.random(n) + 0.05).astype(np.float32)
    g = _guide()
    try:
        _abi.check(L.tr_guide_set_params(g, params.ctypes.data))
        xd = _bits(x)
        dd = _dev(dirs.astype(np.float32), torch.float32)
        wd = _dev(w, torch.float32)
        out = torch.zeros((n, 40), dtype=torch.float32, device="cuda")
        _ready()
        _abi.check(L.tr_guide_set_wait_limit(g, 0))
        assert L.tr_guide_forward(g, C.c_void_p(xd.data_ptr()), n, C.c_void_p(out.data_ptr()), None) == 5
        assert L.tr_guide_train_step(g, C.c_void_p(xd.data_ptr()), C.c_void_p(dd.data_ptr()),
                                     C.c_void_p(wd.data_ptr()), n, 0.0, None, None) == 5
        _abi.check(L.tr_guide_set_wait_limit(g, 1 << 24))
        _abi.check(L.tr_guide_forward(g, C.c_void_p(xd.data_ptr()), n, C.c_void_p(out.data_ptr()), None))
        got = out.cpu().numpy()
    finally:
        L.tr_guide_destroy(g)
    ref, _ = G.forward(params, x)
    scale = np.abs(ref).max() + 1e-6
    assert np.abs(got - ref).max() <= 2e-2 * scale

    sc = S.guided(width=32, height=32, time_bins=128, exposure=0.04, sqrt_spp=2, max_bounces=4)
    sc.flags = S.FLAG_ORTHONORMAL_FRAME
    gd = R.Guide(device=0, seed=1)
    try:
        with R.Context(sc, 0) as ctx:
            ctx.set_guide(gd, mix_prob=0.5, learning_rate=1e-3, train_pool=4096)
            _abi.check(L.tr_guide_set_wait_limit(gd.h, 0))
            with pytest.raises(T.TransientError, match="timed out"):
                ctx.render(0, sc.spp)
            _abi.check(L.tr_guide_set_wait_limit(gd.h, 1 << 24))
            ctx.clear()
            ctx.render(sc.spp, sc.spp)
            f = ctx.film()
            assert np.isfinite(f["streak"]).all() and f["streak"].sum() > 0
    finally:
        gd.close()
