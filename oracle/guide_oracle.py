"""CPU oracle of the learned directional proposal (test infrastructure; no reference counterpart).

numpy restatement of the proposal network and its training step, rounding to BF16 at the same
points as the CUDA kernels: features, weights and hidden activations are BF16, products are
accumulated in FP32 (here: float64, then compared with a tolerance), and the gradients w.r.t.
each layer's outputs are BF16 both where they feed the next backward layer and where they are
the weight-gradient GEMM's operand (the tensor-core kernel k_dw_tc: BF16 x BF16 -> FP32).

Mixture of 8 von Mises-Fisher lobes (per lobe: weight logit, unnormalised mean, concentration
kappa = 0.05 + 2000 sigmoid(k - 8), log-like below a few hundred and smoothly saturating at
2000); density vMF(w; mu, kappa) =
kappa / (2 pi (1 - exp(-2 kappa))) * exp(kappa (mu.w - 1)); sampling follows Jakob 2012
("Numerically stable sampling of the von Mises Fisher distribution on S^2").
"""
from __future__ import annotations

import numpy as np

NP = 16640
KMIN, KMAX = 0.05, 2000.0
KSHIFT = 8.0
LOBES = 8


def bf16(x):
    """Round float32 values to bfloat16 (round to nearest even), returned as float32."""
    a = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    lsb = (a >> 16) & 1
    r = ((a + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(np.shape(x))


def to_bf16_bits(x):
    return (bf16(x).view(np.uint32) >> 16).astype(np.uint16)


def unpack(params):
    p = np.asarray(params, np.float32)
    W = p[:4 * 4096].reshape(4, 64, 64)          # [layer][in][out]
    b = p[4 * 4096:].reshape(4, 64)
    return W, b


def forward(params, x):
    """x: [n][64] float32 already BF16-valued. Returns out [n][40], activations H1..H3 (BF16)."""
    W, b = unpack(params)
    Wb = bf16(W).astype(np.float64)
    h = x.astype(np.float64)
    acts = []
    for l in range(3):
        z = h @ Wb[l] + b[l]
        h = bf16(np.maximum(z, 0.0).astype(np.float32)).astype(np.float64)
        acts.append(h.astype(np.float32))
    out = (h @ Wb[3] + b[3])[:, :40]
    return out.astype(np.float32), acts


def sigmoid(x):
    return 0.5 * (1.0 + np.tanh(0.5 * x))


def decode(out):
    o = np.asarray(out, np.float64).reshape(-1, LOBES, 5)
    a = o[..., 0]
    pi = np.exp(a - a.max(axis=1, keepdims=True))
    pi /= pi.sum(axis=1, keepdims=True)
    m = o[..., 1:4]
    n = np.linalg.norm(m, axis=2, keepdims=True)
    mu = np.where(n > 1e-6, m / np.maximum(n, 1e-30), np.array([0.0, 0.0, 1.0]))
    n = np.maximum(n, 1e-6)
    s = sigmoid(o[..., 4] - KSHIFT)
    kappa = KMIN + KMAX * s
    dkappa = KMAX * s * (1.0 - s)                 # d kappa / d raw
    return pi, mu, n[..., 0], kappa, dkappa


def log_vmf(kappa, c):
    return np.log(kappa) - np.log(2 * np.pi) - np.log1p(-np.exp(-2 * kappa)) + kappa * (c - 1.0)


def mixture_logpdf(out, dirs):
    pi, mu, _, kappa, _ = decode(out)
    c = np.einsum("nld,nd->nl", mu, dirs)
    lg = np.log(np.maximum(pi, 1e-30)) + log_vmf(kappa, c)
    mx = lg.max(axis=1, keepdims=True)
    return (mx + np.log(np.exp(lg - mx).sum(axis=1, keepdims=True)))[:, 0]


def loss_and_dout(out, dirs, w):
    """loss = -sum w log q / sum w; analytic gradient w.r.t. the 40 raw outputs."""
    pi, mu, mnorm, kappa, sig = decode(out)
    dirs = np.asarray(dirs, np.float64)
    c = np.einsum("nld,nd->nl", mu, dirs)
    lg = np.log(np.maximum(pi, 1e-30)) + log_vmf(kappa, c)
    mx = lg.max(axis=1, keepdims=True)
    logq = mx + np.log(np.exp(lg - mx).sum(axis=1, keepdims=True))
    r = np.exp(lg - logq)
    scale = (np.asarray(w, np.float64) / np.sum(w))[:, None]
    loss = float(-(scale[:, 0] * logq[:, 0]).sum())
    g = np.zeros((len(out), LOBES, 5))
    g[..., 0] = -scale * (r - pi)
    cc = r * kappa / mnorm
    g[..., 1:4] = -(scale * cc)[..., None] * (dirs[:, None, :] - c[..., None] * mu)
    e2 = np.exp(-2 * kappa)
    dlogv = 1.0 / kappa - 2 * e2 / (1 - e2) + (c - 1.0)
    g[..., 4] = -scale * r * dlogv * sig
    return loss, g.reshape(len(out), 40)


def gradients(params, x, dirs, w):
    """Gradients of the loss w.r.t. all parameters, quantised like the CUDA kernels."""
    W, b = unpack(params)
    Wb = bf16(W).astype(np.float64)
    out, acts = forward(params, x)
    loss, dout = loss_and_dout(out, dirs, w)
    dy = np.zeros((len(x), 64))
    dy[:, :40] = dout
    dy_b = bf16(dy.astype(np.float32)).astype(np.float64)
    H = [x.astype(np.float64)] + [a.astype(np.float64) for a in acts]
    gW = np.zeros((4, 64, 64))
    gb = np.zeros((4, 64))
    gW[3] = H[3].T @ dy_b
    gb[3] = dy_b.sum(axis=0)
    g_in = dy_b
    for l in (3, 2, 1):
        dh = (g_in @ Wb[l].T) * (H[l] > 0)
        g_in = bf16(dh.astype(np.float32)).astype(np.float64)
        gW[l - 1] = H[l - 1].T @ g_in
        gb[l - 1] = g_in.sum(axis=0)
    return loss, np.concatenate([gW.reshape(-1), gb.reshape(-1)]).astype(np.float32)


def adam(params, grads, m1, m2, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m1 = b1 * m1 + (1 - b1) * grads
    m2 = b2 * m2 + (1 - b2) * grads * grads
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    return params - lr * (m1 / c1) / (np.sqrt(m2 / c2) + eps), m1, m2


def sample_vmf(mu, kappa, u1, u2):
    """Jakob 2012: w = 1 + log(u1 + (1 - u1) exp(-2 kappa)) / kappa, azimuth 2 pi u2."""
    w = 1.0 + np.log(u1 + (1.0 - u1) * np.exp(-2.0 * kappa)) / kappa
    s = np.sqrt(np.maximum(0.0, 1.0 - w * w))
    sg = np.copysign(1.0, mu[..., 2])
    a = -1.0 / (sg + mu[..., 2])
    b = mu[..., 0] * mu[..., 1] * a
    t1 = np.stack([1.0 + sg * mu[..., 0] ** 2 * a, sg * b, -sg * mu[..., 0]], -1)
    t2 = np.stack([b, sg + mu[..., 1] ** 2 * a, -mu[..., 1]], -1)
    phi = 2 * np.pi * u2
    return w[..., None] * mu + s[..., None] * (np.cos(phi)[..., None] * t1 + np.sin(phi)[..., None] * t2)
