"""TEST INFRASTRUCTURE ONLY -- float64 numpy restatement of the surrogate MLP (10 -> 64 -> 64 -> 6,
tanh-form GELU) and of its normalised mean-squared-error loss, with hand-derived gradients.

It checks the library's GPU training kernels (``pm_mlp_loss_grad``) and tensor-core inference
(``pm_mlp_infer``); its own gradients are checked against finite differences.

Parameter vector layout (5286 floats):
    in_mean[10] in_std[10] out_mean[6] out_std[6] W1[64][10] b1[64] W2[64][64] b2[64] W3[6][64] b3[6]
"""
from __future__ import annotations

import numpy as np

NPARAMS = 5286
O_IM, O_IS, O_OM, O_OS = 0, 10, 20, 26
O_W1 = 32
O_B1 = O_W1 + 640
O_W2 = O_B1 + 64
O_B2 = O_W2 + 4096
O_W3 = O_B2 + 64
O_B3 = O_W3 + 384
K0, K1 = 0.7978845608028654, 0.044715


def unpack(p):
    p = np.asarray(p, np.float64)
    return dict(im=p[O_IM:O_IM + 10], isd=p[O_IS:O_IS + 10], om=p[O_OM:O_OM + 6], osd=p[O_OS:O_OS + 6],
                W1=p[O_W1:O_B1].reshape(64, 10), b1=p[O_B1:O_W2], W2=p[O_W2:O_B2].reshape(64, 64), b2=p[O_B2:O_W3],
                W3=p[O_W3:O_B3].reshape(6, 64), b3=p[O_B3:O_B3 + 6])


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(K0 * (z + K1 * z ** 3)))


def gelu_grad(z):
    t = np.tanh(K0 * (z + K1 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * K0 * (1.0 + 3.0 * K1 * z * z)


def forward(p, x):
    """Raw features x[n,10] -> normalised outputs [n,6] and the intermediates."""
    w = unpack(p)
    xn = (np.asarray(x, np.float64) - w["im"]) / w["isd"]
    z1 = xn @ w["W1"].T + w["b1"]
    h1 = gelu(z1)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = gelu(z2)
    y = h2 @ w["W3"].T + w["b3"]
    return y, dict(xn=xn, z1=z1, h1=h1, z2=z2, h2=h2)


def predict(p, x):
    """Raw outputs [n,6]."""
    w = unpack(p)
    y, _ = forward(p, x)
    return y * w["osd"] + w["om"]


def loss_grad(p, x, t):
    """Mean over batch and outputs of (y - (t - out_mean)/out_std)^2 and its gradient."""
    w = unpack(p)
    y, c = forward(p, x)
    tn = (np.asarray(t, np.float64) - w["om"]) / w["osd"]
    d = y - tn
    n = d.size
    loss = float((d * d).sum() / n)
    dy = 2.0 * d / n
    g = np.zeros(NPARAMS)
    g[O_W3:O_B3] = (dy.T @ c["h2"]).ravel()
    g[O_B3:O_B3 + 6] = dy.sum(0)
    dz2 = (dy @ w["W3"]) * gelu_grad(c["z2"])
    g[O_W2:O_B2] = (dz2.T @ c["h1"]).ravel()
    g[O_B2:O_W3] = dz2.sum(0)
    dz1 = (dz2 @ w["W2"]) * gelu_grad(c["z1"])
    g[O_W1:O_B1] = (dz1.T @ c["xn"]).ravel()
    g[O_B1:O_W2] = dz1.sum(0)
    return loss, g


def init_params(x, t, seed=0):
    """Statistics from the data, He-normal weights, zero biases (same recipe as the library)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAMS)
    x = np.asarray(x, np.float64)
    t = np.asarray(t, np.float64)
    p[O_IM:O_IM + 10] = x.mean(0)
    s = x.std(0)
    p[O_IS:O_IS + 10] = np.where(s > 1e-10, s, 1.0)
    p[O_OM:O_OM + 6] = t.mean(0)
    s = t.std(0)
    p[O_OS:O_OS + 6] = np.where(s > 1e-15, s, 1.0)
    p[O_W1:O_B1] = rng.normal(0, np.sqrt(2 / 10), 640)
    p[O_W2:O_B2] = rng.normal(0, np.sqrt(2 / 64), 4096)
    p[O_W3:O_B3] = rng.normal(0, np.sqrt(2 / 64), 384)
    return p.astype(np.float32)
