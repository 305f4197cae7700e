"""FP64 numpy restatement of the warm-start MLP's forward and backward pass -- TEST INFRASTRUCTURE ONLY.

Checks the GPU kernels of taral-lp_b200/csrc/mlp.cu: the same network (W per layer in x out, GELU with the erf
form, mean squared error), with values rounded to bfloat16 at the points where the GPU stores bfloat16 (the input,
the weights, the hidden activations and the back-propagated gradients fed to the GEMMs), and everything else in FP64.
"""
import math

import numpy as np

try:
    from scipy.special import erf as _erf
except ImportError:  # pragma: no cover
    _erf = np.vectorize(math.erf)


def bf16(a):
    """Round to bfloat16 (round to nearest even), returned as float64."""
    x = np.ascontiguousarray(np.asarray(a, np.float32))
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1 + _erf(z / math.sqrt(2)))


def gelu_grad(z):
    return 0.5 * (1 + _erf(z / math.sqrt(2))) + z * np.exp(-0.5 * z * z) / math.sqrt(2 * math.pi)


def split(params, shapes):
    out, k = [], 0
    for (fi, fo), _ in shapes:
        W = params[k:k + fi * fo].reshape(fi, fo)
        k += fi * fo
        b = params[k:k + fo]
        k += fo
        out.append((np.asarray(W, np.float64), np.asarray(b, np.float64)))
    return out


def forward(params, shapes, x):
    layers = split(params, shapes)
    h = bf16(x)
    Zs, Hs = [], [h]
    for k, (W, b) in enumerate(layers):
        z = h @ bf16(W) + b
        Zs.append(z)
        if k < len(layers) - 1:
            h = bf16(gelu(z))
            Hs.append(h)
    return Zs[-1], Zs, Hs


def loss_and_grads(params, shapes, x, t):
    layers = split(params, shapes)
    y, Zs, Hs = forward(params, shapes, x)
    B, P = y.shape
    r = (y - t) * (2.0 / (B * P))
    loss = float(np.mean((y - t) ** 2))
    grads = [None] * len(layers)
    dzf, dzb = r, bf16(r)
    for k in range(len(layers) - 1, -1, -1):
        W, _ = layers[k]
        gW = Hs[k].T @ dzb
        gb = dzf.sum(axis=0)
        grads[k] = (gW, gb)
        if k > 0:
            dh = dzb @ bf16(W).T
            dzf = dh * gelu_grad(Zs[k - 1])
            dzb = bf16(dzf)
    return loss, np.concatenate([np.concatenate([g.ravel(), b]) for g, b in grads])
