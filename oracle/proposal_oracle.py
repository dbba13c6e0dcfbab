"""CPU oracle for the learned pose proposal's network (float64 NumPy).

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` as the checker, never by the product path.

The network has no counterpart in the reference (it is this build's learned stage in front of
the sweep): a circular 1-D CNN over the coarse sweep landscape, x [n][6][36] → conv 6→32 (k 5),
ReLU, conv 32→32 (k 5), ReLU, conv 32→90 (k 3) → [n][90][36], read position-major as 3240
logits (index 90·i + o, position i, channel o), the softmax cross-entropy over them. Each convolution is circular over the 36 positions:
y[c][l] = b[c] + Σ_j Σ_k w[c][j][k] x[j][(l + k − K//2) mod 36]. The parameter vector holds each
layer's weights [co][ci][k] then its bias, layer by layer.
"""
from __future__ import annotations

import numpy as np

L = 36
LAYERS = ((6, 32, 5), (32, 32, 5), (32, 90, 3))


def nparams():
    return sum(co * ci * k + co for ci, co, k in LAYERS)


def unpack(p):
    p = np.asarray(p, np.float64)
    out, o = [], 0
    for ci, co, k in LAYERS:
        w = p[o:o + co * ci * k].reshape(co, ci, k)
        o += co * ci * k
        b = p[o:o + co]
        o += co
        out.append((w, b))
    return out


def _shift_stack(x, K):
    """xs[n][ci][k][l] = x[n][ci][(l + k − K//2) mod L]"""
    return np.stack([np.roll(x, -(k - K // 2), axis=-1) for k in range(K)], axis=2)


def forward(p, x):
    """(logits [n][3240], the layers' inputs and pre-activations for backward)."""
    x = np.asarray(x, np.float64)
    cache = []
    a = x
    layers = unpack(p)
    for li, (w, b) in enumerate(layers):
        xs = _shift_stack(a, w.shape[2])
        z = np.einsum("cjk,njkl->ncl", w, xs) + b[None, :, None]
        cache.append((a, xs, z))
        a = np.maximum(z, 0.0) if li < len(layers) - 1 else z
    return a.transpose(0, 2, 1).reshape(len(x), -1), cache


def loss_grad(p, x, labels):
    """(per-sample loss [n], ∇ of the mean loss over the parameters)."""
    logits, cache = forward(p, x)
    n = len(labels)
    m = logits.max(1, keepdims=True)
    e = np.exp(logits - m)
    se = e.sum(1, keepdims=True)
    loss = (np.log(se) + m)[:, 0] - logits[np.arange(n), labels]
    dz = e / se
    dz[np.arange(n), labels] -= 1.0
    dz /= n
    d = dz.reshape(n, L, LAYERS[-1][1]).transpose(0, 2, 1)
    grads = []
    layers = unpack(p)
    for li in range(len(layers) - 1, -1, -1):
        w, _ = layers[li]
        _, xs, z = cache[li]
        if li < len(layers) - 1:
            d = d * (z > 0)
        grads.append((np.einsum("ncl,njkl->cjk", d, xs), d.sum((0, 2))))
        K = w.shape[2]
        # dx[n][j][m] = Σ_c Σ_k w[c][j][k] d[n][c][(m − k + K//2) mod L]
        dxs = np.einsum("cjk,ncl->njkl", w, d)
        d = sum(np.roll(dxs[:, :, k, :], k - K // 2, axis=-1) for k in range(K))
    g = []
    for dw, db in reversed(grads):
        g += [dw.ravel(), db]
    return loss, np.concatenate(g)


def init_params(seed=0):
    """He-initialised weights and zero biases (a starting point for the tests)."""
    rng = np.random.default_rng(seed)
    out = []
    for ci, co, k in LAYERS:
        out += [rng.standard_normal(co * ci * k) * np.sqrt(2.0 / (ci * k)), np.zeros(co)]
    return np.concatenate(out).astype(np.float32)
