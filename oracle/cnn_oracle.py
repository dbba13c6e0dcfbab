"""Test infrastructure: a float64 NumPy restatement of the 2-D convolutional pose proposal
(zcmir_b200/csrc/cnn.cu), the checker of its GPU forward and backward passes.

The network has no counterpart in the reference (its learned proposal is this build's own
addition). With bf16=True the restatement rounds at the points where the GPU kernels round to
BF16 (weights, each ReLU output, each layer's pre-activation gradient) and sums in float64
where the GPU sums in float32; with bf16=False it is the plain float64 network, whose backward
pass the tests check against central differences.

Layout: samples NHWC [n][128][128][8]; parameters as zcb_cnn_nparams() documents.
"""
import numpy as np

CH = (8, 32, 64, 64, 128)
BINS, FEAT = 216, 128


def n_params():
    n = 0
    for l in range(4):
        n += CH[l + 1] * 9 * CH[l] + CH[l + 1]
    return n + BINS * FEAT + BINS


def unpack(params):
    """[(W [Co][9][Ci], b [Co]) × 4], Wfc [216][128], bfc [216] as float64 views of params."""
    p = np.asarray(params, np.float64)
    out, o = [], 0
    for l in range(4):
        co, ci = CH[l + 1], CH[l]
        W = p[o:o + co * 9 * ci].reshape(co, 9, ci)
        o += co * 9 * ci
        out.append((W, p[o:o + co]))
        o += co
    Wfc = p[o:o + BINS * FEAT].reshape(BINS, FEAT)
    o += BINS * FEAT
    return out, Wfc, p[o:o + BINS]


def bf16_round(x):
    """float → the nearest BF16 value (round to nearest even), as float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits(x):
    """float → BF16 bit patterns (uint16), rounded to nearest even: the GPU's input format."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def from_bits(b):
    return (np.asarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def _taps(a):
    """The nine stride-2 views of a zero-padded [n][H][W][C]: tap (ky, kx) → [n][H/2][W/2][C]."""
    n, H, W, C = a.shape
    ap = np.zeros((n, H + 2, W + 2, C))
    ap[:, 1:H + 1, 1:W + 1] = a
    return [ap[:, ky:ky + H:2, kx:kx + W:2, :] for ky in range(3) for kx in range(3)]


def forward(params, x, bf16=True):
    """Logits [n][216] and the cache for backward(); x: [n][128][128][8] values (BF16-exact when
    bf16, as the GPU reads them)."""
    r = bf16_round if bf16 else (lambda v: np.asarray(v, np.float64))
    layers, Wfc, bfc = unpack(params)
    acts = [np.asarray(x, np.float64)]
    for W, b in layers:
        Wr = r(W)
        z = sum(t @ Wr[:, k, :].T for k, t in enumerate(_taps(acts[-1]))) + b
        acts.append(r(np.maximum(z, 0.0)))
    h = acts[-1].mean(axis=(1, 2))
    logits = h @ r(Wfc).T + bfc
    return logits, (acts, h)


def loss_grad(params, x, labels, bf16=True):
    """Mean softmax cross-entropy and its gradient over params (float64, params' layout)."""
    r = bf16_round if bf16 else (lambda v: np.asarray(v, np.float64))
    layers, Wfc, _ = unpack(params)
    logits, (acts, h) = forward(params, x, bf16)
    n = len(labels)
    z = logits - logits.max(axis=1, keepdims=True)
    p = np.exp(z)
    p /= p.sum(axis=1, keepdims=True)
    loss = float(np.mean(-np.log(p[np.arange(n), labels])))
    d = p.copy()
    d[np.arange(n), labels] -= 1.0
    d /= n
    grads = []
    gWfc, gbfc = d.T @ h, d.sum(axis=0)
    dh = d @ r(Wfc)
    a4 = acts[4]
    dz = r((a4 > 0) * (dh[:, None, None, :] / 64.0))
    for l in range(3, -1, -1):
        W, _ = layers[l]
        taps = _taps(acts[l])
        gW = np.stack([np.einsum("nyxo,nyxi->oi", dz, t) for t in taps], axis=1)
        grads.append((gW, dz.sum(axis=(0, 1, 2))))
        if l == 0:
            break
        n_, H, Wd, Ci = acts[l].shape
        Wr = r(W)
        dap = np.zeros((n_, H + 2, Wd + 2, Ci))
        for k in range(9):
            ky, kx = divmod(k, 3)
            dap[:, ky:ky + H:2, kx:kx + Wd:2, :] += dz @ Wr[:, k, :]
        da = dap[:, 1:H + 1, 1:Wd + 1]
        dz = r((acts[l] > 0) * da)
    grads = grads[::-1]
    flat = []
    for gW, gb in grads:
        flat += [gW.ravel(), gb]
    flat += [gWfc.ravel(), gbfc]
    return loss, np.concatenate(flat)


def init_params(seed=0):
    """He-scaled random weights, zero biases (float32)."""
    rng = np.random.default_rng(seed)
    parts = []
    for l in range(4):
        co, ci = CH[l + 1], CH[l]
        parts += [rng.standard_normal(co * 9 * ci) * np.sqrt(2.0 / (9 * ci)), np.zeros(co)]
    parts += [rng.standard_normal(BINS * FEAT) * np.sqrt(1.0 / FEAT), np.zeros(BINS)]
    return np.concatenate(parts).astype(np.float32)
