"""CPU oracle for zcmir's preprocessing before the SMI features.

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` as the checker, never by the product path.

Restates, in NumPy float32 with the reference's operation order (each elementwise float32
operation rounds once, like the shaders), ZacharyVarley/zcmir's:

* RGBA8 → gray ``shaders/gls_mift.wgsl:283-291`` (``rgba_to_gray_buf``: 0.299 R + 0.587 G +
  0.114 B, channels i/255);
* CLAHE ``src/gls.zig:462-489`` with ``shaders/gls_mift.wgsl:1975-2057`` (reflected padding before
  the image, per-tile histograms, the clipped CDF with the excess spread evenly and the remainder
  to the lowest bins, the bilinear blend of the four nearest tiles);
* the band pass ``src/gls.zig:531-557`` (σ = 1 Gaussian passes ``gauss_h`` / ``gauss_v``
  293-320, clamp to edge; the difference of the fine and coarse blurs rescaled to [0, 1]) and the
  invert ``src/gls.zig:559-566``;
* the order of ``src/engine.zig:322-341`` (``bake``): CLAHE (else the raw texels), band pass,
  invert; with ``half`` every stored texel is rounded to f16.
"""
from __future__ import annotations

import math

import numpy as np

F = np.float32


def texel(a, half):
    a = np.asarray(a, F)
    return a.astype(np.float16).astype(F) if half else a


def rgba_gray(rgba):
    c = np.asarray(rgba, np.uint8).astype(F) / F(255)
    return (F(0.299) * c[..., 0] + F(0.587) * c[..., 1]) + F(0.114) * c[..., 2]


def _reflect(i, n, pad):
    x = i - pad
    if n <= 1:
        return np.zeros_like(x)
    x = np.where(x < 0, -x, x)
    x = np.where(x >= n, 2 * n - 2 - x, x)
    return np.clip(x, 0, n - 1)


def clahe(src, clip=40.0, bins=64, grid=4, half=False):
    a = np.asarray(src, F)
    h, w = a.shape
    hg = min(8, max(2, grid))
    nb = min(256, max(8, bins))
    h_pad, w_pad = (hg - h % hg) % hg, (hg - w % hg) % hg
    ph, pw = h + h_pad, w + w_pad
    h_tile, w_tile = max(1, ph // hg), max(1, pw // hg)
    yy, xx = np.mgrid[0:ph, 0:pw]
    v = np.clip(a[_reflect(yy, h, h_pad), _reflect(xx, w, w_pad)], F(0), F(1))
    bf = np.clip(v * F(nb - 1), F(0), F(nb - 1))
    bins_ = bf.astype(np.int64)
    tile = (yy // h_tile) * hg + xx // w_tile
    hist = np.bincount((tile * nb + bins_).ravel(), minlength=hg * hg * nb).reshape(hg * hg, nb)
    voxels = max(h_tile * w_tile, 1)
    limit = max(F(clip) * F(voxels) / F(nb), F(1))
    cdf = np.zeros((hg * hg, nb), F)
    for t in range(hg * hg):
        sumc = F(0)
        for i in range(nb):
            sumc = F(sumc + min(F(hist[t, i]), limit))
        clipped = F(F(voxels) - sumc)
        fnb = F(nb)
        residual = int(F(clipped - F(fnb * F(math.floor(F(clipped / fnb))))))
        redist = F(F(clipped - F(residual)) / fnb)
        den = max(F(voxels), F(1))
        acc = F(0)
        for i in range(nb):
            c = F(min(F(hist[t, i]), limit) + redist)
            if i < residual:
                c = F(c + F(1))
            acc = F(acc + c)
            cdf[t, i] = min(max(F(acc / den), F(0)), F(1))
    y, x = np.mgrid[0:h, 0:w].astype(F)
    vv = np.clip(a, F(0), F(1))
    gy = (y + F(0.5)) / F(h) * F(hg - 1)
    gx = (x + F(0.5)) / F(w) * F(hg - 1)
    y0, x0 = np.floor(gy).astype(np.int64), np.floor(gx).astype(np.int64)
    y1, x1 = np.minimum(y0 + 1, hg - 1), np.minimum(x0 + 1, hg - 1)
    fy, fx = gy - y0.astype(F), gx - x0.astype(F)
    bfv = vv * F(nb - 1)
    b0 = np.clip(np.floor(bfv), F(0), F(nb - 2)).astype(np.int64)
    fb = bfv - b0.astype(F)
    mix = lambda p, q, t: p * (F(1) - t) + q * t
    look = lambda ty, tx: mix(cdf[ty * hg + tx, b0], cdf[ty * hg + tx, b0 + 1], fb)
    out = mix(mix(look(y0, x0), look(y0, x1), fx), mix(look(y1, x0), look(y1, x1), fx), fy)
    return texel(out, half)


def gauss(src, half):
    a = np.asarray(src, F)
    h, w = a.shape
    ww = [F(np.exp(F(-0.5) * F(k * k))) for k in range(-3, 4)]
    wsum = F(0)
    for v in ww:
        wsum = F(wsum + v)
    xs = np.arange(w)
    acc = np.zeros_like(a)
    for k, v in zip(range(-3, 4), ww):
        acc = acc + a[:, np.clip(xs + k, 0, w - 1)] * v
    mid = texel(acc / wsum, half)
    ys = np.arange(h)
    acc = np.zeros_like(a)
    for k, v in zip(range(-3, 4), ww):
        acc = acc + mid[np.clip(ys + k, 0, h - 1), :] * v
    return texel(acc / wsum, half)


def bandpass(work, fine_px=1.0, coarse_px=6.0, half=False):
    fp = fine_px if fine_px > 0 else 1.0
    cp = coarse_px if coarse_px > 0 else 6.0
    rnd = lambda x: math.floor(x + 0.5)
    fine_n = int(max(1, min(16, rnd(fp * fp))))
    coarse_n = max(fine_n + 1, int(min(64, rnd(cp * cp))))
    fine = np.asarray(work, F)
    for _ in range(fine_n):
        fine = gauss(fine, half)
    coarse = fine
    for _ in range(coarse_n - fine_n):
        coarse = gauss(coarse, half)
    v = np.clip(fine, F(0), F(1)) - np.clip(coarse, F(0), F(1))
    lo, hi = v.min(), v.max()
    sc = F(F(1) / F(hi - lo)) if hi > lo else F(0)
    return texel((v - lo) * sc, half)


def invert(work, half=False):
    return texel(F(1) - np.clip(np.asarray(work, F), F(0), F(1)), half)


def bake(gray, settings, preprocess=True):
    """The work image of a gray f32 image under the settings (before the f16 rounding that the
    features apply when half)."""
    s = settings
    g = np.asarray(gray, F)
    if not preprocess:
        return g
    half = bool(s.get("half", True))
    if s.get("clahe", True):
        w = clahe(g, 40.0, int(s.get("clahe_bins", 64)), int(s.get("clahe_grid", 4)), half)
    else:
        w = texel(g, half)
    if s.get("band", False):
        w = bandpass(w, float(s.get("bp_fine", 1.0)), float(s.get("bp_coarse", 6.0)), half)
    if s.get("invert", False):
        w = invert(w, half)
    return w
