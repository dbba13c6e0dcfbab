"""Seeded synthetic image pairs with the shapes and value distributions of the SMI workloads.

* ``blob_field``: a smooth field of Gaussian blobs (σ 4–20 px, amplitudes ±1) plus two
  sinusoidal gratings, normalised to [0, 1].
* ``pair_remap`` (256² map workload): fixed = the field, moving = 1 − field² (inverted,
  nonlinear contrast) at a known integer shift, plus N(0, 0.02²).
* ``pair_segmented`` (1024² map workload): modality A = a blob field (uint16 range); modality
  B = an 8-level piecewise-constant segmentation of it with a random level → intensity
  permutation plus N(0, 0.03²), shifted by a random integer shift in ±200 px.
* ``pair_similarity`` (512² sweep workload): the same two modalities with the moving image under
  a random similarity about the image centre: rotation in [0°, 360°), scale log-uniform in
  [0.8, 1.25], shift in ±n/8 px.
* ``stack_drift`` (stack workload): slices of one field with sizes uniform in [384, 1024] per side,
  each slice a random similarity drift of the previous one (rotation N(0, 2°), log scale
  N(0, 0.02), shift N(0, 8 px) per step), modalities alternating between the field and its
  inverted nonlinear remap 1 − field², plus N(0, 0.02²).

The true pose maps moving → fixed (1-based pixels): H = translate(dx, dy), i.e. the moving pixel
x shows the fixed content at x + (dx, dy). The shift map at the identity pose then peaks at the
lag (−dx, −dy) and its corrected pose is H.
"""
from __future__ import annotations

import numpy as np


def blob_field(h, w, rng, n_blobs=64, sigma=(4.0, 20.0), gratings=2):
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    f = np.zeros((h, w))
    scale = max(h, w) / 256.0
    for _ in range(int(n_blobs * scale * scale)):
        cx, cy = rng.uniform(0, w), rng.uniform(0, h)
        s = rng.uniform(*sigma)
        a = rng.uniform(-1, 1)
        x0, x1 = int(max(0, cx - 4 * s)), int(min(w, cx + 4 * s + 1))
        y0, y1 = int(max(0, cy - 4 * s)), int(min(h, cy + 4 * s + 1))
        if x1 <= x0 or y1 <= y0:
            continue
        f[y0:y1, x0:x1] += a * np.exp(-((xx[y0:y1, x0:x1] - cx) ** 2 + (yy[y0:y1, x0:x1] - cy) ** 2) / (2 * s * s))
    for _ in range(gratings):
        th = rng.uniform(0, np.pi)
        period = rng.uniform(24, 64)
        f += 0.3 * np.sin(2 * np.pi * (np.cos(th) * xx + np.sin(th) * yy) / period + rng.uniform(0, 2 * np.pi))
    f -= f.min()
    return f / max(f.max(), 1e-12)


def pair_remap(n=256, shift=(17, -9), seed=0, noise=0.02):
    """(moving, fixed, H_true) float32 in [0, 1]: moving = 1 − field² shifted by `shift`."""
    rng = np.random.default_rng(seed)
    dx, dy = shift
    pad = max(abs(dx), abs(dy)) + 8
    big = blob_field(n + 2 * pad, n + 2 * pad, rng)
    fixed = big[pad:pad + n, pad:pad + n]
    mov = big[pad + dy:pad + dy + n, pad + dx:pad + dx + n]
    moving = 1.0 - mov ** 2 + noise * rng.standard_normal((n, n))
    H = np.array([[1, 0, dx], [0, 1, dy], [0, 0, 1.0]])
    return moving.astype(np.float32), fixed.astype(np.float32), H


def pair_segmented(n=1024, seed=1, max_shift=200, levels=8, noise=0.03, shift=None):
    """(moving, fixed, H_true) uint16: fixed = blob field (modality A), moving = its segmented
    modality B at a random integer shift in ±max_shift."""
    rng = np.random.default_rng(seed)
    if shift is None:
        shift = tuple(int(v) for v in rng.integers(-max_shift, max_shift + 1, size=2))
    dx, dy = shift
    pad = max(abs(dx), abs(dy)) + 8
    big = blob_field(n + 2 * pad, n + 2 * pad, rng, n_blobs=64)
    fixed = big[pad:pad + n, pad:pad + n]
    src = big[pad + dy:pad + dy + n, pad + dx:pad + dx + n]
    edges = np.quantile(src, np.linspace(0, 1, levels + 1)[1:-1])
    lab = np.digitize(src, edges)
    perm = rng.permutation(levels)
    moving = perm[lab] / (levels - 1.0) + noise * rng.standard_normal((n, n))
    to16 = lambda a: (np.clip(a, 0, 1) * 65535 + 0.5).astype(np.uint16)
    H = np.array([[1, 0, dx], [0, 1, dy], [0, 0, 1.0]])
    return to16(moving), to16(fixed), H


def similarity(n, deg, scale, tx, ty):
    """Moving → fixed (1-based): rotate by deg and scale about the centre, then shift."""
    c = (n + 1) / 2
    th = np.deg2rad(deg)
    R = np.array([[scale * np.cos(th), -scale * np.sin(th), 0], [scale * np.sin(th), scale * np.cos(th), 0], [0, 0, 1.0]])
    T = lambda x, y: np.array([[1, 0, x], [0, 1, y], [0, 0, 1.0]])
    return T(c + tx, c + ty) @ R @ T(-c, -c)


def pair_similarity(n=512, seed=2, deg=None, scale=None, shift=None, levels=8, noise=0.03):
    """(moving, fixed, H_true) uint16: fixed = blob field (modality A); moving(x) = the segmented
    modality B of the field at H·x, for a random similarity H (unless given)."""
    from scipy.ndimage import map_coordinates

    rng = np.random.default_rng(seed)
    deg = float(rng.uniform(0, 360)) if deg is None else float(deg)
    scale = float(np.exp(rng.uniform(np.log(0.8), np.log(1.25)))) if scale is None else float(scale)
    if shift is None:
        shift = tuple(float(v) for v in rng.integers(-(n // 8), n // 8 + 1, size=2))
    H = similarity(n, deg, scale, *shift)
    pad = n
    big = blob_field(n + 2 * pad, n + 2 * pad, rng, n_blobs=64)
    fixed = big[pad:pad + n, pad:pad + n]
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    X = np.stack([xx + 1, yy + 1, np.ones_like(xx)], -1) @ H.T
    fx, fy = X[..., 0] / X[..., 2] - 1 + pad, X[..., 1] / X[..., 2] - 1 + pad
    src = map_coordinates(big, [fy, fx], order=1, mode="nearest")
    edges = np.quantile(src, np.linspace(0, 1, levels + 1)[1:-1])
    lab = np.digitize(src, edges)
    perm = rng.permutation(levels)
    moving = perm[lab] / (levels - 1.0) + noise * rng.standard_normal((n, n))
    to16 = lambda a: (np.clip(a, 0, 1) * 65535 + 0.5).astype(np.uint16)
    return to16(moving), to16(fixed), H


def stack_drift(n=32, size=(384, 1024), seed=3, drift=(2.0, 0.02, 8.0), noise=0.02):
    """(slices, truths): n uint16 slices; truths[k − 1] maps slice k pixels to slice k − 1 pixels
    (1-based), for k = 1..n−1."""
    from scipy.ndimage import map_coordinates

    rng = np.random.default_rng(seed)
    sizes = [(int(rng.integers(size[0], size[1] + 1)), int(rng.integers(size[0], size[1] + 1))) for _ in range(n)]
    th, ls, t = 0.0, 0.0, np.zeros(2)
    poses = []
    for k in range(n):
        if k:
            th += np.deg2rad(rng.normal(0, drift[0]))
            ls += rng.normal(0, drift[1])
            t = t + rng.normal(0, drift[2], 2)
        poses.append((th, np.exp(ls), t.copy()))
    side = int(1.6 * size[1] + 8 * drift[2] * np.sqrt(n)) + 64
    field = blob_field(side, side, rng)
    cw = (side + 1) / 2
    slices, W = [], []
    for (w, h), (a, sc, tt) in zip(sizes, poses):
        c = np.array([(w + 1) / 2, (h + 1) / 2])
        R = sc * np.array([[np.cos(a), -np.sin(a)], [np.sin(a), np.cos(a)]])
        # slice pixel x (1-based) ↦ field pixel cw + R (x − c) + t
        M = np.eye(3)
        M[:2, :2] = R
        M[:2, 2] = cw + tt - R @ c
        W.append(M)
        yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
        X = np.stack([xx + 1, yy + 1, np.ones_like(xx)], -1) @ M.T
        v = map_coordinates(field, [X[..., 1] - 1, X[..., 0] - 1], order=1, mode="nearest")
        if len(slices) % 2:
            v = 1.0 - v ** 2
        v = v + noise * rng.standard_normal(v.shape)
        slices.append((np.clip(v, 0, 1) * 65535 + 0.5).astype(np.uint16))
    truths = [np.linalg.inv(W[k - 1]) @ W[k] for k in range(1, n)]
    return slices, truths
