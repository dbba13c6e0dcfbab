"""CPU oracle for zcmir's square-loss MI (SMI) shift-map path.

TEST INFRASTRUCTURE ONLY. Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline / reference arm may import this module, and only as the checker or as the timed
CPU baseline. The product path (``libzcmir.so`` and ``zcmir_b200``) never calls into it.

It restates the reference's algorithm for the path (ZacharyVarley/zcmir; cited by the file's
path inside that project) in NumPy:

* the per-image features follow ``shaders/smi.wgsl`` (``zscore_p``, ``hist_bins``,
  ``cdf_scan``, ``rank_eq``, ``feats``, ``feat_moments``, ``chol``, ``whiten``, ``feat_acf``,
  ``acf_norm``, ``corr_area``, ``stack_planes``) in the order ``src/smi.zig:348-400`` runs
  them.  The per-pixel arithmetic is done in float32 with the same operation order as the
  shader (so histogram bins and ranks come out bit-for-bit), the image-wide reductions in
  float64 (the B200 build reduces in float64 too);
* the map plan follows ``src/smi.zig:35-47`` (auto plan), ``src/fft.zig:20-43, 96-114``
  (ladder sizes, ``linearCorrPlanRect``) and ``src/smi.zig:77-159`` (the correlation plan);
* the canvas follows ``src/lie.zig:537-579`` (``regFrame``, ``canvasH``) and
  ``shaders/smi.wgsl:1648-1706`` (``warp_stack``, ``paste_stack``);
* packing follows ``shaders/smi.wgsl:626-728`` (``pack_resample``, ``real_plane``,
  ``pack_pair``);
* the correlations are exact float64 FFTs (``numpy.fft``) of Σ_x a(x + t)·b(x)
  (``shaders/smi.wgsl:747-748``), each inverse scaled by 1/(nx·ny)
  (``src/fft.zig:280-286``);
* the per-shift score follows ``shaders/smi.wgsl:799-931`` (``combine_cell``) in float64;
* the argmax and the lag follow ``shaders/smi.wgsl:1600-1644`` and ``src/engine.zig:789-819``.

``direct_sums`` is an FFT-free check: the 45 correlation sums at one lag as float64 dot
products over the overlap.
"""
from __future__ import annotations

import math

import numpy as np

MIN_N = 12
RIDGE = 1e-4
N_BINS = 256
MAP_CAP = 1024          # src/smi.zig:22
MAP_AUTO_MIN = 128      # src/smi.zig:29
MAP_AUTO_MAX = 512      # src/smi.zig:30
HW_MAX_N = 2048         # src/fft.zig:118-120 (largest line one workgroup transforms)

F32 = np.float32
FEATURE_MODES = ("laplacian", "three", "cubic")   # src/moments.zig:13

# upper triangle of a 4×4, row by row (shaders/smi.wgsl:64-77)
TRI = [(0, 0), (0, 1), (0, 2), (0, 3), (1, 1), (1, 2), (1, 3), (2, 2), (2, 3), (3, 3)]


def tri_k(i, j):
    a, b = min(i, j), max(i, j)
    return a * 4 - (a * (a + 1)) // 2 + b


# ── input ─────────────────────────────────────────────────────────────────────────────────────

def quantize_half(gray):
    """f32 gray → f16 texels → f32, as the default ``half`` upload does
    (``src/gls.zig:433-442``, ``promoteTexels`` 394-408). Round to nearest even."""
    return np.asarray(gray, F32).astype(np.float16).astype(F32)


# ── features (src/smi.zig:348-400) ─────────────────────────────────────────────────────────────

def image_stats(g):
    """Mean and spread of a w×h f32 image (``shaders/smi.wgsl:520-551, 1540-1570``).

    mean = Σg/N; spread = sqrt(max(Σ(g − mean)²/N, 1e-12)) with g − mean rounded to f32 as
    ``zscore_p`` writes it. Both sums are float64 here (and on the B200)."""
    g = np.asarray(g, F32)
    n = g.size
    mean = F32(np.sum(g, dtype=np.float64) / max(n, 1))
    d = (g - mean).astype(np.float64)
    spread = F32(math.sqrt(max(float(np.sum(d * d)) / max(n, 1), 1e-12)))
    return mean, spread


def rank_image(g):
    """Histogram mid-rank of the z-scored image (``shaders/smi.wgsl:393-420, 1548-1554``):
    256 bins over z ∈ [−4, 4], r = (cdf[b] + ½ hist[b]) / N · 2 − 1, in f32."""
    g = np.asarray(g, F32)
    mean, spread = image_stats(g)
    z = (g - mean) / np.maximum(spread, F32(1e-8))
    b = np.clip((z + F32(4.0)) * F32(32.0), F32(0.0), F32(255.0)).astype(np.uint32)
    hist = np.bincount(b.ravel(), minlength=N_BINS).astype(np.int64)
    cdf = np.concatenate([[0], np.cumsum(hist)[:-1]]).astype(np.int64)
    tot = F32(max(int(hist.sum()), 1))
    r = (cdf[b].astype(F32) + F32(0.5) * hist[b].astype(F32)) / tot * F32(2.0) - F32(1.0)
    return r.astype(F32)


def raw_features(r, mode="laplacian"):
    """[r, r², Sobel |∇r|, fourth] of the rank with clamp-to-edge borders
    (``shaders/smi.wgsl:422-462``); fourth: 4-neighbour Laplacian, 0 ("three") or r³."""
    r = np.asarray(r, F32)
    p = np.pad(r, 1, mode="edge")
    t = lambda dx, dy: p[1 + dy: p.shape[0] - 1 + dy, 1 + dx: p.shape[1] - 1 + dx]
    two = F32(2.0)
    gx = -t(-1, -1) + t(1, -1) - two * t(-1, 0) + two * t(1, 0) - t(-1, 1) + t(1, 1)
    gy = -t(-1, -1) - two * t(0, -1) - t(1, -1) + t(-1, 1) + two * t(0, 1) + t(1, 1)
    g = np.sqrt(gx * gx + gy * gy)
    if mode == "laplacian":
        f3 = t(-1, 0) + t(1, 0) + t(0, -1) + t(0, 1) - F32(4.0) * r
    elif mode == "three":
        f3 = np.zeros_like(r)
    elif mode == "cubic":
        f3 = r * r * r
    else:
        raise ValueError(mode)
    feat = np.stack([r, r * r, g, f3]).astype(F32)
    return feat, g.astype(F32)


def whitening(feat):
    """L⁻¹ and μ of the global ridge whitening (``shaders/smi.wgsl:531-585``): the 21 raw
    moments (float64), G = cov + 1e-4·max(tr/4, 1e-12)·I, L = chol(G) with diagonal
    sqrt(max(s, 1e-12)); returned as f32 (X = L⁻¹ row-major, μ)."""
    x = feat.reshape(4, -1).astype(np.float64)
    n = max(float(x.shape[1]), 1.0)
    mu = x.sum(axis=1) / n
    G = (x @ x.T) / n - np.outer(mu, mu)
    tr = float(np.trace(G))
    G = G + np.eye(4) * (RIDGE * max(tr * 0.25, 1e-12))
    L = np.zeros((4, 4))
    for i in range(4):
        for j in range(i + 1):
            s = G[i, j] - sum(L[i, k] * L[j, k] for k in range(j))
            if i == j:
                L[i, i] = math.sqrt(max(s, 1e-12))
            else:
                L[i, j] = s / L[j, j]
    X = np.zeros((4, 4))
    for col in range(4):
        for i in range(4):
            s = (1.0 if i == col else 0.0) - sum(L[i, k] * X[k, col] for k in range(i))
            X[i, col] = s / L[i, i]
    return X.astype(F32), mu.astype(F32)


def whiten(feat, X, mu):
    """x ← L⁻¹(x − μ) per pixel in f32, products rounded one by one in j order
    (``shaders/smi.wgsl:587-599``)."""
    d = [(feat[i] - mu[i]).astype(F32) for i in range(4)]
    out = np.empty_like(feat)
    for i in range(4):
        s = X[i, 0] * d[0]
        for j in range(1, 4):
            s = s + X[i, j] * d[j]
        out[i] = s
    return out


def acf(feat, maxlag=8):
    """Autocorrelation of each plane at |dx|, |dy| ≤ 8 over the valid pairs, normalised by
    the zero lag (``shaders/smi.wgsl:935-975, 1572-1578``); (289, 4) float64, lag index
    (dy + 8)·17 + (dx + 8)."""
    _, h, w = feat.shape
    f = feat.astype(np.float64)
    out = np.zeros((17 * 17, 4))
    for dy in range(-maxlag, maxlag + 1):
        for dx in range(-maxlag, maxlag + 1):
            ys, ye = max(0, -dy), min(h, h - dy)
            xs, xe = max(0, -dx), min(w, w - dx)
            if ye <= ys or xe <= xs:
                continue
            a = f[:, ys:ye, xs:xe]
            b = f[:, ys + dy:ye + dy, xs + dx:xe + dx]
            cnt = max((ye - ys) * (xe - xs), 1)
            out[(dy + 8) * 17 + (dx + 8)] = (a * b).reshape(4, -1).sum(axis=1) / cnt
    z = out[144].copy()
    return out / np.maximum(z, 1e-12)


def pair_area(acf_a, acf_b):
    """Bartlett feature correlation area (px²) of a pair (``shaders/smi.wgsl:1580-1595``)."""
    return max(1.0, float(np.sum(acf_a.sum(axis=1) * acf_b.sum(axis=1))) / 16.0)


def prepare(gray, mode="laplacian", half=False):
    """One image's SMI features, as ``Smi.prepare`` (``src/smi.zig:348-400``) builds them."""
    g = np.asarray(gray, F32)
    if half:
        g = quantize_half(g)
    r = rank_image(g)
    feat, mag = raw_features(r, mode)
    X, mu = whitening(feat)
    wf = whiten(feat, X, mu)
    return {
        "w": g.shape[1], "h": g.shape[0], "mode": mode, "rank": r, "feat": wf, "mag": mag,
        "acf": acf(wf), "X": X, "mu": mu,
        # premultiplied stack [w, w f0 .. w f3], w = 1 (shaders/smi.wgsl:615-624)
        "stack": np.concatenate([np.ones((1,) + g.shape, F32), wf]).astype(F32),
    }


# ── plans ─────────────────────────────────────────────────────────────────────────────────────

def _smooth(n, sizes):
    for p in ((2, 3) if sizes == "ladder" else (2, 3, 5, 7, 11, 13)):
        while n % p == 0:
            n //= p
    return n == 1


def plan_size(target, div=1, sizes="ladder"):
    """Smallest length ≥ target in ``sizes`` (``src/fft.zig:20-25``)."""
    n = max(target, 1)
    while not (n % div == 0 and _smooth(n, sizes)):
        n += 1
    return n


def largest_smooth(max_n, sizes="ladder"):
    """``src/fft.zig:37-43``."""
    n = max(32, max_n)
    while n >= 32:
        if _smooth(n, sizes):
            return n
        n -= 1
    return 32


def _js_round(x):
    return int(math.floor(x + 0.5))


def linear_corr_plan_rect(w, h, max_n0, sizes="ladder"):
    """(nx, ny, cw, ch) of an explicit-resolution map (``src/fft.zig:96-109``)."""
    max_n = largest_smooth(max_n0, sizes)
    s = min(1.0, max(8, max_n >> 1) / max(max(w, h), 1))
    for _ in range(16):
        cw = max(8, _js_round(w * s))
        ch = max(8, _js_round(h * s))
        nx = min(plan_size(max(cw + cw - 1, 32), 1, sizes), max_n)
        ny = min(plan_size(max(ch + ch - 1, 32), 1, sizes), max_n)
        if nx >= cw + cw - 1 and ny >= ch + ch - 1:
            return nx, ny, cw, ch
        s *= 0.85
    m = max(8, (max_n + 1) >> 1)
    return max_n, max_n, m, m


def auto_shift_plan(w, h):
    """(nx, ny, cw, ch) of the automatic map (``src/smi.zig:35-47``)."""
    d = max(w, h, 1)
    g = 1
    while 2 * ((d + g - 1) // g) - 1 > MAP_AUTO_MAX:
        g *= 2
    cw = max(1, (w + g - 1) // g)
    ch = max(1, (h + g - 1) // g)
    pow2 = lambda need: min(max(1 << (max(need, 1) - 1).bit_length(), MAP_AUTO_MIN), MAP_AUTO_MAX)
    return pow2(2 * cw - 1), pow2(2 * ch - 1), cw, ch


def cap_n(cap0, sizes="ladder", hw_max=HW_MAX_N):
    """The FFT-length cap of an explicit map (``src/smi.zig:414-422``); the storage-binding
    halving does not apply (no binding limit on the B200 build)."""
    return largest_smooth(min(cap0, hw_max), sizes)


def corr_plan(exact=True, three=False):
    """The correlation plan (``src/smi.zig:90-158``): the real planes kept (by number) and the
    correlations kept as (moving plane number, fixed plane number, correlation number)."""
    lst = [(0, 0)] + [(1 + i, 0) for i in range(4)] + [(0, 1 + j) for j in range(4)]
    lst += [(1 + i, 1 + j) for i in range(4) for j in range(4)]
    if exact:
        lst += [(5 + k, 0) for k in range(10)] + [(0, 5 + k) for k in range(10)]
    n_planes = 15 if exact else 5
    fourth = {4, 8, 11, 13, 14}
    planes = [p for p in range(n_planes) if not (three and p in fourth)]
    corrs = [(a, b, c) for c, (a, b) in enumerate(lst) if a in planes and b in planes]
    return planes, corrs


# ── canvas (src/lie.zig:537-579, shaders/smi.wgsl:1648-1706) ──────────────────────────────────

def reg_frame(H, lw, lh, rw, rh):
    """(ox, oy, w, h): the fixed image plus the moving image's warped corners, clipped to
    ±2·max(size) (``src/lie.zig:537-574``)."""
    H = np.asarray(H, np.float64).reshape(9)
    xs_min, ys_min, xs_max, ys_max = 0.0, 0.0, float(rw), float(rh)
    lim = max(max(lw, rw), max(max(lh, rh), 8)) * 2.0
    for px, py in ((1, 1), (lw, 1), (lw, lh), (1, lh)):
        x = H[0] * px + H[1] * py + H[2]
        y = H[3] * px + H[4] * py + H[5]
        z = H[6] * px + H[7] * py + H[8]
        zz = 1e-8 if abs(z) < 1e-8 else z
        xs_min = min(xs_min, x / zz - 1)
        xs_max = max(xs_max, x / zz - 1)
        ys_min = min(ys_min, y / zz - 1)
        ys_max = max(ys_max, y / zz - 1)
    clip = lambda v: min(lim, max(-lim, v))
    ox = min(math.floor(clip(xs_min)), 0)
    oy = min(math.floor(clip(ys_min)), 0)
    x1 = max(math.ceil(clip(xs_max)), rw)
    y1 = max(math.ceil(clip(ys_max)), rh)
    return int(ox), int(oy), int(max(8, x1 - ox)), int(max(8, y1 - oy))


def canvas_H(H, ox, oy):
    """Moving → canvas pixels: translate(−ox, −oy)·H (``src/lie.zig:577-579``)."""
    T = np.array([[1, 0, -ox], [0, 1, -oy], [0, 0, 1.0]])
    return T @ np.asarray(H, np.float64).reshape(3, 3)


def warp_stack(stack, Hc, W, Hh):
    """The moving stack on the W×Hh canvas by the canvas pose (bilinear, clamped taps, 0
    outside [0, w−1]×[0, h−1]) (``shaders/smi.wgsl:1655-1688``), float64."""
    _, h, w = stack.shape
    out = np.zeros((stack.shape[0], Hh, W))
    if abs(np.linalg.det(Hc)) < 1e-12:
        return out
    Hi = np.linalg.inv(Hc)
    yy, xx = np.mgrid[0:Hh, 0:W].astype(np.float64)
    q = np.tensordot(Hi, np.stack([xx + 1, yy + 1, np.ones_like(xx)]), 1)
    okz = np.abs(q[2]) >= 1e-8
    qz = np.where(okz, q[2], 1.0)
    fx, fy = q[0] / qz - 1, q[1] / qz - 1
    ok = okz & ~((fx < 0) | (fy < 0) | (fx > w - 1) | (fy > h - 1))
    fx, fy = np.where(ok, fx, 0.0), np.where(ok, fy, 0.0)
    x0, y0 = np.floor(fx).astype(np.int64), np.floor(fy).astype(np.int64)
    tx, ty = fx - x0, fy - y0
    cx = lambda v: np.clip(v, 0, w - 1)
    cy = lambda v: np.clip(v, 0, h - 1)
    s = stack.astype(np.float64)
    for p in range(stack.shape[0]):
        v00, v10 = s[p][cy(y0), cx(x0)], s[p][cy(y0), cx(x0 + 1)]
        v01, v11 = s[p][cy(y0 + 1), cx(x0)], s[p][cy(y0 + 1), cx(x0 + 1)]
        v = (v00 * (1 - tx) + v10 * tx) * (1 - ty) + (v01 * (1 - tx) + v11 * tx) * ty
        out[p] = np.where(ok, v, 0.0)
    return out


def paste_stack(stack, ox, oy, W, Hh):
    """The fixed stack pasted into the canvas at (−ox, −oy) (``shaders/smi.wgsl:1690-1706``)."""
    _, h, w = stack.shape
    out = np.zeros((stack.shape[0], Hh, W))
    out[:, -oy:-oy + h, -ox:-ox + w] = stack
    return out


def pack_resample(canvas, cw, ch):
    """The canvas on the cw×ch grid: k×k box of bilinear taps (k = ⌈W/cw⌉ ≤ 8), identity at
    full resolution (``shaders/smi.wgsl:626-639, 675-705``), float64."""
    P, Hh, W = canvas.shape
    if W == cw and Hh == ch:
        return canvas.copy()
    fx, fy = W / max(cw, 1), Hh / max(ch, 1)
    kx = int(min(max(math.ceil(fx - 1e-4), 1), 8))
    ky = int(min(max(math.ceil(fy - 1e-4), 1), 8))
    out = np.zeros((P, ch, cw))
    gx, gy = np.meshgrid(np.arange(cw, dtype=np.float64), np.arange(ch, dtype=np.float64))
    for j in range(ky):
        py = (gy + (j + 0.5) / ky) * fy
        for i in range(kx):
            px = (gx + (i + 0.5) / kx) * fx
            x, y = px - 0.5, py - 0.5
            x0, y0 = np.floor(x).astype(np.int64), np.floor(y).astype(np.int64)
            ax, ay = x - x0, y - y0
            xa, xb = np.clip(x0, 0, W - 1), np.clip(x0 + 1, 0, W - 1)
            ya, yb = np.clip(y0, 0, Hh - 1), np.clip(y0 + 1, 0, Hh - 1)
            for p in range(P):
                c = canvas[p]
                out[p] += (c[ya, xa] * (1 - ax) + c[ya, xb] * ax) * (1 - ay) + (c[yb, xa] * (1 - ax) + c[yb, xb] * ax) * ay
    return out / (kx * ky)


def real_planes(s, planes):
    """Real correlation planes from premultiplied samples s = [w, w f0..w f3]: 0 → w, 1..4 →
    w f_i, 5..14 → s_i s_j / s_0 (0 where s_0 ≤ 1e-6) (``shaders/smi.wgsl:641-649``)."""
    out = []
    s0 = s[0]
    safe = np.where(s0 > 1e-6, s0, 1.0)
    for r in planes:
        if r < 5:
            out.append(s[r])
        else:
            i, j = TRI[r - 5]
            out.append(np.where(s0 > 1e-6, s[1 + i] * s[1 + j] / safe, 0.0))
    return np.stack(out)


# ── correlations and score ────────────────────────────────────────────────────────────────────

def correlations(planes_a, planes_b, plane_ids, corrs, nx, ny):
    """(45, ny, nx) float64: corr_c(t) = Σ_x a(x + t)·b(x) on the nx×ny torus (zero-padded
    planes), correlations the plan leaves out stay 0. Lag 0 at [0, 0]."""
    slot = {p: k for k, p in enumerate(plane_ids)}
    FA = {p: np.fft.rfft2(planes_a[slot[p]], (ny, nx)) for p in plane_ids}
    FB = {p: np.fft.rfft2(planes_b[slot[p]], (ny, nx)) for p in plane_ids}
    out = np.zeros((45, ny, nx))
    for a, b, c in corrs:
        out[c] = np.fft.irfft2(FA[a] * np.conj(FB[b]), (ny, nx))
    return out


def direct_sums_blocked(grid_a, grid_b, plane_ids, corrs, tx, ty, rows=256):
    """direct_sums from the two 5-plane grids (5, h, w), the real planes formed in float64 a block
    of rows at a time: the 45 sums at lag (tx, ty) as one 15 × 15 product per block, without
    holding the planes of a large image."""
    _, h, w = grid_a.shape
    out = np.zeros(45)
    ys, ye = max(0, -ty), min(h, h - ty)
    xs, xe = max(0, -tx), min(w, w - tx)
    if ye <= ys or xe <= xs:
        return out
    slot = {p: k for k, p in enumerate(plane_ids)}
    P = len(plane_ids)
    G = np.zeros((P, P))
    for r0 in range(ys, ye, rows):
        r1 = min(ye, r0 + rows)
        a5 = np.asarray(grid_a[:, r0 + ty:r1 + ty, xs + tx:xe + tx], np.float64)
        b5 = np.asarray(grid_b[:, r0:r1, xs:xe], np.float64)
        A = real_planes(a5, plane_ids).reshape(P, -1)
        B = real_planes(b5, plane_ids).reshape(P, -1)
        G += A @ B.T
    for a, b, c in corrs:
        out[c] = G[slot[a], slot[b]]
    return out


def direct_sums(planes_a, planes_b, plane_ids, corrs, tx, ty):
    """The correlation sums at one lag (tx, ty) as direct float64 dot products (no FFT)."""
    slot = {p: k for k, p in enumerate(plane_ids)}
    _, h, w = planes_a.shape
    out = np.zeros(45)
    ys, ye = max(0, -ty), min(h, h - ty)
    xs, xe = max(0, -tx), min(w, w - tx)
    if ye <= ys or xe <= xs:
        return out
    for a, b, c in corrs:
        A = planes_a[slot[a]][ys + ty:ye + ty, xs + tx:xe + tx]
        B = planes_b[slot[b]][ys:ye, xs:xe]
        out[c] = float(np.sum(A * B))
    return out


def _wilson_hilferty(f, d1, d2):
    """Normal score of an F(d1, d2) value (``shaders/smi.wgsl:817-823``)."""
    a = 2.0 / (9.0 * d1)
    b = 2.0 / (9.0 * d2)
    c = np.cbrt(np.maximum(f, 0.0))
    return ((1.0 - b) * c - (1.0 - a)) / np.sqrt(b * c * c + a)


def _chol4(G, nf):
    """Vectorised in-place 4×4 Cholesky over cells, failure where a pivot is not > 0
    (``shaders/smi.wgsl:798-813``). G: (4, 4, n)."""
    ok = np.ones(G.shape[2], bool)
    L = np.zeros_like(G)
    for i in range(4):
        for j in range(i + 1):
            s = G[i, j].copy()
            for k in range(j):
                s -= L[i, k] * L[j, k]
            if i == j:
                ok &= s > 0
                L[i, i] = np.sqrt(np.where(s > 0, s, 1.0))
            else:
                L[i, j] = s / L[j, j]
    return L, ok


def combine(corr, exact=True, calibrated=False, min_n=MIN_N, area=1.0, nf=4, ridge=RIDGE, n00=None, dtype=np.float64):
    """Per-shift score from the correlation sums (``shaders/smi.wgsl:825-915``), in float64 (or in
    `dtype`: float32 restates the centring and Cholesky in single precision, as a precision study
    compares).

    corr: (45, ...) sums (already scaled). Global: n·Σ clamp(C_ij, ±1)². Exact: n·‖L_A⁻¹ C
    L_B⁻ᵀ‖². Calibrated (exact only): the Wilson–Hilferty z of Pillai's F. Floors: n < max(min_n,
    8 % of the zero-lag n) (calibrated: n < min_n or n_eff ≤ 10) score 0; failed Cholesky and
    NaN score 0."""
    shape = corr.shape[1:]
    c = corr.reshape(45, -1).astype(dtype)
    n = c[0]
    calib = exact and calibrated
    neff = n / max(area, 1.0)
    # the zero-lag overlap: lag 0 of the map, or where a sweep candidate sits (n00 given)
    n00 = c[0, 0] if n00 is None else float(n00)
    floor_n = float(min_n) if calib else max(float(min_n), 0.08 * max(n00, 0.0))
    dead = (n < floor_n) | (calib & (neff <= 10.0))
    den = np.maximum(n, 1e-8)
    ma = np.stack([c[1 + i] / den for i in range(4)])
    mb = np.stack([c[5 + i] / den for i in range(4)])
    C = np.zeros((4, 4, c.shape[1]), dtype)
    for i in range(nf):
        for j in range(nf):
            C[i, j] = c[9 + 4 * i + j] / den - ma[i] * mb[j]
    if not exact:
        score = n * np.sum(np.clip(C, -1.0, 1.0) ** 2, axis=(0, 1))
        ok = np.ones_like(dead)
    else:
        GA = np.zeros_like(C)
        GB = np.zeros_like(C)
        for i in range(nf):
            for j in range(nf):
                k = tri_k(i, j)
                GA[i, j] = c[25 + k] / den - ma[i] * ma[j]
                GB[i, j] = c[35 + k] / den - mb[i] * mb[j]
        tra = sum(GA[i, i] for i in range(nf))
        trb = sum(GB[i, i] for i in range(nf))
        for i in range(nf):
            GA[i, i] = GA[i, i] + ridge * np.maximum(tra * 0.25, 1e-12)
            GB[i, i] = GB[i, i] + ridge * np.maximum(trb * 0.25, 1e-12)
        for i in range(nf, 4):
            GA[i, i] = 1.0
            GB[i, i] = 1.0
        LA, oka = _chol4(GA, nf)
        LB, okb = _chol4(GB, nf)
        ok = oka & okb
        X = np.zeros_like(C)
        for j in range(nf):
            for i in range(nf):
                s = C[i, j].copy()
                for k in range(i):
                    s -= LA[i, k] * X[k, j]
                X[i, j] = s / LA[i, i]
        acc = np.zeros(c.shape[1], dtype)
        for r in range(nf):
            y = [None] * nf
            for i in range(nf):
                s = X[r, i].copy()
                for k in range(i):
                    s -= LB[i, k] * y[k]
                y[i] = s / LB[i, i]
                acc += y[i] * y[i]
        score = n * acc
        if calib:
            q = float(nf)
            v = np.minimum(acc, q - 1e-4)
            with np.errstate(all="ignore"):
                f = (neff - q - 1.0) / q * v / (q - v)
                score = np.maximum(_wilson_hilferty(f, q * q, q * (neff - q - 1.0)), 0.0)
    score = np.where(dead | ~ok | ~np.isfinite(score), 0.0, score)
    return score.reshape(shape)


def argmax_first(m):
    """Largest value, first flat index on ties (``shaders/smi.wgsl:1597-1644``)."""
    flat = np.asarray(m).ravel()
    i = int(np.argmax(flat))
    return float(flat[i]), i


def peak_lag(idx, nx, ny):
    """``src/engine.zig:789-793``."""
    py, px = divmod(idx, nx)
    return (px if px <= nx // 2 else px - nx, py if py <= ny // 2 else py - ny)


def map_plan(frame_w, frame_h, cap=0, sizes="ladder"):
    """(nx, ny, cw, ch): auto when cap is 0, else the explicit plan (``src/smi.zig:557``)."""
    if cap == 0:
        return auto_shift_plan(frame_w, frame_h)
    return linear_corr_plan_rect(frame_w, frame_h, cap_n(cap, sizes), sizes)


def grid_stacks(prep_a, prep_b, H, cap=0, sizes="ladder"):
    """Both canvas stacks on the map grid and the plan: (grid_a, grid_b, plan, frame)."""
    ox, oy, W, Hh = reg_frame(H, prep_a["w"], prep_a["h"], prep_b["w"], prep_b["h"])
    Hc = canvas_H(H, ox, oy)
    ca = warp_stack(prep_a["stack"], Hc, W, Hh)
    cb = paste_stack(prep_b["stack"], ox, oy, W, Hh)
    nx, ny, cw, ch = map_plan(W, Hh, cap, sizes)
    return pack_resample(ca, cw, ch), pack_resample(cb, cw, ch), (nx, ny, cw, ch), (ox, oy, W, Hh)


def shift_map(prep_a, prep_b, H=None, exact=True, calibrated=True, cap=0, min_overlap=0.0,
              sizes="ladder", return_corr=False):
    """The dense shift map of pose H (moving → fixed, 1-based), as ``Smi.shiftMap`` and
    ``Engine.shiftMapOpts`` compute it (``src/smi.zig:540-572``, ``src/engine.zig:795-819``).

    Returns a dict with the map (ny, nx) and the ShiftResult fields."""
    H = np.eye(3) if H is None else np.asarray(H, np.float64).reshape(3, 3)
    three = prep_a["mode"] == "three"
    ga, gb, (nx, ny, cw, ch), (ox, oy, W, Hh) = grid_stacks(prep_a, prep_b, H, cap, sizes)
    plane_ids, corrs = corr_plan(exact, three)
    pa, pb = real_planes(ga, plane_ids), real_planes(gb, plane_ids)
    corr = correlations(pa, pb, plane_ids, corrs, nx, ny)
    floor_n = math.floor(min_overlap * cw * ch) if min_overlap > 0 else 0
    gcell = W / cw
    area = max(1.0, pair_area(prep_a["acf"], prep_b["acf"]) / (gcell * gcell))
    m = combine(corr, exact, calibrated and exact, max(MIN_N, floor_n), area, 3 if three else 4)
    peak, idx = argmax_first(m)
    lx, ly = peak_lag(idx, nx, ny)
    out = {
        "map": m, "n": nx, "n_y": ny, "cw": cw, "ch": ch, "canvas_w": W, "canvas_h": Hh, "ox": ox, "oy": oy,
        "peak": peak, "peak_index": idx, "dx": lx * (W / cw), "dy": ly * (Hh / ch), "zero": float(m.ravel()[0]),
        "corr_area_px": pair_area(prep_a["acf"], prep_b["acf"]), "exact": exact, "calibrated": calibrated and exact,
    }
    if return_corr:
        out.update(corr=corr, planes_a=pa, planes_b=pb, plane_ids=plane_ids, corrs=corrs)
    return out
