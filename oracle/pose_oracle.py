"""CPU oracle for zcmir's pose scores, gradients and Gauss–Newton step (float64).

TEST INFRASTRUCTURE ONLY (the same rules as oracle/smi_oracle.py: only tests/, smoke() and the
bench's CPU leg use it, as the checker).

Restates, in NumPy:
* the per-pose overlap moments (``shaders/smi.wgsl:977-1057`` overlap_moments, taper 336-351):
  every fixed pixel x samples the moving features bilinearly at H⁻¹(x + 1) − 1, weight = the
  2-px ramp inside the moving image's valid border;
* ``scoreFromMoments`` (``src/moments.zig:91-172``): the score and its gradient coefficients;
* the tangent gradient and Gauss–Newton matrix (``shaders/smi.wgsl:1123-1272``, tangent_grad);
* the cubic B-spline free-form deformation on top of the pose (``shaders/smi.wgsl:198-240``
  cubic_w / dest_half / ffd_disp; its use in overlap_moments 1003-1016 and tangent_grad
  1168-1186: on the fixed image's lattice the displacement moves the fixed pixel before H⁻¹, on
  the moving image's lattice it moves the sample after it) and the score's gradient over the
  control points (``ffd_grad`` 1275-1417; ``src/pair.zig:387-410`` ffdGrad: symmetric
  ½ (g_fwd − g_inv) with the inverse direction's spline negated on the other image);
* the symmetric pair (``src/pair.zig:162-184, 241-268``) and the pose algebra
  (``src/lie.zig``: destN 27-35, inv3 85-117, hat 120-141, expm3 143-163, composeN 182-185,
  vee 187-204, generators 209-224, adjointGrad 227-241).
"""
from __future__ import annotations

import math

import numpy as np

from .smi_oracle import TRI, tri_k

MIN_N = 12
RIDGE = 1e-4
TAPER = 2.0


# ── pose algebra ──────────────────────────────────────────────────────────────────────────────

def dest_n(w, h):
    w, h = max(w, 1), max(h, 1)
    return np.array([[2 / w, 0, -(w + 1) / w], [0, 2 / h, -(h + 1) / h], [0, 0, 1.0]])


def inv3(m):
    """Inverse with one Newton refinement step (src/lie.zig inv3)."""
    m = np.asarray(m, np.float64).reshape(3, 3)
    inv = np.linalg.inv(m)
    return inv @ (2 * np.eye(3) - m @ inv)


def n_keys(homog):
    return 8 if homog else 6


def hat(x, homog=True):
    tx, ty, th, sg, al, ga, px, py = x
    if homog:
        iso, z = sg / 3, -2 * sg / 3
    else:
        iso, z, px, py = sg, 0.0, 0.0, 0.0
    return np.array([[iso + al, ga - th, tx], [ga + th, iso - al, ty], [px, py, z]])


def vee(A, homog=True):
    A = np.asarray(A, np.float64)
    a, e = A[0, 0], A[1, 1]
    if homog:
        tr = (a + e + A[2, 2]) / 3
        a, e = a - tr, e - tr
        iso = (a + e) / 2
        return np.array([A[0, 2], A[1, 2], (A[1, 0] - A[0, 1]) / 2, iso * 3, (a - e) / 2, (A[1, 0] + A[0, 1]) / 2, A[2, 0], A[2, 1]])
    return np.array([A[0, 2], A[1, 2], (A[1, 0] - A[0, 1]) / 2, (a + e) / 2, (a - e) / 2, (A[1, 0] + A[0, 1]) / 2, 0, 0])


def expm3(A):
    from scipy.linalg import expm

    return expm(np.asarray(A, np.float64))


def project_group(H, homog=True):
    H = np.asarray(H, np.float64)
    s = H[2, 2] if abs(H[2, 2]) > 1e-12 else 1.0
    o = H / s
    if not homog:
        o[2] = [0, 0, 1]
    return o


def compose_n(H0, x, homog, dw, dh):
    N = dest_n(dw, dh)
    return project_group(inv3(N) @ expm3(hat(x, homog)) @ N @ H0, homog)


def generators(homog, dw, dh):
    N = dest_n(dw, dh)
    Ni = inv3(N)
    out = [np.zeros((3, 3)) for _ in range(8)]
    for k in range(n_keys(homog)):
        e = np.zeros(8)
        e[k] = 1
        out[k] = Ni @ hat(e, homog) @ N
    return out


def adjoint_grad(g_eta, H, homog, mw, mh, fw, fh):
    M = dest_n(mw, mh) @ inv3(H) @ inv3(dest_n(fw, fh))
    Mi = inv3(M)
    nk = n_keys(homog)
    out = np.zeros(8)
    for i in range(nk):
        e = np.zeros(8)
        e[i] = 1
        cc = vee(M @ hat(e, homog) @ Mi, homog)
        out[i] = -sum(g_eta[j] * cc[j] for j in range(nk))
    return out


# ── one direction ─────────────────────────────────────────────────────────────────────────────

def _ramp(v, lo, hi):
    a, b = (v - lo) / TAPER, (hi - v) / TAPER
    ca, cb = np.clip(a, 0, 1), np.clip(b, 0, 1)
    da = np.where((a > 0) & (a < 1), 1 / TAPER, 0.0)
    db = np.where((b > 0) & (b < 1), -1 / TAPER, 0.0)
    return ca * cb, da * cb + ca * db


def cubic_w(t):
    """The cubic B-spline's four basis weights at t ∈ [0, 1] (smi.wgsl cubic_w)."""
    t2, t3 = t * t, t * t * t
    return np.stack([(1 - t) ** 3 / 6, (3 * t3 - 6 * t2 + 4) / 6, (-3 * t3 + 3 * t2 + 3 * t + 1) / 6, t3 / 6])


def _lattice(xf, yf, rw, rh, g):
    """Per point: the lattice cell (iu, iv) and the 4 + 4 basis weights of a g × g lattice over
    an rw × rh image; spacing (rw − 1)/(g − 1)."""
    spx, spy = max(rw - 1.0, 1.0) / (g - 1), max(rh - 1.0, 1.0) / (g - 1)
    su, sv = xf / spx, yf / spy
    iu, iv = np.floor(su).astype(np.int64), np.floor(sv).astype(np.int64)
    return iu, iv, cubic_w(np.clip(su - iu, 0, 1)), cubic_w(np.clip(sv - iv, 0, 1))


def ffd_disp(xf, yf, rw, rh, ffd):
    """Displacement in pixels at 0-based points (xf, yf) of the lattice's rw × rh image:
    Σ B_i(u) B_j(v) c_ij · (rw/2, rh/2), clamped lattice indices, 0 outside the image."""
    g, cps = int(ffd["g"]), np.asarray(ffd["cps"], np.float64)
    out = np.zeros((2,) + np.shape(xf))
    inside = ~((xf < 0) | (yf < 0) | (xf > rw - 1) | (yf > rh - 1))
    iu, iv, bu, bv = _lattice(xf, yf, rw, rh, g)
    hx, hy = max(rw, 1.0) * 0.5, max(rh, 1.0) * 0.5
    for jj in range(4):
        j = np.clip(iv - 1 + jj, 0, g - 1)
        for ii in range(4):
            i = np.clip(iu - 1 + ii, 0, g - 1)
            w = bu[ii] * bv[jj]
            o = (j * g + i) * 2
            out[0] += w * cps[o] * hx
            out[1] += w * cps[o + 1] * hy
    return np.where(inside, out, 0.0)


def sample(fa, H, bw, bh, ffd=None):
    """Moving features at every fixed pixel under H (and the spline ffd = dict(g, cps, source),
    or None): values, gradients, weight and its gradient, the homogeneous sample position H⁻¹X,
    the pixel vector X (moved by a fixed-image lattice) and the pixel grid."""
    _, ah, aw = fa.shape
    y, x = np.mgrid[0:bh, 0:bw].astype(np.float64)
    X = np.stack([x + 1, y + 1, np.ones_like(x)])
    if ffd is not None and not ffd["source"]:
        d = ffd_disp(x, y, bw, bh, ffd)
        X = np.stack([x + 1 + d[0], y + 1 + d[1], np.ones_like(x)])
    ph = np.tensordot(inv3(H), X, 1)
    okz = np.abs(ph[2]) >= 1e-8
    pz = np.where(okz, ph[2], 1.0)
    fx, fy = ph[0] / pz - 1, ph[1] / pz - 1
    if ffd is not None and ffd["source"]:
        d = ffd_disp(fx, fy, aw, ah, ffd)
        fx, fy = fx + d[0], fy + d[1]
    ok = okz & (fx >= 2) & (fy >= 2) & (fx <= aw - 3) & (fy <= ah - 3)
    tx, dtx = _ramp(fx, 2, aw - 3)
    ty, dty = _ramp(fy, 2, ah - 3)
    x0 = np.clip(np.floor(np.where(ok, fx, 2)).astype(int), 0, aw - 2)
    y0 = np.clip(np.floor(np.where(ok, fy, 2)).astype(int), 0, ah - 2)
    ax, ay = np.where(ok, fx, 2) - x0, np.where(ok, fy, 2) - y0
    A = fa.astype(np.float64)
    v00, v10, v01, v11 = A[:, y0, x0], A[:, y0, x0 + 1], A[:, y0 + 1, x0], A[:, y0 + 1, x0 + 1]
    return {
        "va": (v00 * (1 - ax) + v10 * ax) * (1 - ay) + (v01 * (1 - ax) + v11 * ax) * ay,
        "gx": (v10 - v00) * (1 - ay) + (v11 - v01) * ay,
        "gy": (v01 - v00) * (1 - ax) + (v11 - v10) * ax,
        "w": np.where(ok, tx * ty, 0.0),
        "dw": np.where(ok, np.stack([dtx * ty, tx * dty]), 0.0),
        "ph": ph, "X": X, "ok": ok, "xy": (x, y), "f0": (ph[0] / pz - 1, ph[1] / pz - 1),
    }


def moments(fa, fb, H, ffd=None):
    """The 45 overlap sums of a (moving) onto b (fixed) at H (moments.zig layout)."""
    fb = fb.astype(np.float64)
    S = sample(fa, H, fb.shape[2], fb.shape[1], ffd)
    w, va, vb = S["w"], S["va"], fb
    s = [w.sum()] + [(w * va[i]).sum() for i in range(4)] + [(w * vb[j]).sum() for j in range(4)]
    s += [(w * va[i] * vb[j]).sum() for i in range(4) for j in range(4)]
    s += [(w * va[i] * va[j]).sum() for i, j in TRI] + [(w * vb[i] * vb[j]).sum() for i, j in TRI]
    return np.array(s)


def _chol4(G):
    L = np.zeros((4, 4))
    for i in range(4):
        for j in range(i + 1):
            s = G[i, j] - sum(L[i, k] * L[j, k] for k in range(j))
            if i == j:
                if not s > 0:
                    return None
                L[i, i] = math.sqrt(s)
            else:
                L[i, j] = s / L[j, j]
    return L


def score_from_moments(st, exact=True, ridge=RIDGE):
    """(score, coef[102]) as src/moments.zig:91-172 (coefficients zero when n < 12 or a
    whitening fails)."""
    coef = np.zeros(102)
    n = st[0]
    if not n >= MIN_N:
        return 0.0, coef
    ma, mb = st[1:5] / n, st[5:9] / n
    C = st[9:25].reshape(4, 4) / n - np.outer(ma, mb)
    W, Mh, Nh = C.copy(), np.zeros((4, 4)), np.zeros((4, 4))
    if not exact:
        phi = float(np.sum(C * C))
    else:
        GA, GB = np.zeros((4, 4)), np.zeros((4, 4))
        for i in range(4):
            for j in range(4):
                k = tri_k(i, j)
                GA[i, j] = st[25 + k] / n - ma[i] * ma[j]
                GB[i, j] = st[35 + k] / n - mb[i] * mb[j]
        GA += np.eye(4) * ridge * max(np.trace(GA) / 4, 1e-12)
        GB += np.eye(4) * ridge * max(np.trace(GB) / 4, 1e-12)
        if _chol4(GA) is None or _chol4(GB) is None:
            return 0.0, coef
        GAi, GBi = np.linalg.inv(GA), np.linalg.inv(GB)
        W = GAi @ C @ GBi
        phi = float(np.sum(W * C))
        Mh = W @ C.T @ GAi
        Nh = W.T @ C @ GBi
        Mh += np.eye(4) * np.trace(Mh) * ridge / 4
        Nh += np.eye(4) * np.trace(Nh) * ridge / 4
    score = n * phi
    if not math.isfinite(score):
        return 0.0, coef
    coef[0:16] = W.ravel()
    coef[16:20] = mb
    coef[20:36] = Mh.ravel()
    coef[36:40] = ma
    g = np.zeros(45)
    for i in range(4):
        g[1 + i] = sum(-2 * W[i, j] * mb[j] + 2 * Mh[i, j] * ma[j] for j in range(4))
        g[5 + i] = sum(-2 * W[j, i] * ma[j] + 2 * Nh[i, j] * mb[j] for j in range(4))
        for j in range(4):
            g[9 + i * 4 + j] = 2 * W[i, j]
        for j in range(i, 4):
            f = 1.0 if i == j else 2.0
            g[25 + tri_k(i, j)] = -f * Mh[i, j]
            g[35 + tri_k(i, j)] = -f * Nh[i, j]
    g[0] = (score - float(np.dot(g[1:], st[1:]))) / n
    coef[40:85] = g
    coef[85:101] = (Mh if exact else C @ C.T).ravel()
    return score, coef


def _dva(S, vb, coef):
    """Per pixel ∂S/∂v_a (score_dva) and the taper's boundary value (boundary_value)."""
    va = S["va"]
    W, mb, Mh, ma, g = coef[0:16].reshape(4, 4), coef[16:20], coef[20:36].reshape(4, 4), coef[36:40], coef[40:85]
    tb = vb - mb[:, None, None]
    ta = va - ma[:, None, None]
    ra = 2 * (np.tensordot(W, tb, 1) - np.tensordot(Mh, ta, 1))
    bwv = g[0] + sum(g[1 + i] * va[i] + g[5 + i] * vb[i] for i in range(4))
    bwv = bwv + sum(g[9 + 4 * i + j] * va[i] * vb[j] for i in range(4) for j in range(4))
    bwv = bwv + sum(g[25 + k] * va[i] * va[j] + g[35 + k] * vb[i] * vb[j] for k, (i, j) in enumerate(TRI))
    return ra, bwv


def ffd_grad(fa, fb, H, coef, ffd):
    """∂score/∂(control points) of one direction at H (2·g·g, x then y per point; ffd_grad):
    every valid pixel's (∂S/∂v_a)·∇v_a and taper term, times the sample's motion per control
    point (its basis weight × half the lattice image, through H⁻¹ on a fixed-image lattice)."""
    fb = fb.astype(np.float64)
    _, ah, aw = fa.shape
    bh, bw = fb.shape[1:]
    g = int(ffd["g"])
    S = sample(fa, H, bw, bh, ffd)
    ra, bwv = _dva(S, fb, coef)
    ok, wt, gx, gy = S["ok"], S["w"], S["gx"], S["gy"]
    tpx, tpy = S["dw"][0], S["dw"][1]
    src = bool(ffd["source"])
    lw, lh = (aw, ah) if src else (bw, bh)
    hx, hy = max(lw, 1.0) * 0.5, max(lh, 1.0) * 0.5
    px_, py_ = S["f0"] if src else S["xy"]
    iu, iv, bu, bv = _lattice(px_, py_, lw, lh, g)
    Hi, ph = inv3(H), S["ph"]
    z = np.where(np.abs(ph[2]) >= 1e-8, ph[2], 1.0)
    z2 = np.maximum(z * z, 1e-12)
    ax_ = np.sum(ra * gx, 0)
    ay_ = np.sum(ra * gy, 0)
    grad = np.zeros(2 * g * g)
    for jj in range(4):
        j = np.clip(iv - 1 + jj, 0, g - 1)
        for ii in range(4):
            i = np.clip(iu - 1 + ii, 0, g - 1)
            bk = bu[ii] * bv[jj]
            if src:
                dxx, dyx, dxy, dyy = bk * hx, 0.0 * bk, 0.0 * bk, bk * hy
            else:
                wx = Hi[:, 0][:, None, None] * (bk * hx)
                wy = Hi[:, 1][:, None, None] * (bk * hy)
                dxx = (wx[0] * z - ph[0] * wx[2]) / z2
                dyx = (wx[1] * z - ph[1] * wx[2]) / z2
                dxy = (wy[0] * z - ph[0] * wy[2]) / z2
                dyy = (wy[1] * z - ph[1] * wy[2]) / z2
            gxv = np.where(ok, wt * (ax_ * dxx + ay_ * dyx) + bwv * (tpx * dxx + tpy * dyx), 0.0)
            gyv = np.where(ok, wt * (ax_ * dxy + ay_ * dyy) + bwv * (tpx * dxy + tpy * dyy), 0.0)
            idx = (j * g + i).ravel()
            np.add.at(grad, 2 * idx, gxv.ravel())
            np.add.at(grad, 2 * idx + 1, gyv.ravel())
    return grad


def tangent(fa, fb, H, coef, homog=True, hess=True, ffd=None):
    """(grad[8], GN[8×8]) of one direction at H from its coefficients (tangent_grad)."""
    fb = fb.astype(np.float64)
    bh, bw = fb.shape[1:]
    S = sample(fa, H, bw, bh, ffd)
    va, vb, gx, gy, wt = S["va"], fb, S["gx"], S["gy"], S["w"]
    Q = coef[85:101].reshape(4, 4)
    ra, bwv = _dva(S, vb, coef)
    ok = S["ok"]
    cx = np.where(ok, wt * np.sum(ra * gx, 0) + bwv * S["dw"][0], 0.0)
    cy = np.where(ok, wt * np.sum(ra * gy, 0) + bwv * S["dw"][1], 0.0)
    Hi, ph, X = inv3(H), S["ph"], S["X"]
    pz = np.where(np.abs(ph[2]) >= 1e-8, ph[2], 1.0)
    iz2 = 1 / np.maximum(pz * pz, 1e-12)
    gens = generators(homog, bw, bh)
    px, py = [], []
    for k in range(8):
        v = np.tensordot(-Hi @ gens[k], X, 1)
        px.append((v[0] * pz - ph[0] * v[2]) * iz2)
        py.append((v[1] * pz - ph[1] * v[2]) * iz2)
    grad = np.array([float(np.sum(cx * px[k] + cy * py[k])) for k in range(8)])
    A = np.zeros((8, 8))
    if hess:
        qgx, qgy = np.tensordot(Q, gx, 1), np.tensordot(Q, gy, 1)
        sxx, sxy = np.sum(gx * qgx, 0), np.sum(gx * qgy, 0)
        syx, syy = np.sum(gy * qgx, 0), np.sum(gy * qgy, 0)
        w = np.where(ok, wt, 0.0)
        for k in range(8):
            for l in range(k, 8):
                A[k, l] = A[l, k] = float(np.sum(w * (px[k] * (sxx * px[l] + sxy * py[l]) + py[k] * (syx * px[l] + syy * py[l]))))
    return grad, A


# ── the pair ──────────────────────────────────────────────────────────────────────────────────

def ffd_live(ffd):
    """A spline that moves anything (src/pair.zig:32-36 live): on, some |c| > 1e-12."""
    return ffd is not None and bool(np.any(np.abs(np.asarray(ffd["cps"], np.float64)) > 1e-12))


def ffd_adjoint(ffd):
    """The inverse direction's spline: negated, on the other image (pair.zig invCfg)."""
    return None if ffd is None else dict(g=ffd["g"], cps=-np.asarray(ffd["cps"], np.float64), source=not ffd["source"])


def pair_ffd_grad(fa, fb, H, ffd, exact=True, symmetric=True):
    """(score, ∇ over the control points) at H (src/pair.zig:387-410 ffdGrad): the forward
    direction with the spline as given; when symmetric and the spline is live, the mean with the
    inverse direction, gradient ½ (g_fwd − g_inv)."""
    H = np.asarray(H, np.float64).reshape(3, 3)
    mf = moments(fa, fb, H, ffd)
    sf, cf = score_from_moments(mf, exact)
    gf = ffd_grad(fa, fb, H, cf, ffd) if mf[0] >= MIN_N else np.zeros(2 * ffd["g"] ** 2)
    if not symmetric or not ffd_live(ffd):
        return sf, gf
    Hi = inv3(H)
    adj = ffd_adjoint(ffd)
    mi = moments(fb, fa, Hi, adj)
    si, ci = score_from_moments(mi, exact)
    gi = ffd_grad(fb, fa, Hi, ci, adj) if mi[0] >= MIN_N else np.zeros_like(gf)
    return 0.5 * (sf + si), 0.5 * (gf - gi)


def pair_eval(fa, fb, H, exact=True, symmetric=True, homog=True, grad=False, hess=False, ffd=None):
    """Scores (mean, fwd, inv) and, with grad, the symmetric gradient and GN matrix at H
    (src/pair.zig parts / sym); ffd: the engine's spline (used only when live)."""
    H = np.asarray(H, np.float64).reshape(3, 3)
    nk = n_keys(homog)
    fwd_ffd = ffd if ffd_live(ffd) else None
    inv_ffd = ffd_adjoint(fwd_ffd)
    mf = moments(fa, fb, H, fwd_ffd)
    sf, cf = score_from_moments(mf, exact)
    out = {"fwd": sf, "sums": mf, "n": mf[0]}
    if symmetric:
        Hi = inv3(H)
        mi = moments(fb, fa, Hi, inv_ffd)
        si, ci = score_from_moments(mi, exact)
        out.update(inv=si, mean=0.5 * (sf + si))
    else:
        out.update(inv=None, mean=sf)
    if not grad:
        return out
    gf, Af = tangent(fa, fb, H, cf, homog, hess, fwd_ffd) if mf[0] >= MIN_N else (np.zeros(8), np.zeros((8, 8)))
    gf, Af = gf[:nk], Af[:nk, :nk]
    if not symmetric:
        out.update(grad=gf, hess=Af)
        return out
    gb, Ab = tangent(fb, fa, Hi, ci, homog, hess, inv_ffd) if mi[0] >= MIN_N else (np.zeros(8), np.zeros((8, 8)))
    gb, Ab = gb[:nk], Ab[:nk, :nk]
    _, ah, aw = fa.shape
    _, bh, bw = fb.shape
    pulled = adjoint_grad(np.r_[gb, np.zeros(8 - nk)], H, homog, aw, ah, bw, bh)[:nk]
    PT = np.zeros((nk, nk))
    for j in range(nk):
        e = np.zeros(8)
        e[j] = 1
        PT[:, j] = adjoint_grad(e, H, homog, aw, ah, bw, bh)[:nk]
    out.update(grad=0.5 * (gf + pulled), hess=0.5 * (Af + PT @ Ab @ PT.T))
    return out
