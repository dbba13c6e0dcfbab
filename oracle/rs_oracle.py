"""CPU oracle for zcmir's roto-scale (log-polar) SMI map.

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` as the checker, never by the product path.

Restates the reference's roto-scale map (ZacharyVarley/zcmir) in float64 NumPy:

* the plan ``src/smi.zig:589-630`` (``rsMapFrom``: centre in canvas pixels, radii, angle count,
  n_λ = n/2 rows of log radius);
* the log-polar resampling ``shaders/smi.wgsl:1418-1452`` (``sample_plane_z``,
  ``spatial_logpolar``): bilinear taps of the canvas stacks, zero where the 2×2 footprint leaves
  the canvas;
* the ρ area weight on every real plane ``shaders/smi.wgsl:712-727`` (``pack_pair``, theme 1);
* each correlation scaled by e^{kΔλ}·Δλ·Δθ at log-radius lag k ``shaders/smi.wgsl:777-795``
  (``extract_pair``, scale > 1.5), then the map's score (``combine_cell``) with MIN_N and the
  pair's correlation area in pixels;
* the symmetric average and the scale mask ``shaders/smi.wgsl:1708-1731`` (``rs_finish``), the
  argmax and the result ``src/engine.zig:836-872`` (``rsMap``), the default centre
  ``src/lie.zig:319-329`` (``movingCentroid``).
"""
from __future__ import annotations

import math

import numpy as np

from . import smi_oracle as O

MAP_AUTO_MIN, MAP_AUTO_MAX = 128, 512


def moving_centroid(H, lw, lh):
    H = np.asarray(H, np.float64).reshape(3, 3)
    pts = [(1, 1), (lw, 1), (lw, lh), (1, lh)]
    s = np.zeros(2)
    for x, y in pts:
        q = H @ [x, y, 1.0]
        z = q[2] if abs(q[2]) >= 1e-8 else 1e-8
        s += q[:2] / z
    return s / 4


def rs_plan(W, Hh, ox, oy, c, r0_opt=None, r1_opt=None, cap=0, sizes="ladder"):
    cx = c[0] - 1 - ox
    cy = c[1] - 1 - oy
    r1 = r1_opt or 0.0
    if r1 == 0:
        for px, py in ((0, 0), (W - 1, 0), (W - 1, Hh - 1), (0, Hh - 1)):
            r1 = max(r1, math.hypot(px - cx, py - cy))
    r0 = r0_opt if r0_opt is not None else max(2.0, min(r1 / 16, 8.0))
    r_out = max(r1, 2.0)
    r_in = min(max(r0, 1e-3), r_out / 8)
    n_ring = max(64, math.ceil(2 * math.pi * r_out))
    if cap == 0:
        n = min(max(1 << (n_ring - 1).bit_length(), MAP_AUTO_MIN), MAP_AUTO_MAX)
    else:
        n = min(O.plan_size(n_ring, 1, sizes), O.cap_n(cap, sizes, 8192))
    n_lam = max(16, n >> 1)
    log0 = math.log(r_in)
    span = math.log(r_out) - log0
    return {"n": n, "n_th": n, "n_lam": n_lam, "log0": log0, "span": span, "dlam": span / n_lam,
            "dth": 2 * math.pi / n, "r0": r_in, "r1": r_out, "cx": cx, "cy": cy}


def logpolar(stack, p):
    """(5, n_λ, n_θ) bilinear samples of a canvas stack (5, Hh, W) about (cx, cy). The sample
    points are computed in float32 as the reference's shader computes them (which samples fall
    inside the canvas depends on that rounding at its edge); the interpolation in float64."""
    s = np.asarray(stack, np.float64)
    h, w = s.shape[1:]
    f = np.float32
    yy, xx = np.mgrid[0:p["n_lam"], 0:p["n_th"]].astype(f)
    t = (yy + f(0.5)) / f(max(p["n_lam"], 1))
    rho32 = np.exp(f(p["log0"]) + t * f(p["span"])).astype(f)
    th = ((xx + f(0.5)) / f(p["n_th"]) * f(6.28318530718)).astype(f)
    xs32 = f(p["cx"]) + rho32 * np.cos(th).astype(f)
    ys32 = f(p["cy"]) + rho32 * np.sin(th).astype(f)
    xs, ys, rho = xs32.astype(np.float64), ys32.astype(np.float64), rho32.astype(np.float64)
    x0, y0 = np.floor(xs), np.floor(ys)
    ok = (x0 >= 0) & (y0 >= 0) & (x0 + 1 < w) & (y0 + 1 < h)
    fx, fy = xs - x0, ys - y0
    xi, yi = np.where(ok, x0, 0).astype(np.int64), np.where(ok, y0, 0).astype(np.int64)
    out = np.zeros((5,) + xx.shape)
    for q in range(5):
        a = s[q]
        v = ((1 - fx) * (1 - fy) * a[yi, xi] + fx * (1 - fy) * a[yi, xi + 1] + (1 - fx) * fy * a[yi + 1, xi]
             + fx * fy * a[yi + 1, xi + 1])
        out[q] = np.where(ok, v, 0.0)
    return out, rho[:, :1]


def rs_map_one(prep_a, prep_b, H, c, r0=None, r1=None, exact=True, calibrated=False, cap=0):
    """One direction's raw roto-scale map (n × n, lag 0 at [0, 0]) and its plan."""
    ha, wa = prep_a["stack"].shape[1:]
    hb, wb = prep_b["stack"].shape[1:]
    ox, oy, W, Hh = O.reg_frame(H, wa, ha, wb, hb)
    Hc = O.canvas_H(H, ox, oy)
    ca = O.warp_stack(prep_a["stack"], Hc, W, Hh)
    cb = O.paste_stack(prep_b["stack"], ox, oy, W, Hh)
    p = rs_plan(W, Hh, ox, oy, c, r0, r1, cap)
    p["frame"] = (ox, oy, W, Hh)
    la, rho = logpolar(ca, p)
    lb, _ = logpolar(cb, p)
    three = prep_a.get("mode") == "three"
    ids, corrs = O.corr_plan(exact, three)
    A = O.real_planes(la, ids) * rho
    B = O.real_planes(lb, ids) * rho
    n = p["n"]
    corr = O.correlations(A, B, ids, corrs, n, n)
    k = np.arange(n)
    k = np.where(k > n // 2, k - n, k)
    corr *= (np.exp(k * p["dlam"]) * p["dlam"] * p["dth"])[None, :, None]
    area = max(1.0, O.pair_area(prep_a["acf"], prep_b["acf"]))
    m = O.combine(corr, exact=exact, calibrated=calibrated, min_n=O.MIN_N, area=area, nf=3 if three else 4)
    return m, p, corr


def rs_finish(fwd, inv, mirror, dlam, smin=0.2, smax=5.0):
    n = fwd.shape[0]
    v = np.array(fwd, np.float64)
    if inv is not None:
        y, x = np.mgrid[0:n, 0:n]
        ym = (n - y) % n
        xm = (n - x) % n if mirror else x
        v = 0.5 * (v + inv[ym, xm])
    k = np.arange(n, dtype=np.float64)
    k = np.where(k > n // 2, k - n, k)
    lo = math.log(max(smin if smin > 0 else 0.2, 1e-6))
    hi = math.log(max(smax if smax > 0 else 5, 1.000001))
    sg = -k * dlam
    v[(sg < lo) | (sg > hi), :] = 0.0
    return v


def rs_map(prep_a, prep_b, H, c=None, symmetric=True, exact=True, calibrated=False, cap=0, smin=0.2, smax=5.0):
    """The finished roto-scale map with its peak: dth, dsg as the reference reports them."""
    H = np.asarray(H, np.float64).reshape(3, 3)
    ha, wa = prep_a["stack"].shape[1:]
    if c is None:
        c = moving_centroid(H, wa, ha)
    fwd, p, _ = rs_map_one(prep_a, prep_b, H, c, None, None, exact, calibrated, cap)
    inv = None
    if symmetric:
        Hi = np.linalg.inv(H)
        q = Hi @ [c[0], c[1], 1.0]
        ci = q[:2] / (q[2] if abs(q[2]) >= 1e-8 else 1e-8)
        inv, pi, _ = rs_map_one(prep_b, prep_a, Hi, ci, p["r0"], p["r1"], exact, calibrated, cap)
        assert pi["n"] == p["n"]
    mirror = H[0, 0] * H[1, 1] - H[0, 1] * H[1, 0] > 0
    fin = rs_finish(fwd, inv, mirror, p["dlam"], smin, smax)
    peak, idx = O.argmax_first(fin)
    n = p["n"]
    py, px = divmod(idx, n)
    lx = px if px <= n // 2 else px - n
    ly = py if py <= n // 2 else py - n
    return {"map": fin, "fwd": fwd, "inv": inv, "peak": peak, "peak_index": idx, "plan": p, "center": tuple(c),
            "dth": -(lx / p["n_th"]) * 2 * math.pi, "dsg": -ly * p["dlam"], "zero": float(fin.ravel()[0])}
