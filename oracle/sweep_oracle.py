"""CPU oracle for the rotation × scale (× shear × stretch) sweep of zcmir's SMI path.

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` and ``bench.py``'s CPU legs as the checker or
the timed CPU baseline, never by the product path.

Restates the reference's brute-force sweep (ZacharyVarley/zcmir):

* the candidate grid ``src/search.zig:89-116`` (``sweepGrid``), the linear part
  ``src/search.zig:120-128`` (``candLinear``) about the moving centre ``130-132`` (``aboutC``),
  singular values ``135-142`` (``sv2``);
* the canvas, footprints, ladder plane sizes and box taps ``src/search.zig:300-371``, the plane
  sizes ``src/search.zig:185-190`` (``ladderSize``);
* the packing ``shaders/sweep.wgsl:62-152`` (``tap``, ``real_plane``, ``pack_sweep``): k×k
  bilinear taps per canvas cell, zero where the 2×2 footprint leaves the image;
* the per-shift score ``shaders/sweep.wgsl:226-317`` (``combine_sweep``: the map's combine,
  uncalibrated, the overlap floor taken at the candidate's own zero lag ``zero_lag``), here in
  float64 on float64 FFT correlations;
* the peaks ``shaders/sweep.wgsl:319-371`` (``peaks_sweep``): each of 256 lanes keeps the best
  3×3 local maximum among the shifts t ≡ lane (mod 256), periodic; the top ``n_peak`` lanes by
  score; and their poses ``src/search.zig:460-493``;
* the non-maximum suppression ``src/search.zig:500-529`` (``nms4``).
"""
from __future__ import annotations

import math

import numpy as np

from . import smi_oracle as O

# compact plane lengths (src/search.zig:183)
LADDER_COMPACT = [32, 48, 64, 80, 96, 128, 160, 192, 224, 256, 320, 384, 448, 512]


def linspace(lo, hi, n):
    n = max(1, n)
    if n == 1:
        return [0.5 * (lo + hi)]
    return [lo + (i * (hi - lo)) / (n - 1) for i in range(n)]


def sweep_grid(rot_lo=-180.0, rot_hi=180.0, n_theta=90, s_min=0.5, s_max=2.0, n_sigma=20, shear_max=0.0, n_shear=1,
               aniso_max=0.0, n_aniso=1):
    """θ (rad), σ, shear k, stretch a lists and the wrap flag (``src/search.zig:89-116``)."""
    nT = max(1, n_theta)
    lo_d = min(rot_lo, rot_hi)
    span_d = abs(rot_hi - rot_lo)
    wrap = span_d >= 360 - 1e-9
    th = []
    for i in range(nT):
        if wrap:
            d = -180 + 360 * i / nT
        elif nT == 1:
            d = lo_d + span_d / 2
        else:
            d = lo_d + span_d * i / (nT - 1)
        th.append(d * math.pi / 180.0)
    llo = math.log(max(1e-3, min(s_min, s_max)))
    lhi = math.log(max(1e-3, max(s_min, s_max)))
    sg = [math.exp(v) for v in linspace(llo, lhi, n_sigma)]
    kmax = abs(shear_max)
    sh = linspace(-kmax, kmax, n_shear if kmax > 0 else 1)
    amax = math.log(1 + abs(aniso_max))
    an = [math.exp(v) for v in linspace(-amax, amax, n_aniso if amax > 0 else 1)]
    return {"thetas": th, "sigmas": sg, "shears": sh, "anisos": an, "wrap": wrap}


def cand_linear(th, s, k, a):
    """σ R(θ) diag(a, 1/a) [1 k; 0 1], row-major 2×2."""
    c, sn = s * math.cos(th), s * math.sin(th)
    p00, p01, p11 = a, a * k, 1 / a
    return [c * p00, c * p01 - sn * p11, sn * p00, sn * p01 + c * p11]


def about_c(cc, L):
    return np.array([[L[0], L[1], cc[0] - L[0] * cc[0] - L[1] * cc[1]],
                     [L[2], L[3], cc[1] - L[2] * cc[0] - L[3] * cc[1]], [0, 0, 1.0]])


def sv2(L):
    a = L[0] * L[0] + L[2] * L[2]
    b = L[0] * L[1] + L[2] * L[3]
    d = L[1] * L[1] + L[3] * L[3]
    t = 0.5 * (a + d)
    r = math.sqrt(max(0.0, 0.25 * (a - d) * (a - d) + b * b))
    return math.sqrt(t + r), math.sqrt(max(0.0, t - r))


def map_pt(H, x, y):
    X = H[0, 0] * x + H[0, 1] * y + H[0, 2]
    Y = H[1, 0] * x + H[1, 1] * y + H[1, 2]
    Z = H[2, 0] * x + H[2, 1] * y + H[2, 2]
    z = 1e-8 if abs(Z) < 1e-8 else Z
    return X / z, Y / z


def ladder_size(need, sizes="ladder"):
    if sizes == "compact":
        for L in LADDER_COMPACT:
            if L >= need:
                return L
    return O.plan_size(need, 16, sizes)


def _cells(a, b, o0, c, G):
    lo = min(max(int(math.floor((a - o0) / c)) - 1, 0), G)
    hi = min(max(int(math.ceil((b - o0) / c)) + 1, lo + 1), G)
    return lo, hi


def sweep_setup(mw, mh, fw, fh, H0, gv, G=128, sizes="ladder"):
    """Canvas, the fixed footprint and every candidate (θ-major) with its pose, window origin,
    plane size and taps (``src/search.zig:300-371``), plus the slot order (by plane size)."""
    H0 = np.asarray(H0, np.float64).reshape(3, 3)
    cm = map_pt(H0, (mw + 1) / 2, (mh + 1) / 2)
    s_max = max(sv2(cand_linear(0, s, k, a))[0] for s in gv["sigmas"] for k in gv["shears"] for a in gv["anisos"])
    D = min(2 * max(fw, fh), max(max(fw, fh), s_max * math.hypot(mw, mh)))
    cell = D / G
    ox, oy = (fw + 1) / 2 - D / 2, (fh + 1) / 2 - D / 2
    fcx, fcy = _cells(0.5, fw + 0.5, ox, cell, G), _cells(0.5, fh + 0.5, oy, cell, G)
    Fx, Fy = fcx[1] - fcx[0], fcy[1] - fcy[0]
    s0r = math.sqrt(abs(H0[0, 0] * H0[1, 1] - H0[0, 1] * H0[1, 0]))
    s0 = 1.0 if (s0r == 0 or math.isnan(s0r)) else s0r
    cands = []
    for i, th in enumerate(gv["thetas"]):
        for j, s in enumerate(gv["sigmas"]):
            for ik, kk in enumerate(gv["shears"]):
                for ia, a in enumerate(gv["anisos"]):
                    L = cand_linear(th, s, kk, a)
                    H = about_c(cm, L) @ H0
                    pts = [map_pt(H, *q) for q in ((0.5, 0.5), (mw + 0.5, 0.5), (mw + 0.5, mh + 0.5), (0.5, mh + 0.5))]
                    xs, ys = [p[0] for p in pts], [p[1] for p in pts]
                    ok = all(math.isfinite(v) for v in xs + ys)
                    mcx = _cells(min(xs), max(xs), ox, cell, G) if ok else (0, G)
                    mcy = _cells(min(ys), max(ys), oy, cell, G) if ok else (0, G)
                    cands.append({
                        "it": i, "is": j, "ik": ik, "ia": ia, "th": th, "s": s, "H": H,
                        "gx0": mcx[0], "gy0": mcy[0],
                        "nx": ladder_size(mcx[1] - mcx[0] + Fx - 1, sizes), "ny": ladder_size(mcy[1] - mcy[0] + Fy - 1, sizes),
                        "taps": float(min(6, max(1, math.ceil(cell / (sv2(L)[1] * s0) - 1e-3)))),
                    })
    perm = sorted(range(len(cands)), key=lambda c: ((cands[c]["nx"] << 32) | cands[c]["ny"], c))
    return {"cell": cell, "ox": ox, "oy": oy, "G": G, "fcx": fcx, "fcy": fcy, "Fx": Fx, "Fy": Fy,
            "fixed_taps": float(min(6, max(1, math.ceil(cell - 1e-3)))), "cands": cands, "perm": perm}


def pack_window(stack, Hinv, taps, gx0, gy0, win_x, win_y, nx, ny, ox, oy, cell, G, f32_positions=False):
    """(5, ny, nx) premultiplied samples of a window of canvas cells at the plane origin
    (``shaders/sweep.wgsl:62-152``): each cell the mean of k×k bilinear taps of the source stack
    mapped through Hinv (dest → source, 1-based); a tap whose 2×2 footprint leaves the image adds
    nothing. Zero outside the window and the G×G canvas.

    f32_positions: the tap positions (px, py, the mapped qx, qy, qz and x = qx/qz − 1) in float32,
    one rounding per operation, as the reference's shader computes them
    (``shaders/sweep.wgsl:132-138``); the interpolation stays float64. A tap within ~1e-4 px of
    the image's edge enters or leaves with that rounding, and its whole sample with it."""
    src = np.asarray(stack, np.float64)
    h, w = src.shape[1:]
    k = max(int(taps), 1)
    out = np.zeros((5, ny, nx))
    yy, xx = np.mgrid[0:min(win_y, ny), 0:min(win_x, nx)]
    cx, cy = gx0 + xx, gy0 + yy
    inside = (cx < G) & (cy < G)
    acc = np.zeros((5,) + xx.shape)
    Hi = np.asarray(Hinv, np.float64).reshape(3, 3)
    if f32_positions:
        F = np.float32
        Hi = Hi.astype(F)
        cxf, cyf, kf, oxf, oyf, cellf = cx.astype(F), cy.astype(F), F(k), F(ox), F(oy), F(cell)
    for ty in range(k):
        if f32_positions:
            py = oyf + (cyf + (F(ty) + F(0.5)) / kf) * cellf
        else:
            py = oy + (cy + (ty + 0.5) / k) * cell
        for tx in range(k):
            if f32_positions:
                px = oxf + (cxf + (F(tx) + F(0.5)) / kf) * cellf
            else:
                px = ox + (cx + (tx + 0.5) / k) * cell
            qx = Hi[0, 0] * px + Hi[0, 1] * py + Hi[0, 2]
            qy = Hi[1, 0] * px + Hi[1, 1] * py + Hi[1, 2]
            qz = Hi[2, 0] * px + Hi[2, 1] * py + Hi[2, 2]
            okz = np.abs(qz) >= 1e-8
            qzs = np.where(okz, qz, qz.dtype.type(1))
            x, y = qx / qzs - qz.dtype.type(1), qy / qzs - qz.dtype.type(1)
            x, y = x.astype(np.float64), y.astype(np.float64)
            x0, y0 = np.floor(x), np.floor(y)
            ok = okz & (x0 >= 0) & (y0 >= 0) & (x0 + 1 < w) & (y0 + 1 < h) & inside
            fx, fy = x - x0, y - y0
            xi = np.where(ok, x0, 0).astype(np.int64)
            yi = np.where(ok, y0, 0).astype(np.int64)
            for p in range(5):
                s = src[p]
                v = ((1 - fx) * (1 - fy) * s[yi, xi] + fx * (1 - fy) * s[yi, xi + 1] + (1 - fx) * fy * s[yi + 1, xi]
                     + fx * fy * s[yi + 1, xi + 1])
                acc[p] += np.where(ok, v, 0.0)
    out[:, :xx.shape[0], :xx.shape[1]] = np.where(inside, acc / (k * k), 0.0)
    return out


def zero_lag(c, setup):
    lx = (setup["fcx"][0] - c["gx0"]) % c["nx"]
    ly = (setup["fcy"][0] - c["gy0"]) % c["ny"]
    return ly * c["nx"] + lx


def candidate_map(prep_a, prep_b, setup, c, exact=True, three=False, min_n=12, f32_positions=False):
    """One candidate's shift map (ny × nx, cell units, float64) and its zero-lag overlap."""
    nx, ny, Fx, Fy = c["nx"], c["ny"], setup["Fx"], setup["Fy"]
    sa = pack_window(prep_a["stack"], np.linalg.inv(c["H"]), c["taps"], c["gx0"], c["gy0"], nx - Fx + 1, ny - Fy + 1,
                     nx, ny, setup["ox"], setup["oy"], setup["cell"], setup["G"], f32_positions)
    sb = pack_window(prep_b["stack"], np.eye(3), setup["fixed_taps"], setup["fcx"][0], setup["fcy"][0], Fx, Fy, nx, ny,
                     setup["ox"], setup["oy"], setup["cell"], setup["G"], f32_positions)
    ids, corrs = O.corr_plan(exact, three)
    corr = O.correlations(O.real_planes(sa, ids), O.real_planes(sb, ids), ids, corrs, nx, ny)
    n0 = corr[0].ravel()[zero_lag(c, setup)]
    m = O.combine(corr, exact=exact, calibrated=False, min_n=min_n, nf=3 if three else 4, n00=n0)
    return m, n0


def lane_peaks(m, n_peak=4, lanes=256):
    """Top n_peak (score, index) of the 256 lanes' best 3×3 local maxima (periodic); a lane
    with no positive local maximum gives (0, 0xffffffff)."""
    ny, nx = m.shape
    flat = m.ravel()
    nbr = np.full(m.shape, -np.inf)
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            if dx or dy:
                nbr = np.maximum(nbr, np.roll(np.roll(m, -dy, axis=0), -dx, axis=1))
    is_max = (m >= nbr).ravel() & (flat > 0)
    out = []
    for lane in range(lanes):
        idx = np.arange(lane, flat.size, lanes)
        bv, bi = 0.0, 0xFFFFFFFF
        # the lane's scan keeps the first of equal maxima (strictly greater replaces)
        for t in idx[is_max[idx]]:
            if flat[t] > bv:
                bv, bi = flat[t], int(t)
        out.append((bv, bi))
    out.sort(key=lambda p: -p[0])
    return out[:n_peak]


def peak_pose(c, setup, t):
    """Canvas displacement (cells) and pose T(−d)·H of map index t (``src/search.zig:470-492``)."""
    nx, ny = c["nx"], c["ny"]
    py, px = divmod(t, nx)
    wx, wy = nx - setup["Fx"] + 1, ny - setup["Fy"] + 1
    lx = px if px < wx else px - nx
    ly = py if py < wy else py - ny
    sx = c["gx0"] + lx - setup["fcx"][0]
    sy = c["gy0"] + ly - setup["fcy"][0]
    dx, dy = sx * setup["cell"], sy * setup["cell"]
    return sx, sy, np.array([[1, 0, -dx], [0, 1, -dy], [0, 0, 1.0]]) @ c["H"]


def min_count(min_overlap, fw, fh, cell):
    return int(max(12.0, O._js_round(min_overlap * (fw * fh) / (cell * cell))))


def sweep(prep_a, prep_b, H0, gv, G=128, exact=True, three=False, min_overlap=0.05, n_peak=4, sizes="ladder",
          only=None, f32_positions=False):
    """Every candidate's peaks (slot order, as the reference appends them) and each candidate's
    best score; ``only``: restrict to these candidate indices (for small checks);
    ``f32_positions``: the taps placed in float32 as the reference places them (pack_window)."""
    mh, mw = prep_a["stack"].shape[1:]
    fh, fw = prep_b["stack"].shape[1:]
    st = sweep_setup(mw, mh, fw, fh, H0, gv, G, sizes)
    min_n = min_count(min_overlap, fw, fh, st["cell"])
    c2 = st["cell"] ** 2
    peaks, raw = [], {}
    best = np.zeros(len(st["cands"]))
    for ci in st["perm"]:
        if only is not None and ci not in only:
            continue
        c = st["cands"][ci]
        m, _ = candidate_map(prep_a, prep_b, st, c, exact, three, min_n, f32_positions)
        top = lane_peaks(m, n_peak)
        raw[ci] = top
        for k, (v0, t) in enumerate(top):
            v = v0 * c2
            if not (v > 0) or t >= c["nx"] * c["ny"]:
                continue
            if k == 0:
                best[ci] = v
            sx, sy, H = peak_pose(c, st, t)
            peaks.append({"score": v, "cand": ci, "it": c["it"], "is": c["is"], "ik": c["ik"], "ia": c["ia"],
                          "th": c["th"], "s": c["s"], "sx": sx, "sy": sy, "H": H, "t": t})
    return {"setup": st, "min_n": min_n, "peaks": peaks, "best": best, "raw": raw}


def nms4(peaks, n_theta, keep, wrap):
    """Strongest first (stable); a peak survives unless a kept one lies within ±2 θ steps
    (circular when wrap), ±2 σ steps, ±1 shear and stretch step and 4 cells."""
    kept = []
    for p in sorted(peaks, key=lambda q: -q["score"]):
        ok = True
        for q in kept:
            a = abs(p["it"] - q["it"])
            dt = min(a, n_theta - a) if wrap else a
            if (dt <= 2 and abs(p["is"] - q["is"]) <= 2 and abs(p["ik"] - q["ik"]) <= 1 and abs(p["ia"] - q["ia"]) <= 1
                    and math.hypot(p["sx"] - q["sx"], p["sy"] - q["sy"]) <= 4):
                ok = False
                break
        if ok:
            kept.append(p)
            if len(kept) >= keep:
                break
    return kept
