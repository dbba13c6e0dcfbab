"""CPU oracle for zcmir's NCC overlay metric (the zero-lag NCC score and the NCC shift map).

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` as the checker, never by the product path.

Restates in NumPy, float64 unless noted, ZacharyVarley/zcmir's:

* the union canvas ``src/overlay.zig:127-157`` (``canvas``, ``assemble``): the frame of
  ``src/lie.zig:537-579``, the moving work image warped by the canvas pose
  (``shaders/gls_mift.wgsl:1921-1956`` ``warp_homography``: bilinear, 0 where the source point
  leaves the image, stored as a texel, so rounded to f16 when half) and the fixed work image
  pasted at (−ox, −oy) (``paste_rect`` 1959-1969) on a cleared canvas;
* the zero-lag score ``src/overlay.zig:275-305`` (``nccScore``): Pearson's r over every canvas
  pixel, clamped to ±1.5;
* the map ``src/overlay.zig:209-273`` (``nccShiftMap``) with ``shaders/ncc.wgsl``: the plan
  ``src/fft.zig:70-91`` (``linearCorrPlan``, longest line min(maxFftN, 1024) = 1024), the canvas
  resampled to cw × ch (``pack``: one bilinear tap, clamped to the canvas edge, at
  ((x + ½)·W/cw, (y + ½)·H/ch) in pixel-centre units; positions in float32 as the shader takes
  them), each side made mean-free over the grid, the circular correlation Σ a(x + t)·b(x) of the
  zero-padded n × n planes (``cmul`` A·conj(B), inverse scaled 1/n²) over ‖a‖·‖b‖ (floored at
  1e-12), clamped to ±1.5; the first maximum and its lag in canvas pixels
  (``src/engine.zig:789-793`` ``peakLag``, scaled by W/cw and H/ch).

The reference sums in float32 partials (64 workgroups) and the B200 build in float64; this
oracle sums in float64.
"""
from __future__ import annotations

import numpy as np

from oracle import smi_oracle as O

F32 = np.float32
NCC_MAX_N = 1024   # src/overlay.zig:217: min(maxFftN, 1024)


def canvas(work_a, work_b, H, half=False):
    """(a, b, frame): both sides on the pose's union canvas (moving warped, fixed pasted)."""
    wa = np.asarray(work_a, np.float64)
    wb = np.asarray(work_b, np.float64)
    lh, lw = wa.shape
    rh, rw = wb.shape
    ox, oy, W, Hh = O.reg_frame(H, lw, lh, rw, rh)
    Hc = O.canvas_H(H, ox, oy)
    a = O.warp_stack(wa[None], Hc, W, Hh)[0]
    if half:
        a = a.astype(np.float32).astype(np.float16).astype(np.float64)
    b = O.paste_stack(wb[None], ox, oy, W, Hh)[0]
    return a, b, (ox, oy, W, Hh)


def ncc_score(work_a, work_b, H, half=False):
    a, b, _ = canvas(work_a, work_b, H, half)
    n = a.size
    sa, sb = a.sum(), b.sum()
    cov = (a * b).sum() - sa * sb / n
    va = max((a * a).sum() - sa * sa / n, 0.0)
    vb = max((b * b).sum() - sb * sb / n, 0.0)
    return float(min(1.5, max(-1.5, cov / np.sqrt(max(va * vb, 1e-24)))))


def linear_corr_plan(w, h, max_n0=NCC_MAX_N, sizes="ladder"):
    """(n, cw, ch) with one FFT length for both axes (``src/fft.zig:70-91``)."""
    max_n = O.largest_smooth(max_n0, sizes)
    s = min(1.0, max(8, max_n >> 1) / max(max(w, h), 1))
    n, cw, ch = 8, 8, 8
    for _ in range(16):
        cw = max(8, O._js_round(w * s))
        ch = max(8, O._js_round(h * s))
        n = min(O.plan_size(max(cw + cw - 1, ch + ch - 1, 32), 1, sizes), max_n)
        if n >= cw + cw - 1 and n >= ch + ch - 1:
            return n, cw, ch
        s *= 0.85
    return n, max(8, min(cw, (n + 1) >> 1)), max(8, min(ch, (n + 1) >> 1))


def pack(plane, cw, ch):
    """The canvas plane at cw × ch cells: one bilinear tap per cell, clamped to the edge."""
    Hh, W = plane.shape
    gx = np.arange(cw, dtype=F32)
    gy = np.arange(ch, dtype=F32)
    px = ((gx + F32(0.5)) * F32(W) / F32(max(cw, 1)) - F32(0.5)).astype(np.float64)
    py = ((gy + F32(0.5)) * F32(Hh) / F32(max(ch, 1)) - F32(0.5)).astype(np.float64)
    x0, y0 = np.floor(px).astype(np.int64), np.floor(py).astype(np.int64)
    tx, ty = px - x0, py - y0
    xa, xb = np.clip(x0, 0, W - 1), np.clip(x0 + 1, 0, W - 1)
    ya, yb = np.clip(y0, 0, Hh - 1), np.clip(y0 + 1, 0, Hh - 1)
    r0 = plane[ya][:, xa] * (1 - tx) + plane[ya][:, xb] * tx
    r1 = plane[yb][:, xa] * (1 - tx) + plane[yb][:, xb] * tx
    return r0 * (1 - ty[:, None]) + r1 * ty[:, None]


def ncc_map(work_a, work_b, H, half=False, sizes="ladder"):
    """dict(map (n × n, lag 0 at index 0), n, cw, ch, frame, peak, peak_index, dx, dy, zero)."""
    a, b, fr = canvas(work_a, work_b, H, half)
    ox, oy, W, Hh = fr
    n, cw, ch = linear_corr_plan(W, Hh, NCC_MAX_N, sizes)
    ga, gb = pack(a, cw, ch), pack(b, cw, ch)
    ga = ga - ga.mean()
    gb = gb - gb.mean()
    den = max(np.sqrt((ga * ga).sum()) * np.sqrt((gb * gb).sum()), 1e-12)
    A = np.zeros((n, n))
    B = np.zeros((n, n))
    A[:ch, :cw] = ga
    B[:ch, :cw] = gb
    corr = np.fft.ifft2(np.fft.fft2(A) * np.conj(np.fft.fft2(B))).real
    m = np.clip(corr / den, -1.5, 1.5)
    idx = int(np.argmax(m))
    lx, ly = O.peak_lag(idx, n, n)
    return dict(map=m, n=n, cw=cw, ch=ch, frame=fr, peak=float(m.flat[idx]), peak_index=idx,
                dx=lx * (W / cw), dy=ly * (Hh / ch), zero=float(m[0, 0]))
