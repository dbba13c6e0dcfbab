"""Host driver for libzcmir.so: numpy arrays in, numpy arrays and small records out.

``Engine`` wraps one engine handle of the C ABI (include/zcmir.h for the reference's zc_* calls,
include/zcmir_b200.h for this build's zcb_* extensions). Every method is one C call (or a short
fixed sequence of them); nothing here computes on the CPU. The drop-in front end for users of
the reference is the reference's own unchanged Python package pointed at this library
(``ZCMIR_LIB``); this module is what this repository's tests, bench and extensions drive.

    from zcmir_b200 import Engine
    with Engine(half=False) as eng:
        eng.set_images(moving, fixed, preprocess=False)
        m = eng.shift_map(exact=True, calibrated=True, cap=2048)
        m.peak, m.dx, m.dy, m.map            # map: n_y × n float32, lag (0, 0) at [0, 0]

Poses are 3×3 float64 maps from moving to fixed pixel coordinates, 1-based pixel centres.
Failures raise ``EngineError("<call>: <the engine's message>")``.
"""
from __future__ import annotations

import ctypes
import json
from typing import NamedTuple

import numpy as np

from . import _native as N

LUMA = np.array([0.299, 0.587, 0.114])


class EngineError(RuntimeError):
    """A zc_* / zcb_* call returned its failure value; the text is the engine's message."""


# ── array conversion ─────────────────────────────────────────────────────────────────────────

def gray32(img) -> np.ndarray:
    """img as a C-contiguous float32 gray image: uint8 ÷ 255, uint16 ÷ 65535, colour by luma."""
    a = np.asarray(img)
    scale = {np.dtype(np.uint8): 255.0, np.dtype(np.uint16): 65535.0}.get(a.dtype)
    if a.ndim == 3 and a.shape[2] in (3, 4):
        a = a[..., :3].astype(np.float64) @ LUMA
    if scale is not None:
        a = a / scale
    if a.ndim != 2:
        raise ValueError(f"a gray image is (h, w); got shape {a.shape}")
    return np.ascontiguousarray(a, np.float32)


def rgba8(img) -> np.ndarray:
    """A uint8 gray / RGB / RGBA image as (h, w, 4) RGBA8 (gray replicated, alpha 255)."""
    a = np.asarray(img)
    if a.ndim == 2:
        a = a[:, :, None]
    if a.ndim != 3 or a.shape[2] not in (1, 3, 4):
        raise ValueError(f"a uint8 image is (h, w), (h, w, 3) or (h, w, 4); got shape {a.shape}")
    out = np.empty(a.shape[:2] + (4,), np.uint8)
    out[..., :3] = a[..., :3] if a.shape[2] >= 3 else a
    out[..., 3] = a[..., 3] if a.shape[2] == 4 else 255
    return out


def _f32(a):
    return a.ctypes.data_as(N.f32p)


def _f64(a):
    return a.ctypes.data_as(N.f64p)


def _u32(a):
    return a.ctypes.data_as(N.u32p)


def _pose9(H):
    return np.ascontiguousarray(np.asarray(H, np.float64).reshape(9))


def _mat3(c_arr):
    return np.array(c_arr[:9], np.float64).reshape(3, 3)


def _fields(st) -> dict:
    return {name: getattr(st, name) for name, _ in st._fields_ if not name.startswith("_")}


# ── records ──────────────────────────────────────────────────────────────────────────────────

class Scores(NamedTuple):
    mean: float        # the symmetric score (the forward one when not symmetric)
    fwd: float
    inv: float | None  # None when the score is one-sided


class Grad(NamedTuple):
    score: float
    fwd: float
    inv: float | None
    n: float           # overlap (forward direction)
    grad: np.ndarray   # nk tangent components (8 homography, 6 affine)
    hess: np.ndarray | None


class ClimbOut(NamedTuple):
    H: np.ndarray
    score: float
    iterations: int
    moved: bool


class SearchOut(NamedTuple):
    H: np.ndarray
    score: float
    prev: float
    improved: bool
    count_a: int
    count_b: int


class SweepOut(NamedTuple):
    scores: np.ndarray  # (candidates, lanes) float32, fixed-pixel units
    index: np.ndarray   # (candidates, lanes) uint32 map index, 0xffffffff where empty
    info: dict


class MapResult:
    """A zc_shift_map result: every ShiftResult field as an attribute, plus ``map`` (n_y × n
    float32 or None). A cell spans canvas_w / cw × canvas_h / ch pixels; (dx, dy) is the peak's
    lag in fixed pixels."""

    def __init__(self, st, grid=None):
        self.__dict__.update(_fields(st))
        self.ny = self.n_y or self.n
        self.map = grid

    @property
    def canvas(self):
        return self.canvas_w, self.canvas_h

    @property
    def offset(self):
        return self.ox, self.oy

    def corrected(self, H):
        """The pose moved by the peak's lag: T(−dx, −dy)·H."""
        return np.array([[1, 0, -self.dx], [0, 1, -self.dy], [0, 0, 1.0]]) @ np.asarray(H, np.float64).reshape(3, 3)

    def __repr__(self):
        return f"MapResult(peak={self.peak:.6g}, dx={self.dx}, dy={self.dy}, n={self.n}×{self.ny})"


class RsMapResult:
    """A zc_rs_map result: every RsResult field as an attribute (dth, dsg: the rotation in radians
    and log scale that correct the pose), plus ``map``, ``fwd``, ``inv`` (n × n or None)."""

    def __init__(self, st, maps):
        self.__dict__.update(_fields(st))
        self.map, self.fwd, self.inv = maps

    @property
    def center(self):
        return self.cx, self.cy


SWEEP_INFO = ("candidates", "cell", "ms", "grid", "Fx", "Fy", "fx0", "fy0", "min_n", "n", "groups", "batches",
              "launches", "ox", "oy", "peaks")
BENCH_STAGES = ("canvas", "fwd_rows", "fwd_cols", "inv_cols", "inv_rows_score")


# ── the engine ───────────────────────────────────────────────────────────────────────────────

class Engine:
    """One engine of libzcmir.so: a CUDA context on the current device, one image pair whose
    features stay resident in HBM between calls, the settings and the current pose. Keyword
    arguments are settings. Not thread-safe (one caller at a time, as the C ABI)."""

    def __init__(self, **settings):
        self.lib = N.load()
        self.handle = self.lib.zc_create(b"")
        if not self.handle:
            buf = ctypes.create_string_buffer(512)
            n = self.lib.zc_create_error(buf, 512)
            raise EngineError("create: " + (buf.raw[:n].decode(errors="replace") or "no engine"))
        if settings:
            self.configure(**settings)

    # plumbing
    def message(self) -> str:
        """The engine's last error message (and clears it)."""
        buf = ctypes.create_string_buffer(2048)
        n = self.lib.zc_error(self.handle, buf, len(buf))
        return buf.raw[:n].decode(errors="replace")

    def call(self, name, *args):
        """Call zc_<name> / zcb_<name> (full symbol name) with the handle first; raise on −1."""
        rc = getattr(self.lib, name)(self.handle, *args)
        if rc != 0:
            raise EngineError(f"{name.split('_', 1)[1]}: {self.message() or rc}")

    def _text(self, fn, cap=1 << 14):
        buf = ctypes.create_string_buffer(cap)
        n = fn(self.handle, buf, cap)
        if n > cap:
            buf = ctypes.create_string_buffer(n)
            n = fn(self.handle, buf, n)
        return buf.raw[:n].decode(errors="replace")

    @property
    def adapter(self) -> str:
        return self._text(self.lib.zc_adapter, 512)

    def events(self) -> list:
        """Progress events queued since the last read, as dicts (one JSON object per line)."""
        out = []
        while True:
            chunk = self._text(self.lib.zc_events, 1 << 16)
            if not chunk:
                return out
            out += [json.loads(x) for x in chunk.splitlines() if x]

    # settings
    def configure(self, **kw):
        js = json.dumps(kw).encode()
        self.call("zc_configure", js, len(js))

    @property
    def settings(self) -> dict:
        return json.loads(self._text(self.lib.zc_settings, 1 << 13))

    # images
    def set_image(self, side, img, preprocess=True):
        """Side 0 (moving) or 1 (fixed). uint8 images go up as RGBA8, which the engine always
        preprocesses; anything else as float32 gray, preprocessed (CLAHE / band pass / invert of
        the settings) when ``preprocess``."""
        a = np.asarray(img)
        if a.dtype == np.uint8:
            if not preprocess:
                raise ValueError("uint8 images are always preprocessed; pass a float gray image to skip it")
            px = rgba8(a)
            self.call("zc_set_image_rgba", side, px.ctypes.data_as(N.u8p), px.shape[1], px.shape[0])
            return
        g = gray32(a)
        self.call("zc_set_image_gray", side, _f32(g), g.shape[1], g.shape[0], int(bool(preprocess)))

    def set_images(self, moving, fixed, preprocess=True):
        self.set_image(0, moving, preprocess)
        self.set_image(1, fixed, preprocess)

    def image_size(self, side):
        wh = (ctypes.c_uint32 * 2)()
        self.lib.zc_image_size(self.handle, side, wh)
        return int(wh[0]), int(wh[1])

    def work_image(self, side) -> np.ndarray:
        w, h = self.image_size(side)
        out = np.empty((h, w), np.float32)
        self.call("zc_work_image", side, _f32(out), out.size)
        return out

    def features(self, side) -> np.ndarray:
        """(4, h, w) float32: the whitened feature planes (rank, rank², Sobel magnitude, fourth)."""
        w, h = self.image_size(side)
        out = np.empty((4, h, w), np.float32)
        self.call("zc_features", side, _f32(out), out.size)
        return out

    # pose and spline
    @property
    def pose(self) -> np.ndarray:
        H = np.empty(9)
        self.lib.zc_get_pose(self.handle, _f64(H))
        return H.reshape(3, 3)

    @pose.setter
    def pose(self, H):
        a = _pose9(H)
        self.lib.zc_set_pose(self.handle, _f64(a))

    def _at(self, H):
        return _pose9(self.pose if H is None else H)

    @property
    def ffd(self) -> np.ndarray:
        """Control points of the B-spline (x, y per point, row by row; 2·g² float32)."""
        buf = np.zeros(2 * 16 * 16, np.float32)
        n = self.lib.zc_get_ffd(self.handle, _f32(buf), buf.size)
        return buf[:n].copy()

    @ffd.setter
    def ffd(self, cps):
        a = np.ascontiguousarray(cps, np.float32).ravel()
        self.call("zc_set_ffd", _f32(a), a.size)

    # scores
    def moments(self, H=None) -> np.ndarray:
        a, out = self._at(H), np.empty(45)
        self.call("zc_moments", _f64(a), _f64(out))
        return out

    def score(self, H=None) -> Scores:
        a, out = self._at(H), np.empty(3)
        self.call("zc_score", _f64(a), _f64(out))
        return Scores(float(out[0]), float(out[1]), None if np.isnan(out[2]) else float(out[2]))

    def score_static(self, Hs) -> np.ndarray:
        """zcb_score_static: (n, 3) mean / fwd / inv for n ≤ 64 poses, no device allocation."""
        a = np.ascontiguousarray(np.asarray(Hs, np.float64).reshape(-1, 9))
        out = np.empty((len(a), 3))
        self.call("zcb_score_static", _f64(a), len(a), _f64(out))
        return out

    def gradient(self, H=None, hess=False) -> Grad:
        a, r = self._at(H), N.GradResult()
        self.call("zc_gradient", _f64(a), int(bool(hess)), ctypes.byref(r))
        nk = r.nk
        A = np.array(r.hess[:nk * nk]).reshape(nk, nk) if r.has_hess else None
        return Grad(r.score, r.fwd, None if np.isnan(r.inv) else r.inv, r.n, np.array(r.grad[:nk]), A)

    def ffd_gradient(self, H=None):
        """(score, gradient over the spline's control points) at H."""
        a, s = self._at(H), ctypes.c_double()
        g = np.zeros(2 * 16 * 16)
        self.call("zc_ffd_gradient", _f64(a), ctypes.byref(s), _f64(g), g.size)
        grid = min(max(int(self.settings["ffd_grid"]), 2), 16)
        return s.value, g[:2 * grid * grid].copy()

    def displacement(self) -> np.ndarray:
        """(h, w, 2) float32 over the fixed image: moving − fixed position (0-based pixels)."""
        w, h = self.image_size(1)
        out = np.empty((h, w, 2), np.float32)
        self.call("zc_displacement", _f32(out), out.size)
        return out

    # maps
    def shift_map(self, H=None, *, exact=None, calibrated=None, cap=1024, want_map=True, out=None) -> MapResult:
        """The SMI score of every translation about H. With exact and calibrated both None the
        settings decide everything (zc_shift_map_set); otherwise zc_shift_map with those flags
        (None counts as on) and FFT side cap ``cap``. ``out``: a float32 buffer to write the map
        into (its first n_y·n values), else a fresh array."""
        a, r = self._at(H), N.ShiftResult()
        buf = None
        if want_map:
            side = max(int(cap or 0), int(self.settings.get("map_res", 0) or 0), 1024)
            buf = out if out is not None else np.empty(side * side, np.float32)
        ptr, ln = (_f32(buf), buf.size) if buf is not None else (None, 0)
        if exact is None and calibrated is None:
            self.call("zc_shift_map_set", _f64(a), ctypes.byref(r), ptr, ln)
        else:
            flags = (exact is not False) * 1 + (calibrated is not False) * 2
            self.call("zc_shift_map", _f64(a), flags, int(cap), ctypes.byref(r), ptr, ln)
        grid = None
        if buf is not None:
            grid = buf[:r.n * (r.n_y or r.n)].reshape(r.n_y or r.n, r.n)
            grid = grid if out is not None else grid.copy()
        return MapResult(r, grid)

    def rs_map(self, H=None, *, center=None, symmetric=True, want_maps=True) -> RsMapResult:
        """The roto-scale map about ``center`` (fixed pixels, 1-based; None: the moving image's
        centroid under H)."""
        a, r = self._at(H), N.RsResult()
        res = int(self.settings["map_res"])
        side = 512 if res == 0 else min(res, 8192)
        cap = side * side if want_maps else 0
        bufs = [np.empty(cap, np.float32) if want_maps else None for _ in range(3)]
        if not symmetric:
            bufs[2] = None
        c = (ctypes.c_double * 2)(*center) if center is not None else None
        ptrs = [_f32(b) if b is not None else None for b in bufs]
        self.call("zc_rs_map", _f64(a), c, int(bool(symmetric)), ctypes.byref(r), *ptrs, cap)
        nn = r.n * r.n
        return RsMapResult(r, [b[:nn].reshape(r.n, r.n).copy() if b is not None else None for b in bufs])

    def canvas(self, H=None, inverse=False):
        """((ox, oy), (w, h), Hc): the union frame of the pair at H and the canvas pose."""
        a, c = self._at(H), N.Canvas()
        self.call("zc_canvas", _f64(a), int(bool(inverse)), ctypes.byref(c))
        return (c.ox, c.oy), (c.ow, c.oh), _mat3(c.Hc)

    def stack_maps(self, slices, priors=None, *, exact=True, calibrated=False, cap=0):
        """zcb_stack_maps: slice k (moving) against slice k − 1 (fixed) for k ≥ 1, each slice's
        features built once. Returns the n − 1 MapResults (no maps) and the device ms."""
        imgs = [gray32(s) for s in slices]
        n = len(imgs)
        if n < 2:
            raise ValueError("a stack needs at least 2 slices")
        ptrs = (N.f32p * n)(*[_f32(g) for g in imgs])
        w = np.array([g.shape[1] for g in imgs], np.uint32)
        h = np.array([g.shape[0] for g in imgs], np.uint32)
        pr = None if priors is None else np.ascontiguousarray(np.asarray(priors, np.float64).reshape(n - 1, 9))
        res = (N.ShiftResult * (n - 1))()
        ms = ctypes.c_double()
        self.call("zcb_stack_maps", n, ptrs, _u32(w), _u32(h), None if pr is None else _f64(pr),
                  int(bool(exact)) + 2 * int(bool(calibrated)), int(cap), res, ctypes.byref(ms))
        return [MapResult(x) for x in res], ms.value

    def stack_load(self, slices, priors=None, *, exact=True, calibrated=False, cap=0):
        """zcb_stack_load: the stack's features built and its maps planned, for sweep_stack."""
        imgs = [gray32(s) for s in slices]
        n = len(imgs)
        if n < 2:
            raise ValueError("a stack needs at least 2 slices")
        ptrs = (N.f32p * n)(*[_f32(g) for g in imgs])
        w = np.array([g.shape[1] for g in imgs], np.uint32)
        h = np.array([g.shape[0] for g in imgs], np.uint32)
        pr = None if priors is None else np.ascontiguousarray(np.asarray(priors, np.float64).reshape(n - 1, 9))
        self.call("zcb_stack_load", n, ptrs, _u32(w), _u32(h), None if pr is None else _f64(pr),
                  int(bool(exact)) + 2 * int(bool(calibrated)), int(cap))
        self._stack_n = n

    def sweep_stack(self, H0=None, n_peak=4):
        """zcb_sweep_stack: the sweep of the engine's pair and the loaded stack's maps as two
        branches of one CUDA graph, launched once → (SweepOut, [MapResult] of the stack)."""
        n = getattr(self, "_stack_n", 0)
        if n < 2:
            raise EngineError("sweep_stack: load a stack first (stack_load)")
        nc = self.sweep_size()
        sc = np.zeros((nc, n_peak), np.float32)
        ix = np.zeros((nc, n_peak), np.uint32)
        info = np.zeros(len(SWEEP_INFO))
        res = (N.ShiftResult * (n - 1))()
        h = None if H0 is None else _pose9(H0)
        self.call("zcb_sweep_stack", None if h is None else _f64(h), n_peak, _f32(sc), _u32(ix), sc.size, _f64(info),
                  info.size, res, n - 1)
        return SweepOut(sc, ix, dict(zip(SWEEP_INFO, map(float, info)))), [MapResult(x) for x in res]

    # optimisation
    def climb(self) -> ClimbOut:
        r = N.ClimbResult()
        self.call("zc_climb", ctypes.byref(r))
        return ClimbOut(_mat3(r.H), r.score, r.iterations, bool(r.moved))

    def _search_out(self, r):
        return SearchOut(_mat3(r.H), r.score, r.prev, bool(r.improved), r.count_a, r.count_b)

    def search(self) -> SearchOut:
        r = N.SearchResult()
        self.call("zc_search", ctypes.byref(r))
        return self._search_out(r)

    def sweep_size(self) -> int:
        """Candidates of the sweep under the current sw_* settings (rotations × scales × shears ×
        stretches, each count clamped as the engine clamps it)."""
        s = self.settings
        n = min(max(int(s["sw_nth"]), 1), 720) * min(max(int(s["sw_ns"]), 1), 129)
        for on, mx, cnt in (("sw_shear", "sw_shear_max", "sw_nshear"), ("sw_aniso", "sw_aniso_max", "sw_naniso")):
            if s[on] and float(s[mx]) > 0:
                n *= min(max(int(s[cnt]), 1), 15)
        return n

    def sweep(self, H0=None, n_peak=4, batch=0, shard=0, nshard=1) -> SweepOut:
        """zcb_sweep: the sweep's batched maps and each candidate's lane maxima (the search's first
        stage) at prior pose H0 (None: the engine's pose); shard / nshard: this rank's share."""
        nc = self.sweep_size()
        sc = np.zeros((nc, n_peak), np.float32)
        ix = np.zeros((nc, n_peak), np.uint32)
        info = np.zeros(len(SWEEP_INFO))
        h = None if H0 is None else _pose9(H0)
        self.call("zcb_sweep", None if h is None else _f64(h), n_peak, batch, shard, nshard, _f32(sc), _u32(ix),
                  sc.size, _f64(info), info.size)
        d = dict(zip(SWEEP_INFO, map(float, info)))
        if int(d["candidates"]) != nc:
            raise EngineError(f"sweep: the engine swept {int(d['candidates'])} candidates, expected {nc}")
        return SweepOut(sc, ix, d)

    def tune_sweep(self) -> list:
        """zcb_tune_sweep: the sweep's batch size per plane class, chosen by timing; one dict per
        class (nx, ny, candidates, batch, ms_per_map, options: {batch: ms per map})."""
        used = ctypes.c_size_t()
        self.call("zcb_tune_sweep", None, 0, ctypes.byref(used))
        buf = np.zeros(max(used.value, 1))
        self.call("zcb_tune_sweep", _f64(buf), buf.size, ctypes.byref(used))
        out, i = [], 0
        while i + 6 <= used.value:
            nx, ny, cnt, b, ms, k = buf[i:i + 6]
            opts = {int(buf[i + 6 + 2 * j]): float(buf[i + 7 + 2 * j]) for j in range(int(k))}
            out.append({"nx": int(nx), "ny": int(ny), "candidates": int(cnt), "batch": int(b), "ms_per_map": float(ms),
                        "options": opts})
            i += 6 + 2 * int(k)
        return out

    def search_lanes(self, scores, index) -> SearchOut:
        """zcb_search_lanes: the search finished from (gathered) lane maxima."""
        sc = np.ascontiguousarray(scores, np.float32).ravel()
        ix = np.ascontiguousarray(index, np.uint32).ravel()
        r = N.SearchResult()
        self.call("zcb_search_lanes", _f32(sc), _u32(ix), sc.size, ctypes.byref(r))
        return self._search_out(r)

    def set_dft_stage(self, pieces: int):
        """zcb_set_dft_stage: the maps' forward column FFTs run their first (radix-16) stage on the
        tensor cores in `pieces` (1 to 3) BF16 parts per FP32 value; 0 puts the FP32 stage back."""
        self.call("zcb_set_dft_stage", int(pieces))

    def refine_poses(self, Hs, iters=25):
        """zcb_refine_poses: Gauss–Newton from every pose together → (poses (n, 3, 3), scores)."""
        a = np.ascontiguousarray(np.asarray(Hs, np.float64).reshape(-1, 9))
        out, sc = np.zeros_like(a), np.zeros(len(a))
        self.call("zcb_refine_poses", _f64(a), len(a), int(iters), _f64(out), _f64(sc))
        return out.reshape(-1, 3, 3), sc

    # measurement
    def profile(self, on=True) -> bool:
        return bool(self.lib.zc_profile(self.handle, int(bool(on))))

    def profile_report(self) -> str:
        return self._text(self.lib.zc_profile_report)

    def gpu_counts(self) -> dict:
        c = (ctypes.c_uint32 * 4)()
        self.lib.zc_gpu_counts(self.handle, c)
        return dict(zip(("launches", "submits", "reads", "waits"), map(int, c)))

    def bench_maps(self, H=None, *, flags=3, cap=1024, warmup=3, steps=10) -> dict:
        """zcb_bench_maps: device-timed maps with the inputs resident (L2 flushed between timed
        maps): ms per map replayed from one captured CUDA graph, per-stage ms of
        event-instrumented maps, and the plan."""
        a, o = self._at(H), np.zeros(16)
        self.call("zcb_bench_maps", _f64(a), flags, cap, warmup, steps, _f64(o), o.size)
        return {
            "ms_per_map": float(o[0]), "stages_ms": dict(zip(BENCH_STAGES, map(float, o[1:6]))),
            "ms_per_map_instrumented": float(o[6]), "canvas_h": int(o[7]), "nx": int(o[8]), "ny": int(o[9]),
            "cw": int(o[10]), "ch": int(o[11]), "n_real": int(o[12]), "n_corr": int(o[13]), "split": int(o[14]),
            "canvas_w": int(o[15]),
        }

    # lifetime
    def close(self):
        h, self.handle = getattr(self, "handle", None), None
        if h:
            self.lib.zc_destroy(h)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
