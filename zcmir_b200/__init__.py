"""zcmir_b200: the SMI path of zcmir (square-loss mutual information registration), B200-native.

The Python surface mirrors the reference's (python/zcmir/__init__.py, python/zcmir/api.py) for the
SMI path: the same names, arguments, result types and errors, over the same zc_* C ABI, served by
libzcmir.so (CUDA kernels for sm_100a).

    import zcmir_b200 as zcmir
    sm = zcmir.shift_map(moving, fixed, preprocess=False, map_res=2048)   # dense SMI shift map
    sm.peak, sm.dx, sm.dy, sm.map

Pose convention: H maps MOVING pixel coordinates to FIXED pixel coordinates, row-major, with
(1, 1) the centre of the top-left pixel.
"""
import ctypes
import json
import math
from dataclasses import dataclass

import numpy as np

from . import _native

__all__ = [
    "Registrar", "ShiftMap", "RotoScaleMap", "Score", "Gradient", "Climb", "Search",
    "shift_map", "rs_map", "score", "refine", "register", "register_stack", "stack_maps", "search", "settings", "close",
    "Registration", "StackRegistration", "__version__",
]

__version__ = "0.1.4"


def _mat(H):
    a = np.ascontiguousarray(np.asarray(H, dtype=np.float64).reshape(9))
    return a, a.ctypes.data_as(_native.f64p)


def _fp(a):
    return a.ctypes.data_as(_native.f32p)


@dataclass
class Score:
    """Pose score: the mean of the forward and inverse directions when symmetric."""
    mean: float
    fwd: float
    inv: float | None


@dataclass
class Gradient:
    score: float
    fwd: float
    inv: float | None
    n: float
    grad: np.ndarray
    hess: np.ndarray | None


@dataclass
class ShiftMap:
    """Dense score over every translation of the moving image about a pose.

    map: ny rows × n columns, lag (0, 0) at [0, 0], negative lags wrapped (np.fft.fftshift
    centres it); one cell spans (canvas_w / cw, canvas_h / ch) pixels. dx, dy: the peak's lag in
    fixed pixels; ``corrected(H)`` = translate(−dx, −dy)·H.
    """
    peak: float
    dx: float
    dy: float
    zero: float
    n: int
    cw: int
    ch: int
    canvas: tuple
    offset: tuple
    corr_area_px: float
    exact: bool
    calibrated: bool
    map: np.ndarray | None
    ny: int = 0
    peak_index: int = 0

    def corrected(self, H):
        T = np.array([[1, 0, -self.dx], [0, 1, -self.dy], [0, 0, 1.0]])
        return T @ np.asarray(H, dtype=np.float64).reshape(3, 3)


@dataclass
class Climb:
    H: np.ndarray
    score: float
    iterations: int
    moved: bool


@dataclass
class Search:
    H: np.ndarray
    score: float
    previous: float
    improved: bool
    count_a: int
    count_b: int


@dataclass
class RotoScaleMap:
    """Score over every rotation and scale of the moving image about a centre (fixed pixels,
    1-based). map / fwd / inv: n × n, columns θ (n_th of them over 2π), rows log radius (Δλ each),
    lag 0 at [0, 0]; dth, dsg: the peak as the rotation (rad) and log scale that correct the pose."""
    peak: float
    dth: float
    dsg: float
    zero: float
    center: tuple
    n: int
    n_th: int
    n_lam: int
    dlam: float
    r0: float
    r1: float
    symmetric: bool
    calibrated: bool
    map: np.ndarray | None = None
    fwd: np.ndarray | None = None
    inv: np.ndarray | None = None
    peak_index: int = 0


@dataclass
class Sweep:
    """The sweep's batched maps (zcb_sweep): per candidate (θ-major, then σ, shear, stretch) its
    best lane maxima — scores in fixed pixels, map indices (0xffffffff: none) — and the run's
    figures (candidates, cell, device ms, plane sizes, batches, launches)."""
    scores: np.ndarray
    index: np.ndarray
    info: dict


class Registrar:
    """One GPU engine and one image pair, whose features stay on the GPU between calls.

    Keyword arguments are settings (``configure``). close() releases the engine (also on garbage
    collection; ``with`` works too).
    """

    def __init__(self, on_event=None, **settings):
        lib = _native.load()
        self._lib = lib
        self._e = lib.zc_create(b"")
        self.on_event = on_event
        self._events = []
        if not self._e:
            buf = ctypes.create_string_buffer(1024)
            n = lib.zc_create_error(buf, 1024)
            raise RuntimeError(buf.raw[:n].decode(errors="replace") or "zcmir: could not create the engine")
        if settings:
            self.configure(**settings)

    # ── plumbing ──
    def _error(self):
        buf = ctypes.create_string_buffer(1024)
        n = self._lib.zc_error(self._e, buf, 1024)
        return buf.raw[:n].decode(errors="replace")

    def _check(self, rc, what):
        self._drain()
        if rc != 0:
            raise RuntimeError(f"{what}: {self._error() or rc}")

    def _drain(self):
        buf = ctypes.create_string_buffer(1 << 16)
        while True:
            n = self._lib.zc_events(self._e, buf, len(buf))
            if n == 0:
                break
            for line in buf.raw[:n].decode(errors="replace").splitlines():
                if line:
                    ev = json.loads(line)
                    self._events.append(ev)
                    if self.on_event:
                        self.on_event(ev)

    def events(self):
        self._drain()
        out, self._events = self._events, []
        return out

    @property
    def adapter(self):
        buf = ctypes.create_string_buffer(256)
        n = self._lib.zc_adapter(self._e, buf, 256)
        return buf.raw[:n].decode(errors="replace")

    # ── settings ──
    def configure(self, **settings):
        b = json.dumps(settings).encode()
        self._check(self._lib.zc_configure(self._e, b, len(b)), "configure")

    @property
    def settings(self):
        cap = 8192
        buf = ctypes.create_string_buffer(cap)
        n = self._lib.zc_settings(self._e, buf, cap)
        if n > cap:
            buf = ctypes.create_string_buffer(n)
            n = self._lib.zc_settings(self._e, buf, n)
        return json.loads(buf.raw[:n])

    # ── images ──
    @staticmethod
    def _gray(img):
        """A contiguous float32 gray image (uint16 scaled to [0, 1], RGB(A) to luma)."""
        a = np.asarray(img)
        if a.dtype == np.uint8:
            a = a.astype(np.float32) / np.float32(255)
        if a.ndim == 3 and a.shape[2] in (3, 4):
            a = a[:, :, :3].astype(np.float64) @ np.array([0.299, 0.587, 0.114])
        if a.dtype == np.uint16:
            a = a / 65535.0
        if not (a.dtype == np.float32 and a.flags.c_contiguous):
            a = np.ascontiguousarray(a, dtype=np.float32)
        if a.ndim != 2:
            raise ValueError("expected a gray image (h, w)")
        return a

    def _set(self, side, img, preprocess):
        """python/zcmir/__init__.py:283-307: uint8 images (gray, RGB or RGBA) go up as RGBA8 and are
        always preprocessed; other images as float gray, preprocessed when asked."""
        a = np.asarray(img)
        if a.dtype == np.uint8:
            if a.ndim == 2:
                a = np.repeat(a[:, :, None], 3, axis=2)
            if a.ndim != 3 or a.shape[2] not in (3, 4):
                raise ValueError("uint8 images: (h, w), (h, w, 3) or (h, w, 4)")
            if a.shape[2] == 3:
                a = np.concatenate([a, np.full(a.shape[:2] + (1,), 255, np.uint8)], axis=2)
            a = np.ascontiguousarray(a)
            h, w = a.shape[:2]
            if not preprocess:
                raise ValueError("uint8 images are always preprocessed (pass float gray to skip it)")
            return self._check(self._lib.zc_set_image_rgba(self._e, side, a.ctypes.data_as(_native.u8p), w, h),
                               "set_image")
        a = self._gray(a)
        h, w = a.shape
        rc = self._lib.zc_set_image_gray(self._e, side, _fp(a), w, h, 1 if preprocess else 0)
        self._check(rc, "set_image")

    def set_moving(self, img, preprocess=True):
        self._set(0, img, preprocess)

    def set_fixed(self, img, preprocess=True):
        self._set(1, img, preprocess)

    def set_images(self, moving, fixed, preprocess=True):
        self._set(0, moving, preprocess)
        self._set(1, fixed, preprocess)

    def image_size(self, side):
        out = (ctypes.c_uint32 * 2)()
        self._lib.zc_image_size(self._e, side, out)
        return out[0], out[1]

    def work_image(self, side):
        w, h = self.image_size(side)
        out = np.empty((h, w), np.float32)
        self._check(self._lib.zc_work_image(self._e, side, _fp(out), out.size), "work_image")
        return out

    def features(self, side):
        """The SMI feature planes of side 0 (moving) or 1 (fixed), (4, h, w) float32: the
        whitened rank r, r², |∇r| and the fourth feature."""
        w, h = self.image_size(side)
        out = np.empty((4, h, w), np.float32)
        self._check(self._lib.zc_features(self._e, side, _fp(out), out.size), "features")
        return out

    def moments(self, H=None):
        a, p = self._Hp(H)
        out = np.empty(45, np.float64)
        self._check(self._lib.zc_moments(self._e, p, out.ctypes.data_as(_native.f64p)), "moments")
        return out

    def _map_cap(self, resolution=0):
        n = max(int(resolution or 0), int(self.settings.get("map_res", 0)), 1024)
        return n * n

    # ── pose ──
    @property
    def pose(self):
        H = (ctypes.c_double * 9)()
        self._lib.zc_get_pose(self._e, H)
        return np.array(list(H), np.float64).reshape(3, 3)

    @pose.setter
    def pose(self, H):
        a, p = _mat(H)
        self._lib.zc_set_pose(self._e, p)

    @property
    def ffd(self):
        """The B-spline's control points: 2·g·g float32 (x, y per point, row by row), in half-image
        units of the lattice's image; g = settings["ffd_grid"]."""
        buf = np.zeros(512, np.float32)
        n = self._lib.zc_get_ffd(self._e, _fp(buf), buf.size)
        return buf[:n].copy()

    @ffd.setter
    def ffd(self, cps):
        a = np.ascontiguousarray(cps, dtype=np.float32).ravel()
        self._check(self._lib.zc_set_ffd(self._e, _fp(a), a.size), "set_ffd")

    def _Hp(self, H):
        return _mat(self.pose if H is None else H)

    # ── scores and maps ──
    def score(self, H=None):
        a, p = self._Hp(H)
        out = np.empty(3, np.float64)
        self._check(self._lib.zc_score(self._e, p, out.ctypes.data_as(_native.f64p)), "score")
        return Score(float(out[0]), float(out[1]), None if math.isnan(out[2]) else float(out[2]))

    def gradient(self, H=None, hess=False):
        a, p = self._Hp(H)
        r = _native.GradResult()
        self._check(self._lib.zc_gradient(self._e, p, 1 if hess else 0, ctypes.byref(r)), "gradient")
        nk = r.nk
        g = np.array(r.grad[:nk])
        Hm = np.array(r.hess[: nk * nk]).reshape(nk, nk) if r.has_hess else None
        return Gradient(r.score, r.fwd, None if math.isnan(r.inv) else r.inv, r.n, g, Hm)

    def displacement(self):
        """The composed warp at the engine's pose (and spline, when on) over the fixed image as
        (h, w, 2) float32: x_moving − x_fixed, 0-based pixels."""
        w, h = self.image_size(1)
        out = np.empty((h, w, 2), np.float32)
        self._check(self._lib.zc_displacement(self._e, _fp(out), out.size), "displacement")
        return out

    def ffd_gradient(self, H=None):
        """(score, gradient over the spline's 2·g·g control points) at H; with the spline off
        (settings["ffd"] False) the score is 0 and the gradient zero."""
        a, p = self._Hp(H)
        s = ctypes.c_double()
        g = np.zeros(512, np.float64)
        self._check(self._lib.zc_ffd_gradient(self._e, p, ctypes.byref(s), g.ctypes.data_as(_native.f64p), g.size),
                    "ffd_gradient")
        n = 2 * min(max(int(self.settings["ffd_grid"]), 2), 16) ** 2
        return s.value, g[:n].copy()

    def shift_map(self, H=None, *, exact=None, calibrated=None, resolution=1024, return_map=True, out=None):
        """Score every translation of the moving image about pose H. Without exact / calibrated the
        settings decide (score, resolution, overlap floor); with them those are explicit and there
        is no overlap floor. ``out``: an optional float32 buffer (≥ ny·n) the map is written to."""
        a, p = self._Hp(H)
        r = _native.ShiftResult()
        buf = None
        if return_map:
            buf = out if out is not None else np.empty(self._map_cap(resolution), np.float32)
        mp, ml = (_fp(buf), buf.size) if buf is not None else (None, 0)
        if exact is None and calibrated is None:
            rc = self._lib.zc_shift_map_set(self._e, p, ctypes.byref(r), mp, ml)
        else:
            flags = (1 if (exact is None or exact) else 0) | (2 if (calibrated is None or calibrated) else 0)
            rc = self._lib.zc_shift_map(self._e, p, flags, resolution, ctypes.byref(r), mp, ml)
        self._check(rc, "shift_map")
        ny = r.n_y or r.n
        m = None
        if buf is not None:
            m = buf[: r.n * ny].reshape(ny, r.n)
            if out is None:
                m = m.copy()
        return ShiftMap(
            peak=r.peak, dx=r.dx, dy=r.dy, zero=r.zero, n=r.n, cw=r.cw, ch=r.ch,
            canvas=(r.canvas_w, r.canvas_h), offset=(r.ox, r.oy), corr_area_px=r.corr_area_px,
            exact=bool(r.exact), calibrated=bool(r.calibrated), map=m, ny=ny, peak_index=r.peak_index,
        )

    def stack_maps(self, slices, priors=None, *, exact=True, calibrated=False, resolution=0):
        """Shift maps along a stack: slice k (moving) against slice k − 1 (fixed) for every k ≥ 1,
        each slice's features built once (zcb_stack_maps). priors: n − 1 poses (default: the
        slices' centres aligned). Returns the n − 1 ShiftMaps (without their maps) and the device
        ms of the whole stack. The engine's own images and pose are left as they were."""
        imgs = [self._gray(x) for x in slices]
        n = len(imgs)
        if n < 2:
            raise ValueError("stack_maps: a stack needs at least 2 slices")
        ptrs = (_native.f32p * n)(*[a.ctypes.data_as(_native.f32p) for a in imgs])
        w = np.array([a.shape[1] for a in imgs], np.uint32)
        h = np.array([a.shape[0] for a in imgs], np.uint32)
        pr = None
        if priors is not None:
            pr = np.ascontiguousarray(np.asarray(priors, np.float64).reshape(n - 1, 9))
        out = (_native.ShiftResult * (n - 1))()
        ms = ctypes.c_double(0)
        flags = (1 if exact else 0) | (2 if calibrated else 0)
        self._check(self._lib.zcb_stack_maps(self._e, n, ptrs, w.ctypes.data_as(_native.u32p),
                                             h.ctypes.data_as(_native.u32p),
                                             None if pr is None else pr.ctypes.data_as(_native.f64p), flags, resolution,
                                             out, ctypes.byref(ms)), "stack_maps")
        maps = [ShiftMap(peak=r.peak, dx=r.dx, dy=r.dy, zero=r.zero, n=r.n, cw=r.cw, ch=r.ch,
                         canvas=(r.canvas_w, r.canvas_h), offset=(r.ox, r.oy), corr_area_px=r.corr_area_px,
                         exact=bool(r.exact), calibrated=bool(r.calibrated), map=None, ny=r.n_y or r.n,
                         peak_index=r.peak_index) for r in out]
        return maps, ms.value

    def rs_map(self, H=None, *, center=None, symmetric=True, return_maps=True):
        """Roto-scale map at H about center (fixed pixels, 1-based; default the moving image's
        centroid under H); the settings decide the score and the resolution (map_res)."""
        a, p = self._Hp(H)
        res = int(self.settings["map_res"])
        n_max = 512 if res == 0 else min(res, 8192)  # the auto plan stays within 512 angles
        cap = n_max * n_max if return_maps else 0
        bufs = [np.empty(cap, np.float32) if return_maps else None for _ in range(3)]
        ptr = [_fp(b) if b is not None else None for b in bufs]
        c = (ctypes.c_double * 2)(*center) if center is not None else None
        r = _native.RsResult()
        self._check(self._lib.zc_rs_map(self._e, p, c, 1 if symmetric else 0, ctypes.byref(r), ptr[0], ptr[1],
                                        ptr[2] if symmetric else None, cap), "rs_map")
        nn = r.n * r.n
        get = lambda b: b[:nn].reshape(r.n, r.n).copy() if b is not None else None
        return RotoScaleMap(peak=r.peak, dth=r.dth, dsg=r.dsg, zero=r.zero, center=(r.cx, r.cy), n=r.n, n_th=r.n_th,
                            n_lam=r.n_lam, dlam=r.dlam, r0=r.r0, r1=r.r1, symmetric=bool(r.symmetric),
                            calibrated=bool(r.calibrated), map=get(bufs[0]), fwd=get(bufs[1]),
                            inv=get(bufs[2]) if symmetric else None, peak_index=r.peak_index)

    def canvas(self, H=None, inverse=False):
        a, p = self._Hp(H)
        c = _native.Canvas()
        self._check(self._lib.zc_canvas(self._e, p, 1 if inverse else 0, ctypes.byref(c)), "canvas")
        return (c.ox, c.oy), (c.ow, c.oh), np.array(list(c.Hc)).reshape(3, 3)

    # ── optimisation ──
    def climb(self):
        r = _native.ClimbResult()
        self._check(self._lib.zc_climb(self._e, ctypes.byref(r)), "climb")
        return Climb(np.array(list(r.H)).reshape(3, 3), r.score, r.iterations, bool(r.moved))

    def search(self):
        r = _native.SearchResult()
        self._check(self._lib.zc_search(self._e, ctypes.byref(r)), "search")
        return Search(np.array(list(r.H)).reshape(3, 3), r.score, r.prev, bool(r.improved), r.count_a, r.count_b)

    def _sweep_count(self):
        s = self.settings
        n = min(max(int(s["sw_nth"]), 1), 720) * min(max(int(s["sw_ns"]), 1), 129)
        if s["sw_shear"] and float(s["sw_shear_max"]) > 0:
            n *= min(max(int(s["sw_nshear"]), 1), 15)
        if s["sw_aniso"] and float(s["sw_aniso_max"]) > 0:
            n *= min(max(int(s["sw_naniso"]), 1), 15)
        return n

    def sweep(self, H0=None, n_peak=4, batch=0, shard=0, nshard=1):
        """The sweep's batched maps alone (the first stage of search()) at prior pose H0 (None: the
        one search() uses), with the sw_* settings; shard / nshard: this share of a sweep split
        across ranks (the other candidates' entries stay (0, 0xffffffff))."""
        nc = self._sweep_count()
        sc = np.zeros((nc, n_peak), np.float32)
        ix = np.zeros((nc, n_peak), np.uint32)
        info = np.zeros(16)
        a, h = (None, None) if H0 is None else _mat(H0)
        self._check(self._lib.zcb_sweep(self._e, h, n_peak, batch, shard, nshard, _fp(sc), ix.ctypes.data_as(_native.u32p), sc.size,
                                        info.ctypes.data_as(_native.f64p), 16), "sweep")
        keys = ("candidates", "cell", "ms", "grid", "Fx", "Fy", "fx0", "fy0", "min_n", "n", "groups", "batches",
                "launches", "ox", "oy", "peaks")
        d = {k: float(v) for k, v in zip(keys, info)}
        if int(d["candidates"]) != nc:
            raise RuntimeError(f"sweep: {int(d['candidates'])} candidates, expected {nc}")
        return Sweep(sc, ix, d)

    def refine_poses(self, Hs, iters=25):
        """Gauss–Newton from each pose at once (zcb_refine_poses): (poses (n, 3, 3), scores (n,))."""
        a = np.ascontiguousarray(np.asarray(Hs, np.float64).reshape(-1, 9))
        n = len(a)
        out = np.zeros_like(a)
        sc = np.zeros(n)
        self._check(self._lib.zcb_refine_poses(self._e, a.ctypes.data_as(_native.f64p), n, iters,
                                               out.ctypes.data_as(_native.f64p), sc.ctypes.data_as(_native.f64p)),
                    "refine_poses")
        return out.reshape(n, 3, 3), sc

    def search_lanes(self, scores, index):
        """search() from every candidate's 4 lane maxima gathered from sharded sweeps."""
        sc = np.ascontiguousarray(scores, np.float32).reshape(-1)
        ix = np.ascontiguousarray(index, np.uint32).reshape(-1)
        r = _native.SearchResult()
        self._check(self._lib.zcb_search_lanes(self._e, _fp(sc), ix.ctypes.data_as(_native.u32p), sc.size,
                                               ctypes.byref(r)), "search")
        return Search(np.array(list(r.H)).reshape(3, 3), r.score, r.prev, bool(r.improved), r.count_a, r.count_b)

    # ── profiling ──
    def profile(self, on=True):
        return bool(self._lib.zc_profile(self._e, 1 if on else 0))

    def profile_report(self):
        buf = ctypes.create_string_buffer(1 << 14)
        n = self._lib.zc_profile_report(self._e, buf, len(buf))
        return buf.raw[:n].decode()

    def gpu_counts(self):
        out = (ctypes.c_uint32 * 4)()
        self._lib.zc_gpu_counts(self._e, out)
        return dict(zip(("launches", "submits", "reads", "waits"), list(out)))

    def bench_maps(self, H=None, *, flags=3, cap=1024, warmup=3, steps=10):
        """Device-timed maps (CUDA events, inputs resident, L2 flushed between timed maps): ms per
        map of replays of one captured CUDA graph of the map's passes, per-stage ms (and the total)
        of event-instrumented maps, and the plan."""
        a, p = self._Hp(H)
        out = np.zeros(16, np.float64)
        self._check(self._lib.zcb_bench_maps(self._e, p, flags, cap, warmup, steps, out.ctypes.data_as(_native.f64p), 16),
                    "bench_maps")
        stages = ("canvas", "fwd_rows", "fwd_cols", "inv_cols", "inv_rows_score")
        return {
            "ms_per_map": float(out[0]), "stages_ms": dict(zip(stages, map(float, out[1:6]))),
            "ms_per_map_instrumented": float(out[6]),
            "nx": int(out[8]), "ny": int(out[9]), "cw": int(out[10]), "ch": int(out[11]),
            "n_real": int(out[12]), "n_corr": int(out[13]), "split": int(out[14]), "canvas_w": int(out[15]),
            "canvas_h": int(out[7]),
        }

    # ── lifetime ──
    def close(self):
        if getattr(self, "_e", None):
            self._lib.zc_destroy(self._e)
            self._e = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


from .api import (  # noqa: E402
    Registration, StackRegistration, close, refine, register, register_stack, rs_map, score, search, settings,
    shift_map, stack_maps,
)
