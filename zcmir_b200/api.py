"""The functional API over one shared engine (the reference's python/zcmir/api.py, SMI path).

Every function takes the engine's settings as keyword arguments (``settings()`` lists them) and
starts from the defaults, so one call never changes another. Calls are serialised.
"""
import difflib
import json
import math
import threading
from dataclasses import dataclass

import numpy as np

from . import Registrar

_LOCK = threading.RLock()
_ENGINE = None
_DEFAULTS = None
_LOADED = {}  # side → (key, array) of the image in the engine


def _engine():
    global _ENGINE, _DEFAULTS
    if _ENGINE is None:
        _ENGINE = Registrar()
        _DEFAULTS = _ENGINE.settings
    return _ENGINE


def close():
    """Release the shared engine. The next call makes a new one."""
    global _ENGINE
    with _LOCK:
        if _ENGINE is not None:
            _ENGINE.close()
            _ENGINE = None
            _LOADED.clear()


def settings():
    """Every setting with its default value (enums as strings)."""
    with _LOCK:
        _engine()
        return dict(_DEFAULTS)


_SPELL = {"model": "group", "spline_lattice": "ffd_grid", "spline_stiffness": "ffd_stiffness"}


def _lattice(spline):
    """spline= → the lattice size: True 4, False/0 none, else 2–16 (python/zcmir/api.py:87-95)."""
    if spline is True:
        return 4
    if not spline:
        return 0
    g = int(spline)
    if not 2 <= g <= 16:
        raise ValueError("spline: True (a 4×4 lattice) or the lattice size 2–16")
    return g


def _resolve(model="homography", spline=False, **kw):
    """Keyword arguments → engine settings (defaults + these), with the names checked
    (python/zcmir/api.py:65-84). The spline stays off: register() turns it on for its second
    stage."""
    _engine()
    s = dict(_DEFAULTS)
    if model not in ("affine", "homography"):
        raise ValueError(f'model: "affine" or "homography", not {model!r}')
    s["group"] = model
    lattice = _lattice(spline)
    s["ffd"] = False
    if lattice:
        s["ffd_grid"] = lattice
    for k, v in kw.items():
        k = _SPELL.get(k, k)
        if k not in s:
            near = difflib.get_close_matches(k, s, n=3)
            raise TypeError(f"unknown setting {k!r}" + (f"; did you mean {', '.join(near)}?" if near else " (settings() lists them)"))
        s[k] = v
    return s


_PREP = ("clahe", "clahe_grid", "clahe_bins", "band", "bp_fine", "bp_coarse", "invert", "half", "smi_features")


def _fingerprint(a):
    flat = a.reshape(-1)
    step = max(1, flat.size // 4096)
    return (a.shape, a.dtype.str, hash(flat[::step].tobytes()), float(flat[: min(flat.size, 64)].sum()))


def _load(reg, side, img, preprocess, s):
    key = (id(img), _fingerprint(img), preprocess, tuple(s[k] for k in _PREP))
    cur = _LOADED.get(side)
    if cur and cur[0] == key and cur[1] is img:
        return
    (reg.set_moving if side == 0 else reg.set_fixed)(img, preprocess=preprocess)
    _LOADED[side] = (key, img)


def _prepare(moving, fixed, preprocess, kw):
    reg = _engine()
    s = _resolve(**kw)
    reg.configure(**s)
    m, f = np.asarray(moving), np.asarray(fixed)
    _load(reg, 0, m, preprocess, s)
    _load(reg, 1, f, preprocess, s)
    return reg, s, m, f


def _field_from_H(H, fixed_shape):
    """x_moving − x_fixed (0-based) over the fixed grid for a pose H (moving → fixed, 1-based)."""
    h, w = fixed_shape[:2]
    Hi = np.linalg.inv(np.asarray(H, np.float64))
    Y, X = np.mgrid[1:h + 1, 1:w + 1].astype(np.float64)
    d = Hi[2, 0] * X + Hi[2, 1] * Y + Hi[2, 2]
    out = np.empty((h, w, 2), np.float32)
    out[..., 0] = (Hi[0, 0] * X + Hi[0, 1] * Y + Hi[0, 2]) / d - X
    out[..., 1] = (Hi[1, 0] * X + Hi[1, 1] * Y + Hi[1, 2]) / d - Y
    return out


def warp_image(image, field, fill=0):
    """Resample image (gray or with channels, any dtype) on a displacement field (h, w, 2:
    x_moving − x_fixed, 0-based), bilinear. Returns (warped, mask of fixed pixels inside)."""
    img = np.asarray(image)
    sh, sw = img.shape[:2]
    h, w = field.shape[:2]
    Y, X = np.mgrid[0:h, 0:w].astype(np.float64)
    mx, my = X + field[..., 0], Y + field[..., 1]
    inside = (mx >= 0) & (my >= 0) & (mx <= sw - 1) & (my <= sh - 1)
    x0 = np.clip(np.floor(mx).astype(np.int64), 0, max(sw - 2, 0))
    y0 = np.clip(np.floor(my).astype(np.int64), 0, max(sh - 2, 0))
    fx, fy = np.clip(mx - x0, 0, 1), np.clip(my - y0, 0, 1)
    x1, y1 = np.minimum(x0 + 1, sw - 1), np.minimum(y0 + 1, sh - 1)
    src = img.astype(np.float64)
    if src.ndim == 3:
        fx, fy, inside_c = fx[..., None], fy[..., None], inside[..., None]
    else:
        inside_c = inside
    v = (src[y0, x0] * (1 - fx) + src[y0, x1] * fx) * (1 - fy) + (src[y1, x0] * (1 - fx) + src[y1, x1] * fx) * fy
    v = np.where(inside_c, v, fill)
    if np.issubdtype(img.dtype, np.integer):
        info = np.iinfo(img.dtype)
        v = np.clip(np.rint(v), info.min, info.max)
    return v.astype(img.dtype), inside


@dataclass
class Registration:
    """A registered pair (python/zcmir/api.py:205-290, without the keypoint fields): H maps moving
    pixel coordinates to fixed ones (row-major 3×3, 1-based); with a spline, the full warp is H
    followed by the B-spline (spline: its 2·lattice² control points), which displacement(),
    fixed_to_moving() and warp() include."""
    H: np.ndarray
    score: float
    model: str
    moving_shape: tuple
    fixed_shape: tuple
    method: str = "refine"
    iterations: int = 0
    redetected: bool = False
    spline: np.ndarray | None = None
    lattice: int = 0
    _field: np.ndarray | None = None

    def __repr__(self):
        sp = f", spline {self.lattice}×{self.lattice}" if self.spline is not None else ""
        return f"Registration({self.model}{sp}, score {self.score:.4g}, {self.method})"

    def map_points(self, points):
        """Moving (x, y) points (1-based, (n, 2)) to fixed coordinates by H (the global model; a
        spline's local correction is not included — fixed_to_moving() includes it)."""
        p = np.asarray(points, np.float64).reshape(-1, 2)
        q = np.c_[p, np.ones(len(p))] @ self.H.T
        return q[:, :2] / q[:, 2:]

    def displacement(self):
        """The full warp over the fixed image, (h, w, 2) float32: x_moving − x_fixed, 0-based."""
        if self._field is not None:
            return self._field
        return _field_from_H(self.H, self.fixed_shape)

    def fixed_to_moving(self, points):
        """Fixed (x, y) points (1-based) to moving coordinates through the full warp."""
        d = self.displacement()
        p = np.asarray(points, np.float64).reshape(-1, 2) - 1
        h, w = d.shape[:2]
        x, y = np.clip(p[:, 0], 0, w - 1), np.clip(p[:, 1], 0, h - 1)
        x0, y0 = np.minimum(np.floor(x).astype(int), w - 2), np.minimum(np.floor(y).astype(int), h - 2)
        fx, fy = (x - x0)[:, None], (y - y0)[:, None]
        v = (d[y0, x0] * (1 - fx) + d[y0, x0 + 1] * fx) * (1 - fy) + (d[y0 + 1, x0] * (1 - fx) + d[y0 + 1, x0 + 1] * fx) * fy
        return p + v + 1

    def warp(self, moving, fill=0, mask=False):
        """The moving image resampled into the fixed frame through the full warp (bilinear, fill
        outside); mask=True also returns the fixed pixels the moving image covers."""
        out, m = warp_image(moving, self.displacement(), fill)
        return (out, m) if mask else out

    def to_dict(self):
        return {"H": np.asarray(self.H).tolist(), "score": float(self.score), "model": self.model,
                "moving_shape": list(self.moving_shape), "fixed_shape": list(self.fixed_shape), "method": self.method,
                "iterations": int(self.iterations), "redetected": bool(self.redetected),
                "spline": None if self.spline is None else {"lattice": int(self.lattice),
                                                            "coefficients": np.asarray(self.spline).tolist()}}


def shift_map(moving, fixed, H=None, *, preprocess=True, **settings):
    """The score at every translation of the moving image about pose H (default: identity)."""
    with _LOCK:
        reg, *_ = _prepare(moving, fixed, preprocess, settings)
        return reg.shift_map(np.eye(3) if H is None else np.asarray(H, np.float64))


def rs_map(moving, fixed, H=None, *, center=None, symmetric=True, preprocess=True, **settings):
    """The score at every rotation and scale of the moving image about pose H (default: identity)
    and a centre (default: the moving image's centroid under H)."""
    with _LOCK:
        reg, *_ = _prepare(moving, fixed, preprocess, settings)
        return reg.rs_map(np.eye(3) if H is None else np.asarray(H, np.float64), center=center, symmetric=symmetric)


def score(moving, fixed, H, *, preprocess=True, **settings):
    """The registration score at pose H (the mean of both directions when symmetric)."""
    with _LOCK:
        reg, *_ = _prepare(moving, fixed, preprocess, settings)
        return reg.score(np.asarray(H, np.float64)).mean


def register(moving, fixed, *, init=None, model="homography", spline=False, preprocess=True, **settings):
    """Refine from ``init`` (keypoint detection is not part of this build, so ``init`` is
    required): the climb over the model from H; with spline (True: a 4×4 lattice, or the lattice
    size 2–16; spline_stiffness, default 0.15, the bending penalty's wavelength in fractions of
    the lattice's size), then a second climb of the B-spline together with the model
    (python/zcmir/api.py:291-325)."""
    if init is None:
        raise ValueError("register: keypoint detection is not part of this build; pass init=H (or use search())")
    lattice = _lattice(spline)
    with _LOCK:
        reg, s, m, f = _prepare(moving, fixed, preprocess, dict(model=model, spline=spline, **settings))
        reg.pose = np.asarray(init, np.float64).reshape(3, 3)
        c = reg.climb()
        iters = c.iterations
        cps = fld = None
        if lattice:
            reg.configure(ffd=True, ffd_grid=lattice)
            reg.ffd = np.zeros(2 * lattice * lattice, np.float32)
            c = reg.climb()
            iters += c.iterations
            cps = reg.ffd
            fld = reg.displacement()
        H = reg.pose
        out = Registration(H=H, score=reg.score(H).mean, model=s["group"], moving_shape=m.shape, fixed_shape=f.shape,
                           method="refine", iterations=iters, spline=cps, lattice=lattice, _field=fld)
        if lattice:
            reg.configure(ffd=False)
        return out


def refine(moving, fixed, H, **kw):
    """Refine a pose: register(moving, fixed, init=H, ...)."""
    return register(moving, fixed, init=H, **kw)


def search(moving, fixed, H=None, *, mode="sweep", rotation=None, scale=None, shear=None, stretch=None,
           preprocess=True, **settings):
    """Brute force (python/zcmir/api.py:354-391): "sweep" scores every rotation × scale (× shear
    × stretch) × shift, screens the best peaks by batched Gauss–Newton and climbs the finalists;
    the pose H is kept unless the search scores higher. ("cloud" is not part of this build.)

    Sweep ranges (each also settable through the sw_* settings):
      rotation  degrees: a half-range (30 → ±30°) or a (from, to) range, which may run through
                ±180°; default the full circle
      scale     (min, max) of the moving image's scale; default (0.5, 2)
      shear     largest shear either way, or (largest, values); off by default
      stretch   largest stretch either way as a fraction, or (largest, values); off by default
    """
    if rotation is not None:
        if np.ndim(rotation) == 0:
            settings.update(sw_rot_range=False, sw_rot=float(rotation))
        else:
            lo, hi = rotation
            settings.update(sw_rot_range=True, sw_rot_lo=float(lo), sw_rot_hi=float(hi))
    if scale is not None:
        settings.update(sw_smin=float(scale[0]), sw_smax=float(scale[1]))
    for v, key in ((shear, "shear"), (stretch, "aniso")):
        if v is None:
            continue
        mx, n = (v, None) if np.ndim(v) == 0 else v
        settings[f"sw_{key}"] = float(mx) > 0
        settings[f"sw_{key}_max"] = float(mx)
        if n is not None:
            settings[f"sw_n{key}"] = int(n)
    with _LOCK:
        reg, s, m, f = _prepare(moving, fixed, preprocess, dict(search_mode=mode, **settings))
        reg.pose = np.eye(3) if H is None else np.asarray(H, np.float64)
        reg.search()
        return Registration(H=reg.pose, score=reg.score(reg.pose).mean, model=s["group"], moving_shape=m.shape,
                            fixed_shape=f.shape, method=f"search ({mode})")


# ── stacks (python/zcmir/api.py:430-580) ──────────────────────────────────────────────────────

@dataclass
class StackRegistration:
    """A registered stack: one Registration per slice pair (None where none was made), each
    slice's distance off the trend of its neighbours (fixed px), and the slices flagged as off it."""
    slices: list
    off_trend: list
    flagged: list
    threshold: float

    def __len__(self):
        return len(self.slices)

    def __getitem__(self, i):
        return self.slices[i]

    def __repr__(self):
        n = sum(r is not None for r in self.slices)
        return (f"StackRegistration({n}/{len(self.slices)} registered, {sum(self.flagged)} flagged, "
                f"threshold {self.threshold:.1f} px)")

    @property
    def H(self):
        return [None if r is None else r.H for r in self.slices]

    def to_json(self, path=None):
        d = json.dumps({
            "convention": "H maps moving pixel coordinates to fixed pixel coordinates, row-major 3x3, 1-based pixel centres",
            "threshold_px": self.threshold,
            "slices": [None if r is None else {**r.to_dict(), "off_trend_px": t, "flagged": bool(fl)}
                       for r, t, fl in zip(self.slices, self.off_trend, self.flagged)],
        }, indent=1)
        if path:
            with open(path, "w") as fh:
                fh.write(d)
        return d


def _corners(r):
    h, w = r.moving_shape[:2]
    return np.array([[1, 1], [w, 1], [w, h], [1, h]], np.float64)


def _apply(H, p):
    q = np.c_[p, np.ones(len(p))] @ np.asarray(H).T
    return q[:, :2] / q[:, 2:]


def _pose_gap(r, H, refs):
    """Largest corner distance (fixed px) between pose H and the mean of the reference poses."""
    if not refs:
        return None
    c = _corners(r)
    ref = np.mean([_apply(R, c) for R in refs], axis=0)
    return float(np.max(np.hypot(*(_apply(H, c) - ref).T)))


def _expected(res, k, c):
    """Where slice k's corners c should land given its neighbours: their mean between two, a
    straight-line extrapolation at the ends (a stack that drifts steadily flags nothing)."""
    get = lambda j: res[j] if 0 <= j < len(res) else None
    a, b = get(k - 1), get(k + 1)
    if a is not None and b is not None:
        return (_apply(a.H, c) + _apply(b.H, c)) / 2
    for near, far in ((a, get(k - 2)), (b, get(k + 2))):
        if near is not None:
            return 2 * _apply(near.H, c) - _apply(far.H, c) if far is not None else _apply(near.H, c)
    return None


def _trend(res, jump):
    e = []
    for k, r in enumerate(res):
        ref = None if r is None else _expected(res, k, _corners(r))
        e.append(None if ref is None else float(np.max(np.hypot(*(_apply(r.H, _corners(r)) - ref).T))))
    vals = sorted(v for v in e if v is not None)
    thr = float(jump) if jump is not None else max(2.0, 4 * vals[len(vals) // 2]) if vals else math.inf
    return e, [v is not None and len(vals) >= 3 and v > thr for v in e], thr


def _detect(m, f, kw):
    """A slice pair from scratch: the rotation × scale sweep (this build's global search; keypoint
    detection is not part of it), the pose it returns climbed by its finalists' refine."""
    r = search(m, f, **kw)
    r.method = "search"
    return r


def register_stack(moving, fixed, *, start="previous", drop=0.15, jump=None, polish=False, progress=None,
                   model="homography", preprocess=True, register_pair=None, detect_pair=None, **settings):
    """Register a moving stack to a fixed stack, slice pair by slice pair (serial sections, time
    series): the first pair by the sweep search, then each from the previous pair's pose
    (refined), as python/zcmir/api.py:522-580 does with keypoints for the first pair.

    moving, fixed: sequences of images.
    start: "previous" (carry the previous pose) or "search" (every slice by the sweep search;
        "keypoints" is taken as "search").
    drop: re-detect (by the sweep search) when a slice's score falls more than this fraction below
        the previous slice's (the better of the two poses is kept).
    jump: the same when the pose jumps more than this many fixed px from the previous slice's
        (None: automatic, 4× the median jump so far, at least 2 px); it also flags slices off the
        trend of their neighbours in the result.
    polish: afterwards refine each slice again from the next slice's pose (last to first) and
        keep it when it scores higher.
    progress: callable(i, n, registration) after each slice.
    register_pair / detect_pair: the refine from a pose and the search from scratch (default: this
        module's refine and search on the GPU).
    """
    if start not in ("previous", "search", "keypoints"):
        raise ValueError('start: "previous" or "search"')
    kw = dict(model=model, preprocess=preprocess, **settings)
    refine_ = register_pair or (lambda m, f, H: register(m, f, init=H, **kw))
    detect_ = detect_pair or (lambda m, f: _detect(m, f, kw))
    n = min(len(moving), len(fixed))
    res, jumps = [None] * n, []

    def thr_now():
        if jump is not None:
            return float(jump)
        if len(jumps) < 3:
            return math.inf
        v = sorted(jumps)
        return max(2.0, 4 * v[len(v) // 2])

    for i in range(n):
        m, f = moving[i], fixed[i]
        prev = res[i - 1] if i else None
        if start != "previous" or prev is None:
            r = detect_(m, f)
        else:
            r = refine_(m, f, prev.H)
            r.method = "carry"
            g = _pose_gap(r, r.H, [prev.H])
            dropped = prev.score > 0 and r.score < prev.score * (1 - drop)
            if dropped or g > thr_now():
                k = detect_(m, f)
                r = k if k.score > r.score else r
                r.redetected = True
        if prev is not None:
            jumps.append(_pose_gap(r, r.H, [prev.H]))
        res[i] = r
        if progress:
            progress(i, n, r)
    if polish:
        for i in range(n - 2, -1, -1):
            r = refine_(moving[i], fixed[i], res[i + 1].H)
            if r.score > res[i].score * (1 + 1e-4):
                r.method, r.redetected = "carry", res[i].redetected
                res[i] = r
    e, flags, thr = _trend(res, jump)
    return StackRegistration(res, e, flags, thr)


def stack_maps(slices, priors=None, *, exact=True, calibrated=False, resolution=0, preprocess=False, **settings):
    """Shift maps along one stack — slice k (moving) against slice k − 1 (fixed) — with every
    slice's features built once on the GPU. Returns the n − 1 ShiftMaps and the device ms."""
    if preprocess:
        raise ValueError("stack_maps: preprocessing is not part of this build; pass preprocess=False")
    with _LOCK:
        reg = _engine()
        reg.configure(**_resolve(**settings))
        return reg.stack_maps(slices, priors, exact=exact, calibrated=calibrated, resolution=resolution)
