"""The functional API over one shared engine (the reference's python/zcmir/api.py, SMI path).

Every function takes the engine's settings as keyword arguments (``settings()`` lists them) and
starts from the defaults, so one call never changes another. Calls are serialised.
"""
import difflib
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


def _resolve(model="homography", **kw):
    """Keyword arguments → engine settings (defaults + these), with the names checked
    (python/zcmir/api.py:65-84)."""
    _engine()
    s = dict(_DEFAULTS)
    if model not in ("affine", "homography"):
        raise ValueError(f'model: "affine" or "homography", not {model!r}')
    s["group"] = model
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


@dataclass
class Registration:
    """A registered pair (python/zcmir/api.py:205-222, without the spline and keypoint fields):
    H maps moving pixel coordinates to fixed ones (row-major 3×3, 1-based)."""
    H: np.ndarray
    score: float
    model: str
    moving_shape: tuple
    fixed_shape: tuple
    method: str = "refine"
    iterations: int = 0

    def __repr__(self):
        return f"Registration({self.model}, score {self.score:.4g}, {self.method})"

    def map_points(self, points):
        """Moving (x, y) points (1-based, (n, 2)) to fixed coordinates by H."""
        p = np.asarray(points, np.float64).reshape(-1, 2)
        q = np.c_[p, np.ones(len(p))] @ self.H.T
        return q[:, :2] / q[:, 2:]


def shift_map(moving, fixed, H=None, *, preprocess=True, **settings):
    """The score at every translation of the moving image about pose H (default: identity)."""
    with _LOCK:
        reg, *_ = _prepare(moving, fixed, preprocess, settings)
        return reg.shift_map(np.eye(3) if H is None else np.asarray(H, np.float64))


def score(moving, fixed, H, *, preprocess=True, **settings):
    """The registration score at pose H (the mean of both directions when symmetric)."""
    with _LOCK:
        reg, *_ = _prepare(moving, fixed, preprocess, settings)
        return reg.score(np.asarray(H, np.float64)).mean


def register(moving, fixed, *, init=None, model="homography", preprocess=True, **settings):
    """Refine from ``init`` (keypoint detection is not part of this build, so ``init`` is
    required): the climb from H, then the score at the result."""
    if init is None:
        raise ValueError("register: keypoint detection is not part of this build; pass init=H (or use search())")
    with _LOCK:
        reg, s, m, f = _prepare(moving, fixed, preprocess, dict(model=model, **settings))
        reg.pose = np.asarray(init, np.float64).reshape(3, 3)
        c = reg.climb()
        return Registration(H=reg.pose, score=reg.score(reg.pose).mean, model=s["group"], moving_shape=m.shape,
                            fixed_shape=f.shape, method="refine", iterations=c.iterations)


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
