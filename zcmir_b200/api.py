"""The functional API over one shared engine (the reference's python/zcmir/api.py, SMI path).

Every function takes the engine's settings as keyword arguments (``settings()`` lists them) and
starts from the defaults, so one call never changes another. Calls are serialised.
"""
import difflib
import threading

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
        return {"H": reg.pose, "score": reg.score(reg.pose).mean, "iterations": c.iterations, "moved": c.moved}


def refine(moving, fixed, H, **kw):
    """Refine a pose: register(moving, fixed, init=H, ...)."""
    return register(moving, fixed, init=H, **kw)


def search(moving, fixed, H=None, *, mode="sweep", preprocess=True, **settings):
    """Brute force over rotation × scale × shift about H."""
    with _LOCK:
        reg, s, m, f = _prepare(moving, fixed, preprocess, dict(search_mode=mode, **settings))
        reg.pose = np.eye(3) if H is None else np.asarray(H, np.float64)
        r = reg.search()
        return {"H": reg.pose, "score": r.score, "previous": r.previous, "improved": r.improved}
