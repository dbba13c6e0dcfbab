"""zcb_score_static, the pose-score entry point that allocates no device memory, against zc_score
through the C ABI.

Two calls in a row must each give zc_score's scores within the pose tests' score tolerance
(1e-5 relative), and the second must leave the GPU's free memory unchanged. Oversized batches
and missing feature planes are refused with an error. This file is collected last so that it
also runs after every other GPU test in the same process."""
import ctypes
import gc
import json

import numpy as np
import pytest

from zcmir_b200 import _native, synth

pytestmark = pytest.mark.gpu

MAX_POSES = 64


def _err(lib, e):
    buf = ctypes.create_string_buffer(1024)
    n = lib.zc_error(e, buf, 1024)
    return buf.raw[:n].decode()


def _poses(H, k, seed):
    rng = np.random.default_rng(seed)
    c = 128.5
    out = []
    for _ in range(k):
        a = np.deg2rad(rng.uniform(-4, 4))
        s = np.exp(rng.uniform(-0.03, 0.03))
        t = rng.uniform(-3, 3, 2)
        R = np.array([[s * np.cos(a), -s * np.sin(a), 0], [s * np.sin(a), s * np.cos(a), 0], [0, 0, 1]])
        T = lambda x, y: np.array([[1, 0, x], [0, 1, y], [0, 0, 1.0]])
        out.append(T(c + t[0], c + t[1]) @ R @ T(-c, -c) @ H)
    return np.ascontiguousarray(np.array(out, dtype=np.float64))


@pytest.fixture(scope="module")
def lib():
    return _native.load()


def _engine(lib, settings):
    e = lib.zc_create(None)
    assert e, "zc_create failed"
    js = json.dumps(settings).encode()
    assert lib.zc_configure(e, js, len(js)) == 0, _err(lib, e)
    return e


def _set_images(lib, e, preprocess=0):
    m, f, H = synth.pair_remap(n=256, shift=(17, -9), seed=0)
    for side, img in ((0, m), (1, f)):
        a = np.ascontiguousarray(img, dtype=np.float32)
        h, w = a.shape
        rc = lib.zc_set_image_gray(e, side, a.ctypes.data_as(_native.f32p), w, h, preprocess)
        assert rc == 0, _err(lib, e)
    return H


def _reference_scores(lib, e, Hs):
    out = np.zeros((len(Hs), 3))
    for i, H in enumerate(Hs):
        o = (ctypes.c_double * 3)()
        assert lib.zc_score(e, (ctypes.c_double * 9)(*H.ravel()), o) == 0, _err(lib, e)
        out[i] = list(o)
    return out


def _static_scores(lib, e, Hs):
    out = np.full((len(Hs), 3), -1.0)
    rc = lib.zcb_score_static(e, Hs.ctypes.data_as(_native.f64p), len(Hs), out.ctypes.data_as(_native.f64p))
    assert rc == 0, _err(lib, e)
    return out


def _check(got, ref, symmetric):
    for c in range(3 if symmetric else 2):
        np.testing.assert_allclose(got[:, c], ref[:, c], rtol=1e-5, atol=1e-12)
    if not symmetric:
        assert np.isnan(got[:, 2]).all() and np.isnan(ref[:, 2]).all()


@pytest.mark.parametrize("symmetric", [True, False])
def test_static_scores_match_zc_score_twice(lib, symmetric):
    import torch

    e = _engine(lib, {"half": False, "symmetric": symmetric})
    try:
        H = _set_images(lib, e)
        Hs = _poses(H, 48, seed=3)
        ref = _reference_scores(lib, e, Hs)
        assert np.isfinite(ref[:, :2]).all() and (np.abs(ref[:, 1]) > 0).any()
        first = _static_scores(lib, e, Hs)
        _check(first, ref, symmetric)
        gc.collect()
        gc.disable()
        try:
            free_before = torch.cuda.mem_get_info(0)[0]
            second = _static_scores(lib, e, Hs)
            free_after = torch.cuda.mem_get_info(0)[0]
        finally:
            gc.enable()
        _check(second, ref, symmetric)
        assert free_after == free_before, (free_before, free_after)
        # a shorter batch after a longer one reads only its own poses
        _check(_static_scores(lib, e, Hs[:5]), ref[:5], symmetric)
    finally:
        lib.zc_destroy(e)


def test_static_scores_right_after_the_images(lib):
    """The first call after zc_set_image_gray, with no zc_score before it: side 1's planes build on
    a stream of their own, and the call must wait for that build rather than read planes still
    being written."""
    for rep in range(2):
        e = _engine(lib, {"half": False, "symmetric": True})
        try:
            H = _set_images(lib, e)
            Hs = _poses(H, 16, seed=11 + rep)
            first = _static_scores(lib, e, Hs)
            ref = _reference_scores(lib, e, Hs)
            _check(first, ref, True)
        finally:
            lib.zc_destroy(e)


def test_static_scores_refusals(lib):
    e = _engine(lib, {"half": False})
    try:
        Hs = np.tile(np.eye(3).ravel(), (MAX_POSES + 1, 1))
        out = np.zeros((MAX_POSES + 1, 3))
        # no images yet
        rc = lib.zcb_score_static(e, Hs.ctypes.data_as(_native.f64p), 1, out.ctypes.data_as(_native.f64p))
        assert rc == -1 and "NoImages" in _err(lib, e)
        _set_images(lib, e)
        rc = lib.zcb_score_static(e, Hs.ctypes.data_as(_native.f64p), MAX_POSES + 1, out.ctypes.data_as(_native.f64p))
        assert rc == -1 and "maximum of 64" in _err(lib, e)
        # a count past 2^31 is refused for its size too (it is checked before anything is read)
        rc = lib.zcb_score_static(e, Hs.ctypes.data_as(_native.f64p), 2**31 + 5, out.ctypes.data_as(_native.f64p))
        assert rc == -1 and "maximum of 64" in _err(lib, e)
        # an empty batch is a no-op
        assert lib.zcb_score_static(e, Hs.ctypes.data_as(_native.f64p), 0, out.ctypes.data_as(_native.f64p)) == 0
        # settings that change the feature planes leave them unbuilt: refused, not rebuilt
        js = json.dumps({"smi_features": "three"}).encode()
        assert lib.zc_configure(e, js, len(js)) == 0, _err(lib, e)
        rc = lib.zcb_score_static(e, Hs.ctypes.data_as(_native.f64p), 1, out.ctypes.data_as(_native.f64p))
        assert rc == -1 and "not built" in _err(lib, e)
    finally:
        lib.zc_destroy(e)


def test_static_scores_refuse_stale_preprocessing(lib):
    """Planes baked with one preprocessing (CLAHE) are stale once a preprocessing setting changes:
    the call refuses instead of scoring them (zc_score would re-bake)."""
    e = _engine(lib, {"half": False})
    try:
        H = _set_images(lib, e, preprocess=1)
        Hs = np.ascontiguousarray(H.reshape(1, 9))
        ref = _reference_scores(lib, e, Hs.reshape(1, 3, 3))
        _check(_static_scores(lib, e, Hs), ref, True)
        js = json.dumps({"clahe_grid": 8}).encode()
        assert lib.zc_configure(e, js, len(js)) == 0, _err(lib, e)
        out = np.zeros((1, 3))
        rc = lib.zcb_score_static(e, Hs.ctypes.data_as(_native.f64p), 1, out.ctypes.data_as(_native.f64p))
        assert rc == -1 and "not built" in _err(lib, e)
    finally:
        lib.zc_destroy(e)
