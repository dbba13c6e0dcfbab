"""The reference's own Python package, unmodified, running on this build's libzcmir.so.

baseline/install_reference.py copies the reference's python/zcmir byte for byte into
baseline/_ref (with a manifest of SHA-256 hashes, checked here). ``ZCMIR_LIB`` points that
package's loader (python/zcmir/_native.py:136-146) at zcmir_b200/libzcmir.so; every call below is
the reference's code down to the zc_* C ABI: the functional API (python/zcmir/api.py:291-580:
shift_map, score, rs_map, register / refine, search, register_stack) and ``Registrar``
(python/zcmir/__init__.py:206-622: features, moments, score, shift_map).

Tolerances are the other GPU tests': features within 2e-6 of the float64 oracle's, moments within
1e-5 of the largest sum, scores within 1e-5 relative, maps with the oracle's argmax and every cell
within 1e-4 of the peak where the overlap is at least 20 % of the largest (1e-2 elsewhere),
roto-scale maps with the oracle's peak, refined poses within 1 px of the planted one at every
corner, searches and stacks within the reference's own bounds (5 px, tests/test_api.py:156-166;
2 px per slice pair). Where this package's Engine makes the same call on the same library, the
results must be equal.

This build has no keypoint detector: register() without a start pose and register_stack's first
pair go through zc_detect / zc_match, which here fit the pose by the SMI sweep search."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

import zcmir_b200 as zc
from oracle import pose_oracle as PO
from oracle import rs_oracle as R
from oracle import smi_oracle as O
from zcmir_b200 import synth

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "baseline"))
import install_reference as IR  # noqa: E402

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not IR.verify(), reason="baseline/_ref holds no verified copy of the reference's package "
                                              "(python baseline/install_reference.py --reference <checkout>)"),
]

LIB = ROOT / "zcmir_b200" / "libzcmir.so"


@pytest.fixture(scope="module")
def zcmir():
    os.environ["ZCMIR_LIB"] = str(LIB)
    os.environ["ZCMIR_WGPU"] = str(LIB)  # the loader wants an existing file here; zc_create ignores it
    sys.path.insert(0, str(IR.DEST))
    import zcmir as ref_pkg

    assert Path(ref_pkg.__file__).resolve().parent == (IR.DEST / "zcmir").resolve()
    yield ref_pkg
    ref_pkg.close()


@pytest.fixture(scope="module")
def c1():
    return synth.pair_remap(n=256, shift=(17, -9), seed=0)


def prep_from(feat):
    f = np.asarray(feat, np.float32)
    return {"w": f.shape[2], "h": f.shape[1], "mode": "laplacian", "feat": f, "acf": O.acf(f),
            "stack": np.concatenate([np.ones((1,) + f.shape[1:], np.float32), f])}


def corner_dist(A, B, w, h):
    d = 0.0
    for x, y in [(1, 1), (w, 1), (w, h), (1, h)]:
        a, b = A @ [x, y, 1.0], B @ [x, y, 1.0]
        d = max(d, float(np.hypot(*(a[:2] / a[2] - b[:2] / b[2]))))
    return d


def near_pose(H, deg, scale, t, n):
    c = (n + 1) / 2
    a = np.deg2rad(deg)
    R2 = np.array([[scale * np.cos(a), -scale * np.sin(a), 0], [scale * np.sin(a), scale * np.cos(a), 0], [0, 0, 1]])
    T = lambda x, y: np.array([[1, 0, x], [0, 1, y], [0, 0, 1.0]])
    return T(c + t[0], c + t[1]) @ R2 @ T(-c, -c) @ H


def test_loader_binds_every_symbol(zcmir):
    from zcmir import _native

    lib, _ = _native.load()
    assert Path(lib._name).resolve() == LIB.resolve()
    assert all(hasattr(lib, name) for name in _native._SIGS)


def test_registrar_features_and_moments(zcmir, c1):
    m, f, H = c1
    reg = zcmir.Registrar(half=False)
    try:
        reg.set_images(m, f, preprocess=False)
        fa, fb = reg.features(0), reg.features(1)
        for got, img in ((fa, m), (fb, f)):
            np.testing.assert_allclose(got, O.prepare(img)["feat"], rtol=0, atol=2e-6)
        mom = reg.moments(H)
        want = PO.moments(fa, fb, H)
        assert np.abs(mom - want).max() <= 1e-5 * np.abs(want).max()
        s = reg.score(H)
        ref = PO.pair_eval(fa, fb, H, exact=True, symmetric=True)
        assert abs(s.fwd - ref["fwd"]) <= 1e-5 * abs(ref["fwd"]) and abs(s.inv - ref["inv"]) <= 1e-5 * abs(ref["inv"])
    finally:
        reg.close()
    with zc.Engine(half=False) as eng:
        eng.set_images(m, f, preprocess=False)
        np.testing.assert_array_equal(eng.features(0), fa)
        np.testing.assert_array_equal(eng.moments(H), mom)


def test_functional_score_and_shift_map(zcmir, c1):
    """zcmir.score and zcmir.shift_map with the settings' defaults: exact, calibrated, the
    shift-map overlap floor min_overlap = 0.05 and the auto resolution (a 512² FFT here)."""
    m, f, H = c1
    s = zcmir.score(m, f, H, preprocess=False, half=False)
    sm = zcmir.shift_map(m, f, np.eye(3), preprocess=False, half=False)
    with zc.Engine(half=False) as eng:
        eng.set_images(m, f, preprocess=False)
        pa, pb = prep_from(eng.features(0)), prep_from(eng.features(1))
        mine = eng.shift_map(np.eye(3))
    ref = PO.pair_eval(pa["feat"], pb["feat"], H, exact=True, symmetric=True)
    assert abs(s - ref["mean"]) <= 1e-5 * abs(ref["mean"])
    o = O.shift_map(pa, pb, np.eye(3), exact=True, calibrated=True, cap=0, min_overlap=0.05, return_corr=True)
    assert (sm.n, sm.ny, sm.cw, sm.ch) == (o["n"], o["n_y"], o["cw"], o["ch"]) == (512, 512, 256, 256)
    assert int(np.argmax(sm.map)) == o["peak_index"] and (sm.dx, sm.dy) == (o["dx"], o["dy"]) == (-17.0, 9.0)
    assert abs(sm.peak - o["peak"]) <= 1e-4 * abs(o["peak"])
    n0 = o["corr"][0]
    err = np.abs(sm.map.astype(np.float64) - o["map"]) / abs(o["peak"])
    one_sided = (sm.map == 0) != (o["map"] == 0)
    assert one_sided.mean() < 1e-3
    assert err[(n0 >= 0.2 * n0.max()) & ~one_sided].max() <= 1e-4
    assert err[~one_sided].max() <= 1e-2
    np.testing.assert_array_equal(sm.map, mine.map)


def test_functional_rs_map(zcmir, c1):
    """zcmir.rs_map at the truth turned by 6° and scaled by 1.08 about the moving centroid: the
    oracle's peak (symmetric, calibrated: the settings' defaults) and the correction back."""
    m, f, H = c1
    H1 = near_pose(H, 6.0, 1.08, (0, 0), 256)
    c = R.moving_centroid(H1, 256, 256)
    r = zcmir.rs_map(m, f, H1, preprocess=False, half=False)
    with zc.Engine(half=False) as eng:
        eng.set_images(m, f, preprocess=False)
        pa, pb = prep_from(eng.features(0)), prep_from(eng.features(1))
    o = R.rs_map(pa, pb, H1, symmetric=True, exact=True, calibrated=True)
    assert r.n == o["plan"]["n"]
    assert int(np.argmax(r.map)) == o["peak_index"]
    assert abs(r.dth - o["dth"]) < 1e-9 and abs(r.dsg - o["dsg"]) < 1e-9
    assert abs(np.rad2deg(r.dth) + 6) < 2 and abs(np.exp(-r.dsg) - 1.08) < 0.03
    np.testing.assert_allclose(r.center, c, atol=1e-9)


@pytest.mark.parametrize("model", ["affine", "homography"])
def test_refine_from_a_nearby_pose(zcmir, model):
    """register(init=…) / refine: the reference's climb from 3° and 4 px off the planted
    similarity ends within 1 px of it at every corner."""
    m16, f16, H = synth.pair_similarity(n=256, seed=7)
    m, f = zc.gray32(m16), zc.gray32(f16)
    H0 = near_pose(H, 3.0, 1.02, (4.0, -3.0), 256)
    r = zcmir.register(m, f, init=H0, model=model, preprocess=False, half=False)
    assert r.method == "refine" and r.iterations > 0
    assert corner_dist(r.H, H, 256, 256) < 1, corner_dist(r.H, H, 256, 256)
    r2 = zcmir.refine(m, f, H0, model=model, preprocess=False, half=False)
    np.testing.assert_allclose(r2.H, r.H, atol=1e-9)


def test_search_and_register_without_a_start(zcmir):
    """zcmir.search over the full circle (sweep) and zcmir.register with no start pose (the
    keypoint path, here the SMI sweep) land within 5 px of the planted similarity."""
    m16, f16, H = synth.pair_similarity(n=256, seed=7)
    m, f = zc.gray32(m16), zc.gray32(f16)
    s = zcmir.search(m, f, preprocess=False, half=False)
    assert s.method == "search (sweep)" and corner_dist(s.H, H, 256, 256) < 5, corner_dist(s.H, H, 256, 256)
    r = zcmir.register(m, f, model="affine", preprocess=False, half=False)
    assert r.method == "keypoints" and r.keypoints == (0, 0)
    assert corner_dist(r.H, H, 256, 256) < 2, corner_dist(r.H, H, 256, 256)


def test_search_ranges_shear_stretch_and_misses(zcmir):
    """search()'s rotation range, shear and stretch keywords reach the sw_* settings: a range
    about the truth finds it, a range that misses it does not."""
    m16, f16, H = synth.pair_similarity(n=256, seed=7, deg=25.0, scale=0.9, shift=(10.0, -12.0))
    m, f = zc.gray32(m16), zc.gray32(f16)
    J = H[:2, :2]
    ang = np.degrees(np.arctan2(J[1, 0] - J[0, 1], J[0, 0] + J[1, 1]))
    common = dict(preprocess=False, half=False)
    r = zcmir.search(m, f, rotation=(ang - 40, ang + 40), sw_nth=21, shear=0.05, stretch=(0.05, 3), **common)
    assert corner_dist(r.H, H, 256, 256) < 5, corner_dist(r.H, H, 256, 256)
    miss = zcmir.search(m, f, rotation=(ang + 90, ang + 150), sw_nth=11, **common)
    assert corner_dist(miss.H, H, 256, 256) > 5


def test_register_stack_follows_a_drifting_stack(zcmir):
    """The reference's register_stack loop (python/zcmir/api.py:522-580): the first pair from the
    sweep, the others carried from the previous pose and refined; every pair within 2 px of its
    planted similarity, no slice off the trend."""
    slices, truths = synth.stack_drift(n=6, size=(256, 384), seed=4)
    slices = [zc.gray32(s) for s in slices]
    moving, fixed = slices[1:], slices[:-1]
    seen = []
    r = zcmir.register_stack(moving, fixed, model="affine", preprocess=False, half=False,
                             progress=lambda i, n, x: seen.append(i))
    assert seen == list(range(len(moving)))
    # a pair whose carried score drops by more than 15 % is re-detected (here: the sweep), and
    # keeps whichever pose scores higher
    assert r.slices[0].method == "keypoints"
    assert all(x.method == "carry" or x.redetected for x in r.slices[1:])
    for k, (reg_k, H) in enumerate(zip(r.slices, truths)):
        h, w = moving[k].shape
        assert corner_dist(reg_k.H, H, w, h) < 2, (k, reg_k.method, corner_dist(reg_k.H, H, w, h))
    assert not any(r.flagged)


def _bilinear(img, X, Y):
    h, w = img.shape
    x0 = np.clip(np.floor(X).astype(int), 0, w - 2)
    y0 = np.clip(np.floor(Y).astype(int), 0, h - 2)
    fx, fy = np.clip(X - x0, 0, 1), np.clip(Y - y0, 0, 1)
    return ((img[y0, x0] * (1 - fx) + img[y0, x0 + 1] * fx) * (1 - fy)
            + (img[y0 + 1, x0] * (1 - fx) + img[y0 + 1, x0 + 1] * fx) * fy)


def test_register_with_spline_recovers_a_smooth_warp(zcmir):
    """register(spline=True): a 256² blob field against itself under a smooth non-rigid warp
    (amplitude 3 px) and a small shift; the spline stage moves the control points, raises the
    score over the homography-only result and brings the displacement field closer to the true
    one."""
    rng = np.random.default_rng(8)
    n = 256
    fixed = synth.blob_field(n, n, rng).astype(np.float32)
    Y, X = np.mgrid[0:n, 0:n].astype(np.float64)
    vx = 3.0 * np.sin(2 * np.pi * Y / n) * np.cos(np.pi * X / n) + 1.5
    vy = 3.0 * np.cos(2 * np.pi * X / n) * np.sin(np.pi * Y / n) - 1.0
    moving = _bilinear(fixed.astype(np.float64), X + vx, Y + vy).astype(np.float32)
    true_d = -np.stack([vx, vy], -1)   # fixed x ↔ moving x − v(x), to first order
    r0 = zcmir.register(moving, fixed, init=np.eye(3), preprocess=False, half=False)
    r1 = zcmir.register(moving, fixed, init=np.eye(3), spline=True, preprocess=False, half=False)
    assert r1.spline is not None and r1.spline.shape == (32,) and np.abs(r1.spline).max() > 0
    assert r1.lattice == 4
    assert r1.score > r0.score
    inner = (slice(24, n - 24), slice(24, n - 24))
    e0 = np.linalg.norm(r0.displacement()[inner] - true_d[inner], axis=-1).mean()
    e1 = np.linalg.norm(r1.displacement()[inner] - true_d[inner], axis=-1).mean()
    assert e1 < 0.8 * e0, (e0, e1)
    w = r1.warp(moving)
    assert w.shape == fixed.shape and w.dtype == moving.dtype
