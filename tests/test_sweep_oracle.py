"""The sweep oracle (CPU): its grid and NMS rules, its candidate maps against FFT-free float64
sums, the zero-lag overlap it floors against, and recovery of a planted similarity — the
reference's own check of the sweep is that it lands within 5 px of the pose
(tests/test_api.py:156-166); the coarse peak before any refine must already lie within a few
canvas cells of it."""
import math

import numpy as np
import pytest

from oracle import smi_oracle as O
from oracle import sweep_oracle as S
from zcmir_b200 import synth


def corner_dist(A, B, w, h):
    d = 0.0
    for x, y in [(1, 1), (w, 1), (w, h), (1, h)]:
        a, b = A @ [x, y, 1.0], B @ [x, y, 1.0]
        d = max(d, float(np.hypot(*(a[:2] / a[2] - b[:2] / b[2]))))
    return d


def test_grid_rules():
    g = S.sweep_grid(n_theta=4, n_sigma=3, s_min=0.5, s_max=2)
    assert g["wrap"] and np.allclose(np.degrees(g["thetas"]), [-180, -90, 0, 90])
    assert np.allclose(g["sigmas"], [0.5, 1.0, 2.0])
    assert g["shears"] == [0.0] and g["anisos"] == [1.0]
    g = S.sweep_grid(rot_lo=-30, rot_hi=30, n_theta=3, shear_max=0.1, n_shear=3, aniso_max=0.1, n_aniso=3)
    assert not g["wrap"] and np.allclose(np.degrees(g["thetas"]), [-30, 0, 30])
    assert np.allclose(g["shears"], [-0.1, 0, 0.1]) and np.allclose(g["anisos"], [1 / 1.1, 1, 1.1])
    # σ R(θ) diag(a, 1/a) [1 k; 0 1]
    L = S.cand_linear(0.3, 1.2, 0.05, 1.1)
    R = 1.2 * np.array([[math.cos(0.3), -math.sin(0.3)], [math.sin(0.3), math.cos(0.3)]])
    assert np.allclose(np.array(L).reshape(2, 2), R @ np.diag([1.1, 1 / 1.1]) @ np.array([[1, 0.05], [0, 1]]))
    assert np.allclose(S.sv2(L), np.linalg.svd(np.array(L).reshape(2, 2), compute_uv=False))
    assert S.ladder_size(70) == 96 and S.ladder_size(100) == 128 and S.ladder_size(130) == 144
    assert S.ladder_size(130, "compact") == 160 and S.ladder_size(600, "compact") == 624


def test_nms_rules():
    P = lambda sc, it, is_, sx, sy: {"score": sc, "it": it, "is": is_, "ik": 0, "ia": 0, "sx": sx, "sy": sy}
    peaks = [P(5, 0, 0, 0, 0), P(4, 89, 1, 2, 2), P(3, 3, 0, 0, 0), P(2, 0, 0, 10, 0), P(1, 1, 3, 0, 0)]
    kept = S.nms4(peaks, 90, 8, True)
    # θ 89 is 1 step from θ 0 on the circle: suppressed; θ 3 and 10 cells away and σ 3 steps survive
    assert [p["score"] for p in kept] == [5, 3, 2, 1]
    assert [p["score"] for p in S.nms4(peaks, 90, 8, False)] == [5, 4, 3, 2, 1]
    assert len(S.nms4(peaks, 90, 2, True)) == 2


@pytest.fixture(scope="module")
def small():
    m, f, H = synth.pair_similarity(n=128, seed=5, deg=40.0, scale=1.1, shift=(6.0, -4.0))
    pa, pb = O.prepare(m.astype(np.float32) / 65535), O.prepare(f.astype(np.float32) / 65535)
    return pa, pb, H


def test_candidate_map_equals_direct_sums(small):
    pa, pb, _ = small
    gv = S.sweep_grid(n_theta=6, n_sigma=2, s_min=0.8, s_max=1.25)
    st = S.sweep_setup(128, 128, 128, 128, np.eye(3), gv, G=64)
    c = st["cands"][3]
    nx, ny, Fx, Fy = c["nx"], c["ny"], st["Fx"], st["Fy"]
    sa = S.pack_window(pa["stack"], np.linalg.inv(c["H"]), c["taps"], c["gx0"], c["gy0"], nx - Fx + 1, ny - Fy + 1,
                       nx, ny, st["ox"], st["oy"], st["cell"], st["G"])
    sb = S.pack_window(pb["stack"], np.eye(3), st["fixed_taps"], st["fcx"][0], st["fcy"][0], Fx, Fy, nx, ny, st["ox"],
                       st["oy"], st["cell"], st["G"])
    ids, corrs = O.corr_plan(True, False)
    A, B = O.real_planes(sa, ids), O.real_planes(sb, ids)
    corr = O.correlations(A, B, ids, corrs, nx, ny)
    rng = np.random.default_rng(0)
    for _ in range(6):
        tx, ty = int(rng.integers(-(Fx - 1), nx - Fx + 1)), int(rng.integers(-(Fy - 1), ny - Fy + 1))
        # Σ_x a(x + t) b(x): the lag wraps onto the plane
        direct = np.zeros(45)
        for a, b, k in corrs:
            pa_, pb_ = A[ids.index(a)], B[ids.index(b)]
            sh = np.roll(np.roll(pa_, -ty, axis=0), -tx, axis=1)
            direct[k] = float(np.sum(sh * pb_))
        got = corr[:, ty % ny, tx % nx]
        assert np.allclose(got, direct, rtol=1e-9, atol=1e-9 * np.abs(corr).max())
    # the floor's zero-lag overlap is the weight planes' sum over the cells both windows cover
    zl = S.zero_lag(c, st)
    # fixed cell x' meets moving cell x where gx0 + x = fx0 + x'
    fb = np.roll(np.roll(sb[0], st["fcy"][0] - c["gy0"], 0), st["fcx"][0] - c["gx0"], 1)
    assert abs(corr[0].ravel()[zl] - float(np.sum(sa[0] * fb))) < 1e-6


def test_coarse_peak_near_the_planted_pose(small):
    pa, pb, H = small
    gv = S.sweep_grid(n_theta=36, n_sigma=5, s_min=0.8, s_max=1.25)
    H0 = np.eye(3)
    r = S.sweep(pa, pb, H0, gv, G=64, exact=True)
    top = S.nms4(r["peaks"], 36, 8, gv["wrap"])
    assert top, "no peak"
    cell = r["setup"]["cell"]
    # 10° and 11 % steps and a 3.5 px cell: the best coarse pose within a few cells at the corners
    assert corner_dist(top[0]["H"], H, 128, 128) < 4 * cell, corner_dist(top[0]["H"], H, 128, 128)
    assert abs(math.degrees(top[0]["th"]) - 40) <= 10 and abs(math.log(top[0]["s"] / 1.1)) <= 0.12
