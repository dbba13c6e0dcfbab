"""GPU parity of the NCC overlay metric (settings metric="ncc": zc_score's zero-lag NCC of the
union canvas and zc_shift_map's NCC map, src/overlay.zig:209-305) against the CPU oracle,
through the C ABI.

Tolerances: the score within 1e-6 (float64 sums on both sides; the warp's source positions are
float32 on the GPU and float64 in the oracle). The map within 2e-5 of the oracle's at every lag
(FP32 FFTs of lines ≤ 1024 points, values ≤ 1.5) with its peak at the same lag; with f16
texels 1e-4 (a warped texel may round to the neighbouring f16 value)."""
import numpy as np
import pytest

import zcmir_b200 as zc
from oracle import ncc_oracle as N
from zcmir_b200 import synth

pytestmark = pytest.mark.gpu


def _turn(H, deg, s, c):
    a = np.deg2rad(deg)
    R = np.array([[s * np.cos(a), -s * np.sin(a), 0], [s * np.sin(a), s * np.cos(a), 0], [0, 0, 1]])
    T = lambda x, y: np.array([[1, 0, x], [0, 1, y], [0, 0, 1.0]])
    return T(*c) @ R @ T(-c[0], -c[1]) @ H


@pytest.mark.parametrize("half,crop", [(False, None), (True, (150, 230))])
def test_ncc_score_and_map_match_oracle(half, crop):
    m, f, H = synth.pair_remap(n=240, shift=(11, -7), seed=2)
    if crop:
        m = m[: crop[0], : crop[1]]
        f = f[:190, :170]
    H = _turn(H, 3.0, 1.02, (100.5, 80.5))
    with zc.Engine(half=half, metric="ncc") as reg:
        reg.set_images(np.clip(m, 0, 1), np.clip(f, 0, 1), preprocess=False)
        wa, wb = reg.work_image(0), reg.work_image(1)
        sc = reg.score(H)
        sm = reg.shift_map(H)
    ref_s = N.ncc_score(wa, wb, H, half)
    assert sc.inv is None and sc.mean == sc.fwd
    assert abs(sc.mean - ref_s) <= 1e-6, (sc.mean, ref_s)
    ref = N.ncc_map(wa, wb, H, half)
    assert (sm.n, sm.ny, sm.cw, sm.ch) == (ref["n"], ref["n"], ref["cw"], ref["ch"])
    assert (sm.offset, sm.canvas) == (ref["frame"][:2], ref["frame"][2:])
    tol = 1e-4 if half else 2e-5
    err = np.abs(sm.map - ref["map"]).max()
    assert err <= tol, err
    assert sm.peak_index == ref["peak_index"] and (sm.dx, sm.dy) == (ref["dx"], ref["dy"])
    assert sm.peak == pytest.approx(ref["peak"], abs=tol) and sm.zero == pytest.approx(ref["zero"], abs=tol)
    assert not sm.exact and not sm.calibrated and sm.corr_area_px == 0


def test_ncc_map_finds_a_planted_shift():
    """Same modality, moving = fixed translated by (−19, 12): the NCC map at the identity peaks
    at that lag (in canvas pixels, resampled cells scaled back), NCC near 1."""
    rng = np.random.default_rng(5)
    big = synth.blob_field(400, 400, rng)
    fixed = big[40:340, 40:340]
    tx, ty = -19, 12
    moving = big[40 - ty:340 - ty, 40 - tx:340 - tx]
    with zc.Engine(half=False, metric="ncc") as reg:
        reg.set_images(moving.astype(np.float32), fixed.astype(np.float32), preprocess=False)
        sm = reg.shift_map(np.eye(3))
        s0 = reg.score(np.eye(3)).mean
        s1 = reg.score(np.array([[1, 0, -sm.dx], [0, 1, -sm.dy], [0, 0, 1.0]])).mean
    assert abs(sm.dx - tx) <= 1 and abs(sm.dy - ty) <= 1, (sm.dx, sm.dy)
    assert sm.peak > 0.9
    assert s1 > s0


def test_ncc_metric_leaves_the_smi_paths(golden):
    """With metric "ncc" the pose gradient is SMI's (src/engine.zig:769-779) and the sweep
    search refuses (src/search.zig:666); the reference's own check of the NCC score
    (tests/test_api.py:144): |score| ≤ 1 at the landsat-b truth."""
    d = np.load(golden / "landsat_b.npz")
    mv, fx, truth = d["moving"], d["fixed"], d["truth"]
    with zc.Engine(metric="ncc") as reg:
        reg.set_images(mv, fx)
        s = reg.score(truth).mean
        g_ncc = reg.gradient(truth)
        with pytest.raises(RuntimeError, match="SweepNeedsMomentScore"):
            reg.search()
        reg.configure(metric="smi")
        g_smi = reg.gradient(truth)
    assert 0 < abs(s) <= 1
    assert g_ncc.score == g_smi.score
    np.testing.assert_array_equal(g_ncc.grad, g_smi.grad)
