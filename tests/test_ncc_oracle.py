"""The NCC oracle on its own (CPU): the plan against hand-worked cases of src/fft.zig:70-91, a
planted translation found at its lag with NCC 1, and the zero-lag score's known values."""
import numpy as np

from oracle import ncc_oracle as N


def test_plan_cases():
    # s = 512/640: 512 × 384 cells, 2·512 − 1 = 1023 → the ladder's 1024
    assert N.linear_corr_plan(640, 480) == (1024, 512, 384)
    # small canvases keep their size: 2·100 − 1 = 199 → 216 = 2³·3³
    assert N.linear_corr_plan(100, 60) == (216, 100, 60)
    # the 32-point floor and the 8-cell floor
    assert N.linear_corr_plan(10, 3) == (32, 10, 8)
    # a long thin canvas: the longer side sets the scale
    n, cw, ch = N.linear_corr_plan(3000, 200)
    assert n == 1024 and cw == 512 and ch == 34


def _field(n, seed):
    rng = np.random.default_rng(seed)
    f = rng.standard_normal((n + 16, n + 16))
    k = np.exp(-0.5 * (np.arange(-6, 7) / 2.0) ** 2)
    f = np.apply_along_axis(lambda r: np.convolve(r, k, "same"), 0, f)
    f = np.apply_along_axis(lambda r: np.convolve(r, k, "same"), 1, f)
    return (f - f.min()) / (f.max() - f.min())


def test_planted_shift_and_known_scores():
    big = _field(96, 3)
    fixed = big[8:8 + 96, 8:8 + 96]
    tx, ty = 5, -3
    moving = big[8 - ty:8 - ty + 96, 8 - tx:8 - tx + 96]   # moving(p) = fixed(p − t)
    r = N.ncc_map(moving, fixed, np.eye(3))
    assert (r["dx"], r["dy"]) == (tx, ty)
    assert r["peak"] > 0.9
    # the corrected pose translate(−dx, −dy) scores higher than the identity
    T = np.array([[1, 0, -tx], [0, 1, -ty], [0, 0, 1.0]])
    assert N.ncc_score(moving, fixed, T) > N.ncc_score(moving, fixed, np.eye(3))
    # identical images at the identity: the canvases are equal, r = 1
    assert abs(N.ncc_score(fixed, fixed, np.eye(3)) - 1.0) < 1e-12
    # a constant side has no variance: r = 0 (the 1e-24 floor)
    assert N.ncc_score(np.full((40, 40), 0.5), np.full((40, 40), 0.5), np.eye(3)) == 0.0
