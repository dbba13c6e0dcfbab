"""The oracle against the reference's known answer for the engine's map (examples/03_smi.py:364)
and against itself (FFT correlations vs direct float64 sums). CPU only. The vectors that the
reference's own NumPy code computed are checked in test_golden_03_smi.py."""
import numpy as np
import pytest

from oracle import smi_oracle as O
from zcmir_b200 import synth

@pytest.fixture(scope="module")
def landsat(golden):
    d = np.load(golden / "landsat_b.npz")
    pa = O.prepare(d["moving"].astype(np.float32) / 255, "laplacian")
    pb = O.prepare(d["fixed"].astype(np.float32) / 255, "laplacian")
    return pa, pb, d["truth"]


@pytest.mark.slow
def test_known_answer_engine_map_full_resolution(landsat):
    """The engine-semantics map (canvas, grid, 45 correlations, combine) at full resolution
    peaks at lag (14, −9) for H0 = T(14, −9)·truth (the 03_smi answer; its engine check allows
    2 px, examples/03_smi.py:364), on a 2^3·3^5 = 1944-point ladder FFT."""
    pa, pb, truth = landsat
    H0 = np.array([[1, 0, 14], [0, 1, -9], [0, 0, 1.0]]) @ truth
    r = O.shift_map(pa, pb, H0, exact=True, calibrated=False, cap=2048)
    assert (r["n"], r["cw"]) == (1944, 917)
    assert (r["dx"], r["dy"]) == (14.0, -9.0)
    r = O.shift_map(pa, pb, H0, exact=True, calibrated=False, cap=1024)
    assert np.hypot(r["dx"] - 14, r["dy"] + 9) < 2


def test_fft_correlations_equal_direct_sums():
    m, f, _ = synth.pair_remap(n=64, shift=(5, -3), seed=3)
    pa, pb = O.prepare(m), O.prepare(f)
    ga, gb, (nx, ny, cw, ch), _ = O.grid_stacks(pa, pb, np.eye(3), cap=1024)
    ids, corrs = O.corr_plan(True, False)
    A, B = O.real_planes(ga, ids), O.real_planes(gb, ids)
    corr = O.correlations(A, B, ids, corrs, nx, ny)
    for tx, ty in [(0, 0), (5, -3), (-20, 11), (63, -63), (-7, 0)]:
        d = O.direct_sums(A, B, ids, corrs, tx, ty)
        np.testing.assert_allclose(corr[:, ty % ny, tx % nx], d, rtol=1e-9, atol=1e-9)


def test_plans():
    assert O.linear_corr_plan_rect(917, 917, O.cap_n(2048)) == (1944, 1944, 917, 917)
    assert O.linear_corr_plan_rect(1024, 1024, O.cap_n(2048)) == (2048, 2048, 1024, 1024)
    assert O.linear_corr_plan_rect(256, 256, O.cap_n(1024)) == (512, 512, 256, 256)
    assert O.auto_shift_plan(256, 256) == (512, 512, 256, 256)
    assert O.auto_shift_plan(917, 917) == (512, 512, 230, 230)
    assert O.auto_shift_plan(2000, 300) == (512, 128, 250, 38)
    assert O.largest_smooth(2048) == 2048 and O.largest_smooth(2000) == 1944
    planes, corrs = O.corr_plan(True, True)
    assert len(planes) == 10 and len(corrs) == 28
    planes, corrs = O.corr_plan(False, False)
    assert len(planes) == 5 and len(corrs) == 25


def test_features_three_and_whitening():
    m, f, _ = synth.pair_remap(n=96, seed=5)
    p = O.prepare(f, "three")
    assert np.abs(p["feat"][3]).max() == 0
    p = O.prepare(f, "laplacian")
    x = p["feat"].reshape(4, -1).astype(np.float64)
    cov = np.cov(x, bias=True)
    # the ridge (1e-4·tr/4 of the raw covariance) keeps small variances a little under 1
    np.testing.assert_allclose(cov, np.eye(4), atol=2e-2)
    r = p["rank"]
    assert r.min() > -1 and r.max() < 1


def test_combine_floors_and_failures():
    c = np.zeros((45, 3))
    c[0] = [100.0, 5.0, 100.0]          # n: ok, below MIN_N, ok
    c[25 + 0] = c[35 + 0] = 100.0       # unit variances of plane 0 only → others fail PD? ridge keeps PD
    s = O.combine(c, exact=True, calibrated=False, min_n=12)
    assert s[1] == 0.0
    assert np.all(np.isfinite(s))
