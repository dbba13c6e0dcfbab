"""The oracle against the reference's own known answers (examples/03_smi.py:362-366) and against
itself (FFT correlations vs direct float64 sums). CPU only."""
import numpy as np
import pytest

from oracle import smi_oracle as O
from zcmir_b200 import synth

TRI = O.TRI


@pytest.fixture(scope="module")
def landsat(golden):
    d = np.load(golden / "landsat_b.npz")
    pa = O.prepare(d["moving"].astype(np.float32) / 255, "laplacian")
    pb = O.prepare(d["fixed"].astype(np.float32) / 255, "laplacian")
    return pa, pb, d["truth"]


def _smi_03(s, hf, wf, hm, wm, ridge=1e-4):
    """The SMI of the sums as examples/03_smi.py:124-147 writes it (its own overlap floor)."""
    s = np.asarray(s, np.float64)
    n = s[0]
    ok = n > 0.05 * min(hf * wf, hm * wm)
    n = np.where(ok, n, 1.0)
    ma, mb = s[1:5] / n, s[5:9] / n
    C = s[9:25].reshape((4, 4) + n.shape) / n - ma[:, None] * mb[None]
    Ga, Gb = np.zeros((4, 4) + n.shape), np.zeros((4, 4) + n.shape)
    for k, (i, j) in enumerate(TRI):
        Ga[i, j] = Ga[j, i] = s[25 + k] / n - ma[i] * ma[j]
        Gb[i, j] = Gb[j, i] = s[35 + k] / n - mb[i] * mb[j]
    for G in (Ga, Gb):
        tr = np.trace(G) / 4
        for i in range(4):
            G[i, i] += ridge * tr
    Ga, Gb, C = (np.moveaxis(x, (0, 1), (-2, -1)) for x in (Ga, Gb, C))
    W = np.linalg.solve(Ga, C) @ np.linalg.inv(Gb)
    return np.where(ok, n * np.sum(W * C, axis=(-2, -1)), np.nan)


def _sample_03(A, H, hf, wf):
    """Moving features at every fixed pixel under H with the 2-px taper (examples/03_smi.py:56-80)."""
    hm, wm = A.shape[1:]
    y, x = np.mgrid[0:hf, 0:wf].astype(np.float64)
    ph = np.tensordot(np.linalg.inv(H), np.stack([x + 1, y + 1, np.ones_like(x)]), 1)
    fx, fy = ph[0] / ph[2] - 1, ph[1] / ph[2] - 1
    ok = (fx >= 2) & (fy >= 2) & (fx <= wm - 3) & (fy <= hm - 3)
    ramp = lambda v, lo, hi: np.clip((v - lo) / 2, 0, 1) * np.clip((hi - v) / 2, 0, 1)
    x0 = np.clip(np.floor(fx).astype(int), 0, wm - 2)
    y0 = np.clip(np.floor(fy).astype(int), 0, hm - 2)
    ax, ay = fx - x0, fy - y0
    v00, v10, v01, v11 = A[:, y0, x0], A[:, y0, x0 + 1], A[:, y0 + 1, x0], A[:, y0 + 1, x0 + 1]
    va = (v00 * (1 - ax) + v10 * ax) * (1 - ay) + (v01 * (1 - ax) + v11 * ax) * ay
    return va, np.where(ok, ramp(fx, 2, wm - 3) * ramp(fy, 2, hm - 3), 0.0)


def test_known_answer_03_smi_shift_peak(landsat):
    """examples/03_smi.py:364: the NumPy FFT shift map at H0 = T(14, −9)·truth peaks exactly at
    (14, −9); here on the oracle's features, and the oracle's combine equals 03_smi's smi()."""
    pa, pb, truth = landsat
    A, B = pa["feat"].astype(np.float64), pb["feat"].astype(np.float64)
    hm, wm = A.shape[1:]
    hf, wf = B.shape[1:]
    H0 = np.array([[1, 0, 14], [0, 1, -9], [0, 0, 1.0]]) @ truth
    va, w = _sample_03(A, H0, hf, wf)
    planes_a = [w] + [w * va[i] for i in range(4)] + [w * va[i] * va[j] for i, j in TRI]
    planes_b = [np.ones((hf, wf))] + [B[j] for j in range(4)] + [B[i] * B[j] for i, j in TRI]
    pairs = [(0, 0)] + [(1 + i, 0) for i in range(4)] + [(0, 1 + j) for j in range(4)]
    pairs += [(1 + i, 1 + j) for i in range(4) for j in range(4)]
    pairs += [(5 + k, 0) for k in range(10)] + [(0, 5 + k) for k in range(10)]
    P, L = 1024, 64
    FA = [np.fft.rfft2(a, (P, P)) for a in planes_a]
    FB = [np.fft.rfft2(b, (P, P)) for b in planes_b]
    sums = np.stack([np.fft.irfft2(FA[a] * np.conj(FB[b]), (P, P)) for a, b in pairs])
    idx = np.r_[P - L:P, 0:L + 1]
    sums = sums[:, idx][:, :, idx]
    ref = _smi_03(sums, hf, wf, hm, wm)
    iy, ix = np.unravel_index(np.nanargmax(ref), ref.shape)
    assert (ix - L, iy - L) == (14, -9)
    mine = O.combine(sums, exact=True, calibrated=False, min_n=12, area=1.0)
    both = np.isfinite(ref) & (mine > 0)
    assert both.sum() > 1000
    np.testing.assert_allclose(mine[both], ref[both], rtol=1e-10)


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
