"""The oracle against vectors that the reference's own NumPy code computed (examples/03_smi.py,
executed by tests/golden/make_smi_golden.py on the landsat-b pair with the reference's default
preprocessing). CPU only.

Tolerances: the oracle and 03_smi compute the same float64 sums and score in a different order:
≤ 1e-9 relative. The shift-map window was stored as float32: ≤ 1e-6 of its peak. The gradient:
03_smi takes ∂S/∂sums by central differences (step 1e-6 of each sum), the oracle analytically:
≤ 1e-6 of its norm (they agree to ≈ 1e-8; the reference's own check is 1e-2,
examples/03_smi.py:366). The roto-scale
peak: the reference's bound of 2° (examples/03_smi.py:365), on the oracle's own log-polar plan.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import pose_oracle as PO
from oracle import rs_oracle as R
from oracle import smi_oracle as O

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import make_smi_golden as G  # noqa: E402


@pytest.fixture(scope="module")
def ref(golden):
    return dict(np.load(golden / "smi_03_landsat_b.npz"))


@pytest.fixture(scope="module")
def feats(golden):
    d = np.load(golden / "landsat_b.npz")
    s = G.default_settings()
    return G.features(d["moving"], s), G.features(d["fixed"], s), d["truth"]


def test_moments_and_score_at_the_truth(ref, feats):
    pa, pb, truth = feats
    m = PO.moments(pa["feat"], pb["feat"], truth)
    np.testing.assert_allclose(m, ref["m_np"], rtol=0, atol=1e-9 * np.abs(ref["m_np"]).max())
    s, _ = PO.score_from_moments(ref["m_np"], exact=True)
    assert abs(s - ref["score"]) <= 1e-9 * abs(ref["score"])


def test_score_along_x_shifts(ref, feats):
    pa, pb, truth = feats
    for dx, want in zip(ref["curve_dx"], ref["curve"]):
        H = np.array([[1, 0, dx], [0, 1, 0], [0, 0, 1.0]]) @ truth
        got, _ = PO.score_from_moments(PO.moments(pa["feat"], pb["feat"], H), exact=True)
        assert abs(got - want) <= 1e-9 * abs(want), (dx, got, want)


@pytest.mark.slow
def test_shift_map_window(ref, feats):
    """The oracle's correlations and combine on the planes of 03_smi's map (the moving features
    sampled at H0 with the taper weight, the fixed features with weight 1): the same window of
    lags ±64 and the same peak (14, −9)."""
    pa, pb, _ = feats
    H0 = ref["H0"]
    fb = pb["feat"].astype(np.float64)
    hf, wf = fb.shape[1:]
    S = PO.sample(pa["feat"], H0, wf, hf)
    ga = np.concatenate([S["w"][None], S["w"] * S["va"]])
    gb = np.concatenate([np.ones((1, hf, wf)), fb])
    ids, corrs = O.corr_plan(True, False)
    P, L = 1024, 64
    corr = O.correlations(O.real_planes(ga, ids), O.real_planes(gb, ids), ids, corrs, P, P)
    idx = np.r_[P - L:P, 0:L + 1]
    corr = corr[:, idx][:, :, idx]
    mine = O.combine(corr, exact=True, calibrated=False, min_n=O.MIN_N, area=1.0)
    want = ref["shift_np"].astype(np.float64)
    both = np.isfinite(want) & (mine > 0)
    assert both.sum() > 0.9 * want.size
    peak = np.nanmax(want)
    assert np.abs(mine[both] - want[both]).max() <= 1e-6 * peak
    iy, ix = np.unravel_index(np.argmax(np.where(both, mine, -np.inf)), mine.shape)
    assert (ix - L, iy - L) == tuple(ref["shift_peak"]) == (14, -9)


def test_gradient_near_the_truth(ref, feats):
    pa, pb, _ = feats
    r = PO.pair_eval(pa["feat"], pb["feat"], ref["H2"], exact=True, symmetric=False, homog=True, grad=True)
    g = np.asarray(r["grad"])
    assert np.linalg.norm(g - ref["grad_np"]) <= 1e-6 * np.linalg.norm(ref["grad_np"]), (g, ref["grad_np"])


@pytest.mark.slow
def test_roto_scale_peak(ref, feats):
    """03_smi's log-polar map peaks at 6° and ×1.08 for the truth turned by 6° and scaled by 1.08;
    the oracle's roto-scale map (the engine's plan) puts its peak within the reference's 2° and
    0.02 of scale of that peak."""
    pa, pb, _ = feats
    assert abs(ref["rs_peak"][0] - 6) < 2 and abs(ref["rs_peak"][1] - 1.08) < 0.02
    r = R.rs_map(pa, pb, ref["H1"], c=tuple(ref["rs_center"]), symmetric=False, exact=True, calibrated=False)
    assert abs(-np.rad2deg(r["dth"]) - ref["rs_peak"][0]) < 2, r["dth"]
    assert abs(np.exp(-r["dsg"]) - ref["rs_peak"][1]) < 0.02, r["dsg"]
