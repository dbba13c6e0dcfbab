"""GPU parity of the B-spline on top of the pose (settings ffd, ffd_grid, ffd_source; zc_set_ffd,
zc_get_ffd, zc_ffd_gradient) against the CPU oracle, through the C ABI.

Tolerances as for the spline-free pose path: scores within 1e-5 relative, the tangent gradient
within 1e-3 in norm and the Gauss–Newton matrix within 1e-3 of its largest entry. The gradient
over the control points: most entries within 1e-6 of the largest (median), and within 5e-3 in
norm: each control point sums only its own support, where one pixel whose sample lies within
float32 rounding of the taper's inner end (the taper is 0 there but its slope is not, so the
pixel's boundary term jumps in or out) moves an entry by ~1e-3 of the norm."""
import numpy as np
import pytest

import zcmir_b200 as zc
from oracle import pose_oracle as P
from zcmir_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pair():
    m, f, H = synth.pair_remap(n=200, shift=(9, -6), seed=1)
    return m, f[:180, :190], H


def _close(got, ref):
    d = np.abs(got - ref)
    assert np.median(d) <= 1e-6 * np.abs(ref).max(), (np.median(d), np.abs(ref).max())
    assert np.linalg.norm(d) <= 5e-3 * np.linalg.norm(ref), (np.linalg.norm(d), np.linalg.norm(ref))


def _cps(g, seed, amp=0.01):
    return (amp * np.random.default_rng(seed).standard_normal(2 * g * g)).astype(np.float32)


@pytest.mark.parametrize("source,g", [(False, 4), (True, 5)])
def test_scores_and_pose_gradient_with_a_live_spline(pair, source, g):
    m, f, H = pair
    cps = _cps(g, 7 + g)
    with zc.Engine(half=False, ffd=True, ffd_grid=g, ffd_source=source) as reg:
        reg.set_images(m, f, preprocess=False)
        A, B = reg.features(0), reg.features(1)
        reg.ffd = cps
        np.testing.assert_array_equal(reg.ffd, cps)
        sc = reg.score(H)
        gr = reg.gradient(H, hess=True)
        mom = reg.moments(H)
    ffd = dict(g=g, cps=cps.astype(np.float64), source=source)
    ref = P.pair_eval(A, B, H, grad=True, hess=True, ffd=ffd)
    assert abs(sc.fwd - ref["fwd"]) <= 1e-5 * abs(ref["fwd"])
    assert abs(sc.inv - ref["inv"]) <= 1e-5 * abs(ref["inv"])
    np.testing.assert_allclose(mom, ref["sums"], rtol=0, atol=1e-5 * np.abs(ref["sums"]).max())
    assert np.linalg.norm(gr.grad - ref["grad"]) <= 1e-3 * np.linalg.norm(ref["grad"])
    assert np.abs(gr.hess - ref["hess"]).max() <= 1e-3 * np.abs(ref["hess"]).max()
    # the spline moves the score: the same pose without it scores differently
    plain = P.pair_eval(A, B, H)
    assert abs(plain["mean"] - ref["mean"]) > 1e-4 * abs(ref["mean"])


@pytest.mark.parametrize("source,symmetric", [(False, True), (True, True), (False, False)])
def test_control_point_gradient_matches_oracle(pair, source, symmetric):
    m, f, H = pair
    g = 4
    cps = _cps(g, 3)
    with zc.Engine(half=False, ffd=True, ffd_grid=g, ffd_source=source, symmetric=symmetric) as reg:
        reg.set_images(m, f, preprocess=False)
        A, B = reg.features(0), reg.features(1)
        reg.ffd = cps
        s, gr = reg.ffd_gradient(H)
    ref_s, ref_g = P.pair_ffd_grad(A, B, H, dict(g=g, cps=cps.astype(np.float64), source=source), symmetric=symmetric)
    assert gr.shape == (2 * g * g,)
    assert abs(s - ref_s) <= 1e-5 * abs(ref_s)
    _close(gr, ref_g)


def test_lattices_past_one_chunk_and_spline_rules(pair):
    """A 7 × 7 lattice (98 parameters, four 16-point chunks) matches the oracle; the zero spline
    is not live (scores equal the spline-free ones) but still has a gradient, forward only
    (src/pair.zig:387-398); the spline off gives score 0 and a zero gradient; a wrong number of
    control points is refused; a new lattice size zeroes them; the no-alloc scores refuse a live
    spline."""
    m, f, H = pair
    with zc.Engine(half=False, ffd=True, ffd_grid=7) as reg:
        reg.set_images(m, f, preprocess=False)
        A, B = reg.features(0), reg.features(1)
        assert reg.ffd.shape == (98,) and not reg.ffd.any()
        s0 = reg.score(H)
        ref0 = P.pair_eval(A, B, H)
        assert abs(s0.mean - ref0["mean"]) <= 1e-5 * abs(ref0["mean"])
        sz, gz = reg.ffd_gradient(H)
        rs, rg = P.pair_ffd_grad(A, B, H, dict(g=7, cps=np.zeros(98), source=False))
        assert abs(sz - ref0["fwd"]) <= 1e-5 * abs(ref0["fwd"]) and abs(sz - rs) <= 1e-5 * abs(rs)
        _close(gz, rg)
        cps = _cps(7, 11, 0.006)
        reg.ffd = cps
        s7, g7 = reg.ffd_gradient(H)
        r7s, r7g = P.pair_ffd_grad(A, B, H, dict(g=7, cps=cps.astype(np.float64), source=False))
        assert abs(s7 - r7s) <= 1e-5 * abs(r7s)
        _close(g7, r7g)
        with pytest.raises(RuntimeError, match="BadControlPoints"):
            reg.ffd = np.zeros(10, np.float32)
        with pytest.raises(RuntimeError, match="spline is live"):
            reg.score_static([H])
        reg.configure(ffd_grid=5)
        assert reg.ffd.shape == (50,) and not reg.ffd.any()
        reg.configure(ffd=False)
        s, gv = reg.ffd_gradient(H)
        assert s == 0.0 and gv.shape == (50,) and not gv.any()


@pytest.mark.parametrize("source", [False, True])
def test_displacement_field_with_the_spline(pair, source):
    """zc_displacement (src/export.zig:64-106): the composed warp H then the spline over the fixed
    image against the oracle's displacement, and H alone with the spline off."""
    m, f, H = pair
    g = 5
    cps = _cps(g, 21, 0.02)
    with zc.Engine(half=False, ffd=True, ffd_grid=g, ffd_source=source) as reg:
        reg.set_images(m, f, preprocess=False)
        reg.pose = H
        reg.ffd = cps
        d = reg.displacement()
        reg.configure(ffd=False)
        d0 = reg.displacement()
    fh, fw = f.shape
    mh, mw = m.shape
    y, x = np.mgrid[0:fh, 0:fw].astype(np.float64)
    Hi = np.linalg.inv(H)
    ffd = dict(g=g, cps=cps.astype(np.float64), source=source)
    if source:
        q = np.tensordot(Hi, np.stack([x + 1, y + 1, np.ones_like(x)]), 1)
        sx, sy = q[0] / q[2] - 1, q[1] / q[2] - 1
        dd = P.ffd_disp(sx, sy, mw, mh, ffd)
        px, py = sx + dd[0], sy + dd[1]
    else:
        dd = P.ffd_disp(x, y, fw, fh, ffd)
        q = np.tensordot(Hi, np.stack([x + 1 + dd[0], y + 1 + dd[1], np.ones_like(x)]), 1)
        px, py = q[0] / q[2] - 1, q[1] / q[2] - 1
    np.testing.assert_allclose(d[..., 0], px - x, atol=1e-4)
    np.testing.assert_allclose(d[..., 1], py - y, atol=1e-4)
    q = np.tensordot(Hi, np.stack([x + 1, y + 1, np.ones_like(x)]), 1)
    np.testing.assert_allclose(d0[..., 0], q[0] / q[2] - 1 - x, atol=1e-4)


def test_search_runs_without_the_spline_and_resets_it():
    """The sweep search scores the current pose with the live spline, climbs its peaks without it
    and, when it moves the pose, zeroes the control points (src/search.zig:703-705, 806-815)."""
    m, f, _ = synth.pair_similarity(n=160, seed=5, deg=25.0, scale=1.05, shift=(4.0, -3.0))
    with zc.Engine(half=False, ffd=True, ffd_grid=4, sw_nth=72, sw_ns=3) as reg:
        reg.set_images(m, f, preprocess=False)
        reg.ffd = _cps(4, 2, 0.01)
        r = reg.search()
        logs = [e.get("text", "") for e in reg.events() if e["kind"] == "log"]
        assert r.improved
        assert not reg.ffd.any()
        assert any("spline reset" in t for t in logs), logs
