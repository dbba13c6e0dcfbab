"""GPU parity of the pose path (zc_moments, zc_score, zc_gradient) against the CPU oracle, and the
Gauss–Newton refine (zc_climb), through the C ABI.

Tolerances: moment sums within 1e-5 of the largest (float32 per-pixel sums, float64 across
blocks; examples/03_smi.py:362 allows 1e-4), scores within 1e-5 relative (03_smi: 1e-4),
gradients within 1e-3 in norm and the Gauss–Newton matrix within 1e-3 of its largest entry
(03_smi: 1e-2)."""
import numpy as np
import pytest

import zcmir_b200 as zc
from oracle import pose_oracle as P
from oracle import smi_oracle as O
from zcmir_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pair():
    m, f, H = synth.pair_remap(n=256, shift=(17, -9), seed=0)
    return m, f, H


def _near(H, th=3.0, s=1.02, t=(1.5, -1.0)):
    c = 128.5
    a = np.deg2rad(th)
    R = np.array([[s * np.cos(a), -s * np.sin(a), 0], [s * np.sin(a), s * np.cos(a), 0], [0, 0, 1]])
    T = lambda x, y: np.array([[1, 0, x], [0, 1, y], [0, 0, 1.0]])
    return T(c + t[0], c + t[1]) @ R @ T(-c, -c) @ H


def corner_dist(A, B, w, h):
    d = 0.0
    for x, y in [(1, 1), (w, 1), (w, h), (1, h)]:
        a, b = A @ [x, y, 1.0], B @ [x, y, 1.0]
        d = max(d, float(np.hypot(*(a[:2] / a[2] - b[:2] / b[2]))))
    return d


@pytest.mark.parametrize("group", ["homography", "affine"])
def test_moments_score_gradient_match_oracle(pair, group):
    m, f, H = pair
    Hp = _near(H)
    homog = group == "homography"
    with zc.Engine(half=False, group=group) as reg:
        reg.set_images(m, f, preprocess=False)
        A, B = reg.features(0), reg.features(1)
        mom = reg.moments(Hp)
        sc = reg.score(Hp)
        g = reg.gradient(Hp, hess=True)
    ref = P.pair_eval(A, B, Hp, homog=homog, grad=True, hess=True)
    np.testing.assert_allclose(mom, ref["sums"], rtol=0, atol=1e-5 * np.abs(ref["sums"]).max())
    assert abs(sc.fwd - ref["fwd"]) <= 1e-5 * abs(ref["fwd"])
    assert abs(sc.inv - ref["inv"]) <= 1e-5 * abs(ref["inv"])
    assert abs(sc.mean - ref["mean"]) <= 1e-5 * abs(ref["mean"])
    nk = 8 if homog else 6
    assert g.grad.shape == (nk,) and g.hess.shape == (nk, nk)
    assert abs(g.score - ref["mean"]) <= 1e-5 * abs(ref["mean"])
    assert np.linalg.norm(g.grad - ref["grad"]) <= 1e-3 * np.linalg.norm(ref["grad"])
    assert np.abs(g.hess - ref["hess"]).max() <= 1e-3 * np.abs(ref["hess"]).max()


def test_ragged_images_match_oracle(pair):
    """Image sides that are not multiples of the pose kernels' 8 × 4 pixel tiles (the last tile of
    each tile row and the last tile row reach past the image): sums, scores and gradient as the
    oracle has them."""
    m, f, H = pair
    m2, f2 = np.ascontiguousarray(m[3:160, 5:208]), np.ascontiguousarray(f[:139, 2:183])
    Hp = _near(H)
    with zc.Engine(half=False, group="affine") as reg:
        reg.set_images(m2, f2, preprocess=False)
        A, B = reg.features(0), reg.features(1)
        mom = reg.moments(Hp)
        sc = reg.score(Hp)
        g = reg.gradient(Hp, hess=True)
    ref = P.pair_eval(A, B, Hp, homog=False, grad=True, hess=True)
    assert ref["sums"][0] > 1000
    np.testing.assert_allclose(mom, ref["sums"], rtol=0, atol=1e-5 * np.abs(ref["sums"]).max())
    assert abs(sc.mean - ref["mean"]) <= 1e-5 * abs(ref["mean"])
    assert np.linalg.norm(g.grad - ref["grad"]) <= 1e-3 * np.linalg.norm(ref["grad"])
    assert np.abs(g.hess - ref["hess"]).max() <= 1e-3 * np.abs(ref["hess"]).max()


def test_forward_only_and_edge_cases(pair):
    m, f, H = pair
    with zc.Engine(half=False, symmetric=False) as reg:
        reg.set_images(m, f, preprocess=False)
        A, B = reg.features(0), reg.features(1)
        s = reg.score(H)
        assert s.inv is None
        ref = P.pair_eval(A, B, H, symmetric=False)
        assert abs(s.fwd - ref["fwd"]) <= 1e-5 * abs(ref["fwd"])
        # a pose with no overlap scores 0 (n < 12) and has a zero gradient
        far = np.array([[1, 0, 5000.0], [0, 1, 5000.0], [0, 0, 1]])
        s = reg.score(far)
        g = reg.gradient(far, hess=True)
        assert s.fwd == 0.0 and g.n == 0.0 and not np.any(g.grad)


def test_climb_recovers_pose_and_gn_step_is_small(golden):
    """Refine from a perturbed pose reaches the known pose of the landsat-b pair (the reference's
    refine check: < 1 px at the corners, tests/test_api.py:127-135), and at the result the
    Gauss–Newton step is small (tests/test_api.py:218-221: < 5e-3)."""
    d = np.load(golden / "landsat_b.npz")
    m, f, H = d["moving"].astype(np.float32) / 255, d["fixed"].astype(np.float32) / 255, d["truth"]
    c0 = np.array([320.5, 320.5])
    a, s = np.deg2rad(1.0), 1.01
    R = np.array([[s * np.cos(a), -s * np.sin(a), 0], [s * np.sin(a), s * np.cos(a), 0], [0, 0, 1]])
    T = lambda x, y: np.array([[1, 0, x], [0, 1, y], [0, 0, 1.0]])
    start = T(*(c0 + [2.0, -1.5])) @ R @ T(*-c0) @ H
    mh, mw = m.shape
    assert corner_dist(start, H, mw, mh) > 5
    for group in ("homography", "affine"):
        with zc.Engine(half=False, group=group) as reg:
            reg.set_images(m, f, preprocess=False)
            reg.pose = start
            c = reg.climb()
            assert c.moved and c.iterations >= 1
            assert corner_dist(c.H, H, mw, mh) < 1.0, (group, corner_dist(c.H, H, mw, mh))
            assert c.score > reg.score(start).mean
            np.testing.assert_allclose(reg.pose, c.H)
            g = reg.gradient(hess=True)
            step = np.linalg.solve(g.hess + 1e-4 * np.diag(np.maximum(np.diag(g.hess), 1e-12)), 0.5 * g.grad)
            assert np.linalg.norm(step) < 5e-3, np.linalg.norm(step)
            kinds = {e["kind"] for e in reg.events()}
            assert {"log", "trail", "pose"} <= kinds


def test_climb_ascends_to_a_stationary_point(pair):
    """On the 256² shifted pair the homography climb ends where the score is higher than at the
    start and the Gauss–Newton step vanishes (the score's optimum there is not the planted
    shift: perspective terms trade overlap on this small pair)."""
    m, f, H = pair
    start = _near(H, th=2.0, s=1.015, t=(2.0, -1.5))
    with zc.Engine(half=False) as reg:
        reg.set_images(m, f, preprocess=False)
        s0 = reg.score(start).mean
        reg.pose = start
        c = reg.climb()
        assert c.moved and c.score > s0
        g = reg.gradient(hess=True)
        step = np.linalg.solve(g.hess + 1e-4 * np.diag(np.maximum(np.diag(g.hess), 1e-12)), 0.5 * g.grad)
        assert np.linalg.norm(step) < 5e-3
        # the climb's final score is the pair score at its pose
        assert abs(reg.score(c.H).mean - c.score) <= 1e-9 * abs(c.score)


def test_climb_roto_scale_hop(golden):
    """The roto-scale hop (hop_fm, src/gclimb.zig:417-435): from the landsat-b truth turned by 8°
    and scaled by 1.1 about the moving image's centroid, the climb takes the roto-scale map's
    peak as a step of the pose and ends within 1 px of the truth at the corners."""
    d = np.load(golden / "landsat_b.npz")
    m, f, H = d["moving"].astype(np.float32) / 255, d["fixed"].astype(np.float32) / 255, d["truth"]
    mh, mw = m.shape
    c = np.mean([(H @ [x, y, 1.0])[:2] for x, y in [(1, 1), (mw, 1), (mw, mh), (1, mh)]], axis=0)
    a, s = np.deg2rad(8.0), 1.1
    R = np.array([[s * np.cos(a), -s * np.sin(a), 0], [s * np.sin(a), s * np.cos(a), 0], [0, 0, 1]])
    T = lambda x, y: np.array([[1, 0, x], [0, 1, y], [0, 0, 1.0]])
    start = T(*c) @ R @ T(*-c) @ H
    assert corner_dist(start, H, mw, mh) > 30
    with zc.Engine(half=False, group="affine", hop_fm=True) as reg:
        reg.set_images(m, f, preprocess=False)
        reg.pose = start
        r = reg.climb()
        ev = reg.events()
    labels = [e.get("label") for e in ev if e["kind"] == "trail"]
    logs = [e.get("text", "") for e in ev if e["kind"] == "log"]
    assert "roto-scale hop" in labels, labels
    assert any("roto-scale hop+" in t for t in logs), logs
    assert corner_dist(r.H, H, mw, mh) < 1.0, corner_dist(r.H, H, mw, mh)


def test_tune_parts_changes_the_launch_shape_not_the_scores():
    """zc_tune_parts (the reference's knobs of its per-pixel sum kernels, src/exports.zig:115-121)
    sets the pose kernels' pixels per thread and blocks per pose: the sums are added in another
    order, so the scores agree within the pose tests' 1e-5; the defaults are put back after."""
    from zcmir_b200 import _native

    m, f, H = synth.pair_similarity(n=256, seed=7)
    lib = _native.load()
    with zc.Engine(half=False) as eng:
        eng.set_images(m, f, preprocess=False)
        ref = eng.score(H)
        try:
            for knobs in ((64, 0, 0, 0), (4, 0, 0, 0), (16, 600, 0, 0), (16, 1, 0, 8)):
                lib.zc_tune_parts(*knobs)
                s = eng.score(H)
                assert abs(s.mean - ref.mean) <= 1e-5 * abs(ref.mean), (knobs, s, ref)
        finally:
            lib.zc_tune_parts(16, 1, 0, 4096)
        assert abs(eng.score(H).mean - ref.mean) <= 1e-9 * abs(ref.mean)


def test_device_refine_equals_the_host_loop(monkeypatch):
    """The batched Gauss–Newton refine (zcb_refine_poses, and the search's screening and final
    refines) runs on the device by default; ZCMIR_B200_GN=host runs the same loop on the host.
    The device kernels restate the host's float64 pose algebra without fused multiply-adds, and
    the pose kernels add their blocks' totals in block order, so both take the same steps: the
    poses and scores are equal bit for bit."""
    m, f, H = synth.pair_similarity(n=256, seed=7)
    rng = np.random.default_rng(3)
    starts = [_near(H, th=rng.uniform(-4, 4), s=rng.uniform(0.97, 1.03), t=rng.uniform(-3, 3, 2)) for _ in range(8)]

    def run():
        with zc.Engine(half=False, sw_nth=72, sw_ns=3) as eng:
            eng.set_images(m, f, preprocess=False)
            poses, scores = eng.refine_poses(starts, iters=12)
            s = eng.search()
        return poses, scores, s

    dp, ds, dsr = run()
    monkeypatch.setenv("ZCMIR_B200_GN", "host")
    hp, hs, hsr = run()
    np.testing.assert_array_equal(ds, hs)
    np.testing.assert_array_equal(dp, hp)
    np.testing.assert_array_equal(dsr.H, hsr.H)
    assert dsr.score == hsr.score
    # every start climbed: no score below its start's
    with zc.Engine(half=False) as eng:
        eng.set_images(m, f, preprocess=False)
        s0 = np.array([eng.score(h).mean for h in starts])
    assert np.all(ds >= s0 - 1e-9 * np.abs(s0)), (ds, s0)


@pytest.mark.parametrize("symmetric", [True, False])
def test_pose_sums_are_the_same_in_any_batch(symmetric):
    """A pose's moment and tangent sums are added across its blocks in block order, not by
    atomics: one step of the refine from a pose gives the same pose and score bit for bit whether
    the pose is refined alone, first in a batch of 12 or last in it, and the moments of a pose
    are the same on every call."""
    m, f, H = synth.pair_similarity(n=256, seed=7)
    rng = np.random.default_rng(11)
    starts = [_near(H, th=rng.uniform(-4, 4), s=rng.uniform(0.97, 1.03), t=rng.uniform(-3, 3, 2)) for _ in range(12)]
    with zc.Engine(half=False, symmetric=symmetric) as eng:
        eng.set_images(m, f, preprocess=False)
        alone = [eng.refine_poses([h], iters=1) for h in (starts[0], starts[-1])]
        p, s = eng.refine_poses(starts, iters=1)
        pr, sr = eng.refine_poses(starts[::-1], iters=1)
        mom = [eng.moments(starts[3]) for _ in range(3)]
    np.testing.assert_array_equal(alone[0][0][0], p[0])
    assert alone[0][1][0] == s[0]
    np.testing.assert_array_equal(alone[1][0][0], p[-1])
    assert alone[1][1][0] == s[-1]
    np.testing.assert_array_equal(pr[::-1], p)
    np.testing.assert_array_equal(sr[::-1], s)
    np.testing.assert_array_equal(mom[0], mom[1])
    np.testing.assert_array_equal(mom[0], mom[2])
