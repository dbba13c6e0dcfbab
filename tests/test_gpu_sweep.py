"""GPU parity of the rotation × scale sweep (zcb_sweep, zc_search) against the CPU oracle,
through the C ABI.

Tolerances: per candidate, each of the oracle's lane maxima whose score stands clear of the
others (more than 1e-3 of the candidate's top score apart) is found at the same map index on the
GPU with its score within 1e-4 of the candidate's top score (FP32 FFTs against float64; the map
tests' bound); the top peak's index is exact whenever the oracle's best two lanes stand clear.
The search must land within 5 px of the planted pose at every corner (the reference's own bound,
tests/test_api.py:156-166)."""
import numpy as np
import pytest

import zcmir_b200 as zc
from oracle import smi_oracle as O
from oracle import sweep_oracle as S
from zcmir_b200 import synth

pytestmark = pytest.mark.gpu


def prep_from(feat, mode="laplacian"):
    f = np.asarray(feat, np.float32)
    return {"w": f.shape[2], "h": f.shape[1], "mode": mode, "feat": f,
            "stack": np.concatenate([np.ones((1,) + f.shape[1:], np.float32), f])}


def corner_dist(A, B, w, h):
    d = 0.0
    for x, y in [(1, 1), (w, 1), (w, h), (1, h)]:
        a, b = A @ [x, y, 1.0], B @ [x, y, 1.0]
        d = max(d, float(np.hypot(*(a[:2] / a[2] - b[:2] / b[2]))))
    return d


@pytest.fixture(scope="module")
def small():
    return synth.pair_similarity(n=128, seed=5, deg=40.0, scale=1.1, shift=(6.0, -4.0))


def check_lanes(gs, gi, ref, nc, n_peak, cell, only=None):
    c2 = cell * cell
    clear_top = 0
    for ci in (range(nc) if only is None else sorted(only)):
        top = ref["raw"][ci]
        o_s = np.array([v for v, _ in top]) * c2
        o_i = [t for _, t in top]
        s0 = max(o_s[0], 1e-30)
        if o_s[0] <= 0:
            continue
        for k in range(n_peak):
            if o_s[k] <= 0:
                continue
            gaps = [abs(o_s[k] - o_s[j]) for j in range(n_peak) if j != k and o_s[j] > 0]
            if gaps and min(gaps) <= 1e-3 * s0:
                continue
            hit = np.nonzero(gi[ci] == o_i[k])[0]
            assert hit.size == 1, (ci, k, o_i[k], gi[ci], o_s, gs[ci])
            assert abs(gs[ci, hit[0]] - o_s[k]) <= 1e-4 * s0, (ci, k, gs[ci, hit[0]], o_s[k])
            if k == 0:
                assert hit[0] == 0
                clear_top += 1
    return clear_top


@pytest.mark.parametrize("exact,features", [(True, "laplacian"), (False, "laplacian"), (True, "three")])
def test_sweep_lane_peaks_match_oracle(small, exact, features):
    m, f, H = small
    settings = dict(half=False, exact=exact, smi_features=features, sw_nth=12, sw_ns=3, sw_smin=0.8, sw_smax=1.25,
                    sw_grid=64)
    with zc.Engine(**settings) as reg:
        reg.set_images(m, f, preprocess=False)
        pa, pb = prep_from(reg.features(0), features), prep_from(reg.features(1), features)
        sw = reg.sweep(n_peak=4)
        sw2 = reg.sweep(n_peak=4, batch=5)
    gv = S.sweep_grid(n_theta=12, n_sigma=3, s_min=0.8, s_max=1.25)
    ref = S.sweep(pa, pb, np.eye(3), gv, G=64, exact=exact, three=features == "three", min_overlap=0.05)
    st = ref["setup"]
    nc = len(st["cands"])
    assert int(sw.info["candidates"]) == nc and abs(sw.info["cell"] - st["cell"]) < 1e-12
    assert (sw.info["Fx"], sw.info["Fy"], sw.info["fx0"], sw.info["fy0"]) == (st["Fx"], st["Fy"], st["fcx"][0], st["fcy"][0])
    assert sw.info["min_n"] == ref["min_n"]
    n_clear = check_lanes(sw.scores.astype(np.float64), sw.index, ref, nc, 4, st["cell"])
    assert n_clear >= nc // 2
    # the batch size changes the launch shapes, not the result
    np.testing.assert_array_equal(sw.index, sw2.index)
    np.testing.assert_allclose(sw.scores, sw2.scores, rtol=1e-6, atol=0)


def test_tuned_and_graph_sweeps_equal_the_stream_ordered_sweep(small, monkeypatch):
    """zcb_tune_sweep picks a batch per plane class by timing; the sweep then runs with those
    batches as one replay of a captured CUDA graph. The batch changes the launch shapes, not the
    result, and a replay gives the lanes of a stream-ordered sweep."""
    m, f, _ = small
    settings = dict(half=False, sw_nth=12, sw_ns=3, sw_smin=0.8, sw_smax=1.25, sw_grid=64)
    with zc.Engine(**settings) as eng:
        eng.set_images(m, f, preprocess=False)
        base = eng.sweep(n_peak=4, batch=5)
        rows = eng.tune_sweep()
        assert rows and sum(r["candidates"] for r in rows) == base.info["candidates"]
        for r in rows:
            assert r["batch"] in r["options"] and r["ms_per_map"] == min(r["options"].values())
        tuned = eng.sweep(n_peak=4)
        again = eng.sweep(n_peak=4)
    np.testing.assert_array_equal(tuned.index, base.index)
    np.testing.assert_allclose(tuned.scores, base.scores, rtol=1e-6, atol=0)
    np.testing.assert_array_equal(again.index, tuned.index)
    np.testing.assert_array_equal(again.scores, tuned.scores)
    monkeypatch.setenv("ZCMIR_B200_SWEEP_GRAPH", "0")
    with zc.Engine(**settings) as eng:
        eng.set_images(m, f, preprocess=False)
        plain = eng.sweep(n_peak=4, batch=5)
    np.testing.assert_array_equal(plain.index, base.index)
    np.testing.assert_array_equal(plain.scores, base.scores)


@pytest.mark.slow
def test_sweep_lane_peaks_full_size_sample():
    """The 512² sweep workload: 360 rotations × 9 scales = 3240 candidate maps on the 128-cell
    grid, in plane classes of 192², 256² and 144². Up to 32 candidates of each class, evenly
    spread over the class, are mapped by the float64 oracle (tap positions in float32, as the
    reference computes them); the GPU's full sweep must hold each one's lane maxima as the
    small-grid test requires."""
    m16, f16, _ = synth.pair_similarity(n=512, seed=2)
    m, f = zc.gray32(m16), zc.gray32(f16)
    settings = dict(half=False, sw_nth=360, sw_ns=9, sw_smin=0.8, sw_smax=1.25, sw_grid=128)
    with zc.Engine(**settings) as eng:
        eng.set_images(m, f, preprocess=False)
        pa, pb = prep_from(eng.features(0)), prep_from(eng.features(1))
        sw = eng.sweep(n_peak=4, batch=128)
    gv = S.sweep_grid(n_theta=360, n_sigma=9, s_min=0.8, s_max=1.25)
    st = S.sweep_setup(512, 512, 512, 512, np.eye(3), gv, 128)
    classes = {}
    for ci, c in enumerate(st["cands"]):
        classes.setdefault((c["nx"], c["ny"]), []).append(ci)
    assert sorted(classes) == [(144, 144), (192, 192), (256, 256)], sorted(classes)
    only = set()
    for members in classes.values():
        only.update(members[int(i)] for i in np.linspace(0, len(members) - 1, min(32, len(members))))
    # taps placed in float32 as the reference's shader places them: at this size a few taps sit
    # within 1e-4 px of the image edge, where the rounding decides whether their whole sample
    # counts (with float64 positions one candidate's top score moves by 3e-4)
    ref = S.sweep(pa, pb, np.eye(3), gv, G=128, exact=True, only=only, f32_positions=True)
    nc = len(st["cands"])
    assert int(sw.info["candidates"]) == nc == 3240 and sw.info["min_n"] == ref["min_n"]
    n_clear = check_lanes(sw.scores.astype(np.float64), sw.index, ref, nc, 4, st["cell"], only)
    assert n_clear >= len(only) // 2, (n_clear, len(only))


@pytest.mark.parametrize("seed,near_truth", [(7, True), (11, True), (3, False)])
def test_search_recovers_a_similarity(seed, near_truth):
    """From the identity over the full circle and scales 0.5–2 (the default grid: 1800 maps).
    The search must score at least as well as a climb started at the planted pose; where that
    climb stays at the planted pose, the search lands within 5 px of it. (Seed 3 is a pair whose
    SMI optimum lies a few px off the planted pose: the climb from the truth leaves it.)"""
    m, f, H = synth.pair_similarity(n=256, seed=seed)
    with zc.Engine(half=False) as reg:
        reg.set_images(m, f, preprocess=False)
        s0 = reg.score(np.eye(3)).mean
        r = reg.search()
        assert r.improved and r.count_a > 0 and r.count_b > 0
        assert r.prev == pytest.approx(s0)
        np.testing.assert_allclose(reg.pose, r.H)
        ev = reg.events()
        assert any("search done" in e.get("text", "") for e in ev)
        reg.pose = H
        reg.climb()
        s_truth = reg.score(reg.pose).mean
        assert r.score >= s_truth * (1 - 1e-4), (r.score, s_truth)
        if near_truth:
            assert corner_dist(reg.pose, H, 256, 256) < 1
            assert corner_dist(r.H, H, 256, 256) < 5, corner_dist(r.H, H, 256, 256)


def test_search_refusals():
    m, f, _ = synth.pair_similarity(n=128, seed=5, deg=10.0, scale=1.0, shift=(0.0, 0.0))
    with zc.Engine(half=False, search_mode="cloud") as reg:
        reg.set_images(m, f, preprocess=False)
        with pytest.raises(RuntimeError, match="cloud"):
            reg.search()
        reg.configure(search_mode="sweep", metric="ncc")
        with pytest.raises(RuntimeError, match="ncc"):
            reg.search()


def test_sweep_shards_merge_to_the_whole_sweep(small):
    """Three shards of one sweep (zcb_sweep shard/nshard), merged as the ranks of a split sweep
    merge them (sum of scores, minimum of indices), give the whole sweep; the search finished
    from the merged lanes (zcb_search_lanes) reaches the same pose as search()."""
    m, f, H = small
    with zc.Engine(half=False, sw_nth=12, sw_ns=3, sw_smin=0.8, sw_smax=1.25, sw_grid=64) as reg:
        reg.set_images(m, f, preprocess=False)
        whole = reg.sweep(n_peak=4)
        parts = [reg.sweep(n_peak=4, shard=r, nshard=3) for r in range(3)]
        owned = [(p.index != 0xFFFFFFFF).any(axis=1) for p in parts]
        assert sum(o.astype(int) for o in owned).max() <= 1
        sc = np.sum([p.scores for p in parts], axis=0)
        ix = np.minimum.reduce([p.index for p in parts])
        np.testing.assert_array_equal(ix, whole.index)
        np.testing.assert_allclose(sc, whole.scores, rtol=1e-6, atol=0)
        reg.pose = np.eye(3)
        r1 = reg.search()
        reg.pose = np.eye(3)
        r2 = reg.search_lanes(sc, ix)
        assert r2.count_a == r1.count_a and r2.improved == r1.improved
        assert corner_dist(r2.H, r1.H, 128, 128) < 0.05
        with pytest.raises(RuntimeError, match="lane entries"):
            reg.search_lanes(sc[:-1], ix[:-1])
