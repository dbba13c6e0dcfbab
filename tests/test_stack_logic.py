"""The stack loop (register_stack) against the reference's own decisions: the same scripted
per-slice results fed to both (tests/golden/make_stack_golden.py ran the reference's
python/zcmir/api.py register_stack on them). Every slice's method, re-detection, pose and score,
the off-trend distances, flags and threshold must match. The reference's from-scratch step is
keypoint registration ("keypoints"); this build's is the sweep search ("search")."""
import json
import math

import numpy as np
import pytest

from zcmir_b200 import api


def load_cases(golden):
    return json.loads((golden / "stack_logic.json").read_text())["cases"]


def run_case(c):
    rows, n = c["rows"], c["n"]
    calls = [0] * n
    slot = {}

    def reg_of(i, t, method):
        h, w = rows[i]["shape"]
        return api.Registration(H=np.array(t["H"]), score=t["score"], model="homography", moving_shape=(h, w),
                                fixed_shape=(h, w), method=method)

    def refine(m, f, H):
        i = slot[id(m)]
        t = rows[i]["carry"] if calls[i] == 0 else rows[i]["polish"]
        calls[i] += 1
        return reg_of(i, t, "refine")

    def detect(m, f):
        i = slot[id(m)]
        return reg_of(i, rows[i]["detect"], "search")

    moving = [np.zeros((2, 2)) + i for i in range(n)]
    for i, m in enumerate(moving):
        slot[id(m)] = i
    fixed = [np.zeros((2, 2)) for _ in range(n)]
    return api.register_stack(moving, fixed, register_pair=refine, detect_pair=detect, **c["kwargs"])


def test_stack_loop_matches_reference_decisions(golden):
    cases = load_cases(golden)
    assert len(cases) == 6
    for c in cases:
        out, ref = run_case(c), c["out"]
        assert len(out) == c["n"]
        for k, (r, g) in enumerate(zip(out.slices, ref["slices"])):
            want = "search" if g["method"] == "keypoints" else g["method"]
            assert (r.method, r.redetected) == (want, g["redetected"]), (c["seed"], k)
            np.testing.assert_allclose(r.H, g["H"], rtol=0, atol=0)
            assert r.score == g["score"]
        for a, b in zip(out.off_trend, ref["off_trend"]):
            assert (a is None) == (b is None) and (a is None or math.isclose(a, b, rel_tol=1e-12, abs_tol=1e-12))
        assert out.flagged == ref["flagged"]
        assert out.threshold == pytest.approx(ref["threshold"], rel=1e-12)
    assert any(s["redetected"] for c in cases for s in c["out"]["slices"])
    assert any(any(c["out"]["flagged"]) for c in cases)


def test_stack_json_and_repr(golden):
    out = run_case(load_cases(golden)[1])
    d = json.loads(out.to_json())
    assert len(d["slices"]) == 12 and "off_trend_px" in d["slices"][1]
    assert "registered" in repr(out) and len(out.H) == 12
