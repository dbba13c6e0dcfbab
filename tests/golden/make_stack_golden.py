"""Golden decisions of the reference's stack loop (python/zcmir/api.py:522-580).

Runs the reference's own register_stack, imported from its source tree, with its per-pair
`register` replaced by a scripted one: per slice, a table of what the refine from a pose returns
(first call: the carry; second: the polish) and what the from-scratch registration returns. The
scenarios, the reference's outputs (each slice's method, redetected flag, pose and score, the
off-trend distances, the flags and the threshold) go to stack_logic.json. Run in a checkout where
the reference's source is at ../reference or REFERENCE_ROOT:

    REFERENCE_ROOT=/path/to/zcmir python tests/golden/make_stack_golden.py
"""
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def scenario(seed, n):
    rng = np.random.default_rng(seed)
    shapes = [(int(rng.integers(200, 400)), int(rng.integers(200, 400))) for _ in range(n)]
    drift = np.cumsum(rng.normal(0, 3, (n, 2)), axis=0)
    rows = []
    for i in range(n):
        base = np.array([[1, 0, drift[i, 0]], [0, 1, drift[i, 1]], [0, 0, 1.0]])
        carry_H = base.copy()
        score = float(1000 + rng.normal(0, 20))
        carry_score = score
        kind = rng.choice(["ok", "ok", "ok", "drop", "jump", "jump_small"])
        if kind == "drop":
            carry_score = score * float(rng.uniform(0.5, 0.8))
        if kind == "jump":
            carry_H[:2, 2] += rng.normal(0, 40, 2)
        if kind == "jump_small":
            carry_H[:2, 2] += rng.normal(0, 6, 2)
        det_H = base.copy()
        det_H[:2, 2] += rng.normal(0, 0.5, 2)
        det_score = score * float(rng.uniform(0.9, 1.1))
        pol_H = base.copy()
        pol_H[:2, 2] += rng.normal(0, 0.3, 2)
        pol_score = max(carry_score, det_score) * float(rng.uniform(0.99, 1.01))
        rows.append({"shape": shapes[i], "kind": str(kind),
                     "carry": {"H": carry_H.tolist(), "score": carry_score},
                     "detect": {"H": det_H.tolist(), "score": det_score},
                     "polish": {"H": pol_H.tolist(), "score": pol_score}})
    return rows


def main():
    ref = Path(os.environ.get("REFERENCE_ROOT", HERE.parents[2] / "reference"))
    sys.path.insert(0, str(ref / "python"))
    import zcmir.api as A

    cases = []
    for seed, n, kw in [(1, 12, {}), (2, 12, {"polish": True}), (3, 16, {"jump": 5.0}), (4, 10, {"drop": 0.3}),
                        (5, 12, {"start": "keypoints"}), (6, 20, {"polish": True, "jump": 8.0})]:
        rows = scenario(seed, n)
        calls = [0] * n
        slot = {}

        def fake_register(m, f, init=None, **k):
            i = slot[id(m)]
            if init is None:
                t = rows[i]["detect"]
            else:
                t = rows[i]["carry"] if calls[i] == 0 else rows[i]["polish"]
                calls[i] += 1
            h, w = rows[i]["shape"]
            return A.Registration(H=np.array(t["H"]), score=t["score"], model="homography", moving_shape=(h, w),
                                  fixed_shape=(h, w))

        moving = [np.zeros((2, 2)) + i for i in range(n)]
        for i, m in enumerate(moving):
            slot[id(m)] = i
        fixed = [np.zeros((2, 2)) for _ in range(n)]
        saved = A.register
        A.register = fake_register
        try:
            out = A.register_stack(moving, fixed, **kw)
        finally:
            A.register = saved
        cases.append({
            "seed": seed, "n": n, "kwargs": kw, "rows": rows,
            "out": {"slices": [{"H": np.asarray(r.H).tolist(), "score": r.score, "method": r.method,
                                "redetected": bool(r.redetected)} for r in out.slices],
                    "off_trend": out.off_trend, "flagged": [bool(x) for x in out.flagged],
                    "threshold": out.threshold},
        })
    (HERE / "stack_logic.json").write_text(json.dumps({"source": "python/zcmir/api.py:430-580 register_stack",
                                                       "cases": cases}, indent=1))
    print("wrote", len(cases), "cases")


if __name__ == "__main__":
    main()
