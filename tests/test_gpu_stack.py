"""GPU checks of the stack path: zcb_stack_maps (every slice's features once, one map per
consecutive pair) against one zc_shift_map per pair and the oracle. (register_stack end to end, the
reference's own loop over this library, is in test_gpu_dropin.py.)

Tolerances: stack maps equal the per-pair maps (the same kernels on the same features: peak index
exact, peak score within 1e-6 relative); the first pair's map matches the float64 oracle as the
map tests require (index exact, peak within 1e-4 relative)."""
import numpy as np
import pytest

import zcmir_b200 as zc
from oracle import smi_oracle as O
from zcmir_b200 import synth

pytestmark = pytest.mark.gpu


def corner_dist(A, B, w, h):
    d = 0.0
    for x, y in [(1, 1), (w, 1), (w, h), (1, h)]:
        a, b = A @ [x, y, 1.0], B @ [x, y, 1.0]
        d = max(d, float(np.hypot(*(a[:2] / a[2] - b[:2] / b[2]))))
    return d


@pytest.fixture(scope="module")
def stack():
    return synth.stack_drift(n=6, size=(256, 384), seed=4)


def test_stack_maps_equal_per_pair_maps(stack):
    slices, truths = stack
    n = len(slices)
    priors = [np.array([[1, 0, (s0.shape[1] - s1.shape[1]) / 2], [0, 1, (s0.shape[0] - s1.shape[0]) / 2], [0, 0, 1.0]])
              for s0, s1 in zip(slices[:-1], slices[1:])]
    with zc.Engine(half=False) as reg:
        a, b, _ = synth.pair_remap(n=128, seed=1)
        reg.set_images(a, b, preprocess=False)
        reg.pose = np.diag([1.0, 1.0, 1.0])
        before = reg.score(np.eye(3)).mean
        maps, ms = reg.stack_maps(slices, exact=True, calibrated=False, cap=1024)
        assert len(maps) == n - 1 and ms > 0
        # the engine's own pair is untouched
        assert reg.score(np.eye(3)).mean == pytest.approx(before, rel=1e-9) and tuple(reg.image_size(0)) == (128, 128)
        # explicit priors equal to the default (centres aligned) give the same maps
        maps2, _ = reg.stack_maps(slices, priors, exact=True, calibrated=False, cap=1024)
        for k in range(1, n):
            reg.set_images(slices[k], slices[k - 1], preprocess=False)
            one = reg.shift_map(priors[k - 1], exact=True, calibrated=False, cap=1024, want_map=False)
            for s in (maps[k - 1], maps2[k - 1]):
                assert s.peak_index == one.peak_index and (s.dx, s.dy) == (one.dx, one.dy)
                assert abs(s.peak - one.peak) <= 1e-6 * abs(one.peak)
        # the first pair against the oracle, on the GPU's features
        reg.set_images(slices[1], slices[0], preprocess=False)
        feat = lambda s: np.asarray(reg.features(s), np.float32)
        prep = lambda f: {"w": f.shape[2], "h": f.shape[1], "mode": "laplacian", "feat": f, "acf": O.acf(f),
                          "stack": np.concatenate([np.ones((1,) + f.shape[1:], np.float32), f])}
        ref = O.shift_map(prep(feat(0)), prep(feat(1)), priors[0], exact=True, calibrated=False, cap=1024)
        assert maps[0].peak_index == ref["peak_index"]
        assert abs(maps[0].peak - ref["peak"]) <= 1e-4 * abs(ref["peak"])


def test_stack_maps_errors():
    with zc.Engine(half=False) as reg:
        with pytest.raises(ValueError, match="at least 2"):
            reg.stack_maps([np.zeros((64, 64), np.float32)])
        with pytest.raises(RuntimeError, match="BadImage"):
            reg.stack_maps([np.zeros((64, 64), np.float32), np.zeros((4, 64), np.float32)])


def test_sweep_and_stack_in_one_launch(stack):
    """zcb_stack_load + zcb_sweep_stack: the sweep of the engine's pair and the stack's maps as two
    branches of one CUDA graph, launched once. Each branch computes what it computes alone: the
    lane maxima equal zcb_sweep's, the stack's results equal zcb_stack_maps's, bit for bit; the
    graph is captured once and replayed while nothing changes; a plain sweep or shift map after it
    is unaffected."""
    slices, _ = stack
    m, f, _ = synth.pair_similarity(n=256, seed=5)
    with zc.Engine(half=False, sw_nth=36, sw_ns=3, sw_grid=64) as reg:
        reg.set_images(m, f, preprocess=False)
        alone = reg.sweep(n_peak=4)
        maps, _ = reg.stack_maps(slices, exact=True, calibrated=False, cap=1024)
        with pytest.raises(zc.EngineError, match="load a stack"):
            zc.Engine(half=False).sweep_stack()
        reg.stack_load(slices, exact=True, calibrated=False, cap=1024)
        for rep in range(3):
            sw, st = reg.sweep_stack(n_peak=4)
            np.testing.assert_array_equal(sw.scores, alone.scores)
            np.testing.assert_array_equal(sw.index, alone.index)
            assert len(st) == len(maps)
            for a, b in zip(st, maps):
                assert (a.peak_index, a.dx, a.dy) == (b.peak_index, b.dx, b.dy)
                assert a.peak == b.peak
            assert sw.info["ms"] > 0
            # every kernel of both branches, each launched by the one replay
            assert sw.info["launches"] > alone.info["launches"]
        again = reg.sweep(n_peak=4)
        np.testing.assert_array_equal(again.scores, alone.scores)
        one = reg.shift_map(np.eye(3), exact=True, calibrated=False, cap=512, want_map=False)
        reg.set_images(m, f, preprocess=False)
        ref = reg.shift_map(np.eye(3), exact=True, calibrated=False, cap=512, want_map=False)
        assert (one.peak_index, one.peak) == (ref.peak_index, ref.peak)
