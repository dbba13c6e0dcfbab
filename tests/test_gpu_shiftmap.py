"""GPU parity of the shift-map path against the CPU oracle, through the zc_* C ABI.

Tolerances: features are compared element-wise (the f32 rank/feature arithmetic is restated
operation by operation, so they agree to the last bits); maps must have the same argmax (index
exact), the peak within 1e-4 relative, every cell within 1e-4 of the peak where the overlap is at
least 20 % of the largest, and every other cell within 1e-2 of the peak (FP32 FFT round-off grows
where the overlap is small). Cells that one side zeroes by an overlap floor and the other does not
must lie within 1 % of that floor.
"""
import numpy as np
import pytest

import zcmir_b200 as zc
from oracle import smi_oracle as O
from zcmir_b200 import synth

pytestmark = pytest.mark.gpu


def prep_from(feat, mode="laplacian"):
    """The oracle's per-image record built on given (the GPU's) features."""
    f = np.asarray(feat, np.float32)
    return {"w": f.shape[2], "h": f.shape[1], "mode": mode, "feat": f, "acf": O.acf(f),
            "stack": np.concatenate([np.ones((1,) + f.shape[1:], np.float32), f])}


def check_map(sm, ref, n_corr0=None, tight=1e-4, loose=1e-2):
    g, o = sm.map.astype(np.float64), ref["map"]
    assert g.shape == o.shape
    assert sm.peak_index == ref["peak_index"], (sm.peak_index, ref["peak_index"])
    assert (sm.dx, sm.dy) == (ref["dx"], ref["dy"])
    assert abs(sm.peak - ref["peak"]) <= 1e-4 * abs(ref["peak"])
    err = np.abs(g - o) / max(abs(ref["peak"]), 1e-30)
    disagree = (g == 0) != (o == 0)
    if n_corr0 is not None:
        big = n_corr0 >= 0.2 * n_corr0.max()
        assert err[big & ~disagree].max() <= tight, err[big & ~disagree].max()
    assert err[~disagree].max() <= loose, err[~disagree].max()
    return disagree


@pytest.fixture(scope="module")
def c1_pair():
    return synth.pair_remap(n=256, shift=(17, -9), seed=0)


def test_features_match_oracle(c1_pair):
    m, f, _ = c1_pair
    with zc.Engine(half=False) as reg:
        reg.set_images(m, f, preprocess=False)
        for side, img in ((0, m), (1, f)):
            gpu = reg.features(side)
            ora = O.prepare(img, "laplacian")["feat"]
            np.testing.assert_allclose(gpu, ora, rtol=0, atol=2e-6)
            assert np.mean(gpu == ora) > 0.999
        np.testing.assert_array_equal(reg.work_image(0), m)


def test_features_half_and_modes(c1_pair):
    m, f, _ = c1_pair
    for mode in ("three", "cubic"):
        with zc.Engine(half=True, smi_features=mode) as reg:
            reg.set_images(m, f, preprocess=False)
            gpu = reg.features(1)
            ora = O.prepare(f, mode, half=True)["feat"]
            np.testing.assert_allclose(gpu, ora, rtol=0, atol=2e-6)
            np.testing.assert_array_equal(reg.work_image(1), O.quantize_half(f))
            if mode == "three":
                assert np.abs(gpu[3]).max() == 0


def test_c1_map_exact_uncalibrated(c1_pair):
    """The 256² map workload: 45 correlations zero-padded to 512², exact whitening, no calibration."""
    m, f, H = c1_pair
    with zc.Engine(half=False) as reg:
        reg.set_images(m, f, preprocess=False)
        pa, pb = prep_from(reg.features(0)), prep_from(reg.features(1))
        sm = reg.shift_map(np.eye(3), exact=True, calibrated=False, cap=1024)
    ref = O.shift_map(pa, pb, np.eye(3), exact=True, calibrated=False, cap=1024, return_corr=True)
    assert (sm.n, sm.ny, sm.cw, sm.ch) == (512, 512, 256, 256)
    check_map(sm, ref, ref["corr"][0])
    assert (sm.dx, sm.dy) == (-H[0, 2], -H[1, 2])
    assert np.allclose(sm.corrected(np.eye(3)), H)


def test_c1_map_variants(c1_pair):
    """Global whitening (25 correlations), three features (28), calibrated z, settings maps."""
    m, f, _ = c1_pair
    for kw, mode in (({"exact": False, "calibrated": False}, "laplacian"), ({"exact": True, "calibrated": True}, "laplacian"),
                     ({"exact": True, "calibrated": False}, "three")):
        with zc.Engine(half=False, smi_features=mode) as reg:
            reg.set_images(m, f, preprocess=False)
            pa, pb = prep_from(reg.features(0), mode), prep_from(reg.features(1), mode)
            sm = reg.shift_map(np.eye(3), cap=1024, **kw)
        ref = O.shift_map(pa, pb, np.eye(3), cap=1024, return_corr=True, **kw)
        check_map(sm, ref, ref["corr"][0])


def test_settings_map_auto_resolution(golden):
    """zc_shift_map_set with the defaults (exact, calibrated, min_overlap 0.05, auto resolution:
    a 2-tap resampled grid for the landsat-b canvas)."""
    d = np.load(golden / "landsat_b.npz")
    m, f = d["moving"].astype(np.float32) / 255, d["fixed"].astype(np.float32) / 255
    H0 = np.array([[1, 0, 14], [0, 1, -9], [0, 0, 1.0]]) @ d["truth"]
    with zc.Engine(half=False) as reg:
        reg.set_images(m, f, preprocess=False)
        pa, pb = prep_from(reg.features(0)), prep_from(reg.features(1))
        sm = reg.shift_map(H0)
    ref = O.shift_map(pa, pb, H0, exact=True, calibrated=True, cap=0, min_overlap=0.05, return_corr=True)
    assert (sm.n, sm.cw, sm.canvas) == (ref["n"], ref["cw"], (ref["canvas_w"], ref["canvas_h"]))
    assert sm.offset == (ref["ox"], ref["oy"])
    assert abs(sm.corr_area_px - ref["corr_area_px"]) <= 1e-3 * ref["corr_area_px"]
    check_map(sm, ref, ref["corr"][0], tight=1e-3)
    assert np.hypot(sm.dx - 14, sm.dy + 9) < 2 * 917 / 230  # the 03_smi check, at this grid's cell


@pytest.mark.slow
def test_landsat_full_resolution_ladder_fft(golden):
    """A 1944² (2^3·3^5) map: radix-3 stages and a rotated, scaled canvas; the 03_smi known answer
    (lag (14, −9)) exactly."""
    d = np.load(golden / "landsat_b.npz")
    m, f = d["moving"].astype(np.float32) / 255, d["fixed"].astype(np.float32) / 255
    H0 = np.array([[1, 0, 14], [0, 1, -9], [0, 0, 1.0]]) @ d["truth"]
    with zc.Engine(half=False) as reg:
        reg.set_images(m, f, preprocess=False)
        pa, pb = prep_from(reg.features(0)), prep_from(reg.features(1))
        sm = reg.shift_map(H0, exact=True, calibrated=False, cap=2048)
    assert (sm.n, sm.cw) == (1944, 917)
    assert (sm.dx, sm.dy) == (14.0, -9.0)
    ref = O.shift_map(pa, pb, H0, exact=True, calibrated=False, cap=2048, return_corr=True)
    check_map(sm, ref, ref["corr"][0], tight=1e-3, loose=2e-2)


def test_segmented_1024_full_size_properties():
    """The 1024² workload (2048² FFT, 45 correlations): the argmax is the planted shift, and the
    map at a spread of lags equals the score of the FFT-free float64 direct sums of the same
    planes (the GPU's own features)."""
    m, f, H = synth.pair_segmented(n=1024, seed=1)
    with zc.Engine(half=False) as reg:
        reg.set_images(m, f, preprocess=False)
        pa, pb = prep_from(reg.features(0)), prep_from(reg.features(1))
        sm = reg.shift_map(np.eye(3), exact=True, calibrated=True, cap=2048)
        area = sm.corr_area_px
        sm3 = reg.shift_map(np.eye(3), exact=True, calibrated=False, cap=2048)
    assert (sm.n, sm.ny, sm.cw) == (2048, 2048, 1024)
    assert (sm.dx, sm.dy) == (-H[0, 2], -H[1, 2])
    assert (sm3.dx, sm3.dy) == (-H[0, 2], -H[1, 2])
    ga, gb, _, _ = O.grid_stacks(pa, pb, np.eye(3), cap=2048)
    ids, corrs = O.corr_plan(True, False)
    A, B = O.real_planes(ga, ids), O.real_planes(gb, ids)
    n00 = float(np.sum(A[0] * B[0]))
    rng = np.random.default_rng(0)
    lags = [(0, 0), (int(-H[0, 2]), int(-H[1, 2]))] + [tuple(int(v) for v in rng.integers(-600, 601, 2)) for _ in range(10)]
    for tx, ty in lags:
        s = O.direct_sums(A, B, ids, corrs, tx, ty)
        cells = s.reshape(45, 1)
        want = float(O.combine(cells, exact=True, calibrated=False, min_n=12, area=1.0)[0])
        # the floor at lag 0 uses n(0, 0) of the whole map
        if s[0] < max(12, 0.08 * n00):
            want = 0.0
        got = float(sm3.map[ty % 2048, tx % 2048])
        assert abs(got - want) <= 1e-4 * max(abs(sm3.peak), 1e-30), (tx, ty, got, want)
        wz = float(O.combine(cells, exact=True, calibrated=True, min_n=12, area=max(1.0, area))[0])
        assert abs(float(sm.map[ty % 2048, tx % 2048]) - wz) <= 1e-3 * max(abs(sm.peak), 1.0), (tx, ty)


def test_errors_and_boundaries():
    with zc.Engine(half=False) as reg:
        with pytest.raises(RuntimeError, match="NoImages"):
            reg.shift_map(np.eye(3), exact=True)
        with pytest.raises(RuntimeError, match="BadImage"):
            reg.set_image(0, np.zeros((4, 64), np.float32), preprocess=False)
        with pytest.raises(RuntimeError, match="UnknownSetting"):
            reg.configure(nope=1)
        with pytest.raises(ValueError, match="always preprocessed"):
            reg.set_image(0, np.zeros((64, 64), np.uint8), preprocess=False)
        m, f, _ = synth.pair_remap(n=64, seed=9)
        reg.set_images(m, f, preprocess=False)
        small = np.empty(16, np.float32)
        with pytest.raises(RuntimeError, match="MapTooSmall"):
            reg.shift_map(np.eye(3), exact=True, calibrated=False, out=small)
        # the smallest image (8 × 8) and a ragged rectangle
        for shape in ((8, 8), (37, 91)):
            rng = np.random.default_rng(1)
            a, b = rng.random(shape).astype(np.float32), rng.random(shape).astype(np.float32)
            reg.set_images(a, b, preprocess=False)
            pa, pb = prep_from(reg.features(0)), prep_from(reg.features(1))
            sm = reg.shift_map(np.eye(3), exact=True, calibrated=False, cap=1024)
            ref = O.shift_map(pa, pb, np.eye(3), exact=True, calibrated=False, cap=1024, return_corr=True)
            check_map(sm, ref, ref["corr"][0], tight=1e-3, loose=1e-2)


def test_rotated_pose_canvas(c1_pair):
    """A rotated, scaled pose: warped canvas with bilinear taps, a non-zero canvas offset."""
    m, f, _ = c1_pair
    th, s = np.deg2rad(7.0), 1.05
    c = 128.5
    R = np.array([[s * np.cos(th), -s * np.sin(th), 0], [s * np.sin(th), s * np.cos(th), 0], [0, 0, 1]])
    T = lambda x, y: np.array([[1, 0, x], [0, 1, y], [0, 0, 1.0]])
    H = T(c + 6, c - 4) @ R @ T(-c, -c)
    with zc.Engine(half=False) as reg:
        reg.set_images(m, f, preprocess=False)
        pa, pb = prep_from(reg.features(0)), prep_from(reg.features(1))
        sm = reg.shift_map(H, exact=True, calibrated=False, cap=1024)
        origin, size, Hc = reg.canvas(H)
    ref = O.shift_map(pa, pb, H, exact=True, calibrated=False, cap=1024, return_corr=True)
    assert origin == (ref["ox"], ref["oy"]) and size == (ref["canvas_w"], ref["canvas_h"])
    check_map(sm, ref, ref["corr"][0], tight=1e-3, loose=1e-2)


@pytest.mark.parametrize("n,cap", [(512, 2048), (1024, 2048), (256, 1024)])
def test_row_pass_tensor_memory_matches_split(monkeypatch, n, cap):
    """The last pass with the sums in tensor memory (whole rows) and the shared-memory split pass
    give the same map (FP32 FFTs in a different order: within 1e-5 of the peak) and argmax, except
    cells that the 8 %-of-zero-lag overlap floor zeroes on one side only (their overlap sits on
    the floor to FP32 round-off); those are a few in a million."""
    m, f, H = synth.pair_segmented(n=n, seed=4, max_shift=n // 6)
    maps = {}
    for mode in ("split", "tmem"):
        monkeypatch.setenv("ZCMIR_B200_ROW_PASS", mode)
        with zc.Engine(half=False) as reg:
            reg.set_images(m, f, preprocess=False)
            maps[mode] = reg.shift_map(np.eye(3), exact=True, calibrated=True, cap=cap)
            g3 = reg.shift_map(np.eye(3), exact=True, calibrated=False, cap=cap)
            maps[mode + "3"] = g3
    for a, b in (("split", "tmem"), ("split3", "tmem3")):
        A, B = maps[a], maps[b]
        assert A.peak_index == B.peak_index and (A.dx, A.dy) == (B.dx, B.dy)
        # within a pixel of the planted shift: at 256² the float64 oracle's map of this pair also
        # peaks at (−19, −37) for the planted (−19, −38)
        assert max(abs(A.dx + H[0, 2]), abs(A.dy + H[1, 2])) <= 1
        floor = (A.map == 0) != (B.map == 0)
        assert floor.mean() < 1e-4
        assert np.max(np.abs(A.map - B.map)[~floor]) <= 1e-5 * max(abs(A.peak), 1.0)


def test_bench_maps_graph_replay_leaves_the_map_unchanged(c1_pair):
    """zcb_bench_maps times replays of one captured CUDA graph of the map's passes (and
    event-instrumented maps for the stages): the timings are sane and a map computed after the
    replays is the map computed before them, value for value."""
    m, f, H = c1_pair
    with zc.Engine(half=False) as reg:
        reg.set_images(m, f, preprocess=False)
        before = reg.shift_map(H, exact=True, calibrated=True, cap=512)
        r = reg.bench_maps(H, flags=3, cap=512, warmup=2, steps=4)
        after = reg.shift_map(H, exact=True, calibrated=True, cap=512)
        ev = [e["text"] for e in reg.events() if e.get("kind") == "log"]
    assert 0 < r["ms_per_map"] <= 1.5 * r["ms_per_map_instrumented"], r
    assert abs(sum(r["stages_ms"].values()) - r["ms_per_map_instrumented"]) <= 0.05 * r["ms_per_map_instrumented"]
    assert not any("graph replay unavailable" in t for t in ev), ev
    assert (after.dx, after.dy, after.peak_index) == (before.dx, before.dy, before.peak_index)
    np.testing.assert_array_equal(after.map, before.map)


def test_maps_reuse_each_sides_spectra(c1_pair):
    """A side's canvas and half spectra are built once and reused by the next map whose canvas,
    plan and (for the moving side) canvas pose are the same: the calibrated map after the
    uncalibrated one at the same pose, the map at a pose that keeps the moving image inside the
    fixed frame (the fixed side is reused). Every reused map equals the map of a fresh engine,
    value for value, and launches fewer kernels; new images, a roto-scale map in between and new
    feature settings rebuild what they must."""
    m, f, _ = c1_pair
    c = 128.5
    T = lambda x, y: np.array([[1, 0, x], [0, 1, y], [0, 0, 1.0]])
    a = np.deg2rad(1.5)
    inside = T(c, c) @ np.array([[0.96 * np.cos(a), -0.96 * np.sin(a), 0], [0.96 * np.sin(a), 0.96 * np.cos(a), 0],
                                 [0, 0, 1]]) @ T(-c, -c)

    def fresh(H, **kw):
        with zc.Engine(half=False) as e:
            e.set_images(m, f, preprocess=False)
            return e.shift_map(H, cap=1024, **kw)

    with zc.Engine(half=False) as eng:
        eng.set_images(m, f, preprocess=False)
        first = eng.shift_map(np.eye(3), exact=True, calibrated=False, cap=1024)
        eng.gpu_counts()
        again = eng.shift_map(np.eye(3), exact=True, calibrated=True, cap=1024)
        n_both = eng.gpu_counts()["launches"]
        moved = eng.shift_map(inside, exact=True, calibrated=True, cap=1024)
        n_fixed = eng.gpu_counts()["launches"]
        eng.rs_map(np.eye(3), want_maps=False)
        eng.gpu_counts()
        after_rs = eng.shift_map(inside, exact=True, calibrated=True, cap=1024)
        n_none = eng.gpu_counts()["launches"]
        assert n_both < n_fixed < n_none, (n_both, n_fixed, n_none)
        np.testing.assert_array_equal(first.map, fresh(np.eye(3), exact=True, calibrated=False).map)
        np.testing.assert_array_equal(again.map, fresh(np.eye(3), exact=True, calibrated=True).map)
        ref_moved = fresh(inside, exact=True, calibrated=True)
        np.testing.assert_array_equal(moved.map, ref_moved.map)
        np.testing.assert_array_equal(after_rs.map, ref_moved.map)
        # new images and new feature settings: both sides rebuilt
        eng.set_images(f, m, preprocess=False)
        swapped = eng.shift_map(np.eye(3), exact=True, calibrated=True, cap=1024)
        with zc.Engine(half=False) as e2:
            e2.set_images(f, m, preprocess=False)
            np.testing.assert_array_equal(swapped.map, e2.shift_map(np.eye(3), exact=True, calibrated=True, cap=1024).map)
        eng.configure(smi_features="three")
        three = eng.shift_map(np.eye(3), exact=True, calibrated=True, cap=1024)
        with zc.Engine(half=False, smi_features="three") as e3:
            e3.set_images(f, m, preprocess=False)
            np.testing.assert_array_equal(three.map, e3.shift_map(np.eye(3), exact=True, calibrated=True, cap=1024).map)
