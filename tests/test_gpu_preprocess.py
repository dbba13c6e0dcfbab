"""GPU parity of the preprocessing before the features (CLAHE, band pass, invert, RGBA → gray)
against the CPU oracle, and the reference's known answers in their own setup (uint8 images,
default settings: CLAHE, f16 texels).

Tolerances: CLAHE and RGBA → gray are the same float32 operations in the same order on both
sides: bit-exact. The band pass's Gaussian weights come from expf on the GPU and numpy's float32
exp on the CPU, which may round differently, and the rescale of the band to [0, 1] multiplies
the difference by 1/(hi − lo) (≈ 10 here): within 1e-5 (one f16 step with half)."""
import numpy as np
import pytest

import zcmir_b200 as zc
from oracle import preprocess_oracle as P
from zcmir_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def landsat(golden):
    d = np.load(golden / "landsat_b.npz")
    return d["moving"], d["fixed"], d["truth"]


def rgba_of(u8):
    return np.concatenate([np.repeat(u8[:, :, None], 3, axis=2), np.full(u8.shape + (1,), 255, np.uint8)], axis=2)


@pytest.mark.parametrize("half", [True, False])
def test_clahe_work_image_is_bit_exact(landsat, half):
    mv, fx, _ = landsat
    crop = mv[:333, :517]  # sizes that the 4×4 tiles do not divide: the reflected padding
    with zc.Engine(half=half) as reg:
        reg.set_images(crop, fx)
        got = reg.work_image(0)
        s = reg.settings
    ref = P.bake(P.rgba_gray(rgba_of(crop)), s)
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("clahe,half", [(True, False), (False, False), (True, True)])
def test_band_pass_and_invert(clahe, half):
    m, f, _ = synth.pair_remap(n=150, seed=4)
    m = m[:, :131]
    settings = dict(clahe=clahe, band=True, bp_fine=1.5, bp_coarse=3.0, invert=True, half=half, clahe_grid=6,
                    clahe_bins=100)
    with zc.Engine(**settings) as reg:
        reg.set_images(np.clip(m, 0, 1), np.clip(f, 0, 1), preprocess=True)
        got = reg.work_image(0)
        s = reg.settings
    ref = P.bake(np.clip(m, 0, 1).astype(np.float32), s)
    tol = 1e-3 if half else 1e-5
    assert np.abs(got - ref).max() <= tol, np.abs(got - ref).max()
    assert got.min() >= 0 and got.max() <= 1


def test_rgb_to_gray_and_rebake(landsat):
    mv, fx, _ = landsat
    rgb = np.stack([mv, np.roll(mv, 3, axis=1), 255 - mv], axis=2)
    with zc.Engine(half=False, clahe=False) as reg:
        reg.set_images(rgb, fx)
        np.testing.assert_array_equal(reg.work_image(0), P.rgba_gray(rgb))
        # a preprocessing setting changes the work image the next time it is needed
        reg.configure(clahe=True, clahe_grid=8)
        reg.score(np.eye(3))
        s = reg.settings
        np.testing.assert_array_equal(reg.work_image(0), P.bake(P.rgba_gray(rgb), s))
        with pytest.raises(ValueError, match="always preprocessed"):
            reg.set_images(mv, fx, preprocess=False)


def test_known_answers_in_the_reference_setup(landsat):
    """examples/03_smi.py:364-365 as it runs them: the uint8 landsat-b pair through the default
    preprocessing, the forward direction only; the shift map at T(14, −9)·truth peaks within 2 px
    of (14, −9), and the roto-scale map of the truth turned by 6° and scaled by 1.08 within 2°."""
    mv, fx, truth = landsat
    T = lambda x, y: np.array([[1, 0, x], [0, 1, y], [0, 0, 1.0]])
    with zc.Engine(symmetric=False) as reg:
        reg.set_images(mv, fx)
        sm = reg.shift_map(T(14, -9) @ truth, exact=True, calibrated=False)
        assert np.hypot(sm.dx - 14, sm.dy + 9) < 2, (sm.dx, sm.dy)
        c = reg.rs_map(truth, want_maps=False).center
        a = np.deg2rad(6)
        turn = np.array([[1.08 * np.cos(a), -1.08 * np.sin(a), 0], [1.08 * np.sin(a), 1.08 * np.cos(a), 0], [0, 0, 1]])
        r = reg.rs_map(T(*c) @ turn @ T(-c[0], -c[1]) @ truth)
        assert abs(-np.rad2deg(r.dth) - 6) < 2, np.rad2deg(r.dth)
