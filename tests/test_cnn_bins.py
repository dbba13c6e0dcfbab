"""Host logic of the 2-D proposal network (no GPU): its 24 × 9 rotation × scale bins, the BF16
conversion of its inputs, and its parameter layout against the oracle's."""
import numpy as np

from oracle import cnn_oracle as C
from zcmir_b200 import cnn


def test_bins_round_trip_and_cover_the_grid():
    deg = np.arange(0.0, 360.0, 0.5)
    for s in (0.8, 0.9, 1.0, 1.1, 1.25):
        b = cnn.labels(deg, np.full_like(deg, s))
        assert b.min() >= 0 and b.max() < cnn.BINS
        # each bin's centre falls back in its own bin
        for v in np.unique(b):
            d, sc = cnn.bin_pose(v)
            assert cnn.labels([d], [sc])[0] == v
    # rotation bins are 15° wide from 0°, and wrap at 360°
    assert cnn.labels([14.9], [1.0])[0] // 9 == 0 and cnn.labels([15.0], [1.0])[0] // 9 == 1
    assert cnn.labels([359.9], [1.0])[0] // 9 == 23 and cnn.labels([360.0], [1.0])[0] // 9 == 0
    assert cnn.labels([-10.0], [1.0])[0] // 9 == 23
    # the scale bins: the 9 log-spaced scales of [0.8, 1.25], the ends exact
    assert cnn.labels([0.0], [0.8])[0] % 9 == 0 and cnn.labels([0.0], [1.25])[0] % 9 == 8
    assert abs(cnn.bin_pose(8)[1] - 1.25) < 1e-12 and abs(cnn.bin_pose(0)[1] - 0.8) < 1e-12


def test_bf16_inputs_and_parameter_layout_match_the_oracle():
    x = np.random.default_rng(1).standard_normal(4096).astype(np.float32) * 3
    assert np.array_equal(cnn.to_bf16(x), C.bf16_bits(x))
    p = cnn.init_params(0)
    assert p.size == C.n_params() == 159_480
    layers, Wfc, bfc = C.unpack(p)
    assert [W.shape for W, _ in layers] == [(32, 9, 8), (64, 9, 32), (64, 9, 64), (128, 9, 64)]
    assert Wfc.shape == (216, 128) and bfc.shape == (216,) and not bfc.any()
