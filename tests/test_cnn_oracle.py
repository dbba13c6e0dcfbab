"""The 2-D convolutional proposal's float64 oracle: its backward pass against central differences
(the plain float64 network, no BF16 rounding), and its BF16 rounding rule."""
import numpy as np

from oracle import cnn_oracle as C


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0**-8, 1.0 + 3 * 2.0**-9, -2.5, 1e-3], np.float32)
    r = C.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0  # a tie rounds to the even mantissa
    assert r[2] == 1.0 + 2.0**-7
    assert r[3] == -2.5
    assert abs(r[4] - 1e-3) <= 2.0**-9 * 1e-3
    assert np.array_equal(C.from_bits(C.bf16_bits(x)), r)


def test_backward_matches_central_differences():
    rng = np.random.default_rng(0)
    p = C.init_params(1).astype(np.float64)
    x = rng.standard_normal((2, 128, 128, 8))
    y = np.array([5, 200])
    loss, g = C.loss_grad(p, x, y, bf16=False)
    assert abs(loss - np.log(216)) < 3.0
    # a few coordinates of every block: the four convolutions' weights and biases and the head
    offs, o = [], 0
    for l in range(4):
        nw = C.CH[l + 1] * 9 * C.CH[l]
        offs += [o + 3, o + nw // 2, o + nw + 1]
        o += nw + C.CH[l + 1]
    offs += [o + 17, o + C.BINS * C.FEAT + 5]
    h = 1e-5
    for i in offs:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (C.loss_grad(pp, x, y, bf16=False)[0] - C.loss_grad(pm, x, y, bf16=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])
