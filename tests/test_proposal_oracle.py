"""The proposal network's CPU oracle on its own: its backward pass against central differences
of its loss (CPU only)."""
import numpy as np

from oracle import proposal_oracle as N


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = N.init_params(2).astype(np.float64)
    x = rng.standard_normal((3, 6, 36))
    lab = np.array([5, 1700, 3239])
    loss, g = N.loss_grad(p, x, lab)
    assert g.shape == (N.nparams(),) and loss.shape == (3,)
    # weights and biases of every layer: w1 0–959, b1 960–991, w2 992–6111, b2 6112–6143,
    # w3 6144–14783, b3 14784–14873
    ks = np.concatenate([rng.choice(960, 5, replace=False), 960 + rng.choice(32, 2, replace=False),
                         992 + rng.choice(5120, 4, replace=False), 6112 + rng.choice(32, 2, replace=False),
                         6144 + rng.choice(8640, 5, replace=False), 14784 + rng.choice(90, 3, replace=False)])
    h = 1e-6
    for k in ks:
        e = np.zeros_like(p)
        e[k] = h
        fd = (N.loss_grad(p + e, x, lab)[0].mean() - N.loss_grad(p - e, x, lab)[0].mean()) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])
