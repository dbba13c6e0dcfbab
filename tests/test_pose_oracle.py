"""The pose oracle against the reference's own construction (examples/03_smi.py:169-188,
284-343): the gradient from finite differences of the score over the 45 sums times per-pixel
flows, and the symmetric gradient against finite differences of the pair score. CPU only."""
import numpy as np
import pytest

from oracle import pose_oracle as P
from oracle import smi_oracle as O

TRI = O.TRI


@pytest.fixture(scope="module")
def landsat(golden):
    d = np.load(golden / "landsat_b.npz")
    pa = O.prepare(d["moving"].astype(np.float32) / 255)
    pb = O.prepare(d["fixed"].astype(np.float32) / 255)
    return pa["feat"], pb["feat"], d["truth"]


def test_gradient_matches_03_smi_construction(landsat):
    A, B, truth = landsat
    hf, wf = B.shape[1:]
    N = P.dest_n(wf, hf)
    H2 = np.linalg.inv(N) @ P.expm3(P.hat([0.02, -0.015, 0.02, 0.01, 0, 0, 0, 0])) @ N @ truth
    m2 = P.moments(A, B, H2)
    s2, coef = P.score_from_moments(m2)
    g_an, _ = P.tangent(A, B, H2, coef, hess=False)
    g = np.zeros(45)
    for k in range(45):
        h = 1e-6 * max(abs(m2[k]), 1e-3 * m2[0])
        e = np.zeros(45)
        e[k] = h
        g[k] = (P.score_from_moments(m2 + e)[0] - P.score_from_moments(m2 - e)[0]) / (2 * h)
    np.testing.assert_allclose(coef[40:85], g, rtol=0, atol=1e-6 * np.abs(g).max())
    S = P.sample(A, H2, wf, hf)
    va, vb = S["va"], B.astype(np.float64)
    dS_da = np.zeros_like(va)
    for i in range(4):
        dS_da[i] = g[1 + i] + sum(g[9 + 4 * i + j] * vb[j] for j in range(4))
        for k, (p, q) in enumerate(TRI):
            if p == i:
                dS_da[i] += g[25 + k] * va[q] * (2 if q == i else 1)
            elif q == i:
                dS_da[i] += g[25 + k] * va[p]
    dS_dw = g[0] + sum(g[1 + i] * va[i] for i in range(4)) + sum(g[5 + j] * vb[j] for j in range(4))
    dS_dw += sum(g[9 + 4 * i + j] * va[i] * vb[j] for i in range(4) for j in range(4))
    dS_dw += sum(g[25 + k] * va[p] * va[q] for k, (p, q) in enumerate(TRI))
    dS_dw += sum(g[35 + k] * vb[p] * vb[q] for k, (p, q) in enumerate(TRI))
    dSx = S["w"] * (dS_da * S["gx"]).sum(0) + dS_dw * S["dw"][0]
    dSy = S["w"] * (dS_da * S["gy"]).sum(0) + dS_dw * S["dw"][1]
    Hi, ph, X = np.linalg.inv(H2), S["ph"], S["X"]
    grad_np = []
    for k in range(8):
        Gk = np.linalg.inv(N) @ P.hat(np.eye(8)[k]) @ N
        v = -np.tensordot(Hi @ Gk, X, 1)
        u, w = (v[0] * ph[2] - ph[0] * v[2]) / ph[2] ** 2, (v[1] * ph[2] - ph[1] * v[2]) / ph[2] ** 2
        grad_np.append((dSx * u + dSy * w).sum())
    grad_np = np.array(grad_np)
    assert np.linalg.norm(grad_np - g_an) < 1e-6 * np.linalg.norm(grad_np)


@pytest.mark.slow
def test_symmetric_gradient_finite_differences(landsat):
    A, B, truth = landsat
    hf, wf = B.shape[1:]
    N = P.dest_n(wf, hf)
    H2 = np.linalg.inv(N) @ P.expm3(P.hat([0.02, -0.015, 0.02, 0.01, 0, 0, 0, 0])) @ N @ truth
    r = P.pair_eval(A, B, H2, grad=True, hess=True)
    fd = []
    for k in range(8):
        e = np.zeros(8)
        e[k] = 1e-5
        fd.append((P.pair_eval(A, B, P.compose_n(H2, e, True, wf, hf))["mean"]
                   - P.pair_eval(A, B, P.compose_n(H2, -e, True, wf, hf))["mean"]) / 2e-5)
    fd = np.array(fd)
    assert np.linalg.norm(fd - r["grad"]) < 1e-2 * np.linalg.norm(fd)   # examples/03_smi.py:366
    assert np.all(np.linalg.eigvalsh(r["hess"]) > 0)


def test_pose_algebra():
    H = np.array([[1.01, 0.012, -3.06], [-0.006, 1.008, 4.86], [1e-5, 2e-5, 1]])
    np.testing.assert_allclose(P.inv3(H) @ H, np.eye(3), atol=1e-12)          # src/lie.zig:581-585
    x = np.array([0.1, -0.2, 0.03, 0.02, 0.01, -0.01, 1e-4, -2e-4])
    np.testing.assert_allclose(P.vee(P.hat(x)), x, atol=1e-12)                  # src/lie.zig:587-592
    # adjointGrad pulls a moving-frame increment back: the identity pose of equal frames negates
    g = np.arange(1.0, 9.0)
    np.testing.assert_allclose(P.adjoint_grad(g, np.eye(3), True, 64, 64, 64, 64), -g, atol=1e-12)


@pytest.mark.parametrize("source", [False, True])
def test_ffd_gradient_matches_finite_differences(landsat, source):
    """The control-point gradient of the oracle (smi.wgsl ffd_grad restated) against central
    differences of the pair score over the control points, both lattice placements, symmetric
    (src/pair.zig:387-410). A 4 × 4 lattice with a small random warp on the landsat-b truth."""
    A, B, truth = landsat
    # a 240² window of the fixed image against the whole moving one (the CPU suite stays quick)
    T = np.array([[1, 0, -200.0], [0, 1, -180.0], [0, 0, 1]])
    Bw = B[:, 180:420, 200:440]
    H = T @ truth
    rng = np.random.default_rng(3 if source else 4)
    ffd = dict(g=4, cps=0.004 * rng.standard_normal(32), source=source)
    s0, g_an = P.pair_ffd_grad(A, Bw, H, ffd)
    assert np.isfinite(s0) and np.linalg.norm(g_an) > 0
    h = 2e-5
    ks = np.argsort(-np.abs(g_an))[:8]   # the eight largest components
    g_fd = np.zeros(len(ks))
    for n, k in enumerate(ks):
        for sgn in (1, -1):
            c = ffd["cps"].copy()
            c[k] += sgn * h
            s, _ = P.pair_ffd_grad(A, Bw, H, dict(ffd, cps=c))
            g_fd[n] += sgn * s / (2 * h)
    # bilinear sampling makes the score piecewise smooth: agreement to a few per cent
    assert np.linalg.norm(g_fd - g_an[ks]) < 0.05 * np.linalg.norm(g_fd), (g_fd, g_an[ks])


def test_ffd_off_or_zero_leaves_the_pose_path():
    """A spline with all-zero control points moves nothing: the moments equal the spline-free
    ones (both placements), and the pair scores ignore a spline that is not live."""
    rng = np.random.default_rng(0)
    A = rng.standard_normal((4, 40, 48))
    B = rng.standard_normal((4, 44, 40))
    H = np.array([[1.0, 0.02, 1.5], [-0.01, 0.99, -2.0], [0, 0, 1]])
    for source in (False, True):
        z = dict(g=5, cps=np.zeros(50), source=source)
        np.testing.assert_array_equal(P.moments(A, B, H, z), P.moments(A, B, H))
        assert not P.ffd_live(z)
        assert P.pair_eval(A, B, H, ffd=z)["mean"] == P.pair_eval(A, B, H)["mean"]
