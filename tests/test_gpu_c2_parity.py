"""The 1024² map workload in full against the float64 oracle: a 1024² blob field against its
8-level segmented modality shifted by a seeded integer lag within ±200 px, zero-padded to a 2048²
FFT, with laplacian features (45 correlations) and with "three" (the fourth feature dropped: 28
correlations), each exact with and without the calibrated z. Every cell of the GPU's 2048² map
is compared with the oracle's, which starts from the same images (its own features).

Tolerances (the map tests' rule): the same argmax index, which is the planted lag; the peak
within 1e-4 relative; every cell within 1e-4 of the peak where the overlap is at least 20 % of
the largest and within 1e-2 elsewhere (FP32 FFT round-off grows as the overlap shrinks); cells
that an overlap floor zeroes on one side only are counted and must be rare."""
import numpy as np
import pytest

import zcmir_b200 as zc
from oracle import smi_oracle as O
from zcmir_b200 import synth

pytestmark = pytest.mark.gpu

N, CAP = 1024, 2048


@pytest.fixture(scope="module")
def pair():
    m16, f16, H = synth.pair_segmented(n=N, seed=1)
    # the engine divides uint16 by 65535; the oracle starts from the same float32 values
    return zc.gray32(m16), zc.gray32(f16), H


def oracle_maps(m, f, mode, variants, rows=256):
    """The oracle's maps of the pair at the identity for each (exact, calibrated) variant, the
    correlations formed once and the per-shift combine done a band of rows at a time (the
    zero-lag overlap of the whole map sets the 8 % floor)."""
    pa, pb = O.prepare(m, mode), O.prepare(f, mode)
    ga, gb, (nx, ny, cw, ch), (ox, oy, W, Hh) = O.grid_stacks(pa, pb, np.eye(3), cap=CAP)
    ids, corrs = O.corr_plan(True, mode == "three")
    corr = O.correlations(O.real_planes(ga, ids), O.real_planes(gb, ids), ids, corrs, nx, ny)
    n00 = float(corr[0, 0, 0])
    area = max(1.0, O.pair_area(pa["acf"], pb["acf"]) / (W / cw) ** 2)
    out = {}
    for exact, calibrated in variants:
        mp = np.zeros((ny, nx))
        for r0 in range(0, ny, rows):
            mp[r0:r0 + rows] = O.combine(corr[:, r0:r0 + rows], exact, calibrated, O.MIN_N, area,
                                         3 if mode == "three" else 4, n00=n00)
        peak, idx = O.argmax_first(mp)
        out[(exact, calibrated)] = {"map": mp, "peak": peak, "peak_index": idx}
    return out, corr[0].copy(), (nx, ny, cw, ch)


@pytest.mark.parametrize("mode,n_corr", [("laplacian", 45), ("three", 28)])
def test_full_map_matches_the_oracle(pair, mode, n_corr):
    m, f, H = pair
    variants = [(True, False), (True, True)]
    with zc.Engine(half=False, smi_features=mode) as eng:
        eng.set_images(m, f, preprocess=False)
        got = {v: eng.shift_map(np.eye(3), exact=v[0], calibrated=v[1], cap=CAP) for v in variants}
    ref, n_map, (nx, ny, cw, ch) = oracle_maps(m, f, mode, variants)
    assert (nx, ny, cw, ch) == (2048, 2048, 1024, 1024)
    big = n_map >= 0.2 * n_map.max()
    for v in variants:
        g, o = got[v], ref[v]
        assert (g.n, g.ny, g.cw, g.ch) == (nx, ny, cw, ch)
        assert g.peak_index == o["peak_index"], (v, g.peak_index, o["peak_index"])
        assert (g.dx, g.dy) == (-H[0, 2], -H[1, 2]), (v, g.dx, g.dy)
        assert abs(g.peak - o["peak"]) <= 1e-4 * abs(o["peak"]), (v, g.peak, o["peak"])
        gm, om = g.map.astype(np.float64), o["map"]
        err = np.abs(gm - om) / abs(o["peak"])
        one_sided = (gm == 0) != (om == 0)
        assert one_sided.mean() < 1e-4, one_sided.sum()
        assert err[big & ~one_sided].max() <= 1e-4, (v, err[big & ~one_sided].max())
        assert err[~one_sided].max() <= 1e-2, (v, err[~one_sided].max())
