"""Run a few shift maps, or sweeps, of a workload for a profiler (ncu) to capture.

    python -m zcmir_b200.profile_map [--n 1024] [--cap 2048] [--maps 2] [--features laplacian]
                                     [--dft-stage 0] [--stages]
    python -m zcmir_b200.profile_map --sweep [--n 512] [--maps 1] [--nth 360] [--ns 9] [--batch 0]
    python -m zcmir_b200.profile_map --search [--n 512] [--maps 1]

Maps: builds the seeded segmented pair (zcmir_b200.synth.pair_segmented) at n², uploads it, then
runs `--maps` maps at the identity pose (exact, calibrated) through the C ABI, printing the plan
and the peak. Each map launches, in order: warp_stack, paste_stack, lag0, fwd_rows ×2, cols ×2,
inv_cols, inv_rows. --dft-stage P (1–3): the forward column FFTs' first stage on the tensor
cores in P BF16 pieces (zcb_set_dft_stage; cols ×2 become k_dft16_tc, cols, copy per side).
--stages: per-stage device times of the maps after the first (CUDA events, zc_profile_report).

Sweeps (--sweep): the seeded similarity pair (zcmir_b200.synth.pair_similarity) at n², then
`--maps` sweeps of nth rotations × ns scales in [0.8, 1.25] on a 128² canvas (3240 candidate maps
by default) through zcb_sweep. Each sweep launches interleave ×2 and the fixed window's pack, then
per plane size the fixed window's fwd_rows and cols, then per batch pack, fwd_rows, cols,
inv_cols, rows and peaks.

Searches (--search): the same pair and sweep grid, then `--maps` whole searches from the
identity pose (the sweep, its peaks' non-maximum suppression, the batched Gauss–Newton screen and
the finalists' climbs): after the sweep's launches, each Gauss–Newton step evaluates its poses
with pose_moments (forward and inverse direction), pose_coefs and, for the gradient,
pose_tangent.
"""
import argparse

import numpy as np

import zcmir_b200 as zc
from zcmir_b200 import synth


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=0)
    ap.add_argument("--cap", type=int, default=2048)
    ap.add_argument("--maps", type=int, default=2)
    ap.add_argument("--features", default="laplacian")
    ap.add_argument("--sweep", action="store_true")
    ap.add_argument("--search", action="store_true")
    ap.add_argument("--nth", type=int, default=360)
    ap.add_argument("--ns", type=int, default=9)
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--dft-stage", type=int, default=0)
    ap.add_argument("--stages", action="store_true")
    a = ap.parse_args()
    if a.search:
        n = a.n or 512
        m, f, H = synth.pair_similarity(n=n, seed=2)
        with zc.Engine(half=False, smi_features=a.features, sw_nth=a.nth, sw_ns=a.ns, sw_smin=0.8, sw_smax=1.25,
                          sw_grid=128) as reg:
            reg.set_images(m, f, preprocess=False)
            for _ in range(a.maps):
                reg.pose = np.eye(3)
                r = reg.search()
            print(f"search: score {r.score:.1f}")
        return
    if a.sweep:
        n = a.n or 512
        m, f, H = synth.pair_similarity(n=n, seed=2)
        with zc.Engine(half=False, smi_features=a.features, sw_nth=a.nth, sw_ns=a.ns, sw_smin=0.8, sw_smax=1.25,
                          sw_grid=128) as reg:
            reg.set_images(m, f, preprocess=False)
            for _ in range(a.maps):
                sw = reg.sweep(n_peak=4, batch=a.batch)
            i = sw.info
            print(f"sweep: {i['candidates']:.0f} candidates, {i['groups']:.0f} plane sizes, {i['batches']:.0f} batches, "
                  f"{i['launches']:.0f} launches, {i['ms']:.2f} ms")
        return
    n = a.n or 1024
    m, f, H = synth.pair_segmented(n=n, seed=1, max_shift=min(200, n // 5))
    with zc.Engine(half=False, smi_features=a.features) as reg:
        reg.set_images(m, f, preprocess=False)
        reg.set_dft_stage(a.dft_stage)
        for i in range(a.maps):
            if a.stages and i == 1:
                reg.profile_report()  # drop the first map's times
                reg.profile(True)
            sm = reg.shift_map(np.eye(3), exact=True, calibrated=True, cap=a.cap, want_map=False)
        print(f"n {sm.n}x{sm.ny} grid {sm.cw}x{sm.ch} peak {sm.peak:.3f} at ({sm.dx}, {sm.dy}); truth {-H[0, 2]}, {-H[1, 2]}")
        if a.stages:
            print(reg.profile_report(), end="")


if __name__ == "__main__":
    main()
