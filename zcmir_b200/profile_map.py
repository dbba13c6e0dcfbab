"""Run a few shift maps of a workload for a profiler (ncu) to capture.

    python -m zcmir_b200.profile_map [--n 1024] [--cap 2048] [--maps 2] [--features laplacian]

Builds the seeded segmented pair (zcmir_b200.synth.pair_segmented) at n², uploads it, then runs
`--maps` maps at the identity pose (exact, calibrated) through the C ABI, printing the plan and
the peak. Each map launches, in order: warp_stack, paste_stack, lag0, fwd_rows ×2, cols ×2,
inv_cols, inv_rows.
"""
import argparse

import numpy as np

import zcmir_b200 as zc
from zcmir_b200 import synth


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--cap", type=int, default=2048)
    ap.add_argument("--maps", type=int, default=2)
    ap.add_argument("--features", default="laplacian")
    a = ap.parse_args()
    m, f, H = synth.pair_segmented(n=a.n, seed=1, max_shift=min(200, a.n // 5))
    with zc.Registrar(half=False, smi_features=a.features) as reg:
        reg.set_images(m, f, preprocess=False)
        for _ in range(a.maps):
            sm = reg.shift_map(np.eye(3), exact=True, calibrated=True, resolution=a.cap, return_map=False)
        print(f"n {sm.n}x{sm.ny} grid {sm.cw}x{sm.ch} peak {sm.peak:.3f} at ({sm.dx}, {sm.dy}); truth {-H[0, 2]}, {-H[1, 2]}")


if __name__ == "__main__":
    main()
