"""The 2-D convolutional pose proposal (zcb_cnn_*): a pair's two 128 × 128 feature stacks in,
a distribution over 24 rotation × 9 log-scale bins out, trained and run on the tensor cores with
BF16 weights and FP32 accumulation.

    params = cnn.init_params(seed)
    x = cnn.pair_stacks(pairs)                  # [n][128][128][8] BF16 bits, from the engine
    y = cnn.labels(deg, scale)                  # bin 9·r + s of each pair's rotation and scale
    params, losses, ms = cnn.train(params, x, y, batch=256, steps=2000)
    logits = cnn.forward(params, x_test)

The features are the engine's own (rank, rank², Sobel, Laplacian planes of each image, whitened),
computed on the GPU for pairs at 128² and stacked as 8 channels (moving image's 4, then the
fixed image's 4).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native

BINS, ROT_BINS, SCALE_BINS = 216, 24, 9
SIDE, CHANNELS = 128, 8
S_MIN, S_MAX = 0.8, 1.25
_CH = (8, 32, 64, 64, 128)


def _lib():
    return _native.load()


def _check(rc):
    if rc != 0:
        buf = ctypes.create_string_buffer(1024)
        _lib().zcb_cnn_error(buf, 1024)
        raise RuntimeError(buf.value.decode())


def nparams():
    return int(_lib().zcb_cnn_nparams())


def init_params(seed=0):
    """He-scaled random convolution and head weights, zero biases (float32)."""
    rng = np.random.default_rng(seed)
    parts = []
    for l in range(4):
        co, ci = _CH[l + 1], _CH[l]
        parts += [rng.standard_normal(co * 9 * ci) * np.sqrt(2.0 / (9 * ci)), np.zeros(co)]
    parts += [rng.standard_normal(BINS * 128) * np.sqrt(1.0 / 128), np.zeros(BINS)]
    return np.concatenate(parts).astype(np.float32)


def to_bf16(x):
    """float array → BF16 bit patterns (uint16), round to nearest even."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def labels(deg, scale):
    """Bin 9·r + s: r = the rotation's 15° bin from 0°, s = the nearest of 9 log-spaced scales in
    [0.8, 1.25]."""
    deg = np.asarray(deg, np.float64) % 360.0
    r = np.floor(deg / (360.0 / ROT_BINS)).astype(np.int64) % ROT_BINS
    t = (np.log(np.asarray(scale, np.float64)) - np.log(S_MIN)) / (np.log(S_MAX) - np.log(S_MIN))
    s = np.clip(np.round(t * (SCALE_BINS - 1)), 0, SCALE_BINS - 1).astype(np.int64)
    return (r * SCALE_BINS + s).astype(np.int32)


def bin_pose(b):
    """The centre (degrees, scale) of bin b."""
    r, s = divmod(int(b), SCALE_BINS)
    deg = (r + 0.5) * (360.0 / ROT_BINS)
    return deg, float(np.exp(np.log(S_MIN) + s / (SCALE_BINS - 1) * (np.log(S_MAX) - np.log(S_MIN))))


def pair_stacks(pairs, engine=None):
    """[n][128][128][8] BF16 bits: for each (moving, fixed) pair of 128² images (uint16 or float
    in [0, 1]), the engine's four feature planes of each image, moving first."""
    from .engine import Engine

    own = engine is None
    eng = engine or Engine(half=False)
    try:
        out = np.empty((len(pairs), SIDE, SIDE, CHANNELS), np.uint16)
        for i, (m, f) in enumerate(pairs):
            m = np.asarray(m)
            f = np.asarray(f)
            if m.shape != (SIDE, SIDE) or f.shape != (SIDE, SIDE):
                raise ValueError(f"pair_stacks: images must be {SIDE}×{SIDE}")
            g = lambda a: (a / 65535.0 if a.dtype == np.uint16 else a).astype(np.float32)
            eng.set_images(g(m), g(f), preprocess=False)
            st = np.concatenate([eng.features(0), eng.features(1)])  # [8][h][w]
            out[i] = to_bf16(np.transpose(st, (1, 2, 0)))
        return out
    finally:
        if own:
            eng.close()


def _ptrs(params, x):
    params = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.uint16)
    if params.size != nparams():
        raise ValueError(f"expected {nparams()} parameters, got {params.size}")
    if x.ndim != 4 or x.shape[1:] != (SIDE, SIDE, CHANNELS):
        raise ValueError(f"x must be [n][{SIDE}][{SIDE}][{CHANNELS}] BF16 bits")
    f32 = ctypes.POINTER(ctypes.c_float)
    return params, x, params.ctypes.data_as(f32), x.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))


def forward(params, x):
    """logits [n][216]"""
    params, x, pp, xp = _ptrs(params, x)
    out = np.empty((len(x), BINS), np.float32)
    _check(_lib().zcb_cnn_forward(pp, params.size, xp, len(x), out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
    return out


def grad(params, x, y):
    """(mean cross-entropy, its gradient over params)"""
    params, x, pp, xp = _ptrs(params, x)
    y = np.ascontiguousarray(y, np.int32)
    g = np.empty(params.size, np.float32)
    loss = np.zeros(1, np.float32)
    f32 = ctypes.POINTER(ctypes.c_float)
    _check(_lib().zcb_cnn_grad(pp, params.size, xp, y.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(x),
                               loss.ctypes.data_as(f32), g.ctypes.data_as(f32)))
    return float(loss[0]), g


def train(params, x, y, batch=256, steps=1000, lr=1e-3, seed=0):
    """Adam on the GPU over minibatches drawn from (x, y): (params, per-step losses, ms per step)."""
    params, x, pp, xp = _ptrs(np.array(params, np.float32, copy=True), x)
    y = np.ascontiguousarray(y, np.int32)
    losses = np.empty(steps, np.float32)
    ms = np.zeros(1, np.float32)
    f32 = ctypes.POINTER(ctypes.c_float)
    _check(_lib().zcb_cnn_train(pp, params.size, xp, y.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(x), batch,
                                steps, ctypes.c_float(lr), ctypes.c_uint64(seed), losses.ctypes.data_as(f32),
                                ms.ctypes.data_as(f32)))
    return params, losses, float(ms[0])


def top_k_hits(logits, y, k=8):
    """Fraction of samples whose label is among their k highest logits."""
    top = np.argsort(-logits, axis=1)[:, :k]
    return float(np.mean([y[i] in top[i] for i in range(len(y))]))


def _pose_pair(seed):
    """One seeded similarity pair at 128²: rotation uniform in [0°, 360°), scale log-uniform in
    [0.8, 1.25], shift within ±16 px (the 1024² map workload's generator at 128²)."""
    from . import synth

    rng = np.random.default_rng(1_000_003 * (seed + 1))
    deg = float(rng.uniform(0, 360))
    scale = float(np.exp(rng.uniform(np.log(S_MIN), np.log(S_MAX))))
    m, f, H = synth.pair_similarity(n=SIDE, seed=seed, deg=deg, scale=scale)
    return m, f, deg, scale, H


def pose_dataset(seeds, workers=None):
    """(x BF16 stacks, labels, degrees, scales) of the seeded pairs: images generated on the host
    cores (spawned processes), features on the GPU."""
    import multiprocessing as mp
    import os

    workers = workers or max(1, min(16, os.cpu_count() or 1))
    with mp.get_context("spawn").Pool(workers) as pool:
        res = pool.map(_pose_pair, list(seeds), chunksize=32)
    x = pair_stacks([(r[0], r[1]) for r in res])
    deg = np.array([r[2] for r in res])
    sc = np.array([r[3] for r in res])
    return x, labels(deg, sc), deg, sc


def shipped_params():
    """The network trained by this build (zcmir_b200/data/cnn_params.npy)."""
    from pathlib import Path

    return np.load(Path(__file__).resolve().parent / "data" / "cnn_params.npy").astype(np.float32)


def pose_scores(p, xt, yt):
    """Held-out hit rates of params p on stacks xt with labels yt."""
    z = forward(p, xt)
    r_pred = np.argmax(z, 1) // SCALE_BINS
    r_true = yt // SCALE_BINS
    dr = np.minimum((r_pred - r_true) % ROT_BINS, (r_true - r_pred) % ROT_BINS)
    return {"test_top1": float(np.mean(np.argmax(z, 1) == yt)), "test_top8": top_k_hits(z, yt, 8),
            "test_rotation_within_1_bin": float(np.mean(dr <= 1))}


def evaluate_pose(n_train=6000, n_test=500, steps=3000, batch=256, lr=1e-3, seed=0, save=None):
    """Train on n_train seeded pairs, report on n_test held-out pairs: the label's top-1 / top-8
    hit rates, the rotation bin within one bin (either sense), against chance; save: where to
    write the trained parameters (.npy)."""
    import time

    t0 = time.perf_counter()
    x, y, _, _ = pose_dataset(range(seed, seed + n_train))
    xt, yt, _, _ = pose_dataset(range(10_000_000 + seed, 10_000_000 + seed + n_test))
    t_data = time.perf_counter() - t0
    p, losses, ms = train(init_params(seed), x, y, batch=batch, steps=steps, lr=lr, seed=seed + 1)
    if save:
        np.save(save, p)
    z = forward(p, xt)
    zr = forward(p, x[:n_test])
    r_pred = np.argmax(z, 1) // SCALE_BINS
    r_true = yt // SCALE_BINS
    dr = np.minimum((r_pred - r_true) % ROT_BINS, (r_true - r_pred) % ROT_BINS)
    return {
        "train_pairs": n_train, "test_pairs": n_test, "steps": steps, "batch": batch,
        "loss_first_50": float(losses[:50].mean()), "loss_last_50": float(losses[-50:].mean()),
        "ms_per_step": ms, "data_seconds": t_data,
        "train_top1": float(np.mean(np.argmax(zr, 1) == y[:n_test])),
        "test_top1": float(np.mean(np.argmax(z, 1) == yt)), "test_top8": top_k_hits(z, yt, 8),
        "test_rotation_within_1_bin": float(np.mean(dr <= 1)),
        "chance_top1": 1 / BINS, "chance_top8": 8 / BINS, "chance_rotation_within_1_bin": 3 / ROT_BINS,
    }


def search(reg, params=None, k=8, offsets=(-5.0, 0.0, 5.0), keep=4, iters=25):
    """The network's proposal search on the 128² pair loaded in reg: the network reads the pair's
    feature stacks, its k best bins each give len(offsets) seeds (the bin's centre rotation plus
    each offset in degrees, the bin's scale, about the moving centre), each seed is placed by one
    shift map, the `keep` seeds with the highest map peaks are refined together by the batched
    Gauss–Newton (zcb_refine_poses); the best refined pose becomes the pose when it beats the
    current one. Returns dict(H, score, maps)."""
    from . import proposal

    (mw, mh), (fw, fh) = reg.image_size(0), reg.image_size(1)
    if (mw, mh, fw, fh) != (SIDE, SIDE, SIDE, SIDE):
        raise ValueError(f"cnn.search: the network reads pairs of {SIDE}² images")
    p = shipped_params() if params is None else params
    st = np.concatenate([reg.features(0), reg.features(1)])
    z = forward(p, to_bf16(np.transpose(st, (1, 2, 0)))[None])[0]
    cur = reg.score().mean
    seeds, peaks = [], []
    for b in np.argsort(-z)[:k]:
        deg, sc = bin_pose(b)
        for o in offsets:
            H = proposal.candidate_pose(reg, deg + o, sc)
            sm = reg.shift_map(H, want_map=False)
            seeds.append(np.array([[1, 0, -sm.dx], [0, 1, -sm.dy], [0, 0, 1.0]]) @ H)
            peaks.append(sm.peak)
    top = np.argsort(-np.asarray(peaks))[:keep]
    Hs, scores = reg.refine_poses(np.array([seeds[i] for i in top]), iters)
    i = int(np.argmax(scores))
    best_H, best_s = np.asarray(Hs[i]), float(scores[i])
    if best_s > cur + max(1e-6 * abs(cur), 1e-12):
        reg.pose = best_H
    return dict(H=best_H, score=best_s, maps=len(seeds))


def evaluate_search(n_pairs=64, params=None, forms=((4, 4),), seed=30_000_000):
    """The network's search against the plain search (the full 360 × 9 sweep, its screen and
    finalists) on n_pairs held-out 128² pairs on the same GPU: per form the mean seconds per
    search, the share within 0.5 px corner RMS of the planted pose and the share within 0.5 px of
    the plain search's pose. forms: the network search's (k bins, seeds refined)."""
    import time

    from . import proposal
    from .engine import Engine

    p = shipped_params() if params is None else params
    out = {"pairs": n_pairs}
    names = ["plain"] + [f"cnn_k{k}_keep{kp}" for k, kp in forms]
    rows = {n: [] for n in names}
    with Engine(half=False, sw_nth=360, sw_ns=9, sw_smin=S_MIN, sw_smax=S_MAX, sw_grid=SIDE) as reg:
        for j in range(n_pairs):
            m, f, _, _, Ht = _pose_pair(seed + j)
            reg.set_images(m / 65535.0, f / 65535.0, preprocess=False)
            Hp = None
            for name, form in zip(names, [None] + list(forms)):
                reg.pose = np.eye(3)
                reg.score()
                t0 = time.perf_counter()
                if form is None:
                    H = np.asarray(reg.search().H)
                    Hp = H
                else:
                    H = search(reg, p, k=form[0], keep=form[1])["H"]
                dt = time.perf_counter() - t0
                rows[name].append((dt, proposal.corner_rms(H, Ht, SIDE, SIDE), proposal.corner_rms(H, Hp, SIDE, SIDE)))
    for name, r in rows.items():
        a = np.array(r)
        out[name] = {"seconds_per_search": float(a[1:, 0].mean()) if len(a) > 1 else float(a[0, 0]),
                     "within_0_5_px": float(np.mean(a[:, 1] <= 0.5)),
                     "median_corner_rms_px": float(np.median(a[:, 1])),
                     "plain_pose_within_0_5_px": float(np.mean(a[:, 2] <= 0.5))}
    return out


if __name__ == "__main__":
    import argparse
    import json

    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=6000)
    ap.add_argument("--test", type=int, default=500)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--save", default=None)
    ap.add_argument("--search", type=int, default=0, help="compare the searches on this many held-out pairs")
    a = ap.parse_args()
    if a.search:
        print(json.dumps(evaluate_search(a.search, forms=((2, 2), (4, 4), (8, 4)))))
    else:
        print(json.dumps(evaluate_pose(a.train, a.test, a.steps, a.batch, a.lr, save=a.save)))
