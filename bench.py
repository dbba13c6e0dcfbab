"""SMI shift-map throughput on B200: maps/s for the 1024² pair (2048² FFT, 45 correlations).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One step = one full shift map of the pair at the identity pose (canvas → both sides' real planes
→ forward FFTs → 45 correlation products → inverse FFTs → per-shift exact, calibrated score →
argmax), the images' features resident in HBM. Device time per step is taken with CUDA events
on the engine's stream, W untimed steps first, an L2 flush (a 256 MB write) between timed steps
outside the timed spans. `e2e` is the same metric through the public API (Engine.set_images
from pinned host buffers + Engine.shift_map copying the map back to pinned host memory).

The path does not shard (one map needs all 45 correlations of every shift): N GPUs run N
independent replicas, one process each (torchrun), and `value` is the maps/s of all ranks, timed
as the slowest rank.

The line also carries `sweep`: the rotation × scale sweep of a 512² pair (360 rotations × 9
scales = 3240 candidate maps on a 128² canvas) as poses/s (candidate maps per second, device
time of the batched maps), its `e2e` (set_images + search from host images: sweep, NMS, batched
Gauss–Newton screen and finalists, as searches/s) and a CPU baseline on a sample of 90 candidates.

And `stack`: 32 slices of 384–1024 px, each a drifting similarity of the previous one, mapped
slice against predecessor (features once per slice, 31 maps) as maps/s.

--impl reference: the CPU restatement of the reference's path (the oracle, float64, scipy FFTs on
all host cores) on the same pair; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SMI maps/s at 1024²"
WORKLOAD = "smi_shift_map_1024_fft2048"


def config(extra=None):
    c = {"workload": WORKLOAD, "image": [1024, 1024], "fft": [2048, 2048], "correlations": 45,
         "smi_features": "laplacian", "exact": True, "calibrated": True, "pose": "identity",
         "pair": "blob field vs 8-level segmented modality, seeded shift in ±200 px (seed 1)",
         "l2": "256 MB flush between timed steps (per-step working set 1.3 GB > 126 MB L2)"}
    if extra:
        c.update(extra)
    return c


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return int(os.environ.get("RANK", "0")), ws, int(os.environ.get("LOCAL_RANK", "0"))


def smi_id(local):
    """nvidia-smi's name for CUDA device `local` (its UUID; the CUDA index can differ from
    nvidia-smi's when CUDA_VISIBLE_DEVICES is set)."""
    try:
        import torch

        u = str(torch.cuda.get_device_properties(local).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        return ids[local] if local < len(ids) else str(local)


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons while the timed region runs."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local, interval_ms=20):
        self.index, self.interval, self.lines, self.p, self.first = smi_id(local), interval_ms, [], None, 0

    def _read(self):
        for ln in self.p.stdout:
            self.lines.append(ln)

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", str(self.interval)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the timed region starts once the sampler runs; earlier samples are not counted
            t0 = time.time()
            while not self.lines and time.time() - t0 < 10 and self.p.poll() is None:
                time.sleep(0.005)
            self.first = len(self.lines)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            self.p.wait(timeout=10)
            self.t.join(timeout=5)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines[self.first:]:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 6:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[2:6]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def stage_bytes(p):
    """Algorithmic bytes of each stage of one map (one launch of that kernel per side where it
    runs per side): its compulsory reads and writes in this decomposition."""
    nx, ny, cw, ch, P, C = p["nx"], p["ny"], p["cw"], p["ch"], p["n_real"], p["n_corr"]
    half = (nx // 2 + 1) * 8
    return {
        "canvas": 2 * (5 * p["canvas_w"] * p["canvas_h"] * 4) * 2,
        "fwd_rows": 2 * (5 * cw * ch * 4 + P * ch * half),
        "fwd_cols": 2 * (P * ch * half + P * ny * half),
        "inv_cols": 2 * P * ny * half + C * ny * half,
        "inv_rows_score": C * ny * half + nx * ny * 4,
    }


def reuse_maps(reg, torch, args):
    """Maps through the public call (features resident, map left on the device) when a side's
    spectra are still in place: the moving image turned and shrunk about its centre so it stays
    inside the fixed frame (the fixed side's canvas and spectra reused, the moving side's rebuilt
    at every new pose), and the calibrated map right after the uncalibrated one at one pose (both
    sides reused). Wall time per map, each call synchronised; not the headline, which rebuilds
    both sides in every timed map."""
    c = 512.5
    T = lambda x, y: np.array([[1, 0, x], [0, 1, y], [0, 0, 1.0]])

    def pose(k):
        a, s = np.deg2rad(0.2 * (k % 7 + 1)), 0.97 - 0.001 * (k % 5)
        return T(c, c) @ np.array([[s * np.cos(a), -s * np.sin(a), 0], [s * np.sin(a), s * np.cos(a), 0], [0, 0, 1]]) @ T(-c, -c)

    n = max(5, args.steps // 2)
    for k in range(3):
        reg.shift_map(pose(k), exact=True, calibrated=True, cap=2048, want_map=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(n):
        reg.shift_map(pose(k + 3), exact=True, calibrated=True, cap=2048, want_map=False)
    fixed_s = (time.perf_counter() - t0) / n
    both_s = 0.0
    for k in range(n):
        reg.shift_map(pose(100 + k), exact=True, calibrated=False, cap=2048, want_map=False)
        t1 = time.perf_counter()
        reg.shift_map(pose(100 + k), exact=True, calibrated=True, cap=2048, want_map=False)
        both_s += time.perf_counter() - t1
    both_s /= n
    return {"fixed_side_reused_maps_s": 1.0 / fixed_s, "both_sides_reused_maps_s": 1.0 / both_s,
            "timing": "wall clock per synchronised shift_map call, map not copied back"}


def sweep_work(tuned, Fx, Fy):
    """(bytes, flops) of one whole sweep: per candidate of plane nx × ny (window cw × ch = nx − Fx + 1
    × ny − Fy + 1, P = 15 real planes, C = 45 correlations) the bytes each pass reads and writes once
    (pack → window stacks, forward rows → half spectra, columns in place, inverse columns → the
    correlations' spectra, rows → map, peaks ← map) and the FP32 flops of the survey's counting rule
    (moving side's forward FFT over its rows and columns, 23 inverse 2-D FFTs, products, score)."""
    P, C, NC = 15, 45, 8
    total_b = total_f = 0.0
    for r in tuned:
        nx, ny, k = r["nx"], r["ny"], r["candidates"]
        cw, ch = nx - Fx + 1, ny - Fy + 1
        half = (nx // 2 + 1) * 8
        win = 5 * cw * ch * 4
        b = (win + (win + P * ch * half) + (P * ch * half + P * ny * half) + (P * ny * half + C * ny * half)
             + (C * ny * half + nx * ny * 4) + nx * ny * 4)
        lx, ly = np.log2(nx), np.log2(ny)
        f = (NC * 5 * (nx * lx * ch + ny * ly * nx) + ((C + 1) // 2) * 5 * nx * ny * np.log2(nx * ny)
             + 10 * C * nx * ny + 300 * nx * ny)
        total_b += k * b
        total_f += k * f
    return total_b, total_f


def survey_bytes(p):
    """The whole map's compulsory HBM bytes (both stacks read, both sides' half spectra written and
    read once, the map written)."""
    nx, ny, P = p["nx"], p["ny"], p["n_real"]
    return 2 * 5 * p["canvas_w"] * p["canvas_h"] * 4 + 2 * (2 * P * nx * (ny // 2 + 1) * 8) + nx * ny * 4


def survey_flops(p):
    """The whole map's FP32 flops by the survey's counting rule: both sides' forward FFTs over the
    canvas rows and all columns (packed complex lines), the inverse 2-D FFTs of the packed
    correlations, the conjugate products and about 300 flops of scoring per shift."""
    nx, ny, ch, P, C = p["nx"], p["ny"], p["ch"], p["n_real"], p["n_corr"]
    lx, ly = np.log2(nx), np.log2(ny)
    fwd = 2 * ((P + 1) // 2) * 5 * (nx * lx * ch + ny * ly * nx)
    inv = ((C + 1) // 2) * 5 * nx * ny * np.log2(nx * ny)
    return float(fwd + inv + 10 * C * nx * ny + 300 * nx * ny)


def fp32_peak_tflops():
    """The device's FMA rate measured now by zcb_fp32_peak (TFLOP/s), or None."""
    import ctypes

    from zcmir_b200 import _native

    t = ctypes.c_double(0.0)
    return t.value if _native.load().zcb_fp32_peak(ctypes.byref(t)) == 0 else None


def cpu_map_seconds(m, f):
    """One map of the pair by the CPU restatement (float64; scipy FFTs on every host core)."""
    import scipy.fft as sf

    from oracle import smi_oracle as O

    t0 = time.perf_counter()
    pa, pb = O.prepare(m), O.prepare(f)
    t1 = time.perf_counter()
    ga, gb, (nx, ny, cw, ch), (ox, oy, W, Hh) = O.grid_stacks(pa, pb, np.eye(3), cap=2048)
    ids, corrs = O.corr_plan(True, False)
    A, B = O.real_planes(ga, ids), O.real_planes(gb, ids)
    w = os.cpu_count()
    FA = {p: sf.rfft2(A[k], (ny, nx), workers=w) for k, p in enumerate(ids)}
    FB = {p: sf.rfft2(B[k], (ny, nx), workers=w) for k, p in enumerate(ids)}
    corr = np.zeros((45, ny, nx))
    for a, b, c in corrs:
        corr[c] = sf.irfft2(FA[a] * np.conj(FB[b]), (ny, nx), workers=w)
    area = max(1.0, O.pair_area(pa["acf"], pb["acf"]))
    mp = O.combine(corr, True, True, 12, area)
    O.argmax_first(mp)
    t2 = time.perf_counter()
    return t2 - t1, t1 - t0


def make_pair():
    from zcmir_b200 import synth

    m, f, H = synth.pair_segmented(n=1024, seed=1)
    return (m / 65535.0).astype(np.float32), (f / 65535.0).astype(np.float32), H


SWEEP_SETTINGS = dict(half=False, sw_nth=360, sw_ns=9, sw_smin=0.8, sw_smax=1.25, sw_grid=128)
SWEEP_CONFIG = {"workload": "smi_sweep_512_rot360x9_grid128", "image": [512, 512], "candidates": 3240,
                "rotations": "0-359 deg, 1 deg steps", "scales": "9 log-spaced in [0.8, 1.25]", "grid": 128,
                "pair": "blob field vs 8-level segmented modality under a seeded similarity (seed 2)",
                "l2": "per-sweep working set ~1.3 GB per batch of candidates > 126 MB L2"}


def sweep_cpu_sample(m, f, n_sample=90):
    """Poses/s of the float64 oracle on an evenly spaced sample of the sweep's candidates."""
    from oracle import smi_oracle as O
    from oracle import sweep_oracle as S

    pa, pb = O.prepare(m), O.prepare(f)
    gv = S.sweep_grid(n_theta=360, n_sigma=9, s_min=0.8, s_max=1.25)
    nc = 360 * 9
    only = set(range(0, nc, nc // n_sample))
    t0 = time.perf_counter()
    S.sweep(pa, pb, np.eye(3), gv, G=128, exact=True, only=only)
    return len(only) / (time.perf_counter() - t0), len(only)


def run_sweep(reg_cls, args, barrier, dist, torch, ws):
    """The c3 sweep: 3240 candidate maps per step, device-timed (zcb_sweep), then search end to end
    through the public API from host images."""
    from zcmir_b200 import synth

    m16, f16, H = synth.pair_similarity(n=512, seed=2)
    m, f = (m16 / 65535.0).astype(np.float32), (f16 / 65535.0).astype(np.float32)
    reg = reg_cls(**SWEEP_SETTINGS)
    reg.set_images(m, f, preprocess=False)
    # the batch of every plane class chosen by the engine's autotuner (timed here, untimed below)
    tuned = reg.tune_sweep()
    # N > 1: the candidates split across the ranks (strong scaling of one sweep)
    shard, nshard = (dist.get_rank(), ws) if dist else (0, 1)
    for _ in range(args.warmup):
        reg.sweep(n_peak=4, shard=shard, nshard=nshard)
    barrier()
    with Clocks(torch.cuda.current_device()) as clk:
        ms = [reg.sweep(n_peak=4, shard=shard, nshard=nshard).info["ms"] for _ in range(args.steps)]
    barrier()
    ms_step = float(np.mean(ms))
    info = reg.sweep(n_peak=4, shard=shard, nshard=nshard).info
    if dist:
        t = torch.tensor([ms_step], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_step = float(t.item())
    # e2e: the images from host memory, features, sweep, NMS, Gauss–Newton screen and finalists
    if dist:
        from zcmir_b200 import parallel

        search = lambda: parallel.sharded_search(reg)
    else:
        search = reg.search
    for _ in range(max(1, args.warmup // 2)):
        reg.set_images(m, f, preprocess=False)
        reg.pose = np.eye(3)
        search()
    barrier()
    t0 = time.perf_counter()
    n_e2e = max(3, args.steps // 5)
    for _ in range(n_e2e):
        reg.set_images(m, f, preprocess=False)
        reg.pose = np.eye(3)
        r = search()
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / n_e2e
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    corner = 0.0
    for x, y in [(1, 1), (512, 1), (512, 512), (1, 512)]:
        a, b = r.H @ [x, y, 1.0], H @ [x, y, 1.0]
        corner = max(corner, float(np.hypot(*(a[:2] / a[2] - b[:2] / b[2]))))
    sb, sf = sweep_work(tuned, int(info["Fx"]), int(info["Fy"]))
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = peaks.get("hbm_gbs") or 6650.0
    achieved = sb / nshard / (ms_step * 1e-3) / 1e9
    out = {"metric": "sweep poses/s", "value": info["candidates"] / (ms_step * 1e-3), "unit": "poses/s",
           "ms_per_step": ms_step, "scaling": "strong",
           "tuned": [{k: r[k] for k in ("nx", "ny", "candidates", "batch", "ms_per_map")} for r in tuned],
           "timing": "CUDA events around one replay of the sweep's captured CUDA graph",
           "roofline": {"bound": "hbm", "kernel": "all sweep passes", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                        "frac": achieved / hbm, "traffic": None,
                        "algorithmic_bytes_per_sweep": sb,
                        "what": "bytes every pass of this decomposition reads and writes once per candidate "
                                "(window stacks, half spectra, correlation spectra, maps), summed over the 3240",
                        "peak_source": "measured" if peaks.get("hbm_gbs") else "fallback",
                        "fp32_flops_per_sweep": sf, "fp32_tflops": sf / nshard / (ms_step * 1e-3) / 1e12,
                        "fp32_frac_of_nominal_75_tflops": sf / nshard / (ms_step * 1e-3) / 75e12},
           "config": dict(SWEEP_CONFIG, parallelism=f"candidates split over {ws} GPU(s), lane peaks all-reduced"),
           "launches_per_step": int(info["launches"]), "clocks": clk.summary(), "plane_sizes": int(info["groups"]), "batches": int(info["batches"]),
           "e2e": {"value": 1.0 / e2e_s, "unit": "searches/s", "seconds_per_search": e2e_s,
                   "h2d_bytes_per_step": int(m.nbytes + f.nbytes), "d2h_bytes_per_step": 104,
                   "what": "set_images + search (sweep, NMS, 4-step batched Gauss-Newton screen, 25-step finalists)",
                   "corner_error_px": corner}}
    reg.close()
    return out, m, f


def run_proposal(reg_cls, m, f, H, reps=3):
    """The learned proposal beside the plain search on the sweep's 512² pair, images loaded: the
    plain search (360 × 9 sweep), the coarse search (36 × 3 sweep, no network) and the proposal
    search (36 × 3 sweep, the shipped network's top 4 cells refined); per search its wall time,
    shift maps and corner error against the planted pose."""
    from zcmir_b200 import proposal as P

    net = P.Network.load()
    reg = reg_cls(**SWEEP_SETTINGS)
    reg.set_images(m, f, preprocess=False)
    mh, mw = m.shape
    out = {}
    for name in ("plain", "coarse", "proposal"):
        ts = []
        for _ in range(reps + 1):
            reg.pose = np.eye(3)
            t0 = time.perf_counter()
            fb = False
            if name == "plain":
                Hs, maps = P._with(reg, P.fine_settings(), reg.search).H, P.FINE_NTH * P.FINE_NS
            else:
                r = P.search(reg, net, with_network=name == "proposal")
                Hs, maps, fb = r["H"], r["maps"], r["fallback"]
            ts.append(time.perf_counter() - t0)
        out[name] = {"seconds_per_search": float(np.mean(ts[1:])), "maps": maps, "plain_sweep_fallback": fb,
                     "corner_rms_px": P.corner_rms(np.asarray(Hs), H, mw, mh)}
    reg.close()
    return out


STACK_CONFIG = {"workload": "smi_stack_32_slices_384_1024", "slices": 32,
                "sizes": "per side uniform in [384, 1024] (seed 3)",
                "drift": "per step rotation N(0, 2 deg), log scale N(0, 0.02), shift N(0, 8 px)",
                "maps": "slice k (moving) against slice k-1 (fixed), centres aligned, exact, uncalibrated, cap 1024",
                "modalities": "alternating blob field / 1 - field^2"}


def run_stack(reg_cls, args, barrier, dist, torch, ws):
    """The stack: features of every slice once, then 31 maps, device-timed (zcb_stack_maps); e2e
    the same call from host slices."""
    from zcmir_b200 import synth

    slices, truths = synth.stack_drift(n=32, seed=3)
    imgs = [(s / 65535.0).astype(np.float32) for s in slices]
    reg = reg_cls(half=False)
    for _ in range(args.warmup):
        reg.stack_maps(imgs, exact=True, calibrated=False, cap=1024)
    barrier()
    t0 = time.perf_counter()
    n_steps = max(3, args.steps // 5)
    ms = []
    for _ in range(n_steps):
        maps, m = reg.stack_maps(imgs, exact=True, calibrated=False, cap=1024)
        ms.append(m)
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / n_steps
    ms_step = float(np.mean(ms))
    if dist:
        t = torch.tensor([ms_step, e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_step, e2e_s = float(t[0].item()), float(t[1].item())
    # translation error of each pair's map (the drift's rotation and scale stay in the residual)
    errs = []
    for k, (sm, H) in enumerate(zip(maps, truths)):
        h, w = imgs[k + 1].shape
        c = np.array([(w + 1) / 2, (h + 1) / 2, 1.0])
        P = np.array([[1, 0, (imgs[k].shape[1] - w) / 2 - sm.dx], [0, 1, (imgs[k].shape[0] - h) / 2 - sm.dy], [0, 0, 1.0]])
        a, b = P @ c, H @ c
        errs.append(float(np.hypot(*(a[:2] / a[2] - b[:2] / b[2]))))
    out = {"metric": "stack maps/s", "value": ws * 31 / (ms_step * 1e-3), "unit": "maps/s", "ms_per_step": ms_step,
           "config": dict(STACK_CONFIG, parallelism=f"replicas{ws}"),
           "centre_error_px": {"median": float(np.median(errs)), "max": float(np.max(errs))},
           "e2e": {"value": ws * 31 / e2e_s, "unit": "maps/s", "seconds_per_stack": e2e_s,
                   "h2d_bytes_per_step": int(sum(a.nbytes for a in imgs)), "d2h_bytes_per_step": 31 * 88,
                   "what": "Engine.stack_maps from host slices: 32 uploads, 32 feature builds, 31 maps"}}
    reg.close()
    return out, imgs


def run_sweep_stack(reg_cls, args, m, f, imgs, sweep_ms, stack_ms):
    """The sweep's 3240 candidate maps and the stack's 31 maps as two branches of one CUDA graph,
    launched once per step (zcb_stack_load once, then zcb_sweep_stack), device-timed; beside it
    the two run one after the other (the sweep leg's and the stack leg's device times; the stack's
    includes its 32 feature builds, which the combined launch does not repeat)."""
    reg = reg_cls(**SWEEP_SETTINGS)
    reg.set_images(m, f, preprocess=False)
    reg.tune_sweep()
    reg.stack_load(imgs, exact=True, calibrated=False, cap=1024)
    for _ in range(args.warmup):
        reg.sweep_stack(n_peak=4)
    ms, launches = [], 0
    for _ in range(max(3, args.steps // 5)):
        sw, st = reg.sweep_stack(n_peak=4)
        ms.append(sw.info["ms"])
        launches = int(sw.info["launches"])
    reg.close()
    ms_step = float(np.mean(ms))
    return {"metric": "sweep candidates + stack maps per second, one launch", "unit": "maps/s",
            "value": (3240 + 31) / (ms_step * 1e-3), "ms_per_step": ms_step,
            "kernels_per_launch": launches, "graph_launches_per_step": 1,
            "sweep_alone_ms": sweep_ms, "stack_alone_ms_with_features": stack_ms,
            "timing": "CUDA events around one replay of the combined graph (sweep branch, stack branch)",
            "config": {"workload": "smi_sweep_512_rot360x9 + smi_stack_32_slices_384_1024 in one graph"}}


def stack_cpu_sample(imgs, pairs=2):
    """Maps/s of the float64 oracle on the first pairs of the stack (features included)."""
    from oracle import smi_oracle as O

    t0 = time.perf_counter()
    preps = [O.prepare(a) for a in imgs[:pairs + 1]]
    for k in range(1, pairs + 1):
        h, w = imgs[k].shape
        H = np.array([[1, 0, (imgs[k - 1].shape[1] - w) / 2], [0, 1, (imgs[k - 1].shape[0] - h) / 2], [0, 0, 1.0]])
        O.shift_map(preps[k], preps[k - 1], H, exact=True, calibrated=False, cap=1024)
    return pairs / (time.perf_counter() - t0), pairs


def run_reference(args, rank):
    if rank != 0:
        return
    m, f, _ = make_pair()
    for _ in range(args.warmup):
        cpu_map_seconds(m, f)
    ts = [cpu_map_seconds(m, f)[0] for _ in range(args.steps)]
    sec = float(np.mean(ts))
    v = 1.0 / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "maps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * sec, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config(),
        "cpu_baseline": {"value": v, "unit": "maps/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": "one full 1024² map per step (features excluded, as on the GPU)"},
        "e2e": {"value": v, "unit": "maps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_gpu(args, rank, ws, local):
    import torch

    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    import zcmir_b200 as zc

    m, f, H = make_pair()
    reg = zc.Engine(half=False)
    reg.set_images(m, f, preprocess=False)
    sm = reg.shift_map(np.eye(3), exact=True, calibrated=True, cap=2048)
    assert (sm.dx, sm.dy) == (-H[0, 2], -H[1, 2]), (sm.dx, sm.dy, H)

    # device-timed maps: the 45-correlation workload, and the 28-correlation ("none") one
    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    barrier()
    reg.gpu_counts()
    with Clocks(local) as clk:
        r = reg.bench_maps(np.eye(3), flags=3, cap=2048, warmup=args.warmup, steps=args.steps)
    launches = reg.gpu_counts()["launches"]
    barrier()
    ms = r["ms_per_map"]
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    reg.configure(smi_features="three")
    r28 = reg.bench_maps(np.eye(3), flags=3, cap=2048, warmup=1, steps=max(3, args.steps // 2))
    reg.configure(smi_features="laplacian")
    reuse = reuse_maps(reg, torch, args)

    # e2e: the public API from pinned host buffers, map back into pinned host memory
    pm = torch.empty(m.shape, dtype=torch.float32, pin_memory=True).numpy()
    pf = torch.empty(f.shape, dtype=torch.float32, pin_memory=True).numpy()
    pm[:] = m
    pf[:] = f
    out = torch.empty(2048 * 2048, dtype=torch.float32, pin_memory=True).numpy()
    for _ in range(args.warmup):
        reg.set_images(pm, pf, preprocess=False)
        reg.shift_map(np.eye(3), exact=True, calibrated=True, cap=2048, out=out)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        reg.set_images(pm, pf, preprocess=False)
        e = reg.shift_map(np.eye(3), exact=True, calibrated=True, cap=2048, out=out)
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    assert (e.dx, e.dy) == (sm.dx, sm.dy)

    line = None
    if rank == 0:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
        hbm = peaks.get("hbm_gbs")
        peak_kind = "measured" if hbm else "fallback"
        hbm = hbm or 6650.0
        sb = stage_bytes(r)
        top = max(r["stages_ms"], key=r["stages_ms"].get)
        launches_of = {"canvas": 1, "fwd_rows": 2, "fwd_cols": 2, "inv_cols": 1, "inv_rows_score": 1}
        t_launch = r["stages_ms"][top] / launches_of[top]
        b_launch = sb[top] / launches_of[top]
        achieved = b_launch / (t_launch * 1e-3) / 1e9
        traffic = None
        tf = ROOT / "profiles" / "traffic.json"
        if tf.exists():
            traffic = json.loads(tf.read_text()).get(top)
        fp32 = fp32_peak_tflops()
        line = {
            "metric": METRIC, "value": ws * 1000.0 / ms, "unit": "maps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config({"parallelism": f"replicas{ws}", "none_28_correlations_maps_s": ws * 1000.0 / r28["ms_per_map"],
                              "plan": {k: r[k] for k in ("nx", "ny", "cw", "ch", "n_real", "n_corr", "split")},
                              "stages_ms": r["stages_ms"],
                              "timing": "CUDA events around replays of one captured CUDA graph of the map's passes; "
                                        "stages_ms from event-instrumented maps",
                              "ms_per_map_instrumented": r.get("ms_per_map_instrumented"),
                              "spectra_reuse": reuse}),
            "roofline": {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of this kernel from a capture "
                                           "of an earlier run of this command (profiles/traffic.json), not measured by this run",
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": b_launch, "launch_ms": t_launch,
                         "map_algorithmic_bytes": survey_bytes(r),
                         "map_frac": survey_bytes(r) / (ms * 1e-3) / 1e9 / hbm,
                         "map_fp32": {"flops_per_map": survey_flops(r),
                                      "tflops": survey_flops(r) / (ms * 1e-3) / 1e12,
                                      "peak_tflops": fp32, "peak_source": "measured in this run (zcb_fp32_peak)",
                                      "frac": (survey_flops(r) / (ms * 1e-3) / 1e12 / fp32) if fp32 else None}},
            "e2e": {"value": ws / e2e_s, "unit": "maps/s", "h2d_bytes_per_step": int(pm.nbytes + pf.nbytes),
                    "d2h_bytes_per_step": int(2048 * 2048 * 4 + 88)},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        if ws == 1 and not args.no_cpu:
            sec, _ = cpu_map_seconds(m, f)
            line["cpu_baseline"] = {"value": 1.0 / sec, "unit": "maps/s", "cores": os.cpu_count(), "kind": "port",
                                    "sample": "one full 1024² map of the same pair (float64 oracle, scipy FFTs)"}
    reg.close()
    sweep, sm_, sf_ = run_sweep(zc.Engine, args, barrier, dist, torch, ws)
    stack, st_imgs = run_stack(zc.Engine, args, barrier, dist, torch, ws)
    from zcmir_b200 import synth

    proposal = run_proposal(zc.Engine, sm_, sf_, synth.pair_similarity(n=512, seed=2)[2])
    both = run_sweep_stack(zc.Engine, args, sm_, sf_, st_imgs, sweep["ms_per_step"], stack["ms_per_step"])
    if rank == 0:
        if ws == 1 and not args.no_cpu:
            v, n = sweep_cpu_sample(sm_, sf_)
            sweep["cpu_baseline"] = {"value": v, "unit": "poses/s", "cores": os.cpu_count(), "kind": "port",
                                     "sample": f"{n} evenly spaced candidates of the 3240 (float64 oracle, numpy FFTs)"}
        line["sweep"] = sweep
        if ws == 1 and not args.no_cpu:
            v, n = stack_cpu_sample(st_imgs)
            stack["cpu_baseline"] = {"value": v, "unit": "maps/s", "cores": os.cpu_count(), "kind": "port",
                                     "sample": f"the first {n} pairs of the stack, features included (float64 oracle)"}
        line["stack"] = stack
        line["sweep_stack"] = both
        line["proposal"] = proposal
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    rank, ws, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank)
        return
    run_gpu(args, rank, ws, local)


if __name__ == "__main__":
    main()
