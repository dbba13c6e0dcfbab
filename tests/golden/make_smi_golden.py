"""Golden SMI vectors computed by the reference's own NumPy code (examples/03_smi.py).

    python tests/golden/make_smi_golden.py --reference <path of the zcmir checkout>
    (or set ZCMIR_REFERENCE)

examples/03_smi.py is the reference's independent NumPy statement of the SMI path: the 2-px edge
taper and bilinear sampling (``ramp``, ``sample``, :56-80), the 45 overlap sums (``moments``,
:103-109), the score from the sums (``smi``, :124-147), the FFT shift map over ±64 px (:169-188),
the log-polar roto-scale map (:233-262) and the tangent-space gradient (:265-343). It needs the
engine only for the feature planes (``reg.features``) and the roto-scale centre. This script
parses the file with ``ast``, keeps those functions and the statements that compute the map,
the roto-scale map and the gradient (dropping the plotting and every ``reg`` call), and executes
them unchanged on the landsat-b pair of ``landsat_b.npz`` with feature planes made the way the
reference's example makes them (uint8 → RGBA → default CLAHE with f16 texels, laplacian
features, forward direction), by the oracle. The outputs go to ``smi_03_landsat_b.npz``:

- ``m_np``: the 45 sums at the truth; ``score``: ``smi(m_np)``;
- ``curve_dx``, ``curve``: ``smi`` of the sums at T(d, 0)·truth, d = −30..30 step 2 (:151-155);
- ``shift_np``: the 129 × 129 map of lags ±64 at H0 = T(14, −9)·truth, ``shift_peak`` its argmax
  lag (the reference asserts (14, −9), :364);
- ``rs_np`` and ``rs_peak``: the roto-scale map (rotation × log scale lags) at the truth turned
  by 6° and scaled by 1.08 about ``rs_center``, and its peak (degrees, scale);
- ``H2``, ``grad_np``: the pose near the truth and the 8 gradient components (:265-343).

Only the reference's example is executed; nothing of it is copied into this repository.
"""
from __future__ import annotations

import argparse
import ast
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
OUT = HERE / "smi_03_landsat_b.npz"

KEEP_DEFS = ("ramp", "sample", "moments", "smi", "destN", "hat")
# names whose statements only draw or talk to the engine
SKIP_NAMES = {"plt", "ax", "fig", "reg", "print", "zcmir"}


def _names(node):
    return {n.id for n in ast.walk(node) if isinstance(n, ast.Name)}


def _assigns(node, name):
    if isinstance(node, ast.Assign):
        return any(name in _names(t) for t in node.targets)
    return False


def extract(src):
    """(defs, statements): the kept functions, the TRI table and ``shift`` helper, and the
    module-level statements of the three computations, in file order, as compiled code."""
    tree = ast.parse(src)
    body = tree.body
    keep = []
    for node in body:
        if isinstance(node, ast.FunctionDef) and node.name in KEEP_DEFS:
            keep.append(node)
        elif isinstance(node, ast.Assign) and any(isinstance(t, ast.Name) and t.id in ("TRI", "shift")
                                                  for t in node.targets):
            keep.append(node)
    found = {n.name for n in keep if isinstance(n, ast.FunctionDef)}
    missing = set(KEEP_DEFS) - found
    if missing:
        raise SystemExit(f"03_smi.py no longer defines {sorted(missing)}")

    def span(first, last):
        i = next(k for k, n in enumerate(body) if _assigns(n, first))
        j = next(k for k, n in enumerate(body) if k >= i and _assigns(n, last))
        return [n for n in body[i:j + 1] if not (_names(n) & SKIP_NAMES)]

    blocks = {
        "shift": span("H0", "iy"),                 # :169-188
        "rs": span("a6", "peak_np"),              # :233-262, c supplied
        "grad": span("N", "grad_np"),             # :281-343
    }
    mod = lambda nodes: compile(ast.Module(body=nodes, type_ignores=[]), "examples/03_smi.py", "exec")
    return mod(keep), {k: mod(v) for k, v in blocks.items()}


def features(u8, settings):
    """The feature planes the reference's example reads (reg.features): uint8 gray → RGBA → gray
    (zc_set_image_rgba), the default preprocessing, f16 texels, laplacian features."""
    from oracle import preprocess_oracle as P
    from oracle import smi_oracle as O

    rgba = np.concatenate([np.repeat(u8[:, :, None], 3, axis=2), np.full(u8.shape + (1,), 255, np.uint8)], axis=2)
    work = P.bake(P.rgba_gray(rgba), settings)
    return O.prepare(work, "laplacian", half=bool(settings.get("half", True)))


def default_settings():
    import json

    d = json.loads((HERE / "settings_defaults.json").read_text())
    return {k["name"]: k["default"] for k in d["keys"]}


def main(ref):
    sys.path.insert(0, str(ROOT))
    from scipy.linalg import expm
    from scipy.ndimage import map_coordinates

    from oracle import rs_oracle as R

    src = (Path(ref) / "examples" / "03_smi.py").read_text()
    defs, blocks = extract(src)
    d = np.load(HERE / "landsat_b.npz")
    s = default_settings()
    pa, pb = features(d["moving"], s), features(d["fixed"], s)
    truth = d["truth"]
    A, B = pa["feat"], pb["feat"]
    ns = {"np": np, "expm": expm, "map_coordinates": map_coordinates, "A": A, "B": B, "truth": truth}
    ns["hm"], ns["wm"] = A.shape[1:]
    ns["hf"], ns["wf"] = B.shape[1:]
    exec(defs, ns)
    smi, moments, sample, shift = ns["smi"], ns["moments"], ns["sample"], ns["shift"]

    out = {}
    S = sample(truth)
    out["m_np"] = moments(S["va"], B, S["w"])
    out["score"] = np.float64(smi(out["m_np"]))
    dxs = np.arange(-30, 31, 2)
    curve = []
    for dx in dxs:
        Sd = sample(shift(dx, 0) @ truth)
        curve.append(smi(moments(Sd["va"], B, Sd["w"])))
    out["curve_dx"], out["curve"] = dxs, np.array(curve, np.float64)

    exec(blocks["shift"], ns)
    out["H0"] = ns["H0"]
    out["shift_np"] = ns["shift_np"].astype(np.float32)
    L = ns["L"]
    out["shift_peak"] = np.array([ns["ix"] - L, ns["iy"] - L])

    # the roto-scale centre: the engine's, the moving image's centroid under the pose (the oracle's
    # rs_map default, src/engine.zig:831-872)
    c = np.array(R.moving_centroid(truth, pa["w"], pa["h"]))
    ns["c"] = c
    exec(blocks["rs"], ns)
    out["rs_center"], out["H1"] = c, ns["H1"]
    out["rs_np"] = ns["rs_np"].astype(np.float32)
    out["rs_peak"] = np.array(ns["peak_np"], np.float64)

    exec(blocks["grad"], ns)
    out["H2"], out["grad_np"] = ns["H2"], np.asarray(ns["grad_np"], np.float64)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT.name}: score {out['score']:.4f}, shift peak {tuple(out['shift_peak'])}, "
          f"rs peak {out['rs_peak'][0]:.2f} deg x{out['rs_peak'][1]:.4f}, |grad| {np.linalg.norm(out['grad_np']):.4g}")


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=os.environ.get("ZCMIR_REFERENCE"),
                    help="the zcmir checkout (default: $ZCMIR_REFERENCE)")
    a = ap.parse_args()
    if not a.reference:
        ap.error("give --reference or set ZCMIR_REFERENCE")
    main(a.reference)
