"""Regenerate the golden fixtures in this folder from the reference tree (ZacharyVarley/zcmir).

    python tests/golden/make_golden.py --reference /path/to/zcmir   (or set ZCMIR_REFERENCE)

Run once where the reference is checked out; the fixtures it writes are committed, and
nothing at test time reads the reference tree.

* ``abi.json``: the 52 ``zc_*`` names the reference's ctypes loader binds with their argument
  and result types (``python/zcmir/_native.py:79-133``), and the byte layout of every result
  struct (``python/zcmir/_native.py:14-62``), read by importing that module (it loads no
  library at import time).
* ``settings_defaults.json``: every settings key with its default and type, and the enum
  value sets, parsed from ``src/settings.zig:14-154`` and the enums it names
  (``src/moments.zig:13``, ``src/lie.zig:9``, ``src/fft.zig:17``).
* ``landsat_b.npz``: the landsat-b preset pair (gray uint8, as ``python/zcmir/examples.py:36-44``
  loads it) and its known pose from ``web/app/presets/presets.json``; the fixture of the
  known-answer checks of ``examples/03_smi.py:362-366``.
"""
import ctypes
import importlib.util
import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _ctype_name(t):
    if t is None:
        return "void"
    if isinstance(t, type) and issubclass(t, ctypes._Pointer):
        return "ptr:" + _ctype_name(t._type_)
    if isinstance(t, type) and issubclass(t, ctypes.Array):
        return f"{_ctype_name(t._type_)}[{t._length_}]"
    return t.__name__


def abi(ref):
    spec = importlib.util.spec_from_file_location("_zc_native_ref", ref / "python/zcmir/_native.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    sigs = {name: {"args": [_ctype_name(a) for a in args], "res": _ctype_name(res)} for name, (args, res) in mod._SIGS.items()}
    structs = {}
    for name in ("ShiftResult", "RsResult", "GradResult", "ClimbResult", "DetectResult", "MatchResult", "SearchResult", "Canvas"):
        S = getattr(mod, name)
        structs[name] = {
            "size": ctypes.sizeof(S),
            "fields": [[f, getattr(S, f).offset, getattr(S, f).size] for f, _ in S._fields_],
        }
    return {"symbols": sigs, "structs": structs}


def _enum(text, name):
    m = re.search(r"pub const " + name + r"\s*=\s*enum(?:\([a-z0-9]+\))?\s*\{([^}]*)\}", text)
    return [v.strip().split("=")[0].strip() for v in m.group(1).split(",") if v.strip()]


def settings(ref):
    st = (ref / "src/settings.zig").read_text()
    enums = {
        "Metric": _enum(st, "Metric"), "Detector": _enum(st, "Detector"), "MatchMethod": _enum(st, "MatchMethod"),
        "SearchMode": _enum(st, "SearchMode"),
        "mom.SmiFeatures": _enum((ref / "src/moments.zig").read_text(), "SmiFeatures"),
        "lie.Group": _enum((ref / "src/lie.zig").read_text(), "Group"),
        "fft.Sizes": _enum((ref / "src/fft.zig").read_text(), "Sizes"),
    }
    body = st[st.index("pub const Settings = struct {"):]
    body = body[: body.index("pub fn family")]
    keys = []
    for line in body.splitlines():
        m = re.match(r"\s*([a-z_0-9]+):\s*([A-Za-z0-9_.]+)\s*=\s*([^,]+),\s*$", line)
        if not m:
            continue
        name, typ, dflt = m.groups()
        if typ == "bool":
            val = dflt.strip() == "true"
        elif typ in ("u32",):
            val = int(dflt)
        elif typ == "f64":
            val = float(dflt)
        elif typ in enums:
            val = dflt.strip().lstrip(".")
            assert val in enums[typ], (name, val)
        else:
            raise ValueError(f"unhandled type {typ} of {name}")
        keys.append({"name": name, "type": typ if typ in ("bool", "u32", "f64") else "enum:" + typ, "default": val})
    return {"keys": keys, "enums": enums}


def landsat_b(ref):
    from PIL import Image

    root = ref / "web/app/presets"
    info = next(p for p in json.loads((root / "presets.json").read_text())["presets"] if p["id"] == "landsat-b")
    img = lambda f: np.asarray(Image.open(root / f).convert("L"))
    np.savez_compressed(HERE / "landsat_b.npz", moving=img(info["moving"]), fixed=img(info["fixed"]),
                        truth=np.array(info["truth"], np.float64))


def main(ref):
    ref = Path(ref)
    (HERE / "abi.json").write_text(json.dumps(abi(ref), indent=1) + "\n")
    (HERE / "settings_defaults.json").write_text(json.dumps(settings(ref), indent=1) + "\n")
    landsat_b(ref)


if __name__ == "__main__":
    import argparse
    import os

    ap = argparse.ArgumentParser(description="ABI, settings and landsat-b fixtures from the reference's sources")
    ap.add_argument("--reference", default=os.environ.get("ZCMIR_REFERENCE"),
                    help="the zcmir checkout (default: $ZCMIR_REFERENCE)")
    a = ap.parse_args()
    if not a.reference:
        ap.error("give --reference or set ZCMIR_REFERENCE")
    main(a.reference)
