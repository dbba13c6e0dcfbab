"""The C-ABI library: it loads, exports every name the reference's loader binds and every name
include/*.h declares, and its struct layouts match the reference's. No GPU compute."""
import ctypes
import json
import re
from pathlib import Path

import pytest

from zcmir_b200 import _native

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def lib():
    return _native.load()


def test_reference_symbols_exported(lib, golden):
    abi = json.loads((golden / "abi.json").read_text())
    missing = [n for n in abi["symbols"] if not hasattr(lib, n)]
    assert not missing, missing
    assert len(abi["symbols"]) == 52


def test_header_symbols_exported(lib):
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        names |= set(re.findall(r"\b(zcb?_[a-z0-9_]+)\s*\(", h.read_text()))
    assert len(names) >= 55
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts(lib, golden):
    abi = json.loads((golden / "abi.json").read_text())
    ours = {"ShiftResult": _native.ShiftResult, "RsResult": _native.RsResult, "GradResult": _native.GradResult,
            "ClimbResult": _native.ClimbResult, "SearchResult": _native.SearchResult, "Canvas": _native.Canvas}
    for name, S in ours.items():
        ref = abi["structs"][name]
        assert ctypes.sizeof(S) == ref["size"], name
        assert [[f, getattr(S, f).offset, getattr(S, f).size] for f, _ in S._fields_] == ref["fields"], name
    out = (ctypes.c_uint32 * 4)()
    lib.zc_result_sizes(out)
    assert list(out)[:3] == [abi["structs"]["ShiftResult"]["size"], abi["structs"]["RsResult"]["size"],
                             abi["structs"]["GradResult"]["size"]]


def test_version(lib):
    assert lib.zc_version() == b"0.1.4"


def _apply(lib, obj):
    j = json.dumps(obj).encode() if not isinstance(obj, bytes) else obj
    out, err = ctypes.create_string_buffer(16384), ctypes.create_string_buffer(1024)
    ol, el = ctypes.c_size_t(), ctypes.c_size_t()
    rc = lib.zcb_settings_apply(j, len(j), out, 16384, ctypes.byref(ol), err, 1024, ctypes.byref(el))
    return rc, (json.loads(out.raw[: ol.value]) if rc == 0 else err.raw[: el.value].decode())


def test_settings_defaults_match_reference(lib, golden):
    ref = json.loads((golden / "settings_defaults.json").read_text())
    rc, s = _apply(lib, {})
    assert rc == 0
    assert list(s) == [k["name"] for k in ref["keys"]]
    for k in ref["keys"]:
        v = s[k["name"]]
        if k["type"] == "f64":
            assert isinstance(v, float) and v == k["default"], k
        else:
            assert v == k["default"] and type(v) is type(k["default"]), k


def test_settings_apply_and_errors(lib, golden):
    rc, s = _apply(lib, {"metric": "e4", "g_iters": 5, "symmetric": False, "group": "affine", "min_overlap": 1})
    assert rc == 0 and s["metric"] == "e4" and s["g_iters"] == 5 and s["symmetric"] is False
    assert s["group"] == "affine" and s["min_overlap"] == 1.0
    rc, m = _apply(lib, {"nope": 1})
    assert rc == -1 and "UnknownSetting" in m
    assert _apply(lib, {"metric": "bogus"})[0] == -1
    assert _apply(lib, {"g_iters": 1.5})[0] == -1
    assert _apply(lib, {"g_iters": -1})[0] == -1
    assert _apply(lib, {"exact": 1})[0] == -1
    assert _apply(lib, b"[1, 2]")[0] == -1
    assert _apply(lib, b"{\"map_res\": 2048,}")[0] == -1
    # the whole dict the reference's Python layer sends back round-trips
    rc, d = _apply(lib, {})
    assert _apply(lib, d) == (0, d)


def test_create_without_gpu_fails_cleanly(lib):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert not lib.zc_create(b"")
    buf = ctypes.create_string_buffer(512)
    n = lib.zc_create_error(buf, 512)
    assert b"no CUDA device" in buf.raw[:n]
