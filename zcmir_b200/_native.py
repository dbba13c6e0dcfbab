"""ctypes bindings to libzcmir.so, the B200 build of zcmir's C ABI (include/zcmir.h).

The struct layouts and signatures are the reference's (python/zcmir/_native.py:14-133); the
library is the in-tree build (``python -m zcmir_b200.build``). There is no fallback: when the
library is missing or cannot load, importing this module's ``load()`` raises.
"""
import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libzcmir.so"

U32, I32, I64, F64, SZ, P = ctypes.c_uint32, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_size_t, ctypes.c_void_p
f32p, f64p, u8p, u32p = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint32)
Mat = ctypes.c_double * 9


class ShiftResult(ctypes.Structure):
    _fields_ = [
        ("n", U32), ("cw", U32), ("ch", U32), ("canvas_w", U32), ("canvas_h", U32),
        ("ox", I32), ("oy", I32), ("peak_index", U32),
        ("dx", F64), ("dy", F64), ("peak", F64), ("zero", F64), ("corr_area_px", F64),
        ("exact", U32), ("calibrated", U32), ("n_y", U32), ("_pad", U32),
    ]


class RsResult(ctypes.Structure):
    _fields_ = [
        ("n", U32), ("n_th", U32), ("n_lam", U32), ("peak_index", U32),
        ("dlam", F64), ("r0", F64), ("r1", F64), ("cx", F64), ("cy", F64), ("peak", F64), ("zero", F64),
        ("dth", F64), ("dsg", F64), ("symmetric", U32), ("calibrated", U32),
    ]


class GradResult(ctypes.Structure):
    _fields_ = [
        ("score", F64), ("fwd", F64), ("inv", F64), ("n", F64),
        ("grad", F64 * 8), ("hess", F64 * 64), ("has_hess", U32), ("nk", U32),
    ]


class ClimbResult(ctypes.Structure):
    _fields_ = [("H", Mat), ("score", F64), ("iterations", U32), ("moved", U32)]


class SearchResult(ctypes.Structure):
    _fields_ = [("H", Mat), ("score", F64), ("prev", F64), ("improved", U32), ("count_a", U32), ("count_b", U32), ("_pad", U32)]


class Canvas(ctypes.Structure):
    _fields_ = [("ox", I32), ("oy", I32), ("ow", U32), ("oh", U32), ("Hc", Mat)]


# the SMI path's calls; the library also exports every other zc_* name of the reference
SIGS = {
    "zc_version": ([], ctypes.c_char_p),
    "zc_create": ([ctypes.c_char_p], P),
    "zc_create_error": ([ctypes.c_char_p, SZ], SZ),
    "zc_destroy": ([P], None),
    "zc_adapter": ([P, ctypes.c_char_p, SZ], SZ),
    "zc_error": ([P, ctypes.c_char_p, SZ], SZ),
    "zc_configure": ([P, ctypes.c_char_p, SZ], I32),
    "zc_settings": ([P, ctypes.c_char_p, SZ], SZ),
    "zc_set_image": ([P, U32, f32p, U32, U32], I32),
    "zc_set_image_gray": ([P, U32, f32p, U32, U32, U32], I32),
    "zc_set_image_rgba": ([P, U32, u8p, U32, U32], I32),
    "zc_work_image": ([P, U32, f32p, SZ], I32),
    "zc_features": ([P, U32, f32p, SZ], I32),
    "zc_moments": ([P, f64p, f64p], I32),
    "zc_image_size": ([P, U32, u32p], None),
    "zc_cancel": ([P], None),
    "zc_profile": ([P, U32], I32),
    "zc_gpu_counts": ([P, u32p], None),
    "zc_profile_report": ([P, ctypes.c_char_p, SZ], SZ),
    "zc_swap": ([P], None),
    "zc_search": ([P, ctypes.POINTER(SearchResult)], I32),
    "zc_climb": ([P, ctypes.POINTER(ClimbResult)], I32),
    "zc_set_pose": ([P, f64p], None),
    "zc_get_pose": ([P, f64p], None),
    "zc_events": ([P, ctypes.c_char_p, SZ], SZ),
    "zc_score": ([P, f64p, f64p], I32),
    "zc_gradient": ([P, f64p, U32, ctypes.POINTER(GradResult)], I32),
    "zc_shift_map": ([P, f64p, U32, U32, ctypes.POINTER(ShiftResult), f32p, SZ], I32),
    "zc_shift_map_set": ([P, f64p, ctypes.POINTER(ShiftResult), f32p, SZ], I32),
    "zc_rs_map": ([P, f64p, f64p, U32, ctypes.POINTER(RsResult), f32p, f32p, f32p, SZ], I32),
    "zc_canvas": ([P, f64p, U32, ctypes.POINTER(Canvas)], I32),
    "zc_set_ffd": ([P, f32p, SZ], I32),
    "zc_get_ffd": ([P, f32p, SZ], SZ),
    "zc_ffd_gradient": ([P, f64p, f64p, f64p, SZ], I32),
    "zc_displacement": ([P, f32p, SZ], I32),
    "zc_result_sizes": ([u32p], None),
    "zc_tune_parts": ([U32, U32, U32, U32], None),
    "zcb_bench_maps": ([P, f64p, U32, U32, U32, U32, f64p, SZ], I32),
    "zcb_score_static": ([P, f64p, U32, f64p], I32),
    "zcb_stack_maps": ([P, U32, ctypes.POINTER(f32p), u32p, u32p, f64p, U32, U32, ctypes.POINTER(ShiftResult), f64p], I32),
    "zcb_sweep": ([P, f64p, U32, U32, U32, U32, f32p, u32p, SZ, f64p, SZ], I32),
    "zcb_search_lanes": ([P, f32p, u32p, SZ, ctypes.POINTER(SearchResult)], I32),
    "zcb_tune_sweep": ([P, f64p, SZ, ctypes.POINTER(SZ)], I32),
    "zcb_set_dft_stage": ([P, U32], I32),
    "zcb_stack_load": ([P, U32, ctypes.POINTER(f32p), u32p, u32p, f64p, U32, U32], I32),
    "zcb_sweep_stack": ([P, f64p, U32, f32p, u32p, SZ, f64p, SZ, ctypes.POINTER(ShiftResult), SZ], I32),
    "zcb_refine_poses": ([P, f64p, U32, U32, f64p, f64p], I32),
    "zcb_prop_nparams": ([], SZ),
    "zcb_prop_error": ([ctypes.c_char_p, SZ], SZ),
    "zcb_prop_forward": ([f32p, SZ, f32p, U32, f32p], I32),
    "zcb_prop_grad": ([f32p, SZ, f32p, ctypes.POINTER(ctypes.c_int32), U32, f32p, f32p], I32),
    "zcb_prop_train": ([f32p, SZ, f32p, ctypes.POINTER(ctypes.c_int32), U32, U32, U32, ctypes.c_float, U32, f32p], I32),
    "zcb_cnn_nparams": ([], SZ),
    "zcb_cnn_error": ([ctypes.c_char_p, SZ], SZ),
    "zcb_cnn_forward": ([f32p, SZ, ctypes.POINTER(ctypes.c_uint16), U32, f32p], I32),
    "zcb_cnn_grad": ([f32p, SZ, ctypes.POINTER(ctypes.c_uint16), ctypes.POINTER(ctypes.c_int32), U32, f32p, f32p], I32),
    "zcb_cnn_train": ([f32p, SZ, ctypes.POINTER(ctypes.c_uint16), ctypes.POINTER(ctypes.c_int32), U32, U32, U32,
                       ctypes.c_float, ctypes.c_uint64, f32p, f32p], I32),
    "zcb_fp32_peak": ([f64p], I32),
    "zcb_settings_apply": ([ctypes.c_char_p, SZ, ctypes.c_char_p, SZ, ctypes.POINTER(SZ), ctypes.c_char_p, SZ, ctypes.POINTER(SZ)], I32),
}

_lib = None


def load(path=None):
    """The loaded library (once per process). Raises when it is missing: the B200 path has no
    CPU fallback."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path or os.environ.get("ZCMIR_B200_LIB") or LIB_PATH)
    if not p.exists():
        raise RuntimeError(f"{p} is not built: run `python -m zcmir_b200.build` (needs nvcc)")
    lib = ctypes.CDLL(str(p))
    for name, (args, res) in SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes, fn.restype = args, res
    _lib = lib
    return lib
