"""The forward column FFTs' first stage on the tensor cores (zcb_set_dft_stage): split-BF16
products accumulated in FP32 by tcgen05.mma, the other stages FP32.

Checked on the 512² remap pair (45 correlations zero-padded to 1024², whose 1024-point columns
start with a radix-16 stage) against the float64 oracle with the shift-map tests' rule (same
argmax, peak within 1e-4, cells within 1e-4 of the peak where the overlap is ≥ 20 % of the
largest, 1e-2 elsewhere) for 3 pieces (6 products, about FP32's 24 bits), and against the FP32
map: 3 pieces within 2e-6 of the peak everywhere, 2 pieces (3 products, about 16 bits) within
1e-5, 1 piece (plain BF16) within 1e-2, each with the same argmax. Lengths whose first stage is
not radix 16 and piece counts above 3 are refused."""
import json
import os

import numpy as np
import pytest

import zcmir_b200 as zc
from oracle import smi_oracle as O
from zcmir_b200 import synth

pytestmark = pytest.mark.gpu

from test_gpu_shiftmap import check_map, prep_from  # noqa: E402


@pytest.fixture(scope="module")
def maps():
    m, f, H = synth.pair_remap(n=512, shift=(-37, 21), seed=3)
    out = {}
    with zc.Engine(half=False) as reg:
        reg.set_images(m, f, preprocess=False)
        pa, pb = prep_from(reg.features(0)), prep_from(reg.features(1))
        for p in (0, 3, 2, 1, 0):
            reg.set_dft_stage(p)
            out.setdefault(p, []).append(reg.shift_map(np.eye(3), exact=True, calibrated=False, cap=1024))
    ref = O.shift_map(pa, pb, np.eye(3), exact=True, calibrated=False, cap=1024, return_corr=True)
    return out, ref, H


def errors(sm, base, ref):
    big = ref["corr"][0] >= 0.2 * ref["corr"][0].max()
    both = (sm.map != 0) & (base.map != 0)
    e = np.abs(sm.map.astype(np.float64) - base.map) / abs(base.peak)
    return float(e[big & both].max()), float(e[both].max())


def test_tensor_core_stage_matches_the_oracle(maps):
    out, ref, H = maps
    sm = out[3][0]
    assert (sm.n, sm.ny) == (1024, 1024)
    check_map(sm, ref, ref["corr"][0])
    assert (sm.dx, sm.dy) == (-H[0, 2], -H[1, 2])


def test_tensor_core_stage_against_fp32(maps):
    out, ref, _ = maps
    f32 = out[0][0]
    # the FP32 map is unchanged by a round trip through the tensor-core stage
    np.testing.assert_array_equal(out[0][1].map, f32.map)
    rec = {}
    for p in (3, 2, 1):
        e = errors(out[p][0], f32, ref)
        rec[f"pieces{p}_big_overlap"], rec[f"pieces{p}_all"] = e
        rec[f"pieces{p}_same_argmax"] = bool(out[p][0].peak_index == f32.peak_index)
    path = os.environ.get("ZCMIR_B200_STUDY_OUT")
    if path:
        with open(path.replace(".json", "_dft_tc_512.json"), "w") as fh:
            json.dump(rec, fh, indent=1)
    print(rec)
    assert rec["pieces3_same_argmax"] and rec["pieces2_same_argmax"] and rec["pieces1_same_argmax"], rec
    assert rec["pieces3_all"] <= 2e-6, rec
    assert rec["pieces2_all"] <= 1e-5, rec
    assert rec["pieces1_all"] <= 1e-2, rec


def test_refusals():
    m, f, _ = synth.pair_remap(n=256, shift=(17, -9), seed=0)
    with zc.Engine(half=False) as reg:
        reg.set_images(m, f, preprocess=False)
        with pytest.raises(zc.EngineError, match="pieces"):
            reg.set_dft_stage(4)
        reg.set_dft_stage(3)
        # 512-point columns start with a radix-8 stage
        with pytest.raises(zc.EngineError, match="radix 16"):
            reg.shift_map(np.eye(3), exact=True, calibrated=False, cap=1024)
        reg.set_dft_stage(0)
        assert reg.shift_map(np.eye(3), exact=True, calibrated=False, cap=1024).n == 512
