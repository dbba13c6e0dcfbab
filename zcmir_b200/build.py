"""Build libzcmir.so in-tree (zcmir_b200/libzcmir.so) with nvcc for sm_100a.

    python -m zcmir_b200.build [--force] [--verbose]

Objects go to zcmir_b200/_build/; a source is recompiled when it, or any header in csrc/ or
include/, is newer than its object.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libzcmir.so"
SOURCES = ["features.cu", "preprocess.cu", "shiftmap.cu", "lines_a.cu", "lines_b.cu", "lines_c.cu", "rows_tmem.cu", "inv_cols_tma.cu", "pose.cu", "sweep.cu", "rs.cu", "ncc.cu", "score_static.cu", "gn_device.cu", "dft_tc.cu", "proposal.cu", "cnn.cu", "peak.cu", "engine.cpp", "engine_pose.cpp", "engine_sweep.cpp", "engine_stack.cpp", "engine_rs.cpp", "engine_ncc.cpp", "engine_ffd.cpp", "settings.cpp", "exports.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# the device refine restates the host's float64 pose algebra operation for operation: no fused
# multiply-adds, so both give the same poses bit for bit
PER_FILE = {"gn_device.cu": ["--fmad=false"]}
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr", "-I", str(ROOT / "include")]


def nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found (set NVCC or put CUDA's bin on PATH)")


def _headers_mtime():
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def build(force=False, verbose=False):
    BUILD.mkdir(exist_ok=True)
    cc = nvcc()
    hdr = _headers_mtime()
    srcs = [s for s in SOURCES if (CSRC / s).exists()]
    jobs = []
    for s in srcs:
        src, obj = CSRC / s, BUILD / (s + ".o")
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr):
            extra = ["-Xptxas", "-v"] if verbose and s.endswith(".cu") else []
            if s.endswith(".cpp"):
                extra = ["-x", "cu", *extra]  # host files share the device headers
            extra = [*extra, *PER_FILE.get(s, [])]
            jobs.append([cc, *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose or r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed: {' '.join(cmd[-3:])}")
    objs = [str(BUILD / (s + ".o")) for s in srcs]
    if force or jobs or not LIB.exists() or LIB.stat().st_mtime < max(Path(o).stat().st_mtime for o in objs):
        cmd = [cc, *ARCH, "-shared", "-o", str(LIB), *objs, "-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
