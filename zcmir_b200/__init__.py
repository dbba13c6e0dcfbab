"""zcmir_b200: the square-loss mutual information (SMI) path of zcmir, native to the B200.

``libzcmir.so`` (CUDA for sm_100a, built by ``python -m zcmir_b200.build``) exports the
reference's zc_* C ABI, so the reference's own Python package runs on it unchanged (point its
``ZCMIR_LIB`` at the library), plus this build's zcb_* extensions (sweep shards, stack maps,
device-timed maps, allocation-free pose scores, the learned proposal's network).

This package is the host side of those calls for this repository: ``Engine`` (one engine handle,
numpy in and out), the build, synthetic inputs, the learned proposal and the multi-rank sweep.
"""
from .engine import Engine, EngineError, MapResult, RsMapResult, gray32, rgba8

__all__ = ["Engine", "EngineError", "MapResult", "RsMapResult", "gray32", "rgba8", "__version__"]

__version__ = "0.1.4"  # the reference's version string, as zc_version reports it
