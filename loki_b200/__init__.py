"""loki_b200: B200-native (sm_100a) FFA folding, boxcar scoring, the
frequency sweep over octave regions, the pruning tree (leaf step, whole runs
and their ascend / report end) and the Monte-Carlo threshold stage for pulsar
searches.

The compute path is ``libloki_b200.so`` (hand-written CUDA kernels behind the
C ABI in ``include/loki_b200.h``); this package is its Python face, with the
names of the reference's ``libloki`` / ``libculoki`` modules:

    from loki_b200 import libculoki
    cfg = libculoki.configs.PulsarSearchConfig(...)
    scores, plan = libculoki.ffa.compute_ffa_scores_cuda(ts_e, ts_v, cfg)

Submodules are imported on first use. Every module that computes imports
``_capi``, which loads the native library when it is imported and raises
``ImportError`` if it is missing (there is no fallback path); the synthetic
input generators (``loki_b200.synthetic``) need no native code and do not
load it.
"""

from __future__ import annotations

import importlib

_SUBMODULES = ("batched", "configs", "ffa", "fold", "pipeline", "plans", "prune", "scores", "sweep",
               "thresholds", "libculoki", "synthetic")

__all__ = list(_SUBMODULES) + ["LokiError", "lib"]


def __getattr__(name: str):
    if name in _SUBMODULES:
        return importlib.import_module(f".{name}", __name__)
    if name in ("LokiError", "lib"):
        from . import _capi

        return getattr(_capi, name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
