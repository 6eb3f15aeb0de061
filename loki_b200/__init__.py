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
"""

from __future__ import annotations

from . import _capi
from ._capi import LokiError, lib

# Fail loudly at import time if the native library is missing.
lib()

from . import batched, configs, ffa, fold, pipeline, plans, prune, scores, sweep, thresholds  # noqa: E402
from . import libculoki  # noqa: E402

__all__ = ["configs", "plans", "ffa", "fold", "prune", "scores", "sweep", "thresholds", "batched", "libculoki",
           "LokiError", "lib"]
