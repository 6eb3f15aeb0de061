"""FP64 restatement of the time-domain FFA and boxcar S/N (oracle side).

Test infrastructure: the reference to which the FP32 and BF16-stored device
paths state their fold and S/N error. It follows the same algorithm as the
reference's FP32 path, with every sum in float64:

* brute fold: each (segment, frequency) bucket sums its samples at the phase
  bins of the oracle's phase map (lib/kernels.cpp:550-580, 1132-1154 of the
  reference; the phase indices are the exact reference indices, so the FP64
  fold bins the same samples);
* merges: out[s, c, r, j] = in[2s, tail, r, (j - st) mod n] + in[2s+1, head, r,
  (j - sh) mod n] with the oracle's coordinate tables and the reference's shift
  rounding (lib/kernels.cpp:71-146);
* score: x = E / sqrt(V), circular prefix sum, per-width max window, and
  ((h + b) dmax - b sum) with h = sqrt((n - w) / (n w)), b = w h / (n - w)
  (lib/score.cpp:95-172).

Only tests and the benchmark's error statement import this module.
"""

from __future__ import annotations

import numpy as np

from . import lko


def _shift_bins(shift: np.ndarray, nbins: int) -> np.ndarray:
    # (uint)(phase + 0.5f), with nbins mapped to 0 (FP32, as the reference)
    s = (shift.astype(np.float32) + np.float32(0.5)).astype(np.uint64)
    s[s == nbins] = 0
    return s.astype(np.int64)


def brute_fold64(plan: lko.OraclePlan, ts_e, ts_v) -> np.ndarray:
    nbins = plan.nbins
    seglen = int(plan.segment_lens[0])
    freqs = plan.freqs0()
    nseg = int(plan.nsegments[0])
    pm = lko.phase_map(freqs, seglen, nbins, float(plan.raw.tsamp), plan.t_ref0()).astype(np.int64)
    e = np.asarray(ts_e, dtype=np.float64).reshape(nseg, seglen)
    v = np.asarray(ts_v, dtype=np.float64).reshape(nseg, seglen)
    out = np.zeros((nseg, freqs.size, 2, nbins), dtype=np.float64)
    segoff = (np.arange(nseg, dtype=np.int64) * nbins)[:, None]
    for f in range(freqs.size):
        idx = (pm[f][None, :] + segoff).ravel()
        out[:, f, 0, :] = np.bincount(idx, weights=e.ravel(), minlength=nseg * nbins).reshape(nseg, nbins)
        out[:, f, 1, :] = np.bincount(idx, weights=v.ravel(), minlength=nseg * nbins).reshape(nseg, nbins)
    return out


def merge64(fold_in: np.ndarray, coords: np.ndarray, taylor: bool, nbins: int) -> np.ndarray:
    """fold_in [2 nseg, nprev, 2, nbins] -> [nseg, ncur, 2, nbins]."""
    if taylor:
        it = coords["i_tail"].astype(np.int64)
        ih = coords["i_head"].astype(np.int64)
        st = _shift_bins(coords["shift_tail"], nbins)
        sh = _shift_bins(coords["shift_head"], nbins)
    else:
        it = ih = coords["idx"].astype(np.int64)
        st = np.zeros(coords.size, dtype=np.int64)
        sh = _shift_bins(coords["shift"], nbins)
    j = np.arange(nbins, dtype=np.int64)
    jt = (j[None, :] - st[:, None]) % nbins  # [ncur, nbins]
    jh = (j[None, :] - sh[:, None]) % nbins
    tail = fold_in[0::2][:, it]  # [nseg, ncur, 2, nbins]
    head = fold_in[1::2][:, ih]
    tail = np.take_along_axis(tail, jt[None, :, None, :], axis=3)
    head = np.take_along_axis(head, jh[None, :, None, :], axis=3)
    return tail + head


def ffa64(plan: lko.OraclePlan, ts_e, ts_v, level: int | None = None) -> np.ndarray:
    """FP64 fold of `level` (default: the last), [nseg, ncoords, 2, nbins]."""
    last = plan.n_levels - 1 if level is None else level
    coords = lko.resolve(plan)
    offs = plan.ncoords_offsets
    nc = plan.ncoords
    taylor = plan.nparams > 1
    fold = brute_fold64(plan, ts_e, ts_v)
    for l in range(1, last + 1):
        c = coords[int(offs[l]) : int(offs[l]) + int(nc[l])]
        fold = merge64(fold, c, taylor, plan.nbins)
    return fold


def snr_boxcar64(folds: np.ndarray, widths) -> np.ndarray:
    """[..., 2, nbins] folds -> [..., nwidths] S/N in float64."""
    f = np.asarray(folds, dtype=np.float64)
    nbins = f.shape[-1]
    x = f[..., 0, :] / np.sqrt(f[..., 1, :])
    x = x.reshape(-1, nbins)
    wmax = int(max(widths))
    p = np.cumsum(np.concatenate([x, x[:, :wmax]], axis=1), axis=1)
    total = p[:, nbins - 1]
    out = np.empty((x.shape[0], len(widths)), dtype=np.float64)
    for k, w in enumerate(widths):
        w = int(w)
        h = np.sqrt((nbins - w) / (nbins * w))
        b = w * h / (nbins - w)
        dmax = (p[:, w : w + nbins] - p[:, :nbins]).max(axis=1)
        out[:, k] = (h + b) * dmax - b * total
    return out.reshape(f.shape[:-2] + (len(widths),))


def ffa_scores64(plan: lko.OraclePlan, ts_e, ts_v, widths) -> np.ndarray:
    """FP64 S/N of every final cell and width, [ncoords, nwidths]."""
    fold = ffa64(plan, ts_e, ts_v)
    assert fold.shape[0] == 1, "scores need a single final segment"
    return snr_boxcar64(fold[0], [int(w) for w in widths])
