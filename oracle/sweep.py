"""CPU restatement of the frequency sweep's per-chunk search and result
decode -- test infrastructure only (the product path never imports it).

Follows FFAFreqSweep of the reference: per chunk configuration, the FFA, the
boxcar S/N of every final coordinate and width, the ordered `>= snr_min`
compaction (lib/ffa_freq_sweep.cpp:139-195), then save_results'
decode of every passing index into parameter values by the chunk plan's
final-level counts and Cartesian strides, `get_param_val_at_idx` per
parameter and the width taken from the base configuration's width list
(lib/ffa_freq_sweep.cpp:202-250, lib/loki/psr_utils.hpp:283-293).

The FFA and scoring come from a backend: `lko_backend` (the C oracle) or a
caller-supplied one built on the reference library (the golden-fixture
script uses that).
"""

from __future__ import annotations

import numpy as np

from . import lko


def lko_backend(nsamps, tsamp, nbins, eta, lims, ts_e, ts_v, widths=None):
    """(scores [ncoords * n_widths], final param counts, widths) from the C oracle."""
    plan = lko.plan_create(lko.make_cfg(nsamps, tsamp, nbins, eta, lims))
    w = plan.widths if widths is None else np.asarray(widths, np.uint64)
    fold = lko.ffa(plan, ts_e, ts_v)
    scores = lko.snr_boxcar_3d(fold, w, nbins)
    return scores.ravel(), np.asarray(plan.param_counts[-1], np.uint64), w


def lko_fourier_backend(nsamps, tsamp, nbins, eta, lims, ts_e, ts_v, widths=None):
    """The same from the oracle's FP64 Fourier-domain FFA (FFA<ComplexType>
    back to time, boxcar S/N), scores in float64."""
    plan = lko.plan_create(lko.make_cfg(nsamps, tsamp, nbins, eta, lims))
    w = plan.widths if widths is None else np.asarray(widths, np.uint64)
    scores = lko.ffa_fourier_scores64(plan, ts_e, ts_v, w)
    return scores.ravel(), np.asarray(plan.param_counts[-1], np.uint64), w


def param_val_at_idx(vmin: float, vmax: float, count: int, idx: np.ndarray) -> np.ndarray:
    """psr_utils::get_param_val_at_idx on an index array (IEEE double)."""
    if count <= 1:
        return np.full(idx.shape, (vmax + vmin) / 2.0)
    dv = (vmax - vmin) / float(count)
    return vmin + dv * (idx.astype(np.float64) + 0.5)


def decode(indices: np.ndarray, counts, lims, widths) -> np.ndarray:
    """Rows of (parameter values..., width) for flat `coord * n_widths + w`
    indices, with `widths` the list the decode divides by."""
    counts = [int(c) for c in counts]
    lims = np.asarray(lims, np.float64).reshape(-1, 2)
    npar = len(counts)
    strides = [1] * npar
    for j in range(npar - 2, -1, -1):
        strides[j] = strides[j + 1] * counts[j + 1]
    w = np.asarray(widths, np.uint64)
    idx = np.asarray(indices, np.uint64)
    coord = idx // np.uint64(w.size)
    out = np.zeros((idx.size, npar + 1), np.float64)
    rem = coord.copy()
    for j in range(npar):
        p = rem // np.uint64(strides[j])
        rem = rem - p * np.uint64(strides[j])
        out[:, j] = param_val_at_idx(float(lims[j, 0]), float(lims[j, 1]), counts[j], p)
    out[:, npar] = w[idx % np.uint64(w.size)].astype(np.float64)
    return out


def run(base, chunks, ts_e, ts_v, snr_min, backend=lko_backend, chunk_widths=False, score_widths=None):
    """The sweep on host arrays.

    base: (nsamps, tsamp, nbins, eta, lims) of the base configuration;
    chunks: rows (f_min, f_max, nbins, eta) of the chunk configurations;
    score_widths: an explicit width list for every chunk (None: each chunk's
    generated trials). Returns (param_sets [n, nparams + 1], snr [n],
    per-chunk counts)."""
    nsamps, tsamp, nbins0, eta0, lims0 = base
    lims0 = np.asarray(lims0, np.float64).reshape(-1, 2)
    if score_widths is not None:
        base_w = np.asarray(score_widths, np.uint64)
    else:
        base_w = lko.plan_create(lko.make_cfg(nsamps, tsamp, nbins0, eta0, lims0)).widths
    params, snrs, counts = [], [], []
    for f_min, f_max, nb, eta in chunks:
        lims = lims0.copy()
        lims[-1] = (f_min, f_max)
        scores, pc, w = backend(nsamps, tsamp, int(nb), float(eta), lims, ts_e, ts_v, score_widths)
        keep = np.flatnonzero(scores.astype(np.float64) >= float(snr_min))
        counts.append(keep.size)
        params.append(decode(keep, pc, lims, w if chunk_widths else base_w))
        snrs.append(scores[keep].astype(np.float32))
    npar = lims0.shape[0]
    if not params:
        return np.zeros((0, npar + 1)), np.zeros(0, np.float32), np.zeros(0, np.uint64)
    return np.concatenate(params), np.concatenate(snrs), np.array(counts, np.uint64)
