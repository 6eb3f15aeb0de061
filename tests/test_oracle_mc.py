"""Monte-Carlo threshold stage, CPU side: the oracle's largest S/N (each
width's S/N divided by stdnoise) decides exactly as the reference's
snr_boxcar_threshold_with_cache (run from the reference build), including at
the threshold itself; and the oracle stage's bookkeeping (order, rows,
counts) follows its definition."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import lko
from oracle import ref as R


@pytest.mark.skipif(not R.available(), reason="oracle/_ref (the reference build) is not present")
@pytest.mark.parametrize("nbins,stdnoise", [(64, 1.7320508), (32, 1.0), (100, 4.0)])
def test_threshold_decision_matches_reference(nbins, stdnoise):
    rng = np.random.default_rng(nbins)
    n = 2000
    prof = rng.standard_normal((n, nbins)).astype(np.float32) * 1.5
    prof[:, 10:16] += rng.random((n, 1)).astype(np.float32) * 5
    w = np.array([1, 2, 3, 4, 6, 8, 12, 16], np.uint64)
    sd = np.float32(stdnoise)
    m = lko.snr_max_div(prof, nbins, w, sd)
    for thr in (m, np.nextafter(m, -np.inf, dtype=np.float32), np.full(n, 3.0, np.float32)):
        np.testing.assert_array_equal(R.snr_threshold(prof, nbins, w, thr, sd), m > thr)


def test_mc_stage_bookkeeping():
    rng = np.random.default_rng(1)
    n, nb = 500, 32
    fin = rng.standard_normal((n, nb)).astype(np.float32)
    nz = rng.standard_normal((n, nb)).astype(np.float32)
    sig = np.zeros(nb, np.float32)
    grid = np.array([-1.0, 2.0, 3.0, 100.0], np.float32)
    w = np.array([1, 2, 4], np.uint64)
    f, ids, counts, mx = lko.mc_stage(fin, nz, sig, 1.0, 1.0, w, 2.0, grid)
    keep = np.flatnonzero(mx > 2.0)
    np.testing.assert_array_equal(ids, keep.astype(np.uint32))
    np.testing.assert_array_equal(f, (fin + nz)[keep])
    np.testing.assert_array_equal(counts, [(mx > g).sum() for g in grid])
    assert counts[0] == n and counts[-1] == 0
