"""The C oracle against the golden fixtures generated from the reference's own
code (tests/golden/make_golden.py). Bit-exact comparisons throughout."""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import golden
from oracle import lko

FFA_FIXTURES = ["ffa_freq_nb32.npz", "ffa_freq_nb64.npz", "ffa_accel_nb16.npz", "ffa_jerk_nb16.npz"]


def _plan(g):
    cfg = lko.make_cfg(int(g["nsamps"]), float(g["tsamp"]), int(g["nbins"]), float(g["eta"]), g["param_limits"])
    return lko.plan_create(cfg)


@pytest.mark.parametrize("name", FFA_FIXTURES)
def test_plan_matches_reference(name):
    g = golden(name)
    p = _plan(g)
    assert p.n_levels == int(g["n_levels"])
    assert p.raw.bseg_brute == int(g["bseg_brute"])
    np.testing.assert_array_equal(p.ncoords, g["ncoords"])
    np.testing.assert_array_equal(p.param_counts, g["param_counts"])
    np.testing.assert_array_equal(p.ncoords_offsets, g["ncoords_offsets"])
    assert np.array_equal(p.dparams.view(np.uint64), g["dparams"].view(np.uint64))


@pytest.mark.parametrize("name", FFA_FIXTURES)
def test_coords_match_reference(name):
    g = golden(name)
    coords = lko.resolve(_plan(g))
    got = coords.view(np.uint32).reshape(coords.size, -1)
    np.testing.assert_array_equal(got, g["coords"])


@pytest.mark.parametrize("name", FFA_FIXTURES)
def test_fold_and_scores_match_reference(name):
    g = golden(name)
    p = _plan(g)
    fold = lko.ffa(p, g["ts_e"], g["ts_v"])
    assert fold.size == int(g["fold_size"])
    assert hashlib.sha256(fold.tobytes()).hexdigest() == str(g["fold_sha256"])
    if g["fold"].size:
        np.testing.assert_array_equal(fold.view(np.uint32), g["fold"].view(np.uint32))
    scores = lko.snr_boxcar_3d(fold, g["widths"], int(g["nbins"]))
    np.testing.assert_array_equal(scores.view(np.uint32), g["scores"].view(np.uint32))


def test_brute_fold_matches_reference():
    g = golden("brute_fold_nb64.npz")
    out = lko.brute_fold(g["ts_e"], g["ts_v"], g["freqs"], int(g["segment_len"]), int(g["nbins"]),
                         float(g["tsamp"]), float(g["t_ref"]))
    np.testing.assert_array_equal(out.view(np.uint32), g["fold"].view(np.uint32))


def test_scores_match_reference():
    g = golden("scores_nb48.npz")
    s = lko.snr_boxcar_3d(g["folds"], g["widths"], 48)
    np.testing.assert_array_equal(s.view(np.uint32), g["scores"].view(np.uint32))
    m = lko.snr_boxcar_3d_max(g["folds"], g["widths"], 48)
    np.testing.assert_array_equal(m.view(np.uint32), g["scores_max"].view(np.uint32))
    np.testing.assert_array_equal(lko.box_widths(64), g["trials_64"])
    np.testing.assert_array_equal(lko.box_widths(128), g["trials_128"])
    np.testing.assert_array_equal(lko.box_widths(100, 0.3, 1.5), g["trials_100_03"])


def test_phase_idx_matches_reference():
    cases = golden("phase_idx.npz")["cases"]
    for t, f, nb, d, ph, phu in cases:
        assert lko.phase_idx(t, f, int(nb), d) == np.float32(ph)
        assert lko.phase_idx_uint(t, f, int(nb), d) == int(phu)
