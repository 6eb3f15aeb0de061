"""Chebyshev basis of the pruning leaf step, CPU side: the C oracle against
the reference's own whole pruning runs in that basis (golden fixtures made
by tests/golden/make_golden.py from the reference build) and -- where
oracle/_ref is built -- against the reference's poly_chebyshev_* functions
directly, bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from oracle import lko
from oracle import ref as R

CHEBY_FIXTURES = ["prune_cheby_accel_nb16.npz", "prune_cheby_jerk_nb16.npz"]
STAT_FIELDS = ("level", "seg_idx", "n_branches", "n_leaves", "n_leaves_phy", "n_leaves_surv",
               "threshold", "score_min", "score_max")


def _plan(g):
    cfg = lko.make_cfg(int(g["nsamps"]), float(g["tsamp"]), int(g["nbins"]), float(g["eta"]),
                       g["param_limits"], bseg_ffa=int(g["bseg_ffa"]))
    return lko.plan_create(cfg)


@pytest.mark.parametrize("name", CHEBY_FIXTURES)
def test_oracle_cheby_prune_run_matches_reference_fixture(name):
    g = golden(name)
    assert str(g["basis"]) == "chebyshev"
    plan = _plan(g)
    stats, leaves, folds, scores = lko.prune_run(
        plan, g["ffa_fold"], g["thresholds"], int(g["ref_seg"]), int(g["max_sugg"]), int(g["batch_size"]),
        int(g["branch_max"]), int(plan.nsegments[-1]) - 1, basis="chebyshev")
    np.testing.assert_array_equal(np.stack([stats[k].astype(np.float64) for k in STAT_FIELDS], axis=1), g["stats"])
    np.testing.assert_array_equal(leaves, g["leaves"])
    np.testing.assert_array_equal(folds, g["folds"])
    np.testing.assert_array_equal(scores, g["scores"])


def test_oracle_cheby_rejects_conservative_tile():
    g = golden(CHEBY_FIXTURES[0])
    plan = _plan(g)
    with pytest.raises(RuntimeError):
        lko.prune_run(plan, g["ffa_fold"], g["thresholds"], int(g["ref_seg"]), int(g["max_sugg"]),
                      int(g["batch_size"]), int(g["branch_max"]), 2, conservative=True, basis="chebyshev")


def _leaves(np_, n, seed):
    """Chebyshev-like leaves: coefficients and their errors of several orders
    of magnitude, alpha_0 and f0 as the pruning tree holds them."""
    rng = np.random.default_rng(seed)
    lv = np.zeros((n, np_ + 2, 2))
    for k in range(np_):
        lv[:, k, 0] = rng.normal(0, 10.0 ** (2 - k), n)
        lv[:, k, 1] = 10.0 ** (1 - k) * (0.2 + rng.random(n))
    lv[:, np_, 0] = rng.normal(0, 1e-3, n)
    lv[:, np_, 1] = 1e-3 * rng.random(n)
    lv[:, np_ + 1, 0] = 10.0 + 0.3 * rng.random(n)
    return lv


@pytest.mark.skipif(not R.available(), reason="oracle/_ref (the reference build) is not present")
@pytest.mark.parametrize("np_", [2, 3])
def test_oracle_cheby_functions_match_reference(np_):
    lv = _leaves(np_, 257, 40 + np_)
    ci, cc, cp, cn, ca = (5.0, 2.5), (6.25, 3.75), (5.0, 2.5), (7.5, 5.0), (8.75, 1.25)
    np.testing.assert_array_equal(lko.taylor_to_cheby(lv, np_, ci), R.taylor_to_cheby(lv, np_, ci))
    np.testing.assert_array_equal(lko.cheby_to_taylor(lv, np_, cn), R.cheby_to_taylor(lv, np_, cn))
    idx = np.array([0, 5, 7, 100, 256, 3], np.uint64)
    np.testing.assert_array_equal(lko.cheby_transform(lv, idx, np_, cn, cc), R.cheby_transform(lv, idx, np_, cn, cc))
    # branch: children, origins and the parents transformed in place
    for eta, bmax in ((1.0, 64), (0.5, 256)):
        a = lko.cheby_branch(lv, np_, cc, cp, 16, eta, bmax)
        b = R.cheby_branch(lv, np_, cc, cp, 16, eta, bmax)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
    # resolve on a plan's grid
    lims = [[-1000.0, 1000.0], [10.0, 10.3]] if np_ == 2 else [[-100.0, 100.0], [-900.0, 900.0], [10.0, 10.2]]
    plan = lko.plan_create(lko.make_cfg(16384, 8e-3, 16, 1.0, lims, bseg_ffa=2048))
    rc = R.make_cfg(16384, 8e-3, 16, 1.0, lims, bseg_ffa=2048)
    ch, _, _ = lko.cheby_branch(lv, np_, cc, cp, 16, 1.0, 64)
    got = lko.cheby_resolve(plan, ch, ca, cc, ci)
    want = R.cheby_resolve(rc, ch, ca, cc, ci)
    np.testing.assert_array_equal(got[0], want[0])
    np.testing.assert_array_equal(got[1], want[1])


CHEBY_REF_CASES = [
    # nsamps, tsamp, nbins, eta, limits, bseg_ffa, seed, max_sugg, batch, lo, hi, ref_frac
    (1 << 15, 4e-3, 32, 1.0, [[-500.0, 500.0], [10.0, 10.5]], 2048, 7, 200, 16, 1.0, 3.0, 0.5),
    (1 << 15, 4e-3, 32, 1.0, [[-500.0, 500.0], [10.0, 10.5]], 2048, 8, 1 << 12, 5, 1.0, 3.0, 0.0),
    (1 << 16, 2e-3, 32, 2.0, [[-40.0, 40.0], [-500.0, 500.0], [20.0, 20.6]], 4096, 9, 400, 32, 1.5, 3.5, 0.8),
]


@pytest.mark.skipif(not R.available(), reason="oracle/_ref (the reference build) is not present")
@pytest.mark.parametrize("case", range(len(CHEBY_REF_CASES)))
def test_oracle_cheby_prune_matches_reference_directly(case):
    ns, ts, nb, eta, lim, bf, seed, ms, bs, lo, hi, rf = CHEBY_REF_CASES[case]
    rc = R.make_cfg(ns, ts, nb, eta, lim, bseg_ffa=bf)
    plan = lko.plan_create(lko.make_cfg(ns, ts, nb, eta, lim, bseg_ffa=bf))
    rng = np.random.default_rng(seed)
    e = rng.standard_normal(ns).astype(np.float32)
    v = (1.0 + 0.25 * rng.random(ns)).astype(np.float32)
    fold = lko.ffa(plan, e, v)
    nseg = int(plan.nsegments[-1])
    ref_seg = min(int(nseg * rf), nseg - 1)
    bm = max(int(np.ceil(R.branching_pattern_basis(rc, "chebyshev", 0).max() * 2)), 32)
    thr = np.linspace(lo, hi, nseg - 1).astype(np.float32)
    a = R.prune_run(rc, fold, thr, ref_seg, ms, bs, bm, nseg - 1, nb, basis="chebyshev")
    b = lko.prune_run(plan, fold, thr, ref_seg, ms, bs, bm, nseg - 1, basis="chebyshev")
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("name", CHEBY_FIXTURES)
def test_library_cheby_branching_pattern_matches_reference_fixture(name):
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.prune import branching_pattern

    g = golden(name)
    cfg = PulsarSearchConfig(int(g["nsamps"]), float(g["tsamp"]), int(g["nbins"]), float(g["eta"]),
                             g["param_limits"], use_fourier=False, bseg_ffa=int(g["bseg_ffa"]))
    np.testing.assert_array_equal(branching_pattern(cfg, 0, poly_basis="chebyshev"), g["branching_pattern"])
    np.testing.assert_array_equal(branching_pattern(cfg, int(g["ref_seg"]), poly_basis="chebyshev"),
                                  g["branching_pattern_ref"])
    assert max(int(np.ceil(g["branching_pattern"].max() * 2)), 32) == int(g["branch_max"])


@pytest.mark.skipif(not R.available(), reason="oracle/_ref (the reference build) is not present")
@pytest.mark.parametrize("case", range(len(CHEBY_REF_CASES)))
def test_library_cheby_branching_pattern_matches_reference_directly(case):
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.prune import branching_pattern

    ns, ts, nb, eta, lim, bf = CHEBY_REF_CASES[case][:6]
    rc = R.make_cfg(ns, ts, nb, eta, lim, bseg_ffa=bf)
    cfg = PulsarSearchConfig(ns, ts, nb, eta, np.array(lim), use_fourier=False, bseg_ffa=bf)
    nseg = len(branching_pattern(cfg, 0)) + 1
    for rs in (0, nseg // 2, nseg - 1):
        np.testing.assert_array_equal(branching_pattern(cfg, rs, poly_basis="chebyshev"),
                                      R.branching_pattern_basis(rc, "chebyshev", rs))
