"""Pruning leaf step, CPU side: the C oracle against the reference's own
pruning runs (golden fixtures made by tests/golden/make_golden.py from the
reference build), the library's host-side branching pattern against the same
fixtures, and -- where oracle/_ref is built -- the oracle against the
reference directly on more cases."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import golden
from oracle import lko
from oracle import ref as R

PRUNE_FIXTURES = ["prune_accel_nb16.npz", "prune_jerk_nb16.npz"]
STAT_FIELDS = ("level", "seg_idx", "n_branches", "n_leaves", "n_leaves_phy", "n_leaves_surv",
               "threshold", "score_min", "score_max")


def _plan(g):
    cfg = lko.make_cfg(int(g["nsamps"]), float(g["tsamp"]), int(g["nbins"]), float(g["eta"]),
                       g["param_limits"], bseg_ffa=int(g["bseg_ffa"]))
    return lko.plan_create(cfg)


def _stats_matrix(stats):
    return np.stack([stats[k].astype(np.float64) for k in STAT_FIELDS], axis=1)


@pytest.mark.parametrize("name", PRUNE_FIXTURES)
def test_oracle_prune_run_matches_reference_fixture(name):
    g = golden(name)
    plan = _plan(g)
    stats, leaves, folds, scores = lko.prune_run(
        plan, g["ffa_fold"], g["thresholds"], int(g["ref_seg"]), int(g["max_sugg"]), int(g["batch_size"]),
        int(g["branch_max"]), int(plan.nsegments[-1]) - 1, conservative=bool(g["conservative"]))
    np.testing.assert_array_equal(_stats_matrix(stats), g["stats"])
    np.testing.assert_array_equal(leaves, g["leaves"])
    np.testing.assert_array_equal(folds, g["folds"])
    np.testing.assert_array_equal(scores, g["scores"])


@pytest.mark.parametrize("name", PRUNE_FIXTURES)
def test_library_branching_pattern_matches_reference_fixture(name):
    from loki_b200 import _capi as C
    from loki_b200.configs import PulsarSearchConfig

    g = golden(name)
    cfg = PulsarSearchConfig(int(g["nsamps"]), float(g["tsamp"]), int(g["nbins"]), float(g["eta"]),
                             g["param_limits"], use_fourier=False, bseg_ffa=int(g["bseg_ffa"]))
    cons = int(g["conservative"])
    for rs, key in ((0, "branching_pattern"), (int(g["ref_seg"]), "branching_pattern_ref")):
        out = np.zeros(256)
        n = ctypes.c_uint64()
        C.check(C.lib().lk_plan_branching_pattern(cfg._plan_handle, rs, cons, out.ctypes.data, out.size,
                                                  ctypes.byref(n)))
        np.testing.assert_array_equal(out[: n.value], g[key])
    # EPMultiPass's branch_max rule on the pattern of ref_seg 0
    assert max(int(np.ceil(g["branching_pattern"].max() * 2)), 32) == int(g["branch_max"])


def test_middle_out_order_and_coords():
    # np.argsort(|arange(8) - 4|, kind="stable") = [4, 3, 5, 2, 6, 1, 7, 0]
    order = [lko.middle_out(8, 4, 2.0, lv)[0] for lv in range(8)]
    assert order == [4, 3, 5, 2, 6, 1, 7, 0]
    seg, coord, cur, segc = lko.middle_out(8, 4, 2.0, 2)
    # segments {3, 4, 5}: ref = (3 + 5 + 1) / 2 = 4.5, scale = 1.5 (times tseg 2.0)
    assert coord == (9.0, 3.0)
    assert cur == (lko.middle_out(8, 4, 2.0, 1)[1][0], 3.0)
    assert segc == ((5 + 0.5) * 2.0, 1.0)


def test_determine_ref_segs():
    from loki_b200.prune import determine_ref_segs

    assert determine_ref_segs(32, n_runs=1) == [16]
    assert determine_ref_segs(32, n_runs=4) == [4, 12, 19, 27]
    assert determine_ref_segs(32, ref_segs=[3, 5]) == [3, 5]
    with pytest.raises(RuntimeError):
        determine_ref_segs(32)
    with pytest.raises(RuntimeError):
        determine_ref_segs(8, n_runs=9)


def _series(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n).astype(np.float32), (1.0 + 0.25 * rng.random(n)).astype(np.float32)


REF_CASES = [
    # nsamps, tsamp, nbins, eta, limits, bseg_ffa, seed, max_sugg, batch, lo, hi, ref_frac, cons
    (1 << 15, 4e-3, 32, 1.0, [[-500.0, 500.0], [10.0, 10.5]], 2048, 7, 200, 16, 1.0, 3.0, 0.5, False),
    (1 << 15, 4e-3, 32, 1.0, [[-500.0, 500.0], [10.0, 10.5]], 2048, 8, 1 << 12, 5, 1.0, 3.0, 0.0, True),
    (1 << 16, 2e-3, 32, 2.0, [[-40.0, 40.0], [-500.0, 500.0], [20.0, 20.6]], 4096, 9, 400, 32, 1.5, 3.5, 0.8,
     False),
]


@pytest.mark.skipif(not R.available(), reason="oracle/_ref (the reference build) is not present")
@pytest.mark.parametrize("case", range(len(REF_CASES)))
def test_oracle_prune_matches_reference_directly(case):
    ns, ts, nb, eta, lim, bf, seed, ms, bs, lo, hi, rf, cons = REF_CASES[case]
    rc = R.make_cfg(ns, ts, nb, eta, lim, bseg_ffa=bf)
    plan = lko.plan_create(lko.make_cfg(ns, ts, nb, eta, lim, bseg_ffa=bf))
    e, v = _series(ns, seed)
    fold = lko.ffa(plan, e, v)
    nseg = int(plan.nsegments[-1])
    ref_seg = min(int(nseg * rf), nseg - 1)
    bm = R.branch_max(rc, cons)
    thr = np.linspace(lo, hi, nseg - 1).astype(np.float32)
    a = R.prune_run(rc, fold, thr, ref_seg, ms, bs, bm, nseg - 1, nb, cons)
    b = lko.prune_run(plan, fold, thr, ref_seg, ms, bs, bm, nseg - 1, cons)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


FINAL_FIXTURES = PRUNE_FIXTURES + ["prune_cheby_accel_nb16.npz", "prune_cheby_jerk_nb16.npz"]


@pytest.mark.parametrize("name", FINAL_FIXTURES)
@pytest.mark.parametrize("tag", ["final", "half"])
def test_oracle_ascend_report_matches_reference_fixture(name, tag):
    """The end of a run (PruneImpl::run, lib/prune.cpp:136-139): survivors
    ascended to the middle of the data (folds over every segment so far,
    scores_ep = the scores before) and reported there."""
    g = golden(name)
    plan = _plan(g)
    basis = str(g["basis"])
    nseg = int(plan.nsegments[-1])
    n_iters = nseg - 1 if tag == "final" else (nseg - 1) // 2
    st, lv, fo, sc = lko.prune_run(plan, g["ffa_fold"], g["thresholds"], int(g["ref_seg"]), int(g["max_sugg"]),
                                   int(g["batch_size"]), int(g["branch_max"]), n_iters, bool(g["conservative"]),
                                   basis=basis)
    assert st.size - 1 == int(g[f"{tag}_levels"])
    lv2, fo2, sc2, ep = lko.prune_finalize(plan, g["ffa_fold"], int(g["ref_seg"]), st.size - 1, lv, fo, sc,
                                           basis=basis)
    np.testing.assert_array_equal(lv2.view(np.uint64), g[f"{tag}_leaves"].view(np.uint64))
    np.testing.assert_array_equal(fo2.view(np.uint32), g[f"{tag}_folds"].view(np.uint32))
    np.testing.assert_array_equal(sc2.view(np.uint32), g[f"{tag}_scores"].view(np.uint32))
    np.testing.assert_array_equal(ep.view(np.uint32), g[f"{tag}_scores_ep"].view(np.uint32))
    assert lv2.shape[0] > 0


@pytest.mark.skipif(not R.available(), reason="oracle/_ref (the reference build) is not present")
@pytest.mark.parametrize("case", range(len(REF_CASES)))
@pytest.mark.parametrize("basis", ["taylor", "chebyshev"])
def test_oracle_ascend_report_matches_reference_directly(case, basis):
    ns, ts, nb, eta, lim, bf, seed, ms, bs, lo, hi, rf, cons = REF_CASES[case]
    if basis == "chebyshev" and cons:
        pytest.skip("the conservative tile has no Chebyshev form")
    rc = R.make_cfg(ns, ts, nb, eta, lim, bseg_ffa=bf)
    plan = lko.plan_create(lko.make_cfg(ns, ts, nb, eta, lim, bseg_ffa=bf))
    e, v = _series(ns, seed)
    fold = lko.ffa(plan, e, v)
    nseg = int(plan.nsegments[-1])
    ref_seg = min(int(nseg * rf), nseg - 1)
    bm = max(R.branch_max(rc, cons), int(np.ceil(R.branching_pattern_basis(rc, basis, 0, cons).max() * 2)), 32)
    thr = np.linspace(lo, hi, nseg - 1).astype(np.float32)
    for n_iters in (nseg - 1, 2):
        st, lv, fo, sc, ep = R.prune_run_full(rc, fold, thr, ref_seg, ms, bs, bm, n_iters, nb, cons, basis=basis)
        st2, lv2, fo2, sc2 = lko.prune_run(plan, fold, thr, ref_seg, ms, bs, bm, n_iters, cons, basis=basis)
        out = lko.prune_finalize(plan, fold, ref_seg, st2.size - 1, lv2, fo2, sc2, basis=basis)
        for x, y in zip((lv, fo, sc, ep), out):
            np.testing.assert_array_equal(x.view(np.uint8), y.view(np.uint8))
