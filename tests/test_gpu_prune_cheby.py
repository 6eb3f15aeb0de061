"""Chebyshev-basis pruning on the GPU (through the C ABI) against the C
oracle and the reference's own pruning runs: whole runs (per-level
statistics and final trees bit for bit, overload pruning included) and every
single step (basis conversions, branch with its in-place re-centring of the
parents, resolve, transform)."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import golden
from oracle import lko

pytestmark = pytest.mark.gpu

STAT_FIELDS = ("level", "seg_idx", "n_branches", "n_leaves", "n_leaves_phy", "n_leaves_surv",
               "threshold", "score_min", "score_max")

# nsamps, tsamp, nbins, eta, limits, bseg_ffa, seed, max_sugg, batch, thr_lo, thr_hi, ref_frac
CASES = {
    "accel_nb32_overload": (1 << 17, 1e-3, 32, 1.0, [[-20.0, 20.0], [5.0, 6.0]], 1 << 13, 1, 160, 16,
                            1.0, 3.0, 0.5),
    "accel_nb64_eta2": (1 << 19, 5e-4, 64, 2.0, [[-200.0, 200.0], [20.0, 25.0]], 1 << 14, 2, 4096, 64,
                        2.0, 5.0, 0.3),
    "accel_nb32_wrap": (1 << 17, 1e-3, 32, 1.0, [[-20.0, 20.0], [5.0, 7.0]], 1 << 13, 3, 301, 37,
                        0.5, 2.5, 1.0),
    "jerk_nb32": (1 << 18, 1e-3, 32, 1.0, [[-0.2, 0.2], [-20.0, 20.0], [5.0, 6.0]], 1 << 14, 4, 400, 32,
                  1.0, 3.0, 0.2),
    "jerk_nb32_big": (1 << 19, 5e-4, 32, 1.0, [[-0.5, 0.5], [-30.0, 30.0], [20.0, 21.0]], 1 << 14, 5, 4133,
                      100, 2.0, 4.0, 0.7),
}


def _series(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n).astype(np.float32), (1.0 + 0.25 * rng.random(n)).astype(np.float32)


def _setup(name):
    from loki_b200.configs import PulsarSearchConfig

    ns, ts, nb, eta, lim, bf, seed, ms, bs, lo, hi, rf = CASES[name]
    plan = lko.plan_create(lko.make_cfg(ns, ts, nb, eta, lim, bseg_ffa=bf))
    cfg = PulsarSearchConfig(ns, ts, nb, eta, np.array(lim), use_fourier=False, bseg_ffa=bf)
    e, v = _series(ns, seed)
    fold = lko.ffa(plan, e, v)
    nseg = int(plan.nsegments[-1])
    ref_seg = min(int(nseg * rf), nseg - 1)
    thr = np.linspace(lo, hi, nseg - 1).astype(np.float32)
    return plan, cfg, fold, nseg, ref_seg, thr, ms, bs


def _stats_matrix(stats):
    return np.stack([stats[k].astype(np.float64) for k in STAT_FIELDS], axis=1)


def _branch_max(cfg):
    from loki_b200.prune import branching_pattern

    return max(int(np.ceil(branching_pattern(cfg, 0, poly_basis="chebyshev").max() * 2)), 32)


@pytest.mark.parametrize("name", sorted(CASES))
def test_cheby_prune_run_bit_exact(cuda, name):
    from loki_b200.prune import PruneCUDA

    plan, cfg, fold, nseg, ref_seg, thr, ms, bs = _setup(name)
    bm = _branch_max(cfg)
    want = lko.prune_run(plan, fold, thr, ref_seg, ms, bs, bm, nseg - 1, basis="chebyshev")
    pr = PruneCUDA(cfg, max_sugg=ms, batch_size=bs, poly_basis="chebyshev")
    stats = pr.run(fold, ref_seg, thr)
    np.testing.assert_array_equal(_stats_matrix(stats), _stats_matrix(want[0]))
    leaves, folds, scores = pr.tree()
    np.testing.assert_array_equal(leaves, want[1])
    np.testing.assert_array_equal(folds, want[2])
    np.testing.assert_array_equal(scores, want[3])


@pytest.mark.parametrize("name", sorted(CASES))
def test_cheby_finalize_bit_exact(cuda, name):
    """Ascend + report in the Chebyshev basis (leaves converted to Taylor at
    the middle coordinate before the report)."""
    from loki_b200.prune import PruneCUDA

    plan, cfg, fold, nseg, ref_seg, thr, ms, bs = _setup(name)
    bm = _branch_max(cfg)
    pr = PruneCUDA(cfg, max_sugg=ms, batch_size=bs, poly_basis="chebyshev")
    for n_iters in (nseg - 1, max(1, (nseg - 1) // 2)):
        want = lko.prune_run(plan, fold, thr, ref_seg, ms, bs, bm, n_iters, basis="chebyshev")
        lv, fo, sc, ep = lko.prune_finalize(plan, fold, ref_seg, want[0].size - 1, *want[1:], basis="chebyshev")
        pr.run(fold, ref_seg, thr, n_iters=n_iters)
        pr.finalize(fold)
        leaves, folds, scores = pr.tree()
        np.testing.assert_array_equal(leaves.view(np.uint64), lv.view(np.uint64))
        np.testing.assert_array_equal(folds.view(np.uint32), fo.view(np.uint32))
        np.testing.assert_array_equal(scores.view(np.uint32), sc.view(np.uint32))
        np.testing.assert_array_equal(pr.scores_ep().view(np.uint32), ep.view(np.uint32))


@pytest.mark.parametrize("name", ["prune_cheby_accel_nb16.npz", "prune_cheby_jerk_nb16.npz"])
def test_cheby_prune_reference_golden_fixtures(cuda, name):
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.prune import PruneCUDA

    g = golden(name)
    cfg = PulsarSearchConfig(int(g["nsamps"]), float(g["tsamp"]), int(g["nbins"]), float(g["eta"]),
                             g["param_limits"], use_fourier=False, bseg_ffa=int(g["bseg_ffa"]))
    pr = PruneCUDA(cfg, max_sugg=int(g["max_sugg"]), batch_size=int(g["batch_size"]),
                   branch_max=int(g["branch_max"]), poly_basis="chebyshev")
    stats = pr.run(g["ffa_fold"], int(g["ref_seg"]), g["thresholds"])
    np.testing.assert_array_equal(_stats_matrix(stats), g["stats"])
    leaves, folds, scores = pr.tree()
    np.testing.assert_array_equal(leaves, g["leaves"])
    np.testing.assert_array_equal(folds, g["folds"])
    np.testing.assert_array_equal(scores, g["scores"])


def test_cheby_rejects_conservative_and_unknown_basis(cuda):
    from loki_b200 import _capi as C
    from loki_b200.prune import PruneCUDA

    _, cfg, _, _, _, _, ms, bs = _setup("accel_nb32_overload")
    with pytest.raises(C.LokiError):
        PruneCUDA(cfg, max_sugg=ms, batch_size=bs, use_conservative_tile=True, poly_basis="chebyshev")
    with pytest.raises(ValueError):
        PruneCUDA(cfg, max_sugg=ms, batch_size=bs, poly_basis="legendre")


def _dev(t, a, dtype=None):
    return t.from_numpy(np.ascontiguousarray(a if dtype is None else a.astype(dtype))).cuda()


@pytest.mark.parametrize("name", ["accel_nb32_overload", "jerk_nb32"])
def test_cheby_steps_bit_exact(cuda, name):
    from loki_b200 import _capi as C

    t = cuda
    L = C.lib()
    plan, cfg, fold, nseg, ref_seg, thr, ms, bs = _setup(name)
    np_ = plan.nparams
    nb = plan.nbins
    h = cfg._plan_handle
    s = t.cuda.current_stream().cuda_stream
    tseg = float(cfg.tseg_ffa)
    _, c_init, _, _ = lko.middle_out(nseg, ref_seg, tseg, 0)

    # seed, then the basis conversion of the seeds
    seed = lko.taylor_seed(plan)
    want = lko.taylor_to_cheby(seed, np_, c_init)
    d = _dev(t, seed)
    C.check(L.lk_taylor_to_cheby(d.data_ptr(), seed.shape[0], np_, c_init[1], s))
    np.testing.assert_array_equal(d.cpu().numpy(), want)
    back = lko.cheby_to_taylor(want, np_, c_init)
    C.check(L.lk_cheby_to_taylor(d.data_ptr(), seed.shape[0], np_, c_init[1], s))
    np.testing.assert_array_equal(d.cpu().numpy(), back)

    leaves = want
    bm = _branch_max(cfg)
    for level in (1, 2, 3):
        _, coord, cur, segc = lko.middle_out(nseg, ref_seg, tseg, level)
        _, prev, _, _ = lko.middle_out(nseg, ref_seg, tseg, level - 1)
        want_l, want_o, want_par = lko.cheby_branch(leaves, np_, cur, prev, nb, float(cfg.eta), bm)
        d_in = _dev(t, leaves)
        cap = want_l.shape[0] + 5
        d_out = t.empty((cap, np_ + 2, 2), dtype=t.float64, device="cuda")
        d_org = t.empty(cap, dtype=t.int32, device="cuda")
        n = ctypes.c_uint64()
        C.check(L.lk_cheby_branch(h, d_in.data_ptr(), leaves.shape[0], cur[0], cur[1], prev[0], prev[1], bm,
                                  d_out.data_ptr(), d_org.data_ptr(), cap, ctypes.byref(n), s))
        assert n.value == want_l.shape[0]
        np.testing.assert_array_equal(d_in.cpu().numpy(), want_par)
        np.testing.assert_array_equal(d_out[: n.value].cpu().numpy(), want_l)
        np.testing.assert_array_equal(d_org[: n.value].cpu().numpy().astype(np.uint64), want_o)

        coords = np.array([*segc, *cur, *c_init], np.float64)
        pidx_w, ph_w = lko.cheby_resolve(plan, want_l, segc, cur, c_init)
        d_pidx = t.empty(n.value, dtype=t.int32, device="cuda")
        d_ph = t.empty(n.value, dtype=t.float32, device="cuda")
        C.check(L.lk_cheby_resolve(h, d_out.data_ptr(), n.value, coords.ctypes.data, d_pidx.data_ptr(),
                                   d_ph.data_ptr(), s))
        np.testing.assert_array_equal(d_pidx.cpu().numpy().astype(np.uint64), pidx_w)
        np.testing.assert_array_equal(d_ph.cpu().numpy(), ph_w)

        idx = np.arange(0, n.value, 2, dtype=np.uint64)
        tw = lko.cheby_transform(want_l, idx, np_, coord, cur)
        d_t = _dev(t, want_l)
        d_idx = _dev(t, idx, np.int32)
        C.check(L.lk_cheby_transform(h, d_t.data_ptr(), n.value, d_idx.data_ptr(), idx.size, coord[0], coord[1],
                                     cur[0], cur[1], s))
        np.testing.assert_array_equal(d_t.cpu().numpy(), tw)
        leaves = lko.cheby_transform(want_l, np.arange(n.value, dtype=np.uint64), np_, coord, cur)
